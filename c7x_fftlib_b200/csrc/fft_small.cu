// fft_small.cu -- FP32 c2c of lengths 2..32 and 45 with one transform per
// thread.
//
// For these lengths every exchange-based schedule spends its time on
// shared-memory traffic and barriers around a few butterflies (the
// pipelined kernel's two passes ran N = 8 at 2.6 TB/s and N = 16 at
// 3.3 TB/s). Here a CTA of 256 (128 above N = 16, 64 above 32) threads takes
// as many consecutive transforms (their values contiguous): the threads copy them into shared memory with
// coalesced 8- or 16-byte accesses (rows padded to an odd number of values,
// so that one row per lane is conflict-free), each thread runs the
// in-register DFT codelet dft<N> (natural order in and out) on its row, and
// the block goes back out coalesced.
#include <algorithm>

#include "fft_engine.h"
#include "fft_stockham.cuh"
#include "plan.h"

namespace fftb200 {

namespace {

// transforms (threads) per CTA: 256, 128 above N = 16, 64 above N = 32 (the
// padded rows stay within 48 KB of static shared memory)
template <int N>
constexpr int small_rows() { return N <= 16 ? 256 : (N <= 32 ? 128 : 64); }

template <int N>
__global__ void __launch_bounds__(small_rows<N>()) k_fft_small(const __grid_constant__ FftArgs a, bool vec)
{
    constexpr int kSmallRows = small_rows<N>();
    constexpr int S = N | 1;  // padded row length
    __shared__ float2 rows[kSmallRows * S];
    // a launch that follows with programmatic stream serialization may start
    // now (a no-op otherwise)
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const uint32_t tid = threadIdx.x;
    const uint64_t blocks = (a.batch + kSmallRows - 1u) / kSmallRows;
    for (uint64_t blk = blockIdx.x; blk < blocks; blk += gridDim.x) {
        const uint64_t b0 = blk * kSmallRows;
        const uint32_t cnt = (uint32_t)min((uint64_t)kSmallRows, a.batch - b0);
        const uint32_t vals = cnt * (uint32_t)N;
        const float2* src = a.in + b0 * (uint64_t)N;
        float2* dst = a.out + b0 * (uint64_t)N;
        // in: value i of the block -> row i / N, column i % N
        if (vec && (vals % 2u) == 0u) {
            for (uint32_t p = tid; p < vals / 2u; p += kSmallRows) {
                const float4 q = __ldg(reinterpret_cast<const float4*>(src) + p);
                const uint32_t i = 2u * p;
                rows[(i / N) * S + i % N] = make_float2(q.x, q.y);
                rows[((i + 1u) / N) * S + (i + 1u) % N] = make_float2(q.z, q.w);
            }
        } else {
            for (uint32_t i = tid; i < vals; i += kSmallRows) rows[(i / N) * S + i % N] = __ldg(src + i);
        }
        __syncthreads();
        if (tid < cnt) {
            float2 v[N];
            static_for<N>([&](auto k) FFT_INL { v[k] = rows[tid * S + decltype(k)::value]; });
            if (a.conjIn) {
                static_for<N>([&](auto k) FFT_INL { v[k] = cconj(v[k]); });
            }
            dft<N>(v);
            if (a.conjOut || a.scale != 1.0f) {
                static_for<N>([&](auto k) FFT_INL { v[k] = finish(a, v[k]); });
            }
            static_for<N>([&](auto k) FFT_INL { rows[tid * S + decltype(k)::value] = v[k]; });
        }
        __syncthreads();
        if (vec && (vals % 2u) == 0u) {
            for (uint32_t p = tid; p < vals / 2u; p += kSmallRows) {
                const uint32_t i = 2u * p;
                const float2 x = rows[(i / N) * S + i % N], y = rows[((i + 1u) / N) * S + (i + 1u) % N];
                reinterpret_cast<float4*>(dst)[p] = make_float4(x.x, x.y, y.x, y.y);
            }
        } else {
            for (uint32_t i = tid; i < vals; i += kSmallRows) dst[i] = rows[(i / N) * S + i % N];
        }
        __syncthreads();  // the rows are refilled for the next block
    }
}

template <int N>
cudaError_t launch_small_n(const FftArgs& a, cudaStream_t s)
{
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    constexpr int kSmallRows = small_rows<N>();
    const uint64_t blocks = (a.batch + kSmallRows - 1u) / kSmallRows;
    const uint32_t grid = (uint32_t)std::min<uint64_t>(blocks, (uint64_t)std::max(sms, 1) * 8u);
    const bool vec = ((((uintptr_t)a.in) | ((uintptr_t)a.out)) & 15u) == 0;
    if (a.overlapPrev) {  // see FftArgs::overlapPrev
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(grid);
        lc.blockDim = dim3((unsigned)kSmallRows);
        lc.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        lc.attrs = attr;
        lc.numAttrs = 1;
        return cudaLaunchKernelEx(&lc, k_fft_small<N>, a, vec);
    }
    k_fft_small<N><<<grid, kSmallRows, 0, s>>>(a, vec);
    return cudaGetLastError();
}

} // namespace

bool small_fft_length(uint32_t n)
{
    switch (n) {
    case 2: case 3: case 4: case 5: case 6: case 8: case 9: case 10: case 12: case 15: case 16:
    case 18: case 20: case 24: case 25: case 27: case 30: case 32:
    case 45:  // its two-pass schedule ran at 2.7 TB/s (here 4.7; 50, 60 and 75 measured
              // slower here than their 3.5-3.8 TB/s two-pass schedules)
        return true;
    default:
        return false;
    }
}

bool small_fft_eligible(const FftArgs& a)
{
    return small_fft_length(a.N) && a.ioMode == IO_C2C && !a.perCh && !a.batchMinor && a.inElem == 1 &&
           a.outElem == 1 && a.inBatch == (int64_t)a.N && a.outBatch == (int64_t)a.N;
}

cudaError_t launch_fft_small(const FftArgs& a, cudaStream_t s)
{
    if (a.batch == 0) return cudaSuccess;
    switch (a.N) {
    case 2: return launch_small_n<2>(a, s);
    case 3: return launch_small_n<3>(a, s);
    case 4: return launch_small_n<4>(a, s);
    case 5: return launch_small_n<5>(a, s);
    case 6: return launch_small_n<6>(a, s);
    case 8: return launch_small_n<8>(a, s);
    case 9: return launch_small_n<9>(a, s);
    case 10: return launch_small_n<10>(a, s);
    case 12: return launch_small_n<12>(a, s);
    case 15: return launch_small_n<15>(a, s);
    case 16: return launch_small_n<16>(a, s);
    case 18: return launch_small_n<18>(a, s);
    case 20: return launch_small_n<20>(a, s);
    case 24: return launch_small_n<24>(a, s);
    case 25: return launch_small_n<25>(a, s);
    case 27: return launch_small_n<27>(a, s);
    case 30: return launch_small_n<30>(a, s);
    case 32: return launch_small_n<32>(a, s);
    case 45: return launch_small_n<45>(a, s);
    default: return cudaErrorInvalidValue;
    }
}

} // namespace fftb200
