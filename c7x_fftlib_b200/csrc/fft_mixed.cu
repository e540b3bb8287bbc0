// fft_mixed.cu -- persistent kernel for batches of FP32 c2c transforms of
// uneven lengths (K6).
//
// The host groups the transforms by length; every group has its own
// schedule (FftArgs: radices, threads per transform T, transforms per tile
// M, twiddle table) and its transforms are cut into tiles of M. Tiles are
// ordered by cost, largest first. A grid of resident CTAs pulls tiles from a
// global counter (atomicAdd; no waiting involved) and runs the group's
// schedule with the runtime-planned engine code, reading and writing each
// transform at its own offset in the packed input/output arrays.
#include <algorithm>
#include <mutex>

#include "fft_mixed.h"
#include "fft_stockham.cuh"

namespace fftb200 {

template <int EMAX, int BLK>
__global__ void __launch_bounds__(BLK) k_fft_mixed(const MixedGroup* __restrict__ groups,
                                                   const MixedTile* __restrict__ tiles, uint32_t numTiles,
                                                   const uint64_t* __restrict__ offsets, const float2* x, float2* y,
                                                   uint32_t* counter)
{
    extern __shared__ __align__(16) float2 smem[];
    __shared__ uint32_t s_tile;
    // the group's schedule is read many times per pass: keep a copy in
    // shared memory for the tile instead of re-reading it from global memory
    __shared__ __align__(16) FftArgs s_args;
    static_assert(sizeof(FftArgs) % 4 == 0 && sizeof(FftArgs) / 4 <= BLK, "FftArgs copy");
    const uint32_t tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t ti = s_tile;
        if (ti >= numTiles) break;
        const MixedTile tl = tiles[ti];
        if (tid < sizeof(FftArgs) / 4)
            reinterpret_cast<uint32_t*>(&s_args)[tid] = reinterpret_cast<const uint32_t*>(&groups[tl.group].args)[tid];
        __syncthreads();
        const FftArgs& a = s_args;
        const uint32_t T = a.T, used = T * a.M;
        // threads beyond T*M get a lane index past every butterfly: they only
        // take part in the barriers
        uint32_t m = 0, t = 0xFFFFu;
        if (tid < used) {
            m = tid / T;
            t = tid - m * T;
        }
        const bool active = tid < used && m < tl.count;
        const uint64_t off = active ? offsets[tl.first + m] : 0;
        const float2* rowIn = x + off;
        float2* rowOut = y + off;
        float2* sm = smem + m * a.slen;
        float2 v[EMAX];
        for (int p = 0; p < (int)a.P; ++p) {
            dispatch_radix<EMAX>(a.pass[p].R, [&](auto r) {
                run_pass<EMAX, decltype(r)::value>(a, a.pass[p], p == 0, p + 1 == (int)a.P, T, v, sm, t, active,
                                                   rowIn, rowOut);
            });
        }
        __syncthreads(); // shared memory and s_tile are reused by the next tile
    }
}

namespace {
constexpr int kMixedEmax = 20;
constexpr int kMixedBlock = 256;
} // namespace

int mixed_emax() { return kMixedEmax; }
int mixed_block() { return kMixedBlock; }

cudaError_t mixed_configure(size_t smem, int* residentPerSm)
{
    auto k = k_fft_mixed<kMixedEmax, kMixedBlock>;
    if (smem > 48u * 1024u) {
        // the limit only ever grows, so launches planned earlier stay valid
        static std::mutex mu;
        static size_t configured[64] = {};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        std::lock_guard<std::mutex> lock(mu);
        if (dev >= 64 || configured[dev] < smem) {
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            if (dev < 64) configured[dev] = smem;
        }
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(residentPerSm, k, kMixedBlock, smem);
}

void* mixed_kernel_symbol() { return (void*)k_fft_mixed<kMixedEmax, kMixedBlock>; }

cudaError_t launch_mixed(const MixedLaunch& L, cudaStream_t s)
{
    if (L.numTiles == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(L.counter, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    k_fft_mixed<kMixedEmax, kMixedBlock><<<L.grid, kMixedBlock, L.smem, s>>>(L.groups, L.tiles, L.numTiles,
                                                                               L.offsets, L.x, L.y, L.counter);
    return cudaGetLastError();
}

} // namespace fftb200
