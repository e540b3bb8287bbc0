// tables.cu -- the reference's table generators on the GPU, bit-identical
// to the host generators of capi_ext.cu and capi_mma.cu (same formulas, pi
// truncated to 3.141592654, the same order of double operations; cos and
// sin are CUDA's double functions):
//   stage-twiddle tables (c2c / ifft / r2c / c2r, the half-length c2c table)
//     test/fft_c7x/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/..._d.c:30-96,
//     src/fft_c7x/FFTLIB_fft1dBatched_i32f_c32fc_o32fc/..._tw_gen.cpp:9-78,
//     src/fft_c7x/FFTLIB_ifft1dBatched_i32fc_c32fc_o32f/..._tw_gen.cpp:9-79;
//   the int16 Q15 table (test/fft_c7x/FFTLIB_fft1dBatched_i16sc_c16sc_o16sc/..._d.c:29-61);
//   the r2c / c2r split factors (..._tw_gen.cpp:80-97 and :81-95);
//   the coordinator's dense dftLarge matrix (c71/FFTLIB_FFT_dftLarge_ixX_cxX_oxX_ci.cpp:122-138).
// One thread per table entry (or entry pair); the stage structure of the
// twiddle tables is flattened on the host into segments, one per stage.
#include <math.h>

#include "capi_common.h"
#include "fftlib_b200_ext.h"
#include "tables.h"

namespace fftb200 {

namespace {

constexpr double kTablePi = 3.141592654;
constexpr int kMaxSegs = 48;

// One stage of a stage-twiddle table: entries i = 0, j, 2j, ... < m0/r, each
// writing r-1 complex values W^(m i), m = 1..r-1, at k0 + 2 idx + 2 (m-1) t.
struct TwSeg {
    uint32_t k0, m0, r, j, t, count;
    uint64_t firstItem;  // items (entry, m) before this segment
};
struct TwPlan {
    int nseg;
    uint64_t items;
    TwSeg seg[kMaxSegs];
};

// The loop of one radix block of the FP32 table (capi_ext.cu twiddle_block).
uint32_t plan_block(TwPlan& p, uint32_t* k, uint32_t m0, uint32_t r)
{
    uint32_t rest = m0, t = m0 / r;
    for (uint32_t j = 1; j <= m0 / r && rest % r == 0; j *= r) {
        const uint32_t count = (m0 / r + j - 1) / j;
        if (p.nseg < kMaxSegs) p.seg[p.nseg++] = TwSeg{*k, m0, r, j, t, count, p.items};
        p.items += (uint64_t)count * (r - 1u);
        *k += 2u * count;
        *k += 2u * t * (r - 2u);
        t /= r;
        rest /= r;
    }
    return rest;
}

TwPlan plan_f32(uint32_t n)
{
    TwPlan p{};
    uint32_t k = 0;
    if (n % 5u == 0u) n = plan_block(p, &k, n, 5u);
    if (n % 3u == 0u) n = plan_block(p, &k, n, 3u);
    if (n % 4u == 0u) plan_block(p, &k, n, 4u);
    return p;
}

// The Q15 table: radix-4 stages over the full length.
TwPlan plan_i16(uint32_t n)
{
    TwPlan p{};
    uint32_t k = 0, t = n >> 2;
    for (uint32_t j = 1; j <= (n >> 2); j <<= 2) {
        const uint32_t count = ((n >> 2) + j - 1) / j;
        if (p.nseg < kMaxSegs) p.seg[p.nseg++] = TwSeg{k, n, 4u, j, t, count, p.items};
        p.items += (uint64_t)count * 3u;
        k += 2u * count + 4u * t;
        t >>= 2;
    }
    return p;
}

__device__ __forceinline__ int16_t round_q15(double x)
{
    x = floor(0.5 + x);
    if (x >= 32767.0) return 32767;
    if (x <= -32768.0) return -32768;
    return (int16_t)x;
}

template <bool Q15>
__global__ void k_stage_twiddles(TwPlan p, void* out)
{
    const uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= p.items) return;
    int s = 0;
    while (s + 1 < p.nseg && p.seg[s + 1].firstItem <= item) ++s;
    const TwSeg g = p.seg[s];
    const uint32_t within = (uint32_t)(item - g.firstItem);
    const uint32_t idx = within / (g.r - 1u), m = within % (g.r - 1u) + 1u;
    const uint32_t i = idx * g.j;
    const double ang = (double)(2u * m) * kTablePi * (double)i / (double)g.m0;
    const size_t e = (size_t)g.k0 + 2u * idx + 2u * (m - 1u) * g.t;
    if (Q15) {
        int16_t* w = static_cast<int16_t*>(out);
        w[e] = round_q15(32767.5 * cos(ang));
        w[e + 1] = round_q15(32767.5 * (-sin(ang)));
    } else {
        float* w = static_cast<float*>(out);
        w[e] = (float)cos(ang);
        w[e + 1] = (float)-sin(ang);
    }
}

// r2c (c2r = false) and c2r split factors of n points.
template <bool C2R>
__global__ void k_split_factors(float* sf, int32_t n)
{
    const int32_t i = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= n / 2) return;
    const double ang = 2.0 * kTablePi * (double)i / (double)n;
    if (!C2R) {
        sf[2 * i] = (float)(0.5 * (1.0 - sin(ang)));
        sf[2 * i + 1] = (float)(0.5 * (-cos(ang)));
        sf[2 * n - 2 * i - 2] = (float)(0.5 * (1.0 + sin(ang)));
        sf[2 * n - 2 * i - 1] = (float)(0.5 * cos(ang));
    } else {
        sf[2 * i] = (float)(0.5 * (1.0 - sin(ang)));
        sf[2 * i + 1] = (float)(0.5 * cos(ang));
        sf[2 * i + n] = (float)(0.5 * (1.0 + sin(ang)));
        sf[2 * i + n + 1] = (float)(0.5 * (-cos(ang)));
    }
}

// Round half up of scale * v with saturation, scale = 2^(bits-1) - 0.5
// (the host table_entry of dft_int.cu).
__device__ __forceinline__ int32_t table_entry(double v, int bits)
{
    const double scale = (double)((1u << (bits - 2)) - 1u) + (double)(1u << (bits - 2)) + 0.5;
    const long long x = (long long)floor(0.5 + scale * v);
    const long long mx = (1ll << (bits - 1)) - 1;
    return (int32_t)(x >= mx ? mx : (x <= -mx - 1 ? -mx - 1 : x));
}

// The dftLarge matrix: for (j, k) < n, the 2 x 2 real block of W_n^(j k).
template <class T>
__global__ void k_dft_large_matrix(T* w, uint32_t n, uint32_t interleave, int bits)
{
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint64_t)n * n) return;
    const uint32_t j = (uint32_t)(e / n), k = (uint32_t)(e % n);
    const double a = 2 * kTablePi * j * k / n;
    const T c = (T)table_entry(cos(a), bits), sn = (T)table_entry(sin(a), bits);
    if (interleave) {
        w[(size_t)j * 4u * n + 2 * k] = c;
        w[(size_t)j * 4u * n + 2 * k + 1] = (T)-sn;
        w[(size_t)(2 * j + 1) * 2u * n + 2 * k] = sn;
        w[(size_t)(2 * j + 1) * 2u * n + 2 * k + 1] = c;
    } else {
        w[(size_t)j * 2u * n + k] = c;
        w[(size_t)j * 2u * n + n + k] = (T)-sn;
        w[(size_t)2u * n * n + j * 2u * n + k] = sn;
        w[(size_t)2u * n * n + j * 2u * n + n + k] = c;
    }
}

unsigned blocks_for(uint64_t items) { return (unsigned)((items + 255u) / 256u); }

} // namespace

cudaError_t stage_twiddles_device(void* out, uint32_t n, bool q15, cudaStream_t s)
{
    const TwPlan p = q15 ? plan_i16(n) : plan_f32(n);
    if (p.nseg >= kMaxSegs) return cudaErrorInvalidValue;
    if (p.items == 0) return cudaSuccess;
    if (q15) k_stage_twiddles<true><<<blocks_for(p.items), 256, 0, s>>>(p, out);
    else k_stage_twiddles<false><<<blocks_for(p.items), 256, 0, s>>>(p, out);
    return cudaGetLastError();
}

cudaError_t split_factors_device(float* sf, int32_t n, bool c2r, cudaStream_t s)
{
    if (n / 2 <= 0) return cudaSuccess;
    if (c2r) k_split_factors<true><<<blocks_for((uint64_t)(n / 2)), 256, 0, s>>>(sf, n);
    else k_split_factors<false><<<blocks_for((uint64_t)(n / 2)), 256, 0, s>>>(sf, n);
    return cudaGetLastError();
}

cudaError_t dft_large_matrix_device(void* w, int bits, uint32_t n, uint32_t interleave, cudaStream_t s)
{
    const uint64_t items = (uint64_t)n * n;
    if (items == 0) return cudaSuccess;
    if (blocks_for(items) > 0x7FFFFFFFu) return cudaErrorInvalidValue;
    if (bits == 16)
        k_dft_large_matrix<int16_t><<<blocks_for(items), 256, 0, s>>>(static_cast<int16_t*>(w), n, interleave, 16);
    else
        k_dft_large_matrix<int32_t><<<blocks_for(items), 256, 0, s>>>(static_cast<int32_t*>(w), n, interleave, 32);
    return cudaGetLastError();
}

} // namespace fftb200

using namespace fftb200;

namespace {

FFTLIB_STATUS device_result(cudaError_t e, const char* what)
{
    return e == cudaSuccess ? FFTLIB_SUCCESS : cuda_fail(e, what);
}

FFTLIB_STATUS need_device(const void* p)
{
    if (!p) return FFTLIB_ERR_NULL_POINTER;
    if (!is_device_ptr(p)) {
        set_error("the device table generators write device memory");
        return FFTLIB_ERR_INVALID_VALUE;
    }
    return FFTLIB_SUCCESS;
}

} // namespace

extern "C" {

FFTLIB_STATUS FFTLIB_b200_tw_gen_c2c_device(FFTLIB_F32* pW, uint32_t numPoints, void* stream)
{
    FFTLIB_STATUS st = need_device(pW);
    if (st != FFTLIB_SUCCESS) return st;
    return device_result(stage_twiddles_device(pW, numPoints, false, (cudaStream_t)stream), "tw_gen_c2c_device");
}

FFTLIB_STATUS FFTLIB_b200_tw_gen_i16_device(int16_t* pW, uint32_t numPoints, void* stream)
{
    FFTLIB_STATUS st = need_device(pW);
    if (st != FFTLIB_SUCCESS) return st;
    // the int16 kernel's lengths; for others the host generator's blocks
    // overlap and its result depends on its write order
    if (numPoints & (numPoints - 1u)) {
        set_error("tw_gen_i16_device: numPoints %u is not a power of two", numPoints);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    return device_result(stage_twiddles_device(pW, numPoints, true, (cudaStream_t)stream), "tw_gen_i16_device");
}

FFTLIB_STATUS FFTLIB_b200_tw_gen_r2c_device(FFTLIB_F32* pW, int32_t numPoints, void* stream)
{
    FFTLIB_STATUS st = need_device(pW);
    if (st != FFTLIB_SUCCESS) return st;
    if (numPoints < 0) return FFTLIB_ERR_INVALID_DIMENSION;
    return device_result(stage_twiddles_device(pW, (uint32_t)numPoints >> 1, false, (cudaStream_t)stream),
                         "tw_gen_r2c_device");
}

FFTLIB_STATUS FFTLIB_b200_split_factor_gen_r2c_device(FFTLIB_F32* pSFactor, int32_t numPoints, void* stream)
{
    FFTLIB_STATUS st = need_device(pSFactor);
    if (st != FFTLIB_SUCCESS) return st;
    if (numPoints < 0) return FFTLIB_ERR_INVALID_DIMENSION;
    return device_result(split_factors_device(pSFactor, numPoints, false, (cudaStream_t)stream),
                         "split_factor_gen_r2c_device");
}

FFTLIB_STATUS FFTLIB_b200_ifft_c2r_tw_gen_device(FFTLIB_F32* pW, int32_t numPoints, void* stream)
{
    return FFTLIB_b200_tw_gen_r2c_device(pW, numPoints, stream);
}

FFTLIB_STATUS FFTLIB_b200_ifft_c2r_split_factor_gen_device(FFTLIB_F32* pSFactor, int32_t numPoints, void* stream)
{
    FFTLIB_STATUS st = need_device(pSFactor);
    if (st != FFTLIB_SUCCESS) return st;
    if (numPoints < 0) return FFTLIB_ERR_INVALID_DIMENSION;
    return device_result(split_factors_device(pSFactor, numPoints, true, (cudaStream_t)stream),
                         "ifft_c2r_split_factor_gen_device");
}

} // extern "C"
