// tc_dft.cu -- tensor-core DFT: supported lengths, the FP32 computational
// matrix (FP64 generation), launch dispatch.
#include <math.h>

#include "tc_dft.h"

namespace fftb200 {

bool tc_dft_supported(uint32_t n)
{
    return n >= 8 && n <= 4096 && (n & (n - 1u)) == 0;
}

void tc_dft_factors(uint32_t n, uint32_t* n1, uint32_t* n2)
{
    switch (n) {
    case 128: *n1 = 16, *n2 = 8; return;
    case 256: *n1 = 16, *n2 = 16; return;
    case 512: *n1 = 32, *n2 = 16; return;
    case 1024: *n1 = 32, *n2 = 32; return;
    case 2048: *n1 = 64, *n2 = 32; return;
    case 4096: *n1 = 64, *n2 = 64; return;
    default: *n1 = n, *n2 = 1; return;
    }
}

size_t tc_dft_w_floats(uint32_t n)
{
    uint32_t n1, n2;
    tc_dft_factors(n, &n1, &n2);
    if (n2 == 1) return (size_t)4u * n * n;
    return (size_t)4u * n1 * n1 + (size_t)4u * n2 * n2 + 2u * (size_t)n;
}

namespace {

// Element i of the matrix buffer as (index within a block, block kind):
// the real embedding of an m-point DFT occupies (2m)^2 floats, the twiddle
// block 2n floats.
struct WLayout {
    uint32_t n, n1, n2;
    size_t e1, e2, total;
};

WLayout wlayout(uint32_t n)
{
    WLayout L;
    L.n = n;
    tc_dft_factors(n, &L.n1, &L.n2);
    L.e1 = (size_t)4u * L.n1 * L.n1;
    L.e2 = L.n2 == 1 ? 0 : (size_t)4u * L.n2 * L.n2;
    L.total = tc_dft_w_floats(n);
    return L;
}

// Value of element i: embedding entries are cos / -sin / sin / cos of
// 2 pi ((j k) mod m) / m, twiddles cos / -sin of 2 pi j / n.
__host__ __device__ inline void w_angle(const WLayout& L, size_t i, uint64_t* num, uint64_t* den, int* kind)
{
    size_t off = i;
    uint32_t m = L.n1;
    if (off >= L.e1) {
        off -= L.e1;
        m = L.n2;
        if (L.n2 == 1 || off >= L.e2) {
            off -= L.e2;
            *num = off / 2;
            *den = L.n;
            *kind = (off & 1) ? 1 : 0;  // re = cos, im = -sin
            return;
        }
    }
    const size_t w2 = 2u * (size_t)m;
    const uint32_t rowIdx = (uint32_t)(off / w2), colIdx = (uint32_t)(off % w2);
    const uint32_t j = rowIdx >> 1, cin = rowIdx & 1u, k = colIdx >> 1, cout = colIdx & 1u;
    *num = ((uint64_t)j * k) % m;
    *den = m;
    // [cos, -sin | sin, cos]
    *kind = cin == cout ? 0 : (cin == 0 ? 1 : 2);
}

__global__ void k_tc_gen_w(float* w, WLayout L)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.total) return;
    uint64_t num, den;
    int kind;
    w_angle(L, i, &num, &den, &kind);
    double s, c;
    sincospi(2.0 * (double)num / (double)den, &s, &c);
    w[i] = (float)(kind == 0 ? c : (kind == 1 ? -s : s));
}

} // namespace

cudaError_t tc_dft_gen_w_device(float* w, uint32_t n, cudaStream_t s)
{
    if (!tc_dft_supported(n)) return cudaErrorInvalidValue;
    const WLayout L = wlayout(n);
    k_tc_gen_w<<<(unsigned)((L.total + 255) / 256), 256, 0, s>>>(w, L);
    return cudaGetLastError();
}

void tc_dft_gen_w_host(float* w, uint32_t n)
{
    if (!tc_dft_supported(n)) return;
    const WLayout L = wlayout(n);
    const double twoPi = 6.283185307179586476925286766559;
    for (size_t i = 0; i < L.total; ++i) {
        uint64_t num, den;
        int kind;
        w_angle(L, i, &num, &den, &kind);
        const double a = twoPi * (double)num / (double)den;
        w[i] = (float)(kind == 0 ? cos(a) : (kind == 1 ? -sin(a) : sin(a)));
    }
}

cudaError_t launch_tc_dft(uint32_t n, const float2* x, float2* y, const float* w, uint32_t batch, uint32_t* err,
                          cudaStream_t s)
{
    if (!tc_dft_supported(n)) return cudaErrorInvalidValue;
    if (n <= 64) return launch_tc_one(n, x, y, w, batch, err, s);
    return launch_tc_two(n, x, y, w, batch, err, s);
}

} // namespace fftb200
