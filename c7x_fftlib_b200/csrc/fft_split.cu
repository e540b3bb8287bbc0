// fft_split.cu -- stand-alone split passes of the real-input kernels, used
// when the half-length complex transform is too long for one CTA (global
// passes); shorter transforms fuse these into the FFT kernel.
//   r2c post-process: FFTLIB_fft1dBatched_i32f_c32fc_o32fc_cn.c:40-121
//   c2r pre-process:  FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_cn.c:35-83
#include "fft_device.cuh"
#include "fft_split.h"

namespace fftb200 {

// One thread per pair (i, h-i), i in [0, h/2]; z: batch x h complex,
// y: batch x (h+1) (outmode 0) or batch x 2h (outmode 1).
__global__ void k_r2c_post(const float2* __restrict__ z, float2* __restrict__ y, const float2* __restrict__ wsp,
                           uint32_t h, uint32_t batch, int outmode)
{
    const uint32_t pairs = h / 2u + 1u;
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)pairs * batch) return;
    const uint32_t b = (uint32_t)(g / pairs), i = (uint32_t)(g - (uint64_t)b * pairs);
    const float2* zr = z + (size_t)b * h;
    float2* row = y + (size_t)b * (outmode ? 2u * h : h + 1u);
    if (i == 0) {
        const float2 z0 = zr[0];
        row[0] = make_float2(z0.x + z0.y, 0.f);
        row[h] = make_float2(z0.x - z0.y, 0.f);
        return;
    }
    const uint32_t ip = h - i;
    const float2 zi = zr[i], zp = zr[ip];
    auto split = [](float2 a, float2 ap, float2 w) {
        const float2 ac = cconj(ap);
        const float2 e = cscale(cadd(a, ac), 0.5f), o = cscale(csub(a, ac), 0.5f);
        return cadd(e, cmul(make_float2(w.y, -w.x), o));
    };
    const float2 yi = split(zi, zp, wsp[i]);
    row[i] = yi;
    if (outmode) row[2u * h - i] = cconj(yi);
    if (ip != i) {
        const float2 yp = split(zp, zi, wsp[ip]);
        row[ip] = yp;
        if (outmode) row[2u * h - ip] = cconj(yp);
    }
}

// z[i] = 0.5 [(X[i] + b) + i conj(W) (X[i] - b)], b = conj(X[h-i]) or X[i+h].
FFT_DEV float2 c2r_pre_point(float2 xi, float2 bb, float2 w)
{
    const float2 s = cadd(xi, bb), d = csub(xi, bb);
    return cscale(cadd(s, cmul(make_float2(w.y, w.x), d)), 0.5f);
}

// inMode 0 (h + 1 bins per row): one thread per pair (i, h-i), i in
// [0, h/2], so each bin is read once (X[i] and X[h-i] serve both outputs).
__global__ void k_c2r_pre_pairs(const float2* __restrict__ x, float2* __restrict__ z, const float2* __restrict__ wsp,
                                uint32_t h, uint32_t batch)
{
    const uint32_t pairs = h / 2u + 1u;
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)pairs * batch) return;
    const uint32_t b = (uint32_t)(g / pairs), i = (uint32_t)(g - (uint64_t)b * pairs);
    const float2* row = x + (size_t)b * (h + 1u);
    float2* zr = z + (size_t)b * h;
    const uint32_t ip = h - i;
    const float2 xi = row[i], xp = row[ip];
    zr[i] = c2r_pre_point(xi, cconj(xp), wsp[i]);
    if (i != 0u && ip != i) zr[ip] = c2r_pre_point(xp, cconj(xi), wsp[ip]);
}

// inMode 1 (2h bins per row): one thread per output point.
__global__ void k_c2r_pre(const float2* __restrict__ x, float2* __restrict__ z, const float2* __restrict__ wsp,
                          uint32_t h, uint32_t batch, int inmode)
{
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (uint64_t)h * batch) return;
    const uint32_t b = (uint32_t)(g / h), i = (uint32_t)(g - (uint64_t)b * h);
    const float2* row = x + (size_t)b * (inmode ? 2u * h : h + 1u);
    const float2 xi = row[i];
    const float2 bb = inmode ? row[i + h] : cconj(row[h - i]);
    z[(size_t)b * h + i] = c2r_pre_point(xi, bb, wsp[i]);
}

cudaError_t launch_r2c_post(const float2* z, float2* y, const float2* wsp, uint32_t h, uint32_t batch,
                            int outmode, cudaStream_t s)
{
    const uint64_t total = (uint64_t)(h / 2u + 1u) * batch;
    if (total == 0) return cudaSuccess;
    k_r2c_post<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(z, y, wsp, h, batch, outmode);
    return cudaGetLastError();
}

cudaError_t launch_c2r_pre(const float2* x, float2* z, const float2* wsp, uint32_t h, uint32_t batch,
                           int inmode, cudaStream_t s)
{
    if (!inmode) {
        const uint64_t pairs = (uint64_t)(h / 2u + 1u) * batch;
        if (pairs == 0 || h == 0) return cudaSuccess;
        k_c2r_pre_pairs<<<(unsigned)((pairs + 255) / 256), 256, 0, s>>>(x, z, wsp, h, batch);
        return cudaGetLastError();
    }
    const uint64_t total = (uint64_t)h * batch;
    if (total == 0) return cudaSuccess;
    k_c2r_pre<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(x, z, wsp, h, batch, inmode);
    return cudaGetLastError();
}

} // namespace fftb200
