// fft_f64.cu -- FP64 oracle FFT on the GPU (the harness's FP64 reference).
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/ as the checker for the
// benchmark-size batches (millions of transforms), where numpy's FP64 FFT on
// the host would need minutes. Never linked into libfftlib_b200.so.
//
// The transform is the DFT the reference's tests define,
// X[k] = sum_n x[n] exp(-2 pi i n k / N) (test generator
// test/fft_c7x/FFTLIB_idat_gen/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/
// fft1dBatched_i32fc_c32fc_o32fc.py:33-34, np.fft.fft), and for the inverse
// x[n] = (1/N) sum_k X[k] exp(+2 pi i n k / N)
// (FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_cn.c:209-227).
//
// Algorithm: textbook Stockham autosort passes in FP64, one launch per pass,
// global-memory ping-pong, radices 4, 2, 3, 5 (and a direct O(N^2) DFT for
// lengths with another prime factor). Every twiddle is computed where it is
// used as sincospi(2 e / m) with the exponent e reduced exactly in integers,
// so no rounding accumulates across passes. Accuracy is that of FP64
// arithmetic (rel-L2 ~1e-16 against the exact DFT); speed does not matter.
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// exp(sign * 2 pi i e / m), 0 <= e < m
__device__ __forceinline__ double2 unit(uint64_t e, uint64_t m, double sign)
{
    double s, c;
    sincospi(2.0 * (double)e / (double)m, &s, &c);
    return make_double2(c, sign * s);
}

// One Stockham pass of radix R: butterfly j < n/R reads x[j + q n/R],
// multiplies input q by W_{ns R}^{q (j mod ns)}, takes the R-point DFT and
// writes output p to y[(j / ns) ns R + (j mod ns) + p ns].
template <int R>
__global__ void k_pass(const double2* __restrict__ in, double2* __restrict__ out, uint32_t n, uint32_t ns,
                       uint64_t batch, double sign)
{
    const uint32_t nb = n / R;
    const uint64_t total = batch * nb;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = t / nb;
        const uint32_t j = (uint32_t)(t - b * nb);
        const double2* x = in + b * n;
        double2* y = out + b * n;
        const uint32_t k = j % ns;
        double2 v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            v[q] = x[j + (uint64_t)q * nb];
            if (q) v[q] = cmul(v[q], unit((uint64_t)q * k, (uint64_t)ns * R, sign));
        }
        const uint64_t base = (uint64_t)(j / ns) * ns * R + k;
#pragma unroll
        for (int p = 0; p < R; ++p) {
            double2 acc = v[0];
#pragma unroll
            for (int q = 1; q < R; ++q) {
                const double2 m = cmul(v[q], unit((uint64_t)((p * q) % R), R, sign));
                acc.x += m.x;
                acc.y += m.y;
            }
            y[base + (uint64_t)p * ns] = acc;
        }
    }
}

// Direct DFT (lengths with a prime factor other than 2, 3, 5).
__global__ void k_direct(const double2* __restrict__ in, double2* __restrict__ out, uint32_t n, uint64_t batch,
                         double sign)
{
    const uint64_t total = batch * n;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = t / n;
        const uint32_t k = (uint32_t)(t - b * n);
        const double2* x = in + b * n;
        double2 acc = make_double2(0.0, 0.0);
        for (uint32_t i = 0; i < n; ++i) {
            const double2 m = cmul(x[i], unit(((uint64_t)i * k) % n, n, sign));
            acc.x += m.x;
            acc.y += m.y;
        }
        out[t] = acc;
    }
}

__global__ void k_scale(double2* __restrict__ y, uint64_t count, double s)
{
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < count;
         t += (uint64_t)gridDim.x * blockDim.x) {
        y[t].x *= s;
        y[t].y *= s;
    }
}

unsigned grid_for(uint64_t work)
{
    const uint64_t g = (work + 255) / 256;
    return (unsigned)(g < 148ull * 64 ? (g ? g : 1) : 148ull * 64);
}

} // namespace

extern "C" {

// y = DFT (inverse != 0: the scaled inverse DFT) of `batch` contiguous rows of
// n interleaved complex doubles. x is preserved; work holds n * batch complex
// values. All pointers are device pointers; the passes run on `stream`.
// Returns 0, or the CUDA error code of a failed launch.
int orc_gpu_fft_f64(const double* x, double* y, double* work, uint32_t n, uint64_t batch, int inverse,
                    void* stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    const double sign = inverse ? 1.0 : -1.0;
    const double2* in = (const double2*)x;
    double2* out = (double2*)y;
    double2* tmp = (double2*)work;
    if (n == 0 || batch == 0) return 0;
    // radix sequence
    int rad[64];
    int P = 0;
    uint32_t r = n;
    while (r % 4 == 0) rad[P++] = 4, r /= 4;
    while (r % 2 == 0) rad[P++] = 2, r /= 2;
    while (r % 3 == 0) rad[P++] = 3, r /= 3;
    while (r % 5 == 0) rad[P++] = 5, r /= 5;
    if (r != 1 || n == 1) {
        if (n == 1) {
            cudaError_t e = cudaMemcpyAsync(out, in, batch * sizeof(double2), cudaMemcpyDeviceToDevice, s);
            return (int)e;
        }
        k_direct<<<grid_for(batch * n), 256, 0, s>>>(in, out, n, batch, sign);
    } else {
        const double2* src = in;
        uint32_t ns = 1;
        for (int p = 0; p < P; ++p) {
            double2* dst = ((P - p) % 2 == 1) ? out : tmp;
            const uint64_t work_items = batch * (n / (uint32_t)rad[p]);
            const unsigned g = grid_for(work_items);
            switch (rad[p]) {
            case 4: k_pass<4><<<g, 256, 0, s>>>(src, dst, n, ns, batch, sign); break;
            case 2: k_pass<2><<<g, 256, 0, s>>>(src, dst, n, ns, batch, sign); break;
            case 3: k_pass<3><<<g, 256, 0, s>>>(src, dst, n, ns, batch, sign); break;
            default: k_pass<5><<<g, 256, 0, s>>>(src, dst, n, ns, batch, sign); break;
            }
            src = dst;
            ns *= (uint32_t)rad[p];
        }
    }
    if (inverse) k_scale<<<grid_for(batch * n), 256, 0, s>>>(out, batch * n, 1.0 / (double)n);
    return (int)cudaGetLastError();
}

} // extern "C"
