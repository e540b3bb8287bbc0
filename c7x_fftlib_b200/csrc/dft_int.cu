// dft_int.cu -- integer (INT16 / INT32) DFT of the coordinator, bit-exact
// with the reference's natural-C arithmetic (see dft_int.h for the sources
// each part follows). Exact integer products and sums on CUDA cores: the
// results depend on every rounding step, so the data never leaves integers.
#include <math.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "dft_int.h"
#include "int_arith.cuh"

namespace fftb200 {

namespace {

// The reference table generators use this truncated value of pi.
constexpr double kTablePi = 3.141592654;

// ---- dftSmall / dftLarge: Y = round_shift(X W) -------------------------------

// Persistent CTAs: each stages W (n2 x n2 of the caller's table, row stride
// ld) in shared memory once, then walks tiles of kGemmRows rows of X, stored
// transposed so that element k of 4 consecutive rows is one vector; every
// thread forms the exact dot products of one output column for 4 rows (one
// W load and one vector X load per 4 multiply-adds). In place when x == y
// (a tile is read completely before it is written).
constexpr uint32_t kGemmRows = 32;
constexpr size_t kIntGemmMaxSmem = 200u * 1024u;

template <class T> struct Vec4;
template <> struct Vec4<int8_t> { using type = char4; };
template <> struct Vec4<int16_t> { using type = short4; };
template <> struct Vec4<int32_t> { using type = int4; };

template <class T>
__global__ void __launch_bounds__(256) k_int_gemm(const T* x, const T* __restrict__ w, T* y, uint32_t n2,
                                                  uint32_t ld, uint32_t rows, uint32_t shift)
{
    using V = typename Vec4<T>::type;
    extern __shared__ __align__(16) unsigned char s_raw[];
    T* ws = reinterpret_cast<T*>(s_raw);
    T* xt = ws + n2 * n2;  // [k][row], kGemmRows rows
    for (uint32_t e = threadIdx.x; e < n2 * n2; e += blockDim.x) {
        const uint32_t k = e / n2;
        ws[e] = w[k * ld + (e - k * n2)];
    }
    const V* xv = reinterpret_cast<const V*>(xt);
    const uint32_t tiles = (rows + kGemmRows - 1) / kGemmRows;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t r0 = tile * kGemmRows;
        const uint32_t nr = min(kGemmRows, rows - r0);
        const T* xr = x + (size_t)r0 * n2;
        __syncthreads();  // the previous tile's reads of xt are done
        for (uint32_t e = threadIdx.x; e < kGemmRows * n2; e += blockDim.x) {
            const uint32_t r = e / n2, k = e - r * n2;
            xt[k * kGemmRows + r] = r < nr ? xr[e] : (T)0;
        }
        __syncthreads();
        T* yr = y + (size_t)r0 * n2;
        for (uint32_t e = threadIdx.x; e < (kGemmRows / 4) * n2; e += blockDim.x) {
            const uint32_t g = e / n2, j = e - g * n2;  // rows 4g..4g+3, column j
            typename IntT<T>::Acc a0 = 0, a1 = 0, a2 = 0, a3 = 0;
            for (uint32_t k = 0; k < n2; ++k) {
                const T wk = ws[k * n2 + j];
                const V v = xv[k * (kGemmRows / 4) + g];
                a0 = mac(a0, v.x, wk);
                a1 = mac(a1, v.y, wk);
                a2 = mac(a2, v.z, wk);
                a3 = mac(a3, v.w, wk);
            }
            const uint32_t r = 4 * g;
            if (r < nr) yr[(size_t)r * n2 + j] = shift_round<T>(a0, shift);
            if (r + 1 < nr) yr[(size_t)(r + 1) * n2 + j] = shift_round<T>(a1, shift);
            if (r + 2 < nr) yr[(size_t)(r + 2) * n2 + j] = shift_round<T>(a2, shift);
            if (r + 3 < nr) yr[(size_t)(r + 3) * n2 + j] = shift_round<T>(a3, shift);
        }
    }
}

// ---- general matrix multiply: C = round_shift(A B) ---------------------------------

// The LINALG multiply (..._matrixMatrixMultiply_ixX_ixX_oxX_cn.cpp:27-62) for
// any M x K by K x N with row strides in elements. A CTA owns a 64 x 64 tile
// of C and walks K in steps of 32: the A slice is stored transposed in shared
// memory ([k][m]) so that four rows of one column k are one vector, the B
// slice row by row; each of the 256 threads keeps the exact sums of a 4 x 4
// block of C. Ragged edges are zero-filled on load and skipped on store.
constexpr uint32_t kMmTile = 64, kMmK = 32, kMmPad = 4;

template <class T>
__global__ void __launch_bounds__(256) k_int_mm(const T* __restrict__ a, size_t lda, const T* __restrict__ b,
                                                size_t ldb, T* __restrict__ c, size_t ldc, uint32_t M, uint32_t K,
                                                uint32_t N, uint32_t shift)
{
    using V = typename Vec4<T>::type;
    using Acc = typename IntT<T>::Acc;
    __shared__ __align__(16) T as[kMmK][kMmTile + kMmPad];
    __shared__ __align__(16) T bs[kMmK][kMmTile + kMmPad];
    const uint32_t tx = threadIdx.x % 16u, ty = threadIdx.x / 16u;
    const size_t m0 = (size_t)blockIdx.x * kMmTile;
    const uint32_t n0 = blockIdx.y * kMmTile;
    Acc acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0;
    for (uint32_t k0 = 0; k0 < K; k0 += kMmK) {
        for (uint32_t e = threadIdx.x; e < kMmTile * kMmK; e += blockDim.x) {
            const uint32_t r = e / kMmK, k = e % kMmK;  // A: consecutive threads along k
            const size_t m = m0 + r;
            as[k][r] = (m < M && k0 + k < K) ? a[m * lda + k0 + k] : (T)0;
            const uint32_t kb = e / kMmTile, n = e % kMmTile;  // B: consecutive threads along n
            bs[kb][n] = (k0 + kb < K && n0 + n < N) ? b[(size_t)(k0 + kb) * ldb + n0 + n] : (T)0;
        }
        __syncthreads();
#pragma unroll 4
        for (uint32_t k = 0; k < kMmK; ++k) {
            const V av = *reinterpret_cast<const V*>(&as[k][4u * ty]);
            const V bv = *reinterpret_cast<const V*>(&bs[k][4u * tx]);
            const T ar[4] = {av.x, av.y, av.z, av.w}, br[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = mac(acc[i][j], ar[i], br[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const size_t m = m0 + 4u * ty + i;
        if (m >= M) break;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t n = n0 + 4u * tx + j;
            if (n < N) c[m * ldc + n] = shift_round<T>(acc[i][j], shift);
        }
    }
}

template <class T>
cudaError_t matmul_typed(uint32_t M, uint32_t K, uint32_t N, const void* a, size_t lda, const void* b, size_t ldb,
                         void* c, size_t ldc, uint32_t shift, cudaStream_t s)
{
    if (M == 0 || N == 0) return cudaSuccess;
    if constexpr (IntT<T>::kBits <= 16) {
        // square products of dense rows of at most 128 values (the DFT
        // shape): the super-row kernel keeps the whole B in shared memory
        if (IntT<T>::kBits == 16 && int_tensor_cores() && K == N && lda == K && ldc == N &&
            int16_tc_supported(K, a, c) && a != c)
            return launch_int16_tc(static_cast<const int16_t*>(a), static_cast<int16_t*>(c),
                                   static_cast<const int16_t*>(b), K, (uint32_t)ldb, M, shift, s);
        if (int_mm_tc_supported(IntT<T>::kBits, M, K, N, a, lda, b, ldb))
            return launch_int_mm_tc(IntT<T>::kBits, M, K, N, a, lda, b, ldb, c, ldc, shift, s);
    }
    const uint64_t gx = ((uint64_t)M + kMmTile - 1) / kMmTile, gy = ((uint64_t)N + kMmTile - 1) / kMmTile;
    if (gx > 0x7FFFFFFFull || gy > 65535ull) return cudaErrorInvalidValue;
    k_int_mm<T><<<dim3((unsigned)gx, (unsigned)gy), 256, 0, s>>>(static_cast<const T*>(a), lda,
                                                                 static_cast<const T*>(b), ldb, static_cast<T*>(c),
                                                                 ldc, M, K, N, shift);
    return cudaGetLastError();
}

// ---- highRadix -----------------------------------------------------------------

// One decimation stage, in place: inside each block of s points, butterfly q
// (< s/rad) takes x[q + m s/rad], m < rad, forms y_l = sum_m F[l][m] x_m
// exactly (F the rad-point DFT from the internal table, rows of MMA entries;
// the imaginary part negated with saturation as the reference does), rounds
// by `shift`, multiplies by its twiddle (the caller's (-sin, cos) pair of
// (q, l)) and rounds by bits - 1, and writes the result to q + l s/rad.
template <class T, uint32_t RAD>
__global__ void __launch_bounds__(256) k_int_stage(T* buf, uint32_t n, uint32_t s, uint32_t radRt, uint32_t shift,
                                                   const T* __restrict__ F, const T* __restrict__ tw, uint32_t rows,
                                                   int planar)
{
    constexpr uint32_t MMA = IntT<T>::kMma, R = MMA / 2;
    // a radix fixed at compile time (2, 4, 8, MMA/2) drops the unused terms; 0: radRt
    const uint32_t rad = RAD ? RAD : radRt;
    const uint32_t per = n / rad;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint64_t)rows * per) return;
    const uint32_t row = (uint32_t)(t / per), bf = (uint32_t)(t - (uint64_t)row * per);
    const uint32_t stride = s / rad, blk = bf / stride, q = bf - blk * stride;
    T* rp = buf + (size_t)row * 2u * n;
    const uint32_t p0 = blk * s + q;
    T ar[R], ai[R];
#pragma unroll
    for (uint32_t m = 0; m < R; ++m) {
        if (m < rad) {
            const uint32_t p = p0 + m * stride;
            ar[m] = planar ? rp[p] : rp[2 * p];
            ai[m] = planar ? rp[n + p] : rp[2 * p + 1];
        }
    }
    const T* twq = tw + (q / R) * MMA * rad + 2u * (q % R);
    for (uint32_t l = 0; l < rad; ++l) {
        typename IntT<T>::Acc yr = 0, yi = 0;
        const T* f = F + l * MMA;
#pragma unroll
        for (uint32_t m = 0; m < R; ++m) {
            if (m < rad) {
                const T c0 = f[2 * m], c1 = f[2 * m + 1];
                yi = mac(mac(yi, c0, ai[m]), c1, ar[m]);
                yr = mac(mac(yr, c0, ar[m]), c1, neg_sat<T>(ai[m]));
            }
        }
        const T tr = shift_round<T>(yr, shift), ti = shift_round<T>(yi, shift);
        const T e0 = twq[l * MMA], e1 = twq[l * MMA + 1];
        const T re = shift_round<T>(mul<T>(e1, tr) + mul<T>(neg_sat<T>(e0), ti), IntT<T>::kBits - 1);
        const T im = shift_round<T>(mul<T>(e0, tr) + mul<T>(e1, ti), IntT<T>::kBits - 1);
        const uint32_t p = p0 + l * stride;
        if (planar) {
            rp[p] = re;
            rp[n + p] = im;
        } else {
            rp[2 * p] = re;
            rp[2 * p + 1] = im;
        }
    }
}

// Final stage: the R-point DFT (rows of the caller's last table block) of
// every group of R consecutive points; group (k, m, i, h) starts at
// k n/d0 + m n/(d0 R) + i n/(d0 R^2) + h R and its output l goes to the
// digit-reversed position l G + h d0 mC iC + i d0 mC + m d0 + k, G = n / R.
template <class T>
__global__ void __launch_bounds__(256) k_int_final(const T* buf, T* y, uint32_t n, uint32_t d0, uint32_t mC,
                                                   uint32_t iC, uint32_t hC, uint32_t shift,
                                                   const T* __restrict__ D, uint32_t rows, int planar)
{
    constexpr uint32_t MMA = IntT<T>::kMma, R = MMA / 2;
    const uint32_t G = n / R;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint64_t)rows * G) return;
    const uint32_t row = (uint32_t)(t / G);
    uint32_t g = (uint32_t)(t - (uint64_t)row * G);
    const uint32_t h = g % hC;
    g /= hC;
    const uint32_t i = g % iC;
    g /= iC;
    const uint32_t m = g % mC;
    const uint32_t k = g / mC;
    const uint32_t start = k * (n / d0) + m * (n / (d0 * R)) + i * (n / (d0 * R * R)) + h * R;
    const T* rp = buf + (size_t)row * 2u * n;
    T ar[R], ai[R];
#pragma unroll
    for (uint32_t q = 0; q < R; ++q) {
        const uint32_t p = start + q;
        ar[q] = planar ? rp[p] : rp[2 * p];
        ai[q] = planar ? rp[n + p] : rp[2 * p + 1];
    }
    T* yp = y + (size_t)row * 2u * n;
    const uint32_t dst0 = h * d0 * mC * iC + i * d0 * mC + m * d0 + k;
    for (uint32_t l = 0; l < R; ++l) {
        typename IntT<T>::Acc xr = 0, xi = 0;
        const T* dr = D + l * 2u * MMA;
        const T* di = D + (2u * l + 1u) * MMA;
#pragma unroll
        for (uint32_t q = 0; q < R; ++q) {
            xr = mac(mac(xr, dr[2 * q], ai[q]), dr[2 * q + 1], ar[q]);
            xi = mac(mac(xi, di[2 * q], ai[q]), di[2 * q + 1], ar[q]);
        }
        const uint32_t p = l * G + dst0;
        const T vr = shift_round<T>(xr, shift), vi = shift_round<T>(xi, shift);
        if (planar) {
            yp[p] = vr;
            yp[n + p] = vi;
        } else {
            yp[2 * p] = vr;
            yp[2 * p + 1] = vi;
        }
    }
}

// ---- tables ------------------------------------------------------------------------

// Round half up of scale * v with saturation, scale = 2^(bits-1) - 0.5
// (FFTLIB_utility.h:672-722).
int32_t table_entry(double v, int bits)
{
    const double scale = (double)((1u << (bits - 2)) - 1u) + (double)(1u << (bits - 2)) + 0.5;
    const long long x = (long long)floor(0.5 + scale * v);
    const long long mx = (1ll << (bits - 1)) - 1;
    return (int32_t)(x >= mx ? mx : (x <= -mx - 1 ? -mx - 1 : x));
}

uint32_t first_factor(uint32_t n, uint32_t r)
{
    while (n > r) n /= r;
    return n;
}

template <class T>
void put(void* w, size_t i, int32_t v)
{
    static_cast<T*>(w)[i] = (T)v;
}

// Fills the highRadix internal table (MMA x MMA entries): the first-stage
// d0-point DFT as block-diagonal copies in the first MMA/2 rows, the
// MMA/2-point DFT in the rest, (cos, -sin) pairs.
void fill_w1(int bits, uint32_t n, std::vector<int32_t>& w1)
{
    const uint32_t mma = (uint32_t)int_mma_size(bits), r = mma / 2, d0 = first_factor(n, r);
    w1.assign((size_t)mma * mma, 0);
    for (uint32_t j = 0; j < mma / (2 * d0); ++j)
        for (uint32_t k = 0; k < d0; ++k)
            for (uint32_t l = 0; l < d0; ++l) {
                const double a = (2 * kTablePi * k * l) / d0;
                const size_t e = (size_t)j * d0 * mma + j * d0 * 2u + k * mma + 2u * l;
                w1[e] = table_entry(cos(a), bits);
                w1[e + 1] = -table_entry(sin(a), bits);
            }
    for (uint32_t k = 0; k < r; ++k)
        for (uint32_t l = 0; l < r; ++l) {
            const double a = (2 * kTablePi * k * l * 2) / mma;
            const size_t e = (size_t)mma * mma / 2 + k * mma + 2u * l;
            w1[e] = table_entry(cos(a), bits);
            w1[e + 1] = -table_entry(sin(a), bits);
        }
}

// Device copies of the internal tables, per (device, bits, n).
const void* device_w1(int bits, uint32_t n, cudaError_t* err)
{
    static std::mutex mu;
    static std::map<std::tuple<int, int, uint32_t>, void*> cache;
    int dev = 0;
    *err = cudaGetDevice(&dev);
    if (*err != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    void*& slot = cache[std::make_tuple(dev, bits, n)];
    if (!slot) {
        std::vector<int32_t> w1;
        fill_w1(bits, n, w1);
        const size_t es = bits == 16 ? 2 : 4;
        std::vector<unsigned char> host(w1.size() * es);
        for (size_t i = 0; i < w1.size(); ++i) {
            if (bits == 16) put<int16_t>(host.data(), i, w1[i]);
            else put<int32_t>(host.data(), i, w1[i]);
        }
        void* d = nullptr;
        *err = cudaMalloc(&d, host.size());
        if (*err == cudaSuccess) *err = cudaMemcpy(d, host.data(), host.size(), cudaMemcpyHostToDevice);
        if (*err != cudaSuccess) {
            cudaFree(d);
            cache.erase(std::make_tuple(dev, bits, n));
            return nullptr;
        }
        slot = d;
    }
    return slot;
}

template <class T>
cudaError_t launch_typed(int v, uint32_t n, uint32_t batch, uint32_t interleave, const uint32_t* shifts, void* xv,
                         const void* wv, void* yv, cudaStream_t s)
{
    constexpr int bits = IntT<T>::kBits;
    constexpr uint32_t MMA = IntT<T>::kMma, R = MMA / 2;
    T* x = static_cast<T*>(xv);
    T* y = static_cast<T*>(yv);
    const T* w = static_cast<const T*>(wv);
    if (v == INT_DFT_SMALL || v == INT_DFT_LARGE) {
        const uint32_t n2 = 2u * n, ld = v == INT_DFT_SMALL ? MMA : n2;
        if constexpr (IntT<T>::kBits == 16) {
            if (int_tensor_cores() && int16_tc_supported(n2, x, y))
                return launch_int16_tc(x, y, w, n2, ld, batch, shifts[0], s);
        }
        const size_t smem = ((size_t)n2 * n2 + kGemmRows * n2) * sizeof(T);  // x tile 16-byte aligned: n2 is even
        if (smem > kIntGemmMaxSmem) {
            // a table too large to stay in shared memory: the tiled multiply,
            // whose CTAs read rows that others write, so in place goes
            // through a temporary output
            if (x != y) return matmul_typed<T>(batch, n2, n2, x, n2, w, ld, y, n2, shifts[0], s);
            const size_t bytes = (size_t)batch * n2 * sizeof(T);
            void* tmp = nullptr;
            cudaError_t e = cudaMallocAsync(&tmp, bytes, s);
            if (e != cudaSuccess) return e;
            e = matmul_typed<T>(batch, n2, n2, x, n2, w, ld, tmp, n2, shifts[0], s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(y, tmp, bytes, cudaMemcpyDeviceToDevice, s);
            const cudaError_t f = cudaFreeAsync(tmp, s);
            return e != cudaSuccess ? e : f;
        }
        if (smem > 48u * 1024u) {
            cudaError_t e = cudaFuncSetAttribute(k_int_gemm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        int dev = 0, sms = 0, per = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_int_gemm<T>, 256, smem);
        if (e != cudaSuccess) return e;
        const uint32_t tiles = (batch + kGemmRows - 1) / kGemmRows;
        const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)std::max(1, per * sms));
        k_int_gemm<T><<<grid, 256, smem, s>>>(x, w, y, n2, ld, batch, shifts[0]);
        return cudaGetLastError();
    }
    if (!int_high_radix_covered(bits, n) || x == y) return cudaErrorInvalidValue;
    cudaError_t e;
    const T* w1 = static_cast<const T*>(device_w1(bits, n, &e));
    if (!w1) return e;
    const uint32_t d0 = first_factor(n, R);
    const int planar = interleave ? 0 : 1;
    const T* tw = w;
    uint32_t len = n, rad = d0;
    // INT16 radix-16 stages and the final stage of interleaved rows run on the
    // tensor cores (dft_int_hr_tc.cu), the rest on the CUDA cores
    bool tcHr = false;
    if constexpr (IntT<T>::kBits == 16) tcHr = int_tensor_cores() && !planar && int16_hr_tc_supported(n, x, y, w);
    for (int st = 0; len > R; ++st) {
        const T* F = st == 0 ? w1 : w1 + MMA * MMA / 2;
        bool done = false;
        if constexpr (IntT<T>::kBits == 16) {
            if (tcHr && rad == R) {
                if ((e = launch_int16_hr_stage(x, F, tw, n, len, batch, shifts[st], s)) != cudaSuccess) return e;
                done = true;
            }
        }
        if (!done) {
            const uint64_t threads = (uint64_t)batch * (n / rad);
            const unsigned grid = (unsigned)((threads + 255) / 256);
            if (rad == 2) k_int_stage<T, 2><<<grid, 256, 0, s>>>(x, n, len, rad, shifts[st], F, tw, batch, planar);
            else if (rad == 4) k_int_stage<T, 4><<<grid, 256, 0, s>>>(x, n, len, rad, shifts[st], F, tw, batch, planar);
            else if (rad == 8) k_int_stage<T, 8><<<grid, 256, 0, s>>>(x, n, len, rad, shifts[st], F, tw, batch, planar);
            else if (rad == R) k_int_stage<T, R><<<grid, 256, 0, s>>>(x, n, len, rad, shifts[st], F, tw, batch, planar);
            else k_int_stage<T, 0><<<grid, 256, 0, s>>>(x, n, len, rad, shifts[st], F, tw, batch, planar);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        tw += 2u * len;
        len /= rad;
        rad = R;
    }
    const uint32_t g1 = n / (d0 * R);
    const uint32_t mC = g1 > R ? R : g1;
    const uint32_t iC = g1 > R ? (g1 / R > R ? R : g1 / R) : 1u;
    const uint32_t hC = g1 / R > R ? g1 / (R * R) : 1u;
    if constexpr (IntT<T>::kBits == 16) {
        if (tcHr) return launch_int16_hr_final(x, y, tw, n, d0, mC, iC, hC, batch, shifts[4], s);
    }
    const uint64_t threads = (uint64_t)batch * (n / R);
    k_int_final<T><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(x, y, n, d0, mC, iC, hC, shifts[4], tw, batch,
                                                                   planar);
    return cudaGetLastError();
}

} // namespace

namespace {
std::atomic<bool> g_int_tc{true};
} // namespace

void int_set_tensor_cores(bool on) { g_int_tc.store(on); }
bool int_tensor_cores() { return g_int_tc.load(); }

int int_mma_size(int bits) { return bits == 16 ? 32 : 16; }

int int_dft_variant(int bits, uint32_t n, uint32_t batch, uint32_t interleave)
{
    const uint32_t mma = (uint32_t)int_mma_size(bits);
    if (n <= mma / 2) return INT_DFT_SMALL;
    if (n == mma) return INT_DFT_LARGE;
    if (n == 2u * mma) {
        if (batch < mma / 2) return INT_HIGH_RADIX;
        if (batch == mma / 2) return interleave ? INT_HIGH_RADIX : INT_DFT_LARGE;
        return INT_DFT_LARGE;
    }
    return INT_HIGH_RADIX;
}

uint32_t int_dft_w_size(int bits, uint32_t n, uint32_t batch, uint32_t interleave)
{
    return int_dft_w_size_v(bits, int_dft_variant(bits, n, batch, interleave), n);
}

uint32_t int_dft_w_size_v(int bits, int variant, uint32_t n)
{
    const uint32_t mma = (uint32_t)int_mma_size(bits), r = mma / 2;
    switch (variant) {
    case INT_DFT_SMALL: return mma * mma;
    case INT_DFT_LARGE: return 4u * n * n;
    default: {
        const uint32_t d0 = first_factor(n, r);
        uint32_t w = 2u * n;
        for (uint32_t len = n / d0; len > r; len /= r) w += 2u * len;
        return w + mma * mma;
    }
    }
}

bool int_high_radix_covered(int bits, uint32_t n)
{
    const uint32_t r = (uint32_t)int_mma_size(bits) / 2;
    if (n < 4u * r) return false;
    const uint32_t d0 = first_factor(n, r);
    if (d0 == 0 || n % d0) return false;
    uint32_t len = n / d0;
    int stages = 1;
    while (len > r) {
        if (len % r) return false;
        len /= r;
        ++stages;
    }
    return len == r && stages <= 4;
}

void int_dft_twgen_host(int bits, uint32_t n, uint32_t batch, uint32_t interleave, void* w)
{
    int_dft_twgen_host_v(bits, int_dft_variant(bits, n, batch, interleave), n, batch, interleave, w);
}

void int_dft_twgen_host_v(int bits, int v, uint32_t n, uint32_t batch, uint32_t interleave, void* w)
{
    const uint32_t mma = (uint32_t)int_mma_size(bits), r = mma / 2;
    const size_t total = int_dft_w_size_v(bits, v, n);
    auto set = [&](size_t i, int32_t val) {
        if (bits == 16) put<int16_t>(w, i, val);
        else put<int32_t>(w, i, val);
    };
    for (size_t i = 0; i < total; ++i) set(i, 0);
    if (v == INT_DFT_SMALL) {
        // r/n block-diagonal copies of the 2n x 2n real embedding, row stride MMA
        // (planar: only the copies j < batch, as the reference generates them)
        for (uint32_t j = 0; j < r / n; ++j)
            for (uint32_t k = 0; k < n; ++k)
                for (uint32_t m = 0; m < n; ++m) {
                    const double a = 2 * kTablePi * k * m / n;
                    const int32_t c = table_entry(cos(a), bits), sn = table_entry(sin(a), bits);
                    if (interleave) {
                        const size_t b = (size_t)(j * n + k) * 2u * mma + j * n * 2u;
                        set(b + 2 * m, c);
                        set(b + 2 * m + 1, -sn);
                        set(b + mma + 2 * m, sn);
                        set(b + mma + 2 * m + 1, c);
                    } else if (j < batch) {
                        const size_t b = (size_t)(j * n * 2u + k) * mma + j * n * 2u;
                        set(b + m, c);
                        set(b + n + m, -sn);
                        set(b + (size_t)n * mma + m, sn);
                        set(b + (size_t)n * mma + n + m, c);
                    }
                }
        return;
    }
    if (v == INT_DFT_LARGE) {
        for (uint32_t j = 0; j < n; ++j)
            for (uint32_t k = 0; k < n; ++k) {
                const double a = 2 * kTablePi * j * k / n;
                const int32_t c = table_entry(cos(a), bits), sn = table_entry(sin(a), bits);
                if (interleave) {
                    set((size_t)j * 4u * n + 2 * k, c);
                    set((size_t)j * 4u * n + 2 * k + 1, -sn);
                    set((size_t)(2 * j + 1) * 2u * n + 2 * k, sn);
                    set((size_t)(2 * j + 1) * 2u * n + 2 * k + 1, c);
                } else {
                    set((size_t)j * 2u * n + k, c);
                    set((size_t)j * 2u * n + n + k, -sn);
                    set((size_t)2u * n * n + j * 2u * n + k, sn);
                    set((size_t)2u * n * n + j * 2u * n + n + k, c);
                }
            }
        return;
    }
    // highRadix: each stage's twiddles W_len^(q l) as (-sin, cos) pairs at
    // [q / R][l][q mod R], then the rows of the final R-point DFT
    const uint32_t d0 = first_factor(n, r);
    size_t off = 0;
    uint32_t len = n, rad = d0;
    for (;;) {
        for (uint32_t b = 0; b < (2u * len) / (mma * rad); ++b)
            for (uint32_t l = 0; l < rad; ++l)
                for (uint32_t k = 0; k < r; ++k) {
                    const double a = (2 * kTablePi * (b * mma / 2 + k) * l) / len;
                    const size_t e = off + (size_t)b * mma * rad + l * mma + 2u * k;
                    set(e + 1, table_entry(cos(a), bits));
                    set(e, -table_entry(sin(a), bits));
                }
        off += 2u * len;
        len /= rad;
        rad = r;
        if (len <= r) break;
    }
    for (uint32_t k = 0; k < r; ++k)
        for (uint32_t l = 0; l < r; ++l) {
            const double a = (2 * kTablePi * k * l * 2) / mma;
            set(off + (size_t)k * 2u * mma + 2 * l, table_entry(sin(a), bits));
            set(off + (size_t)k * 2u * mma + 2 * l + 1, table_entry(cos(a), bits));
            set(off + (size_t)(2 * k + 1) * mma + 2 * l, table_entry(cos(a), bits));
            set(off + (size_t)(2 * k + 1) * mma + 2 * l + 1, -table_entry(sin(a), bits));
        }
}

cudaError_t int_dft_launch(int bits, uint32_t n, uint32_t batch, uint32_t interleave, const uint32_t* shifts,
                           void* x, const void* w, void* y, cudaStream_t s)
{
    return int_dft_launch_v(bits, int_dft_variant(bits, n, batch, interleave), n, batch, interleave, shifts, x, w, y,
                            s);
}

cudaError_t int_dft_launch_v(int bits, int variant, uint32_t n, uint32_t batch, uint32_t interleave,
                             const uint32_t* shifts, void* x, const void* w, void* y, cudaStream_t s)
{
    if (batch == 0) return cudaSuccess;
    return bits == 16 ? launch_typed<int16_t>(variant, n, batch, interleave, shifts, x, w, y, s)
                      : launch_typed<int32_t>(variant, n, batch, interleave, shifts, x, w, y, s);
}

void int_dft_w1_host(int bits, uint32_t n, void* out)
{
    std::vector<int32_t> w1;
    fill_w1(bits, n, w1);
    for (size_t i = 0; i < w1.size(); ++i) {
        if (bits == 16) put<int16_t>(out, i, w1[i]);
        else put<int32_t>(out, i, w1[i]);
    }
}

cudaError_t int_matmul_launch(int bits, uint32_t M, uint32_t K, uint32_t N, const void* a, size_t lda, const void* b,
                              size_t ldb, void* c, size_t ldc, uint32_t shift, cudaStream_t s)
{
    switch (bits) {
    case 8: return matmul_typed<int8_t>(M, K, N, a, lda, b, ldb, c, ldc, shift, s);
    case 16: return matmul_typed<int16_t>(M, K, N, a, lda, b, ldb, c, ldc, shift, s);
    case 32: return matmul_typed<int32_t>(M, K, N, a, lda, b, ldb, c, ldc, shift, s);
    default: return cudaErrorInvalidValue;
    }
}

} // namespace fftb200
