/*
 * mma_int_oracle.c -- CPU oracle for the integer (INT16 / INT32) paths of the
 * DFT coordinator FFTLIB_FFT_fft_ixX_cxX_oxX (dftSmall, dftLarge and
 * highRadixDecompositions variants).
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference's
 * natural-C arithmetic and table generators, used by tests/ as the checker.
 * The product library never links, loads or calls it.
 *
 * Values are passed as int32 arrays whatever the data type (bits = 16 or 32);
 * every sum is formed exactly in 128 bits, so the results equal those of the
 * reference's int64 (int16 data) and 128-bit (int32 data) accumulators.
 *
 * Reference sources restated here:
 *   variant choice   src/fft_c7xmma/FFTLIB_FFT_fft_ixX_cxX_oxX/FFTLIB_FFT_fft_ixX_cxX_oxX.cpp:13-50
 *   integer helpers  src/common/FFTLIB_utility.h:229-249 (negate), 492-568 (saturate),
 *                    576-594, 643-661 (shiftAndRound), 672-722 (table entries)
 *   dftSmall         .../FFTLIB_FFT_dftSmall_ixX_cxX_oxX_cn.cpp:18-46; getSizes/twGen
 *                    .../c71/FFTLIB_FFT_dftSmall_ixX_cxX_oxX_ci.cpp:74-212
 *   dftLarge and the LINALG matrix multiply (INT8 too)
 *                    src/linalg_c7xmma/FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX/..._cn.cpp:27-62;
 *                    getSizes/twGen .../c71/FFTLIB_FFT_dftLarge_ixX_cxX_oxX_ci.cpp:43-156
 *   highRadix        .../FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_cn.cpp:20-455;
 *                    getSizes/twGen .../c71/..._ci.cpp:1975-2168
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef __int128 i128;

/* The reference table generators use this truncated value of pi. */
static const double MMA_PI = 3.141592654;

static int mma_size(int bits) { return bits == 16 ? 32 : 16; }
static int64_t mma_max(int bits) { return ((int64_t)1 << (bits - 1)) - 1; }

/* Arithmetic right shift of the exact sum; counts past its width give the
 * sign (the reference's shift of its accumulator is undefined there). */
static i128 mma_sra(i128 x, uint32_t k) { return k >= 127u ? (x < 0 ? -1 : 0) : x >> k; }

/* Saturate to the data type. The reference's 128-bit saturation
 * (FFTLIB_utility.h:546-566) tests only the low 64 bits of a non-negative
 * value, so one of 2^64 or more keeps its low 32 bits when those fit: kept
 * here as the reference computes it. */
static int32_t mma_sat(i128 x, int bits)
{
    const int64_t mx = mma_max(bits);
    if (x < 0) return x < (i128)(-mx - 1) ? (int32_t)(-mx - 1) : (int32_t)x;
    if (bits == 32) {
        const uint64_t lo = (uint64_t)x;
        return (lo & 0xFFFFFFFF80000000ull) ? (int32_t)mx : (int32_t)lo;
    }
    return x > (i128)mx ? (int32_t)mx : (int32_t)x;
}

/* Round half up after an arithmetic right shift by s (s = 0: saturate
 * only); the shift amount is the reference's uint8_t parameter. */
static int32_t mma_shift_round(i128 x, uint32_t shift, int bits)
{
    const uint32_t s = shift & 0xFFu;
    if (s == 0) return mma_sat(x, bits);
    return mma_sat(mma_sra(mma_sra(x, s - 1) + 1, 1), bits);
}

/* Negation that maps the most negative value to the most positive. */
static int32_t mma_neg(int32_t a, int bits)
{
    return (int64_t)a == -mma_max(bits) - 1 ? (int32_t)mma_max(bits) : -a;
}

/* Table entry: round half up of scale * f, saturated (scale 2^(bits-1) - 0.5). */
static int32_t mma_q(double v, int bits)
{
    const double scale = (double)((1u << (bits - 2)) - 1u) + (double)(1u << (bits - 2)) + 0.5;
    const int64_t x = (int64_t)floor(0.5 + scale * v);
    const int64_t mx = mma_max(bits);
    if (x >= mx) return (int32_t)mx;
    if (x <= -mx - 1) return (int32_t)(-mx - 1);
    return (int32_t)x;
}

/* 1 dftSmall, 2 dftLarge, 3 highRadixDecompositions. */
int orc_mma_variant(int bits, uint32_t fftSize, uint32_t batchSize, uint32_t interleave)
{
    const uint32_t mma = (uint32_t)mma_size(bits);
    if (fftSize <= mma / 2) return 1;
    if (fftSize == mma) return 2;
    if (fftSize == 2 * mma) {
        if (batchSize < mma / 2) return 3;
        if (batchSize == mma / 2) return interleave ? 3 : 2;
        return 2;
    }
    return 3;
}

/* First decomposition factor: fftSize reduced by MMA/2 while above MMA/2. */
static uint32_t stage0_factor(uint32_t fftSize, uint32_t r)
{
    uint32_t f = fftSize;
    while (f > r) f /= r;
    return f;
}

/* Caller's table size (elements) of a variant, as its getSizes reports it. */
uint32_t orc_mma_w_size_v(int bits, int variant, uint32_t fftSize)
{
    const uint32_t mma = (uint32_t)mma_size(bits), r = mma / 2;
    switch (variant) {
    case 1: return mma * mma;
    case 2: return 4u * fftSize * fftSize;
    default: {
        const uint32_t d0 = stage0_factor(fftSize, r);
        uint32_t w = 2u * fftSize, s = fftSize / d0;
        while (s > r) {
            w += 2u * s;
            s /= r;
        }
        return w + mma * mma;
    }
    }
}

uint32_t orc_mma_w_size(int bits, uint32_t fftSize, uint32_t batchSize, uint32_t interleave)
{
    return orc_mma_w_size_v(bits, orc_mma_variant(bits, fftSize, batchSize, interleave), fftSize);
}

/* The caller's table (twGen) of a variant, int values in int32 slots. */
void orc_mma_twgen_v(int bits, int v, uint32_t fftSize, uint32_t batchSize, uint32_t interleave, int32_t *W)
{
    const uint32_t mma = (uint32_t)mma_size(bits), r = mma / 2;
    const uint32_t n = fftSize;
    memset(W, 0, sizeof(int32_t) * orc_mma_w_size_v(bits, v, fftSize));
    if (v == 1) {
        /* block-diagonal copies of the 2N x 2N real embedding, row stride MMA */
        const uint32_t copies = r / n;
        for (uint32_t j = 0; j < copies; ++j) {
            for (uint32_t k = 0; k < n; ++k) {
                for (uint32_t m = 0; m < n; ++m) {
                    const double a = 2 * MMA_PI * k * m / n;
                    const int32_t c = mma_q(cos(a), bits), sn = mma_q(sin(a), bits);
                    if (interleave) {
                        const uint32_t base = (j * n + k) * 2u * mma + j * n * 2u;
                        W[base + 2 * m] = c;
                        W[base + 2 * m + 1] = -sn;
                        W[base + mma + 2 * m] = sn;
                        W[base + mma + 2 * m + 1] = c;
                    } else if (j < batchSize) {
                        const uint32_t base = (j * n * 2u + k) * mma + j * n * 2u;
                        W[base + m] = c;
                        W[base + n + m] = -sn;
                        W[base + n * mma + m] = sn;
                        W[base + n * mma + n + m] = c;
                    }
                }
            }
        }
        return;
    }
    if (v == 2) {
        for (uint32_t j = 0; j < n; ++j) {
            for (uint32_t k = 0; k < n; ++k) {
                const double a = 2 * MMA_PI * j * k / n;
                const int32_t c = mma_q(cos(a), bits), sn = mma_q(sin(a), bits);
                if (interleave) {
                    W[j * 4u * n + 2 * k] = c;
                    W[j * 4u * n + 2 * k + 1] = -sn;
                    W[(2 * j + 1) * 2u * n + 2 * k] = sn;
                    W[(2 * j + 1) * 2u * n + 2 * k + 1] = c;
                } else {
                    W[j * 2u * n + k] = c;
                    W[j * 2u * n + n + k] = -sn;
                    W[2u * n * n + j * 2u * n + k] = sn;
                    W[2u * n * n + j * 2u * n + n + k] = c;
                }
            }
        }
        return;
    }
    /* highRadix: per-stage twiddles as (-sin, cos) pairs, then the final
     * R-point DFT rows */
    const uint32_t d0 = stage0_factor(n, r);
    int32_t *w = W;
    uint32_t s = n, rad = d0;
    for (;;) {
        /* entry (block b, output l, lane k): pair at b*rad*MMA/... laid out
         * as [b][l][k] with k the fastest index; angle 2 pi (b R + k) l / s */
        const uint32_t blocks = (2u * s) / (mma * rad);
        for (uint32_t b = 0; b < blocks; ++b) {
            for (uint32_t l = 0; l < rad; ++l) {
                for (uint32_t k = 0; k < r; ++k) {
                    const double a = (2 * MMA_PI * (b * mma / 2 + k) * l) / s;
                    const uint32_t e = b * mma * rad + l * mma + 2u * k;
                    w[e + 1] = mma_q(cos(a), bits);
                    w[e] = -mma_q(sin(a), bits);
                }
            }
        }
        w += 2u * s;
        s /= rad;
        rad = r;
        if (s <= r) break;
    }
    for (uint32_t k = 0; k < r; ++k) {
        for (uint32_t l = 0; l < r; ++l) {
            const double a = (2 * MMA_PI * k * l * 2) / mma;
            w[k * 2u * mma + 2 * l] = mma_q(sin(a), bits);
            w[k * 2u * mma + 2 * l + 1] = mma_q(cos(a), bits);
            w[(2 * k + 1) * mma + 2 * l] = mma_q(cos(a), bits);
            w[(2 * k + 1) * mma + 2 * l + 1] = -mma_q(sin(a), bits);
        }
    }
}

/* Y[row][j] = round_shift(sum_k X[row][k] W[k ld + j]) for j, k < 2N. */
static void mma_gemm(int bits, uint32_t n2, uint32_t rows, uint32_t ld, uint32_t shift, const int32_t *W,
                     const int32_t *x, int32_t *y)
{
    for (uint32_t b = 0; b < rows; ++b) {
        for (uint32_t j = 0; j < n2; ++j) {
            i128 acc = 0;
            for (uint32_t k = 0; k < n2; ++k) acc += (i128)((int64_t)x[b * n2 + k] * (int64_t)W[k * ld + j]);
            y[b * n2 + j] = mma_shift_round(acc, shift, bits);
        }
    }
}

/* One decimation stage of highRadix on a row of n complex values (re, im
 * arrays): inside every block of s points, for q < s/rad:
 *   y_l = sum_m F[l][m] x[q + m s/rad]   (F the rad-point DFT from the
 *         internal table, the imaginary part of x negated with saturation),
 *   t   = round_shift(y, shift), z = t * conj-stored twiddle, rounded by
 *         bits - 1, stored at q + l s/rad. */
static void hr_stage(int bits, uint32_t n, uint32_t s, uint32_t rad, uint32_t shift, const int32_t *F, uint32_t fld,
                     const int32_t *tw, uint32_t mma, const int32_t *re, const int32_t *im, int32_t *ore, int32_t *oim)
{
    const uint32_t r = mma / 2, stride = s / rad;
    for (uint32_t base = 0; base < n; base += s) {
        for (uint32_t q = 0; q < stride; ++q) {
            for (uint32_t l = 0; l < rad; ++l) {
                i128 yr = 0, yi = 0;
                for (uint32_t m = 0; m < rad; ++m) {
                    const int32_t c0 = F[l * fld + 2 * m], c1 = F[l * fld + 2 * m + 1];
                    const int32_t ar = re[base + q + m * stride], ai = im[base + q + m * stride];
                    yi += (i128)((int64_t)c0 * ai) + (i128)((int64_t)c1 * ar);
                    yr += (i128)((int64_t)c0 * ar) + (i128)((int64_t)c1 * mma_neg(ai, bits));
                }
                const int32_t tr = mma_shift_round(yr, shift, bits), ti = mma_shift_round(yi, shift, bits);
                /* twiddle pair of (q, l): [q / R][l][q mod R] */
                const uint32_t e = (q / r) * mma * rad + l * mma + 2u * (q % r);
                const int32_t e0 = tw[e], e1 = tw[e + 1];
                ore[base + q + l * stride] =
                    mma_shift_round((i128)((int64_t)e1 * tr) + (i128)((int64_t)mma_neg(e0, bits) * ti), bits - 1, bits);
                oim[base + q + l * stride] =
                    mma_shift_round((i128)((int64_t)e0 * tr) + (i128)((int64_t)e1 * ti), bits - 1, bits);
            }
        }
    }
}

/* The highRadix internal table (MMA x MMA entries): the first-stage
 * decomposition DFT (d0 points) in rows 0..MMA/2-1 and the MMA/2-point DFT in
 * rows MMA/2..MMA-1, as (cos, -sin) pairs; the reference's twGen writes the
 * first one as block-diagonal copies (c71/..._ci.cpp:2084-2112). */
void orc_mma_w1(int bits, uint32_t fftSize, int32_t *W1)
{
    const uint32_t mma = (uint32_t)mma_size(bits), r = mma / 2;
    const uint32_t d0 = stage0_factor(fftSize, r);
    memset(W1, 0, sizeof(int32_t) * mma * mma);
    for (uint32_t j = 0; j < mma / (2 * d0); ++j)
        for (uint32_t k = 0; k < d0; ++k)
            for (uint32_t l = 0; l < d0; ++l) {
                const double a = (2 * MMA_PI * k * l) / d0;
                const uint32_t e = j * d0 * mma + j * d0 * 2u + k * mma + 2u * l;
                W1[e] = mma_q(cos(a), bits);
                W1[e + 1] = -mma_q(sin(a), bits);
            }
    int32_t *F1 = W1 + mma * mma / 2;
    for (uint32_t k = 0; k < r; ++k)
        for (uint32_t l = 0; l < r; ++l) {
            const double a = (2 * MMA_PI * k * l * 2) / mma;
            F1[k * mma + 2 * l] = mma_q(cos(a), bits);
            F1[k * mma + 2 * l + 1] = -mma_q(sin(a), bits);
        }
}

void orc_mma_twgen(int bits, uint32_t fftSize, uint32_t batchSize, uint32_t interleave, int32_t *W)
{
    orc_mma_twgen_v(bits, orc_mma_variant(bits, fftSize, batchSize, interleave), fftSize, batchSize, interleave, W);
}

/* One variant's transform. Returns 0 on success, 1 for a length the
 * decomposition does not cover. */
int orc_mma_exec_v(int bits, int v, uint32_t fftSize, uint32_t batchSize, uint32_t interleave,
                   const uint32_t *shifts, const int32_t *W, const int32_t *x, int32_t *y)
{
    const uint32_t mma = (uint32_t)mma_size(bits), r = mma / 2, n = fftSize;
    if (v == 1) {
        mma_gemm(bits, 2u * n, batchSize, mma, shifts[0], W, x, y);
        return 0;
    }
    if (v == 2) {
        mma_gemm(bits, 2u * n, batchSize, 2u * n, shifts[0], W, x, y);
        return 0;
    }
    if (n < 2u * mma) return 1;
    const uint32_t d0 = stage0_factor(n, r);
    uint32_t check = n / d0, nstages = 1;
    while (check > r) {
        if (check % r) return 1;
        check /= r;
        ++nstages;
    }
    if (check != r || d0 * (n / d0) != n || nstages > 4) return 1;

    /* internal table: the d0-point and R-point DFTs as (cos, -sin) pairs */
    int32_t *W1 = (int32_t *)calloc((size_t)mma * mma, sizeof(int32_t));
    orc_mma_w1(bits, n, W1);
    const int32_t *F0 = W1, *F1 = W1 + mma * mma / 2;
    int32_t *re = (int32_t *)malloc(sizeof(int32_t) * n), *im = (int32_t *)malloc(sizeof(int32_t) * n);
    int32_t *re2 = (int32_t *)malloc(sizeof(int32_t) * n), *im2 = (int32_t *)malloc(sizeof(int32_t) * n);
    for (uint32_t b = 0; b < batchSize; ++b) {
        const int32_t *xr = x + (size_t)b * 2u * n;
        for (uint32_t p = 0; p < n; ++p) {
            re[p] = interleave ? xr[2 * p] : xr[p];
            im[p] = interleave ? xr[2 * p + 1] : xr[n + p];
        }
        const int32_t *tw = W;
        uint32_t s = n, rad = d0;
        for (uint32_t st = 0; st < nstages; ++st) {
            hr_stage(bits, n, s, rad, shifts[st], st == 0 ? F0 : F1, mma, tw, mma, re, im, re2, im2);
            int32_t *t = re; re = re2; re2 = t;
            t = im; im = im2; im2 = t;
            tw += 2u * s;
            s /= rad;
            rad = r;
        }
        /* final R-point DFTs of consecutive groups, outputs in digit-reversed
         * order: group start k n/d0 + m n/(d0 R) + i n/(d0 R^2) + h R */
        const int32_t *D = tw;
        const uint32_t g1 = n / (d0 * r);
        const uint32_t mC = g1 > r ? r : g1;
        const uint32_t iC = g1 > r ? (g1 / r > r ? r : g1 / r) : 1u;
        const uint32_t hC = g1 / r > r ? g1 / (r * r) : 1u;
        int32_t *yr = y + (size_t)b * 2u * n;
        for (uint32_t k = 0; k < d0; ++k)
            for (uint32_t m = 0; m < mC; ++m)
                for (uint32_t i = 0; i < iC; ++i)
                    for (uint32_t h = 0; h < hC; ++h) {
                        const uint32_t g = k * (n / d0) + m * (n / (d0 * r)) + i * (n / (d0 * r * r)) + h * r;
                        for (uint32_t l = 0; l < r; ++l) {
                            i128 ar = 0, ai = 0;
                            for (uint32_t q = 0; q < r; ++q) {
                                ar += (i128)((int64_t)D[l * 2u * mma + 2 * q] * im[g + q]) +
                                      (i128)((int64_t)D[l * 2u * mma + 2 * q + 1] * re[g + q]);
                                ai += (i128)((int64_t)D[(2 * l + 1) * mma + 2 * q] * im[g + q]) +
                                      (i128)((int64_t)D[(2 * l + 1) * mma + 2 * q + 1] * re[g + q]);
                            }
                            const uint32_t p = l * d0 * mC * iC * hC + h * d0 * mC * iC + i * d0 * mC + m * d0 + k;
                            const int32_t vr = mma_shift_round(ar, shifts[4], bits), vi = mma_shift_round(ai, shifts[4], bits);
                            if (interleave) {
                                yr[2 * p] = vr;
                                yr[2 * p + 1] = vi;
                            } else {
                                yr[p] = vr;
                                yr[n + p] = vi;
                            }
                        }
                    }
    }
    free(W1);
    free(re);
    free(im);
    free(re2);
    free(im2);
    return 0;
}

int orc_mma_exec(int bits, uint32_t fftSize, uint32_t batchSize, uint32_t interleave, const uint32_t *shifts,
                 const int32_t *W, const int32_t *x, int32_t *y)
{
    return orc_mma_exec_v(bits, orc_mma_variant(bits, fftSize, batchSize, interleave), fftSize, batchSize, interleave,
                          shifts, W, x, y);
}

/* The LINALG matrix multiply (src/linalg_c7xmma/FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX/
 * ..._cn.cpp:27-62): C[m][n] = shiftAndRound(sum_k A[m][k] B[k][n], shift) for
 * bits = 8, 16 or 32, row strides in elements, values in int32 slots. The
 * shift is the InitArgs int8_t, passed on as the uint8_t of shiftAndRound.
 * INT8 sums are kept in 32 bits with two's-complement wrap (the reference's
 * int32 accumulator; its overflow is undefined in C). */
void orc_linalg_mm(int bits, uint32_t M, uint32_t K, uint32_t N, const int32_t *A, uint64_t lda, const int32_t *B,
                   uint64_t ldb, int32_t *Cm, uint64_t ldc, int32_t shift)
{
    const uint32_t s = (uint32_t)(uint8_t)(int8_t)shift;
    for (uint32_t m = 0; m < M; ++m)
        for (uint32_t n = 0; n < N; ++n) {
            i128 acc = 0;
            for (uint32_t k = 0; k < K; ++k) {
                acc += (i128)((int64_t)A[m * lda + k] * (int64_t)B[k * ldb + n]);
                if (bits == 8) acc = (i128)(int32_t)(uint32_t)(uint64_t)acc;
            }
            Cm[m * ldc + n] = mma_shift_round(acc, s, bits);
        }
}
