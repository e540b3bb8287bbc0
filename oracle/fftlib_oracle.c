/*
 * fftlib_oracle.c -- CPU oracle for the FFTLIB batched FFT hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see fftlib_oracle.h). A restatement, in this
 * repository's own code, of the reference natural-C kernels. Every function
 * names the reference lines it follows; paths are relative to the
 * TexasInstruments/c7x_fftlib tree.
 *
 * FP32 paths reproduce the reference algorithm (same DIF stage order
 * 5,3,4,2, same twiddle-table layout, same final digit reversal) but not its
 * exact expression order, so they agree with the reference to FP32 rounding.
 * The int16 path and the table generators reproduce the reference
 * bit-for-bit.
 */
#include "fftlib_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* The reference generators use this truncated value of pi
 * (test/fft_c7x/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/..._d.c:33). */
static const double REF_PI = 3.141592654;

/* ------------------------------------------------------------------------ */
/* Radix schedule                                                            */
/* ------------------------------------------------------------------------ */

/* DIF stage radices in execution order: every 5, then every 3, then 4 while
 * divisible by 4, then one trailing 2.
 * src/fft_c7x/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/..._cn.c:240-260.
 * Returns the stage count, or -1 if numPoints has another prime factor. */
static int stage_radices(uint32_t n, int *radix)
{
   int s = 0;
   while (n > 1u) {
      if (n % 5u == 0u) { radix[s++] = 5; n /= 5u; }
      else if (n % 3u == 0u) { radix[s++] = 3; n /= 3u; }
      else if (n % 4u == 0u) { radix[s++] = 4; n /= 4u; }
      else if (n % 2u == 0u) { radix[s++] = 2; n /= 2u; }
      else { return -1; }
   }
   return s;
}

/* Position in the DIF work buffer that holds frequency k. Each radix-4 stage
 * counts as two radix-2 digits because the radix-4 butterfly stores its
 * outputs in bit-reversed slot order.
 * src/fft_c7x/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/..._cn.c:412-491. */
static uint32_t dif_position(uint32_t k, const int *radix, int nStages)
{
   int digitRadix[64];
   int nd = 0;
   for (int s = 0; s < nStages; s++) {
      if (radix[s] == 4) { digitRadix[nd++] = 2; digitRadix[nd++] = 2; }
      else { digitRadix[nd++] = radix[s]; }
   }
   /* k = d0 + r0*(d1 + r1*(d2 + ...)); position = d0*(N/r0) + d1*(N/(r0 r1)) + ... */
   uint32_t weight = 1u;
   for (int d = 0; d < nd; d++) weight *= (uint32_t) digitRadix[d];
   uint32_t pos = 0u;
   for (int d = 0; d < nd; d++) {
      weight /= (uint32_t) digitRadix[d];
      pos += (k % (uint32_t) digitRadix[d]) * weight;
      k /= (uint32_t) digitRadix[d];
   }
   return pos;
}

/* ------------------------------------------------------------------------ */
/* Twiddle tables                                                            */
/* ------------------------------------------------------------------------ */

/* One radix block of the FP32 table: for each stage of this radix, (r-1)
 * sub-blocks of M/r complex twiddles W_M^{m*i}, m = 1..r-1, i = 0..M/r-1.
 * Restates test/fft_c7x/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/..._d.c:30-96
 * (identical in src/fft_c7x/FFTLIB_fft1dBatched_i32f_c32fc_o32fc/..._tw_gen.cpp:9-78
 * for N/2). Angles are evaluated as ((2m*PI)*i)/M0 in double, where M0 is the
 * size at the start of the radix block and i steps by the stage stride. */
static uint32_t tw_block_f32(float *pW, uint32_t *k, uint32_t m0, uint32_t r)
{
   uint32_t stage = m0;
   uint32_t t = m0 / r;
   for (uint32_t j = 1u; j <= m0 / r && stage % r == 0u; j *= r) {
      for (uint32_t i = 0u; i < m0 / r; i += j) {
         for (uint32_t m = 1u; m < r; m++) {
            double ang = (double) (2u * m) * REF_PI * (double) i / (double) m0;
            pW[*k + 2u * (m - 1u) * t]      = (float) cos(ang);
            pW[*k + 2u * (m - 1u) * t + 1u] = (float) -sin(ang);
         }
         *k += 2u;
      }
      *k += 2u * t * (r - 2u);
      t /= r;
      stage /= r;
   }
   return stage;
}

void orc_tw_gen_f32(float *pW, uint32_t numPoints)
{
   uint32_t k = 0u;
   uint32_t n = numPoints;
   if (n % 5u == 0u) n = tw_block_f32(pW, &k, n, 5u);
   if (n % 3u == 0u) n = tw_block_f32(pW, &k, n, 3u);
   if (n % 4u == 0u) (void) tw_block_f32(pW, &k, n, 4u);
}

/* Round-half-up to int16 with saturation.
 * test/fft_c7x/FFTLIB_fft1dBatched_i16sc_c16sc_o16sc/..._d.c:29-37. */
static int16_t to_q15(double x)
{
   x = floor(0.5 + x);
   if (x >= 32767.0) return 32767;
   if (x <= -32768.0) return -32768;
   return (int16_t) x;
}

/* Q15 radix-4 table: 3 sub-blocks per stage, scaled by 32767.5.
 * test/fft_c7x/FFTLIB_fft1dBatched_i16sc_c16sc_o16sc/..._d.c:39-61. */
void orc_tw_gen_i16(int16_t *pW, uint32_t numPoints)
{
   const double scale = 32767.5;
   uint32_t k = 0u;
   uint32_t t = numPoints >> 2;
   for (uint32_t j = 1u; j <= (numPoints >> 2); j <<= 2) {
      for (uint32_t i = 0u; i < (numPoints >> 2); i += j) {
         for (uint32_t m = 1u; m < 4u; m++) {
            double ang = (double) (2u * m) * REF_PI * (double) i / (double) numPoints;
            pW[k + 2u * (m - 1u) * t]      = to_q15(scale * cos(ang));
            pW[k + 2u * (m - 1u) * t + 1u] = to_q15(scale * (-sin(ang)));
         }
         k += 2u;
      }
      k += 4u * t;
      t >>= 2;
   }
}

/* A[i] = 0.5(1 - sin) - 0.5i cos at [2i]; B[i] = 0.5(1 + sin) + 0.5i cos stored
 * reversed at [2N-2i-2].
 * src/fft_c7x/FFTLIB_fft1dBatched_i32f_c32fc_o32fc/..._tw_gen.cpp:80-97. */
void orc_split_factor_r2c(float *pSf, uint32_t numPoints)
{
   for (uint32_t i = 0u; i < numPoints / 2u; i++) {
      double ang = 2.0 * REF_PI * (double) i / (double) numPoints;
      pSf[2u * i]                         = (float) (0.5 * (1.0 - sin(ang)));
      pSf[2u * i + 1u]                    = (float) (0.5 * (-cos(ang)));
      pSf[2u * numPoints - 2u * i - 2u]   = (float) (0.5 * (1.0 + sin(ang)));
      pSf[2u * numPoints - 2u * i - 1u]   = (float) (0.5 * cos(ang));
   }
}

/* A'[i] at [2i] = 0.5(1 - sin) + 0.5i cos; B'[i] at [2i+N] = 0.5(1 + sin) - 0.5i cos.
 * src/fft_c7x/FFTLIB_ifft1dBatched_i32fc_c32fc_o32f/..._tw_gen.cpp:81-95. */
void orc_split_factor_c2r(float *pSf, uint32_t numPoints)
{
   for (uint32_t i = 0u; i < numPoints / 2u; i++) {
      double ang = 2.0 * REF_PI * (double) i / (double) numPoints;
      pSf[2u * i]                   = (float) (0.5 * (1.0 - sin(ang)));
      pSf[2u * i + 1u]              = (float) (0.5 * cos(ang));
      pSf[2u * i + numPoints]       = (float) (0.5 * (1.0 + sin(ang)));
      pSf[2u * i + numPoints + 1u]  = (float) (0.5 * (-cos(ang)));
   }
}

/* ------------------------------------------------------------------------ */
/* FP32 c2c                                                                  */
/* ------------------------------------------------------------------------ */

/* Forward r-point DFT, r in {3,4,5}, X[m] = sum_n a[n] exp(-2 pi i n m / r). */
static void small_dft(int r, const float *are, const float *aim, float *xre, float *xim)
{
   for (int m = 0; m < r; m++) {
      float sr = 0.0f, si = 0.0f;
      for (int n = 0; n < r; n++) {
         int e = (n * m) % r;
         double ang = 2.0 * M_PI * (double) e / (double) r;
         float c = (float) cos(ang);
         float s = (float) sin(ang);
         /* (a.re + i a.im) (c - i s) */
         sr += are[n] * c + aim[n] * s;
         si += aim[n] * c - are[n] * s;
      }
      xre[m] = sr;
      xim[m] = si;
   }
}

/* One channel, in place on x (numPoints complex). DIF stages with the
 * twiddle multiply after each butterfly, reading twiddles from the caller's
 * table in the tw_gen layout.
 * src/fft_c7x/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/..._cn.c:262-407. */
static void dif_channel_f32(float *x, const float *pW, uint32_t n, const int *radix, int nStages)
{
   const float *tw = pW;
   uint32_t m = n;
   for (int s = 0; s < nStages; s++) {
      int r = radix[s];
      uint32_t q = m / (uint32_t) r;
      if (r == 2) {
         /* trailing radix-2 on adjacent pairs, no twiddle (_cn.c:388-407) */
         for (uint32_t b = 0; b < n; b += 2u) {
            float ar = x[2u * b], ai = x[2u * b + 1u];
            float br = x[2u * b + 2u], bi = x[2u * b + 3u];
            x[2u * b] = ar + br;       x[2u * b + 1u] = ai + bi;
            x[2u * b + 2u] = ar - br;  x[2u * b + 3u] = ai - bi;
         }
      }
      else {
         /* radix-4 stores X1 at slot 2q and X2 at slot q (_cn.c:368-381) */
         static const int slot4[4] = {0, 2, 1, 3};
         for (uint32_t b = 0; b < n; b += m) {
            for (uint32_t k = 0; k < q; k++) {
               float are[5], aim[5], xre[5], xim[5];
               for (int i = 0; i < r; i++) {
                  are[i] = x[2u * (b + k + (uint32_t) i * q)];
                  aim[i] = x[2u * (b + k + (uint32_t) i * q) + 1u];
               }
               small_dft(r, are, aim, xre, xim);
               for (int i = 1; i < r; i++) {
                  float wr = tw[2u * ((uint32_t) (i - 1) * q + k)];
                  float wi = tw[2u * ((uint32_t) (i - 1) * q + k) + 1u];
                  float tr = xre[i] * wr - xim[i] * wi;
                  float ti = xre[i] * wi + xim[i] * wr;
                  xre[i] = tr;
                  xim[i] = ti;
               }
               for (int i = 0; i < r; i++) {
                  uint32_t sl = (r == 4) ? (uint32_t) slot4[i] : (uint32_t) i;
                  x[2u * (b + k + sl * q)]      = xre[i];
                  x[2u * (b + k + sl * q) + 1u] = xim[i];
               }
            }
         }
         tw += 2u * (uint32_t) (r - 1) * q;
      }
      m = q;
   }
}

/* Forward: src/fft_c7x/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/..._cn.c:210-495.
 * Inverse: src/fft_c7x/FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc/..._cn.c:233-495,
 * computed as conj(FFT(conj(x) * (1/N))) with the forward table; the scale
 * is the float (1.0f/(float)N) of ..._cn.c:220-228. */
int orc_fft_c2c_f32(float *pX, const float *pW, float *pY,
                    uint32_t numPoints, uint32_t numChannels, int inverse)
{
   int radix[64];
   int ns = stage_radices(numPoints, radix);
   if (ns < 0) return -1;
   uint32_t *perm = (uint32_t *) malloc(sizeof(uint32_t) * (numPoints ? numPoints : 1u));
   if (!perm) return -2;
   for (uint32_t k = 0; k < numPoints; k++) perm[k] = dif_position(k, radix, ns);
   const float scale = 1.0f / (float) numPoints;
   for (uint32_t ch = 0; ch < numChannels; ch++) {
      float *x = pX + (size_t) ch * numPoints * 2u;
      float *y = pY + (size_t) ch * numPoints * 2u;
      if (inverse) {
         for (uint32_t k = 0; k < numPoints; k++) {
            x[2u * k + 1u] = -x[2u * k + 1u];
            x[2u * k]      = scale * x[2u * k];
            x[2u * k + 1u] = scale * x[2u * k + 1u];
         }
      }
      dif_channel_f32(x, pW, numPoints, radix, ns);
      for (uint32_t k = 0; k < numPoints; k++) {
         y[2u * k]      = x[2u * perm[k]];
         y[2u * k + 1u] = inverse ? -x[2u * perm[k] + 1u] : x[2u * perm[k] + 1u];
      }
   }
   free(perm);
   return 0;
}

/* N/2-point c2c on the packed reals, then the split post-process.
 * src/fft_c7x/FFTLIB_fft1dBatched_i32f_c32fc_o32fc/..._cn.c:9-125. */
int orc_fft_r2c_f32(float *pX, const float *pW, float *pXFFT, const float *pSf,
                    float *pY, uint32_t numPoints, uint32_t numChannels, int outmode)
{
   uint32_t h = numPoints / 2u;
   uint32_t nOut = outmode ? numPoints : h + 1u;
   int rc = orc_fft_c2c_f32(pX, pW, pXFFT, h, numChannels, 0);
   if (rc) return rc;
   for (uint32_t ch = 0; ch < numChannels; ch++) {
      const float *z = pXFFT + (size_t) ch * numPoints;
      float *y = pY + (size_t) ch * nOut * 2u;
      for (uint32_t i = 0; i < h; i++) {
         uint32_t j = (i == 0u) ? 0u : h - i;
         float ar = z[2u * i], ai = z[2u * i + 1u];
         float br = z[2u * j], bi = z[2u * j + 1u];
         float Ar = pSf[2u * i], Ai = pSf[2u * i + 1u];
         float Br = pSf[2u * numPoints - 2u * i - 2u], Bi = pSf[2u * numPoints - 2u * i - 1u];
         /* Z[i] A[i] + conj(Z[h-i]) B[i] */
         float re = (ar * Ar - ai * Ai) + (br * Br + bi * Bi);
         float im = (ar * Ai + ai * Ar) + (br * Bi - bi * Br);
         y[2u * i] = re;
         y[2u * i + 1u] = im;
         if (outmode && i > 0u) {
            y[2u * (numPoints - i)] = re;
            y[2u * (numPoints - i) + 1u] = -im;
         }
      }
      /* Nyquist bin (_cn.c:113-118) */
      y[2u * h] = z[0] - z[1];
      y[2u * h + 1u] = 0.0f;
   }
   return 0;
}

/* Split pre-process, then the N/2-point inverse c2c.
 * src/fft_c7x/FFTLIB_ifft1dBatched_i32fc_c32fc_o32f/..._cn.c:7-91. */
int orc_fft_c2r_f32(const float *pX, const float *pW, float *pXFFT, const float *pSf,
                    float *pY, uint32_t numPoints, uint32_t numChannels, int inMode)
{
   uint32_t h = numPoints / 2u;
   uint32_t inStride = inMode ? 2u * numPoints : 2u * (h + 1u);
   for (uint32_t ch = 0; ch < numChannels; ch++) {
      const float *x = pX + (size_t) ch * inStride;
      float *z = pXFFT + (size_t) ch * numPoints;
      for (uint32_t i = 0; i < h; i++) {
         float ar = x[2u * i], ai = x[2u * i + 1u];
         float br, bi;
         if (inMode == 0) { br = x[2u * (h - i)]; bi = -x[2u * (h - i) + 1u]; }
         else { br = x[2u * (i + h)]; bi = x[2u * (i + h) + 1u]; }
         float Ar = pSf[2u * i], Ai = pSf[2u * i + 1u];
         float Br = pSf[2u * i + numPoints], Bi = pSf[2u * i + numPoints + 1u];
         z[2u * i]      = (ar * Ar - ai * Ai) + (br * Br - bi * Bi);
         z[2u * i + 1u] = (ar * Ai + ai * Ar) + (br * Bi + bi * Br);
      }
   }
   return orc_fft_c2c_f32(pXFFT, pW, pY, h, numChannels, 1);
}

/* ------------------------------------------------------------------------ */
/* int16 c2c (bit-exact)                                                     */
/* ------------------------------------------------------------------------ */

/* Two's-complement narrowing, as every int16 assignment in the reference. */
static inline int16_t wrap16(int v) { return (int16_t) (uint16_t) (unsigned) v; }

/* Q15 product scaling with saturation, the VCMPYR1HH model:
 * ((x + 0x4000) << 1) clamped to [-2^31, 0x7FFF0000], then >> 16.
 * src/fft_c7x/FFTLIB_fft1dBatched_i16sc_c16sc_o16sc/..._cn.c:13-25. */
static int16_t q15_scale(int64_t x)
{
   int64_t t = (x + 0x4000) * 2;
   if (t > 0x7FFF0000LL) t = 0x7FFF0000LL;
   if (t < -0x80000000LL) t = -0x80000000LL;
   return (int16_t) (t >> 16);
}

/* Multiply by j with the VCROT90H saturation of -(-32768) to 32767:
 * (re, im) -> (-im, re). ..._cn.c:27-34. */
static inline int16_t rot90_re(int16_t im) { return (im == (int16_t) -32768) ? (int16_t) 32767 : (int16_t) -im; }

/* Arithmetic right shift that rounds by the last bit shifted out. The mask
 * is formed exactly as the reference forms it (a 32-bit shift by shift-1,
 * x86 masking the count, narrowed to int16), so shift == 0 is a no-op.
 * ..._cn.c:36-45. */
static inline int16_t shift_round(int16_t v, uint32_t shift)
{
   int16_t mask = (int16_t) (uint16_t) (1u << ((shift - 1u) & 31u));
   int vi = v;
   int s = (int) (shift & 31u);
   return wrap16(((vi & mask) != 0) ? ((vi >> s) + 1) : (vi >> s));
}

/* 4-point DIF butterfly with int16 intermediates (..._cn.c:47-168).
 * Outputs in natural bin order y[0..3]; twiddled when tw != NULL. */
static void bfly4_i16(const int16_t *pr, const int16_t *pi, const int16_t *tw,
                      int16_t *yr, int16_t *yi)
{
   int16_t s1r = wrap16(pr[0] + pr[2]), s1i = wrap16(pi[0] + pi[2]);
   int16_t s2r = wrap16(pr[1] + pr[3]), s2i = wrap16(pi[1] + pi[3]);
   int16_t d1r = wrap16(pr[0] - pr[2]), d1i = wrap16(pi[0] - pi[2]);
   int16_t d2r = wrap16(pr[1] - pr[3]), d2i = wrap16(pi[1] - pi[3]);
   int16_t jr = rot90_re(d2i), ji = d2r; /* j * d2 */
   int16_t tr[4], ti[4];
   tr[0] = wrap16(s1r + s2r); ti[0] = wrap16(s1i + s2i);
   tr[1] = wrap16(d1r - jr);  ti[1] = wrap16(d1i - ji);
   tr[2] = wrap16(s1r - s2r); ti[2] = wrap16(s1i - s2i);
   tr[3] = wrap16(d1r + jr);  ti[3] = wrap16(d1i + ji);
   if (!tw) {
      for (int i = 0; i < 4; i++) { yr[i] = tr[i]; yi[i] = ti[i]; }
      return;
   }
   yr[0] = q15_scale((int64_t) tr[0] * 32768);
   yi[0] = q15_scale((int64_t) ti[0] * 32768);
   for (int i = 1; i < 4; i++) {
      int64_t wr = tw[2 * (i - 1)], wi = tw[2 * (i - 1) + 1];
      yr[i] = q15_scale((int64_t) tr[i] * wr - (int64_t) ti[i] * wi);
      yi[i] = q15_scale((int64_t) tr[i] * wi + (int64_t) ti[i] * wr);
   }
}

/* src/fft_c7x/FFTLIB_fft1dBatched_i16sc_c16sc_o16sc/..._cn.c:191-338. */
int orc_fft_c2c_i16(int16_t *pX, const int16_t *pW, int16_t *pY,
                    const uint32_t *pShift, uint32_t numShifts,
                    uint32_t numPoints, uint32_t numChannels)
{
   if (numPoints == 0u || (numPoints & (numPoints - 1u)) != 0u) return -1;
   uint32_t nBits = 0u;
   while ((1u << nBits) < numPoints) nBits++;
   for (uint32_t ch = 0; ch < numChannels; ch++) {
      int16_t *x = pX + (size_t) ch * numPoints * 2u;
      int16_t *y = pY + (size_t) ch * numPoints * 2u;
      const int16_t *tw = pW;
      uint32_t m = numPoints, stage = 0u, shift = 0u;
      while (m > 2u) {
         if (stage >= numShifts) return -3;
         shift = pShift[stage];
         uint32_t q = m / 4u;
         for (uint32_t b = 0; b < numPoints; b += m) {
            for (uint32_t k = 0; k < q; k++) {
               int16_t pr[4], pi[4], yr[4], yi[4];
               for (int i = 0; i < 4; i++) {
                  pr[i] = x[2u * (b + k + (uint32_t) i * q)];
                  pi[i] = x[2u * (b + k + (uint32_t) i * q) + 1u];
               }
               int noTw = (m == 4u) || (m == 8u && k == 0u);
               int16_t w[6];
               for (int i = 0; i < 3; i++) {
                  w[2 * i]     = tw[2u * ((uint32_t) i * q + k)];
                  w[2 * i + 1] = tw[2u * ((uint32_t) i * q + k) + 1u];
               }
               bfly4_i16(pr, pi, noTw ? NULL : w, yr, yi);
               if (m != 8u) {
                  for (int i = 0; i < 4; i++) {
                     yr[i] = shift_round(yr[i], shift);
                     yi[i] = shift_round(yi[i], shift);
                  }
               }
               /* bins 0,1,2,3 -> slots 0,2,1,3 */
               static const uint32_t slot[4] = {0u, 2u, 1u, 3u};
               for (int i = 0; i < 4; i++) {
                  x[2u * (b + k + slot[i] * q)]      = yr[i];
                  x[2u * (b + k + slot[i] * q) + 1u] = yi[i];
               }
            }
         }
         tw += 2u * 3u * q;
         m = q;
         stage++;
      }
      if (m == 2u) {
         /* trailing radix-2 shares the 8-point stage's shift (..._cn.c:302-323) */
         for (uint32_t b = 0; b < numPoints; b += 2u) {
            int16_t ar = x[2u * b], ai = x[2u * b + 1u];
            int16_t br = x[2u * b + 2u], bi = x[2u * b + 3u];
            x[2u * b]      = shift_round(wrap16(ar + br), shift);
            x[2u * b + 1u] = shift_round(wrap16(ai + bi), shift);
            x[2u * b + 2u] = shift_round(wrap16(ar - br), shift);
            x[2u * b + 3u] = shift_round(wrap16(ai - bi), shift);
         }
      }
      /* bit reversal into pY (..._cn.c:326-334) */
      for (uint32_t k = 0; k < numPoints; k++) {
         uint32_t rk = 0u;
         for (uint32_t bit = 0; bit < nBits; bit++) rk |= ((k >> bit) & 1u) << (nBits - 1u - bit);
         if (nBits == 0u) rk = 0u;
         y[2u * k]      = x[2u * rk];
         y[2u * k + 1u] = x[2u * rk + 1u];
      }
   }
   return 0;
}
