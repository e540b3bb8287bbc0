/*
 * fft1d_c7x.h -- the FFTLIB single-transform 1-D FFT kernels
 * (FFTLIB_{fft,ifft}1d_*), served by the same B200 CUDA kernels as the
 * batched family in libfftlib_b200.so.
 *
 * Every function keeps the reference name, signature, argument meaning and
 * status codes; each block cites the reference declaration it replaces.
 * The calling convention (_checkParams, _init, _kernel, _cn,
 * _checkParams_cn) and the buffer rules (device or host memory; pX may be
 * used as a work buffer; FP32 twiddles are computed on the GPU, pW and pSf
 * are validated but not read; the int16 kernel reads its Q15 table pW) are
 * those of fft_c7x.h.
 *
 * The transform length comes from bufParamsX->dim_x, as in the reference:
 *   c2c, ifft, int16 : numPoints = dim_x / 2 complex points
 *   r2c              : numPoints = dim_x reals in, numPoints complex bins out
 *                      (the full spectrum; bins numPoints/2+1.. are the
 *                      conjugates of bins numPoints/2-1..1)
 *   c2r              : numPoints complex bins in (the full spectrum),
 *                      numPoints reals out
 * and the results are the batched kernels' with one channel:
 *   fft1d  c2c  = fft1dBatched c2c                 (numChannels 1)
 *   ifft1d c2c  = ifft1dBatched c2c, scaled 1/numPoints
 *   fft1d  r2c  = fft1dBatched r2c, outmode 1
 *   ifft1d c2r  = ifft1dBatched c2r, inMode 1 (scaled 1/(numPoints/2) inside
 *                 its half-length inverse, i.e. real(ifft) of the spectrum)
 *   fft1d int16 = fft1dBatched int16               (bit-exact, same table and
 *                 shift vector)
 * The reference's natural-C r2c (FFTLIB_fft1d_i32f_c32fc_o32fc_cn.c:137-138,
 * i = 0) also stores the conjugate of bin 0 one bin past the output; this
 * library writes exactly numPoints bins.
 */
#ifndef FFTLIB_B200_FFT1D_C7X_H_
#define FFTLIB_B200_FFT1D_C7X_H_

#include "FFTLIB_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* pBlock sizes: src/fft_c7x/<kernel>/<kernel>.h (c2c :27, ifft :27, r2c :32,
 * c2r :32, int16 :26). The reference's ifft header reuses the c2c macro name
 * with the larger size; both names here carry that larger size. */
#define FFTLIB_FFT1D_I32FC_C32FC_O32FC_PBLOCK_SIZE  (27 * SE_PARAM_SIZE + 16 * sizeof(uint32_t))
#define FFTLIB_IFFT1D_I32FC_C32FC_O32FC_PBLOCK_SIZE (27 * SE_PARAM_SIZE + 16 * sizeof(uint32_t))
#define FFTLIB_FFT1D_I32F_C32FC_O32FC_PBLOCK_SIZE   (35 * SE_PARAM_SIZE + 18 * sizeof(uint32_t))
#define FFTLIB_IFFT1D_I32FC_C32FC_O32F_PBLOCK_SIZE  (34 * SE_PARAM_SIZE + 16 * sizeof(uint32_t))
#define FFTLIB_FFT1D_I16SC_C16SC_O16SC_PBLOCK_SIZE  (9 * SE_PARAM_SIZE)

/* ---- FP32 complex-to-complex forward ------------------------------------
 * src/fft_c7x/FFTLIB_fft1d_i32fc_c32fc_o32fc/FFTLIB_fft1d_i32fc_c32fc_o32fc.h:56-120
 * src/fft_c7x/FFTLIB_fft1d_i32fc_c32fc_o32fc/FFTLIB_fft1d_i32fc_c32fc_o32fc_cn.h:11-23 */
FFTLIB_STATUS FFTLIB_fft1d_i32fc_c32fc_o32fc_init(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_F32 *pW,
                                                  FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_F32 *pY,
                                                  FFTLIB_bufParams1D_t *bufParamsY, void *pBlock);
FFTLIB_STATUS FFTLIB_fft1d_i32fc_c32fc_o32fc_kernel(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_F32 *pW,
                                                    FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_F32 *pY,
                                                    FFTLIB_bufParams1D_t *bufParamsY, void *pBlock);
FFTLIB_STATUS FFTLIB_fft1d_i32fc_c32fc_o32fc_checkParams(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                         FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                         FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                         void *pBlock);
FFTLIB_STATUS FFTLIB_fft1d_i32fc_c32fc_o32fc_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_F32 *pW,
                                                FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_F32 *pY,
                                                FFTLIB_bufParams1D_t *bufParamsY);
FFTLIB_STATUS FFTLIB_fft1d_i32fc_c32fc_o32fc_checkParams_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                            FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                            FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY);

/* ---- FP32 complex-to-complex inverse (scaled 1/numPoints) -----------------
 * src/fft_c7x/FFTLIB_ifft1d_i32fc_c32fc_o32fc/FFTLIB_ifft1d_i32fc_c32fc_o32fc.h:56-120
 * src/fft_c7x/FFTLIB_ifft1d_i32fc_c32fc_o32fc/FFTLIB_ifft1d_i32fc_c32fc_o32fc_cn.h:11-23 */
FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32fc_init(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_F32 *pW,
                                                   FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_F32 *pY,
                                                   FFTLIB_bufParams1D_t *bufParamsY, void *pBlock);
FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32fc_kernel(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_F32 *pW,
                                                     FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_F32 *pY,
                                                     FFTLIB_bufParams1D_t *bufParamsY, void *pBlock);
FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32fc_checkParams(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                          FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                          FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                          void *pBlock);
FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32fc_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_F32 *pW,
                                                 FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_F32 *pY,
                                                 FFTLIB_bufParams1D_t *bufParamsY);
FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32fc_checkParams_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                             FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                             FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY);

/* ---- FP32 real-to-complex forward (full spectrum) ------------------------
 * src/fft_c7x/FFTLIB_fft1d_i32f_c32fc_o32fc/FFTLIB_fft1d_i32f_c32fc_o32fc.h:67-146
 * src/fft_c7x/FFTLIB_fft1d_i32f_c32fc_o32fc/FFTLIB_fft1d_i32f_c32fc_o32fc_cn.h:12-30
 * Table generators (..._i32f_c32fc_o32fc.h:152,160): split_factor_gen_r2c and
 * tw_gen_r2c, declared in fft_c7x.h (the tables are the batched kernel's). */
FFTLIB_STATUS FFTLIB_fft1d_i32f_c32fc_o32fc_init(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_F32 *pW,
                                                 FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_F32 *pXFFT,
                                                 FFTLIB_bufParams1D_t *bufParamsXFFT, FFTLIB_F32 *pSf,
                                                 FFTLIB_bufParams1D_t *bufParamsSf, FFTLIB_F32 *pY,
                                                 FFTLIB_bufParams1D_t *bufParamsY, void *pBlock);
FFTLIB_STATUS FFTLIB_fft1d_i32f_c32fc_o32fc_kernel(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_F32 *pW,
                                                   FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_F32 *pXFFT,
                                                   FFTLIB_bufParams1D_t *bufParamsXFFT, FFTLIB_F32 *pSf,
                                                   FFTLIB_bufParams1D_t *bufParamsSf, FFTLIB_F32 *pY,
                                                   FFTLIB_bufParams1D_t *bufParamsY, void *pBlock);
FFTLIB_STATUS FFTLIB_fft1d_i32f_c32fc_o32fc_checkParams(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                        FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                        FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                        void *pBlock);
FFTLIB_STATUS FFTLIB_fft1d_i32f_c32fc_o32fc_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_F32 *pW,
                                               FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_F32 *pXFFT,
                                               FFTLIB_bufParams1D_t *bufParamsXFFT, FFTLIB_F32 *pSf,
                                               FFTLIB_bufParams1D_t *bufParamsSf, FFTLIB_F32 *pY,
                                               FFTLIB_bufParams1D_t *bufParamsY);
FFTLIB_STATUS FFTLIB_fft1d_i32f_c32fc_o32fc_checkParams_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                           FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                           FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY);

/* ---- FP32 complex-to-real inverse (full spectrum in) ---------------------
 * src/fft_c7x/FFTLIB_ifft1d_i32fc_c32fc_o32f/FFTLIB_ifft1d_i32fc_c32fc_o32f.h:68-149
 * src/fft_c7x/FFTLIB_ifft1d_i32fc_c32fc_o32f/FFTLIB_ifft1d_i32fc_c32fc_o32f_cn.h:12-30
 * Table generators (..._i32fc_c32fc_o32f.h:154,159): ifft_c2r_split_factor_gen
 * and ifft_c2r_tw_gen, declared in fft_c7x.h. */
FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32f_init(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_F32 *pW,
                                                  FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_F32 *pXFFT,
                                                  FFTLIB_bufParams1D_t *bufParamsXFFT, FFTLIB_F32 *pSf,
                                                  FFTLIB_bufParams1D_t *bufParamsSf, FFTLIB_F32 *pY,
                                                  FFTLIB_bufParams1D_t *bufParamsY, void *pBlock);
FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32f_kernel(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_F32 *pW,
                                                    FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_F32 *pXFFT,
                                                    FFTLIB_bufParams1D_t *bufParamsXFFT, FFTLIB_F32 *pSf,
                                                    FFTLIB_bufParams1D_t *bufParamsSf, FFTLIB_F32 *pY,
                                                    FFTLIB_bufParams1D_t *bufParamsY, void *pBlock);
FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32f_checkParams(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                         FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                         FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                         void *pBlock);
FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32f_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_F32 *pW,
                                                FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_F32 *pXFFT,
                                                FFTLIB_bufParams1D_t *bufParamsXFFT, FFTLIB_F32 *pSf,
                                                FFTLIB_bufParams1D_t *bufParamsSf, FFTLIB_F32 *pY,
                                                FFTLIB_bufParams1D_t *bufParamsY);
FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32f_checkParams_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                            FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                            FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY);

/* ---- int16 complex-to-complex forward, per-stage shift --------------------
 * src/fft_c7x/FFTLIB_fft1d_i16sc_c16sc_o16sc/FFTLIB_fft1d_i16sc_c16sc_o16sc.h:60-137
 * src/fft_c7x/FFTLIB_fft1d_i16sc_c16sc_o16sc/FFTLIB_fft1d_i16sc_c16sc_o16sc_cn.h:11-28
 * Bit-exact with the reference _cn (..._cn.c:189-306). */
FFTLIB_STATUS FFTLIB_fft1d_i16sc_c16sc_o16sc_init(int16_t *pX, FFTLIB_bufParams1D_t *bufParamsX, int16_t *pW,
                                                  FFTLIB_bufParams1D_t *bufParamsW, int16_t *pY,
                                                  FFTLIB_bufParams1D_t *bufParamsY, uint32_t *pShift,
                                                  FFTLIB_bufParams1D_t *bufParamsShift, void *pBlock);
FFTLIB_STATUS FFTLIB_fft1d_i16sc_c16sc_o16sc_kernel(int16_t *pX, FFTLIB_bufParams1D_t *bufParamsX, int16_t *pW,
                                                    FFTLIB_bufParams1D_t *bufParamsW, int16_t *pY,
                                                    FFTLIB_bufParams1D_t *bufParamsY, uint32_t *pShift,
                                                    FFTLIB_bufParams1D_t *bufParamsShift, void *pBlock);
FFTLIB_STATUS FFTLIB_fft1d_i16sc_c16sc_o16sc_checkParams(int16_t *pX, FFTLIB_bufParams1D_t *bufParamsX, int16_t *pW,
                                                         FFTLIB_bufParams1D_t *bufParamsW, int16_t *pY,
                                                         FFTLIB_bufParams1D_t *bufParamsY, uint32_t *pShift,
                                                         FFTLIB_bufParams1D_t *bufParamsShift, void *pBlock);
FFTLIB_STATUS FFTLIB_fft1d_i16sc_c16sc_o16sc_cn(int16_t *pX, FFTLIB_bufParams1D_t *bufParamsX, int16_t *pW,
                                                FFTLIB_bufParams1D_t *bufParamsW, int16_t *pY,
                                                FFTLIB_bufParams1D_t *bufParamsY, uint32_t *pShift,
                                                FFTLIB_bufParams1D_t *bufParamsShift);
FFTLIB_STATUS FFTLIB_fft1d_i16sc_c16sc_o16sc_checkParams_cn(int16_t *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                            int16_t *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                            int16_t *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                            uint32_t *pShift, FFTLIB_bufParams1D_t *bufParamsShift);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* FFTLIB_B200_FFT1D_C7X_H_ */
