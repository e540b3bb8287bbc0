/*
 * fft_c7x.h -- the FFTLIB batched 1-D FFT kernels, served by B200 CUDA
 * kernels in libfftlib_b200.so.
 *
 * Every function keeps the reference name, signature, argument meaning and
 * status codes; each block cites the reference declaration it replaces.
 *
 * Calling convention (same as the reference):
 *   _checkParams : validates the arguments, returns a FFTLIB_STATUS.
 *   _init        : validates, builds the plan (radix schedule, FP64-generated
 *                  twiddles resident in HBM) and records it in pBlock
 *                  (caller-allocated, *_PBLOCK_SIZE bytes).
 *   _kernel      : runs the transform and returns when the result is in pY.
 *   _cn          : the reference's "natural C" entry point; here it runs the
 *                  same CUDA path (there is no CPU implementation in the
 *                  library).
 *   _checkParams_cn : the natural-C parameter check (no pBlock argument).
 *
 * Buffers may be device memory (the fast path; cudaMalloc/managed) or host
 * memory (staged through the device, host<->device copies included in the
 * call). Like the reference, the kernels may overwrite pX, which they use as
 * a work buffer for transforms too long for one CTA's shared memory.
 * FP32 kernels compute their own twiddles in FP64 on the GPU; pW (and pSf)
 * are validated as in the reference but their values are not read. The int16
 * kernel reads the caller's Q15 table pW, as its result is defined by it.
 */
#ifndef FFTLIB_B200_FFT_C7X_H_
#define FFTLIB_B200_FFT_C7X_H_

#include "FFTLIB_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* exported from libfftlib_b200.so (built with hidden default visibility) */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* pBlock sizes: src/fft_c7x/<kernel>/<kernel>.h (c2c :27, ifft :27, r2c :34,
 * c2r :34, int16 :29). */
#define FFTLIB_FFT1DBATCHED_I32FC_C32FC_O32FC_PBLOCK_SIZE  (31 * SE_PARAM_SIZE + 18 * sizeof(uint32_t))
#define FFTLIB_IFFT1DBATCHED_I32FC_C32FC_O32FC_PBLOCK_SIZE (31 * SE_PARAM_SIZE + 18 * sizeof(uint32_t))
#define FFTLIB_FFT1DBATCHED_I32F_C32FC_O32FC_PBLOCK_SIZE   (41 * SE_PARAM_SIZE + 18 * sizeof(uint32_t))
#define FFTLIB_IFFT1DBATCHED_I32FC_C32FC_O32F_PBLOCK_SIZE  (41 * SE_PARAM_SIZE + 18 * sizeof(uint32_t))
#define FFTLIB_FFT1DBATCHED_I16SC_C16SC_O16SC_PBLOCK_SIZE  (13 * SE_PARAM_SIZE)

/* ---- FP32 complex-to-complex forward ------------------------------------
 * src/fft_c7x/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc.h:58-135
 * src/fft_c7x/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_cn.h */
FFTLIB_STATUS FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_init(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                         FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                         FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                         uint32_t numPoints, uint32_t numChannels, void *pBlock);
FFTLIB_STATUS FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_kernel(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                           FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                           FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                           uint32_t numPoints, uint32_t numChannels, void *pBlock);
FFTLIB_STATUS FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_checkParams(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                                FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                                FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                                uint32_t numPoints, uint32_t numChannels,
                                                                void *pBlock);
FFTLIB_STATUS FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                       FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                       FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                       uint32_t numPoints, uint32_t numChannels);
FFTLIB_STATUS FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_checkParams_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                                   FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                                   FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                                   uint32_t numPoints, uint32_t numChannels);

/* ---- FP32 complex-to-complex inverse ------------------------------------
 * src/fft_c7x/FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc/FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc.h:58-135 */
FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_init(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                          FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                          FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                          uint32_t numPoints, uint32_t numChannels, void *pBlock);
FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_kernel(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                            FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                            FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                            uint32_t numPoints, uint32_t numChannels, void *pBlock);
FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_checkParams(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                                 FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                                 FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                                 uint32_t numPoints, uint32_t numChannels,
                                                                 void *pBlock);
FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                        FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                        FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                        uint32_t numPoints, uint32_t numChannels);
FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_checkParams_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                                    FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                                    FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                                    uint32_t numPoints, uint32_t numChannels);

/* ---- FP32 real-to-complex forward ----------------------------------------
 * src/fft_c7x/FFTLIB_fft1dBatched_i32f_c32fc_o32fc/FFTLIB_fft1dBatched_i32f_c32fc_o32fc.h:71-180
 * outmode 0: numPoints/2+1 bins per channel; 1: numPoints bins. */
FFTLIB_STATUS FFTLIB_fft1dBatched_i32f_c32fc_o32fc_init(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                        FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                        FFTLIB_F32 *pXFFT, FFTLIB_bufParams1D_t *bufParamsXFFT,
                                                        FFTLIB_F32 *pSf, FFTLIB_bufParams1D_t *bufParamsSf,
                                                        FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                        uint32_t numPoints, uint32_t numChannels, uint8_t outmode,
                                                        void *pBlock);
FFTLIB_STATUS FFTLIB_fft1dBatched_i32f_c32fc_o32fc_kernel(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                          FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                          FFTLIB_F32 *pXFFT, FFTLIB_bufParams1D_t *bufParamsXFFT,
                                                          FFTLIB_F32 *pSf, FFTLIB_bufParams1D_t *bufParamsSf,
                                                          FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                          uint32_t numPoints, uint32_t numChannels, uint8_t outmode,
                                                          void *pBlock);
FFTLIB_STATUS FFTLIB_fft1dBatched_i32f_c32fc_o32fc_checkParams(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                               FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                               FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                               uint32_t numPoints, uint32_t numChannels,
                                                               uint8_t outmode, void *pBlock);
FFTLIB_STATUS FFTLIB_fft1dBatched_i32f_c32fc_o32fc_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                      FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                      FFTLIB_F32 *pXFFT, FFTLIB_bufParams1D_t *bufParamsXFFT,
                                                      FFTLIB_F32 *pSf, FFTLIB_bufParams1D_t *bufParamsSf,
                                                      FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                      uint32_t numPoints, uint32_t numChannels, uint8_t outmode);
FFTLIB_STATUS FFTLIB_fft1dBatched_i32f_c32fc_o32fc_checkParams_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                                  FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                                  FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                                  uint32_t numPoints, uint32_t numChannels,
                                                                  uint8_t outmode);
/* Table generators of the r2c kernel (..._i32f_c32fc_o32fc.h:172,180;
 * ..._tw_gen.cpp:9-97), bit-identical to the reference tables. */
void split_factor_gen_r2c(FFTLIB_F32 *pSFactor, int32_t numPoints);
void tw_gen_r2c(FFTLIB_F32 *pW, int32_t numPoints);

/* ---- FP32 complex-to-real inverse ----------------------------------------
 * src/fft_c7x/FFTLIB_ifft1dBatched_i32fc_c32fc_o32f/FFTLIB_ifft1dBatched_i32fc_c32fc_o32f.h:72-179
 * inMode 0: numPoints/2+1 input bins per channel; 1: numPoints bins. */
FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_init(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                         FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                         FFTLIB_F32 *pXFFT, FFTLIB_bufParams1D_t *bufParamsXFFT,
                                                         FFTLIB_F32 *pSf, FFTLIB_bufParams1D_t *bufParamsSf,
                                                         FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                         uint32_t numPoints, uint32_t numChannels, uint8_t inMode,
                                                         void *pBlock);
FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_kernel(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                           FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                           FFTLIB_F32 *pXFFT, FFTLIB_bufParams1D_t *bufParamsXFFT,
                                                           FFTLIB_F32 *pSf, FFTLIB_bufParams1D_t *bufParamsSf,
                                                           FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                           uint32_t numPoints, uint32_t numChannels, uint8_t inMode,
                                                           void *pBlock);
FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_checkParams(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                                FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                                FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                                uint32_t numPoints, uint32_t numChannels,
                                                                uint8_t inMode, void *pBlock);
FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                       FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                       FFTLIB_F32 *pXFFT, FFTLIB_bufParams1D_t *bufParamsXFFT,
                                                       FFTLIB_F32 *pSf, FFTLIB_bufParams1D_t *bufParamsSf,
                                                       FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                       uint32_t numPoints, uint32_t numChannels, uint8_t inMode);
FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_checkParams_cn(FFTLIB_F32 *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                                   FFTLIB_F32 *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                                   FFTLIB_F32 *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                                   uint32_t numPoints, uint32_t numChannels,
                                                                   uint8_t inMode);
/* Table generators of the c2r kernel (..._i32fc_c32fc_o32f.h:174,179;
 * ..._tw_gen.cpp:9-95). */
void ifft_c2r_split_factor_gen(FFTLIB_F32 *pSFactor, int32_t numPoints);
void ifft_c2r_tw_gen(FFTLIB_F32 *pW, int32_t numPoints);

/* ---- int16 complex-to-complex forward, per-stage shift --------------------
 * src/fft_c7x/FFTLIB_fft1dBatched_i16sc_c16sc_o16sc/FFTLIB_fft1dBatched_i16sc_c16sc_o16sc.h:64-152
 * Bit-exact with the reference _cn (..._cn.c:191-338). */
FFTLIB_STATUS FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_init(int16_t *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                         int16_t *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                         int16_t *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                         uint32_t *pShift, FFTLIB_bufParams1D_t *bufParamsShift,
                                                         uint32_t numPoints, uint32_t numChannels, void *pBlock);
FFTLIB_STATUS FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_kernel(int16_t *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                           int16_t *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                           int16_t *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                           uint32_t *pShift, FFTLIB_bufParams1D_t *bufParamsShift,
                                                           uint32_t numPoints, uint32_t numChannels, void *pBlock);
FFTLIB_STATUS FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_checkParams(int16_t *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                                int16_t *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                                int16_t *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                                uint32_t *pShift,
                                                                FFTLIB_bufParams1D_t *bufParamsShift,
                                                                uint32_t numPoints, uint32_t numChannels,
                                                                void *pBlock);
FFTLIB_STATUS FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_cn(int16_t *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                       int16_t *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                       int16_t *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                       uint32_t *pShift, FFTLIB_bufParams1D_t *bufParamsShift,
                                                       uint32_t numPoints, uint32_t numChannels);
FFTLIB_STATUS FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_checkParams_cn(int16_t *pX, FFTLIB_bufParams1D_t *bufParamsX,
                                                                   int16_t *pW, FFTLIB_bufParams1D_t *bufParamsW,
                                                                   int16_t *pY, FFTLIB_bufParams1D_t *bufParamsY,
                                                                   uint32_t *pShift,
                                                                   FFTLIB_bufParams1D_t *bufParamsShift,
                                                                   uint32_t numPoints, uint32_t numChannels);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* FFTLIB_B200_FFT_C7X_H_ */
