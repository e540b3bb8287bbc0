/*
 * fft_c7xmma.h -- the DFT coordinator of libfftlib_b200.so, a drop-in for
 * the reference's src/fft_c7xmma/FFTLIB_FFT_fft_ixX_cxX_oxX/
 * FFTLIB_FFT_fft_ixX_cxX_oxX.h:37-234 (same names, InitArgs layout, call
 * order and status codes).
 *
 * Data types. The reference implements INT16 and INT32 and answers
 * FFTLIB_ERR_NOT_IMPLEMENTED for anything else. This library implements
 * INT16 and INT32 exactly as the reference does, and adds FLOAT32
 * (interleaved complex); other types answer FFTLIB_ERR_NOT_IMPLEMENTED.
 *
 * INT16 / INT32 (interleaved or planar, both as in the reference): the
 * reference's variant choice for its C7120 MMA widths (32 for INT16, 16 for
 * INT32; FFTLIB_FFT_fft_ixX_cxX_oxX.cpp:13-50), its getSizes and twGen
 * tables, and its natural-C arithmetic bit for bit, on the GPU:
 *   fftSize <= MMA/2          dftSmall: Y = round_shift(X W, shiftVector[0])
 *   fftSize == MMA (or 2 MMA  dftLarge: the same product through the dense
 *     with a large batch)     2N x 2N embedding
 *   larger                    highRadixDecompositions: decimation stages
 *                             (shiftVector[0..3]) and a final MMA/2-point
 *                             DFT stage (shiftVector[4]).
 * highRadix covers fftSize = d0 (MMA/2)^L with d0 <= MMA/2 and L <= 4 (the
 * reference's stage structure; init answers FFTLIB_ERR_NOT_IMPLEMENTED for
 * other lengths, where the reference's loops do not compute a DFT). As in
 * the reference, highRadix uses pX as its work buffer (pX is overwritten and
 * must differ from pY).
 *
 * FLOAT32 paths (chosen by init, from InitArgs):
 *   funcStyle OPTIMIZED, fftSize a power of two in [8, 4096]:
 *     split-precision tensor-core DFT. fftSize <= 64 is one DFT-GEMM (the
 *     reference's dftSmall / dftLarge variants); larger sizes are two
 *     DFT-GEMM stages with the twiddle multiply fused between them (the
 *     highRadixDecompositions variant). pW holds the FP32 computational
 *     matrix written by twGen:
 *       fftSize <= 64:  the real 2N x 2N embedding of the DFT, interleaved
 *                       rows [cos, -sin | sin, cos] exactly as the
 *                       reference's dftLarge twGen lays out its integer
 *                       matrix (FFTLIB_FFT_dftLarge_ixX_cxX_oxX_ci.cpp:122-138);
 *       fftSize  > 64:  the embeddings of the two factor DFTs
 *                       (N = N1 * N2; (2 N1)^2 then (2 N2)^2 floats) and the
 *                       N twiddles (cos, -sin)(2 pi j / N).
 *   any other fftSize of the form 2^a 3^b 5^c, or funcStyle NATC:
 *     the CUDA-core FP32 FFT of FFTLIB_fft1dBatched_i32fc_c32fc_o32fc; pW is
 *     2N floats (the c2c twiddle table, FFTLIB_b200_tw_gen_c2c layout).
 * Both paths return X[k] = sum_n x[n] e^{-2 pi i n k / N} per channel, in
 * natural order, within 2e-6 relative L2 of an FP64 DFT.
 *
 * The handle is caller-allocated (getHandleSize bytes) and holds no device
 * memory of its own. pX, pW and pY may be device or host memory; exec is
 * synchronous. FFTLIB_b200_FFT_fft_execAsync is the stream-ordered form for
 * device buffers.
 */
#ifndef FFTLIB_B200_FFT_C7XMMA_H_
#define FFTLIB_B200_FFT_C7XMMA_H_

#include "FFTLIB_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* reference: FFTLIB_FFT_fft_ixX_cxX_oxX.h:37 */
#define FFTLIB_FFT_FFT_IXX_CXX_OXX_NUMSHIFTS 5

/* reference: FFTLIB_FFT_fft_ixX_cxX_oxX.h:42-64 (same fields and order) */
typedef struct {
    int8_t funcStyle;    /* FFTLIB_FUNCTION_NATC or FFTLIB_FUNCTION_OPTIMIZED */
    uint32_t fftSize;    /* complex points per channel */
    uint32_t batchSize;  /* channels */
    uint32_t interleave; /* 1: |R0|I0|R1|I1|...; 0: |R0|R1|...|I0|I1|... */
    uint32_t shiftVector[FFTLIB_FFT_FFT_IXX_CXX_OXX_NUMSHIFTS]; /* integer paths only; unused for FLOAT32 */
} FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs;

/* reference: FFTLIB_FFT_fft_ixX_cxX_oxX.h:76 */
int32_t FFTLIB_FFT_fft_ixX_cxX_oxX_getHandleSize(FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs *pKerInitArgs);

/* reference: FFTLIB_FFT_fft_ixX_cxX_oxX.h:97-100. Data type from
 * bufParamsX->data_type; fills the three dim_x values. */
FFTLIB_STATUS FFTLIB_FFT_fft_ixX_cxX_oxX_getSizes(const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs *pKerInitArgs,
                                                  FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_bufParams1D_t *bufParamsW,
                                                  FFTLIB_bufParams1D_t *bufParamsY);

/* reference: FFTLIB_FFT_fft_ixX_cxX_oxX.h:118-120. FP64 generation with the
 * angle reduced exactly ((j k) mod N), rounded to FP32; pW may be device or
 * host memory. */
FFTLIB_STATUS FFTLIB_FFT_fft_ixX_cxX_oxX_twGen(const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs *pKerInitArgs, void *pW,
                                               const FFTLIB_bufParams1D_t *bufParamsW);

/* reference: FFTLIB_FFT_fft_ixX_cxX_oxX.h:144-148 */
FFTLIB_STATUS FFTLIB_FFT_fft_ixX_cxX_oxX_init(FFTLIB_kernelHandle handle, FFTLIB_bufParams1D_t *bufParamsX,
                                              FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_bufParams1D_t *bufParamsY,
                                              const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs *pKerInitArgs);

/* reference: FFTLIB_FFT_fft_ixX_cxX_oxX.h:173-177 */
FFTLIB_STATUS FFTLIB_FFT_fft_ixX_cxX_oxX_init_checkParams(FFTLIB_kernelHandle handle,
                                                          const FFTLIB_bufParams1D_t *bufParamsX,
                                                          const FFTLIB_bufParams1D_t *bufParamsW,
                                                          const FFTLIB_bufParams1D_t *bufParamsY,
                                                          const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs *pKerInitArgs);

/* reference: FFTLIB_FFT_fft_ixX_cxX_oxX.h:208-209 */
FFTLIB_STATUS FFTLIB_FFT_fft_ixX_cxX_oxX_exec(FFTLIB_kernelHandle handle, void *pX, void *pW, void *pY);

/* reference: FFTLIB_FFT_fft_ixX_cxX_oxX.h:230-234 */
FFTLIB_STATUS FFTLIB_FFT_fft_ixX_cxX_oxX_exec_checkParams(FFTLIB_kernelHandle handle, const void *pX, const void *pW,
                                                          const void *pY);

/* Extension (no counterpart in the reference): exec enqueued on `stream`
 * (a cudaStream_t; NULL = legacy default stream) without synchronizing.
 * pX, pW and pY must be device memory. Timeouts of the kernel's internal
 * waits are reported by the next synchronous call or by
 * FFTLIB_b200_FFT_fft_sync. */
FFTLIB_STATUS FFTLIB_b200_FFT_fft_execAsync(FFTLIB_kernelHandle handle, void *pX, void *pW, void *pY, void *stream);
/* Synchronizes `stream` and reports a device-side failure of earlier
 * execAsync calls (FFTLIB_ERR_FAILURE, text in FFTLIB_b200_lastError). */
FFTLIB_STATUS FFTLIB_b200_FFT_fft_sync(void *stream);
/* Which path init chose: 1 = tensor-core DFT, 2 = CUDA-core FFT (FLOAT32),
 * 3 = the integer path (INT16 / INT32), 0 = none. */
int32_t FFTLIB_b200_FFT_fft_path(FFTLIB_kernelHandle handle);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif
