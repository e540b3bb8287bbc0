/*
 * linalg_c7xmma.h -- the integer matrix multiply of libfftlib_b200.so, a
 * drop-in for the reference's src/linalg_c7xmma/
 * FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX/
 * FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX.h:35-196 (same names,
 * InitArgs layout, call order and status codes).
 *
 * C = round_shift(A B): A is dim_y x dim_x of src0 (M x K), B of src1
 * (K x N), C of dst (M x N), row strides stride_y in bytes. Types INT8,
 * INT16 and INT32, the same for all three; products and sums are exact (the
 * reference's int32, int64 and 128-bit accumulators; an INT8 sum that leaves
 * the int32 range wraps, where the reference's C is undefined), then
 * shiftAndRound by InitArgs.shift (round half up, saturated to the type;
 * 0: saturate only), bit for bit as the reference's natural C
 * (..._cn.cpp:27-62). Runs on the GPU whatever funcStyle says.
 *
 * Differences: init always runs init_checkParams (the reference does so
 * when built with FFTLIB_CHECK_PARAMS) and also refuses a dst stride that
 * makes rows of C overlap (FFTLIB_ERR_INVALID_DIMENSION). Buffers may be
 * device or host memory; exec is synchronous. C must not overlap A or B
 * (the reference assumes the same). perfEst (C7x cycles) is not provided.
 */
#ifndef FFTLIB_B200_LINALG_C7XMMA_H_
#define FFTLIB_B200_LINALG_C7XMMA_H_

#include "FFTLIB_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* reference: FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX.h:35-38 */
typedef enum {
    FFTLIB_LINALG_MATRIXMATRIXMULTIPLY_IXX_IXX_OXX_ERR_SMALL_K = FFTLIB_ERROR_MAX,
    FFTLIB_LINALG_MATRIXMATRIXMULTIPLY_IXX_IXX_OXX_ERR_MAX
} FFTLIB_LINALG_MATRIXMATRIXMULTIPLY_IXX_IXX_OXX_STATUS_NAME;

/* reference: FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX.h:48-51 (same fields and order) */
typedef struct {
    int8_t funcStyle; /* FFTLIB_FUNCTION_NATC or FFTLIB_FUNCTION_OPTIMIZED */
    int8_t shift;     /* output shift */
} FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_InitArgs;

/* reference: FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX.h:64-65 */
int32_t FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_getHandleSize(
    FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_InitArgs *pKerInitArgs);

/* reference: FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX.h:89-94 */
FFTLIB_STATUS FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_init(
    FFTLIB_kernelHandle handle, const FFTLIB_bufParams2D_t *src0_addr, const FFTLIB_bufParams2D_t *src1_addr,
    const FFTLIB_bufParams2D_t *dst_addr, const FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_InitArgs *pKerInitArgs);

/* reference: FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX.h:117-122; the
 * checks of ..._oxX.cpp:14-62 in the same order */
FFTLIB_STATUS FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_init_checkParams(
    FFTLIB_kernelHandle handle, const FFTLIB_bufParams2D_t *src0_addr, const FFTLIB_bufParams2D_t *src1_addr,
    const FFTLIB_bufParams2D_t *dst_addr, const FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_InitArgs *pKerInitArgs);

/* reference: FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX.h:156-160 */
FFTLIB_STATUS FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_exec(FFTLIB_kernelHandle handle, const void *src0,
                                                                  const void *src1, void *dst);

/* reference: FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX.h:181-184 */
FFTLIB_STATUS FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_exec_checkParams(FFTLIB_kernelHandle handle,
                                                                              const void *src0, const void *src1,
                                                                              const void *dst);

/* Extension (no counterpart in the reference): exec enqueued on `stream`
 * (a cudaStream_t) without synchronizing; src0, src1 and dst must be device
 * memory. */
FFTLIB_STATUS FFTLIB_b200_LINALG_matrixMatrixMultiply_execAsync(FFTLIB_kernelHandle handle, const void *src0,
                                                                const void *src1, void *dst, void *stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif
