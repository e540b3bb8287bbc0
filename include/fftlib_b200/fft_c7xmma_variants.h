/*
 * fft_c7xmma_variants.h -- the three integer DFT kernels behind the
 * coordinator, callable on their own as in the reference:
 *   FFTLIB_FFT_dftSmall_ixX_cxX_oxX_*                (src/fft_c7xmma/FFTLIB_FFT_dftSmall_ixX_cxX_oxX/
 *                                                    FFTLIB_FFT_dftSmall_ixX_cxX_oxX.h:35-230)
 *   FFTLIB_FFT_dftLarge_ixX_cxX_oxX_*                (.../FFTLIB_FFT_dftLarge_ixX_cxX_oxX.h:37-238)
 *   FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_* (.../FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX.h:45-262)
 * Same names, InitArgs layouts, call order and status codes. INT16 and INT32
 * (interleaved or planar) with the C7120 MMA widths (32 and 16), bit-exact
 * with the reference's natural C; other types answer
 * FFTLIB_ERR_NOT_IMPLEMENTED. The arithmetic, tables and buffer rules are
 * those of the coordinator (fft_c7xmma.h) with the variant fixed:
 *   dftSmall   fftSize <= MMA/2 (getSizes: FFTLIB_ERR_INVALID_DIMENSION above),
 *              W = MMA x MMA;
 *   dftLarge   fftSize  > MMA/2 (FFTLIB_ERR_INVALID_DIMENSION at or below),
 *              W = the dense 2N x 2N embedding, the product through the
 *              LINALG multiply (a shiftVector[0] above 64 for INT16, 128 for
 *              INT32 read as int8_t: FFTLIB_ERR_INVALID_SHIFT);
 *   highRadix  fftSize >= 2 MMA (init_checkParams: FFTLIB_ERR_INVALID_VALUE
 *              below), fftSize = d0 (MMA/2)^L with d0 <= MMA/2 and at most
 *              four decimation stages (init: FFTLIB_ERR_NOT_IMPLEMENTED
 *              otherwise); pX is its work buffer and must differ from pY.
 * Handles are caller-allocated (getHandleSize bytes); buffers may be device
 * or host memory, exec is synchronous, and FFTLIB_b200_FFT_fft_execAsync
 * (fft_c7xmma.h) runs any of these handles on a stream.
 * The reference's perfEst functions estimate C7x cycles and are not provided.
 */
#ifndef FFTLIB_B200_FFT_C7XMMA_VARIANTS_H_
#define FFTLIB_B200_FFT_C7XMMA_VARIANTS_H_

#include "FFTLIB_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---- dftSmall ------------------------------------------------------------ */

/* reference: FFTLIB_FFT_dftSmall_ixX_cxX_oxX.h:35 */
#define FFTLIB_FFT_DFTSMALL_IXX_CXX_OXX_NUMSHIFTS 1

/* reference: FFTLIB_FFT_dftSmall_ixX_cxX_oxX.h:40-62 (same fields and order) */
typedef struct {
    int8_t funcStyle;
    uint32_t fftSize;
    uint32_t batchSize;
    uint32_t interleave;
    uint32_t shiftVector[FFTLIB_FFT_DFTSMALL_IXX_CXX_OXX_NUMSHIFTS];
} FFTLIB_FFT_dftSmall_ixX_cxX_oxX_InitArgs;

/* reference: FFTLIB_FFT_dftSmall_ixX_cxX_oxX.h:72 */
int32_t FFTLIB_FFT_dftSmall_ixX_cxX_oxX_getHandleSize(FFTLIB_FFT_dftSmall_ixX_cxX_oxX_InitArgs *pKerInitArgs);
/* reference: FFTLIB_FFT_dftSmall_ixX_cxX_oxX.h:93-96 */
FFTLIB_STATUS FFTLIB_FFT_dftSmall_ixX_cxX_oxX_getSizes(const FFTLIB_FFT_dftSmall_ixX_cxX_oxX_InitArgs *pKerInitArgs,
                                                       FFTLIB_bufParams1D_t *bufParamsX,
                                                       FFTLIB_bufParams1D_t *bufParamsW,
                                                       FFTLIB_bufParams1D_t *bufParamsY);
/* reference: FFTLIB_FFT_dftSmall_ixX_cxX_oxX.h:114-116 */
FFTLIB_STATUS FFTLIB_FFT_dftSmall_ixX_cxX_oxX_twGen(const FFTLIB_FFT_dftSmall_ixX_cxX_oxX_InitArgs *pKerInitArgs,
                                                    void *pW, const FFTLIB_bufParams1D_t *bufParamsW);
/* reference: FFTLIB_FFT_dftSmall_ixX_cxX_oxX.h:140-144 */
FFTLIB_STATUS FFTLIB_FFT_dftSmall_ixX_cxX_oxX_init(FFTLIB_kernelHandle handle, FFTLIB_bufParams1D_t *bufParamsX,
                                                   FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_bufParams1D_t *bufParamsY,
                                                   FFTLIB_FFT_dftSmall_ixX_cxX_oxX_InitArgs *pKerInitArgs);
/* reference: FFTLIB_FFT_dftSmall_ixX_cxX_oxX.h:168-173 */
FFTLIB_STATUS FFTLIB_FFT_dftSmall_ixX_cxX_oxX_init_checkParams(
    FFTLIB_kernelHandle handle, const FFTLIB_bufParams1D_t *bufParamsX, const FFTLIB_bufParams1D_t *bufParamsW,
    const FFTLIB_bufParams1D_t *bufParamsY, const FFTLIB_FFT_dftSmall_ixX_cxX_oxX_InitArgs *pKerInitArgs);
/* reference: FFTLIB_FFT_dftSmall_ixX_cxX_oxX.h:203-206 */
FFTLIB_STATUS FFTLIB_FFT_dftSmall_ixX_cxX_oxX_exec(FFTLIB_kernelHandle handle, void *pX, void *pW, void *pY);
/* reference: FFTLIB_FFT_dftSmall_ixX_cxX_oxX.h:226-230 */
FFTLIB_STATUS FFTLIB_FFT_dftSmall_ixX_cxX_oxX_exec_checkParams(FFTLIB_kernelHandle handle, const void *pX,
                                                               const void *pW, const void *pY);

/* ---- dftLarge ------------------------------------------------------------ */

/* reference: FFTLIB_FFT_dftLarge_ixX_cxX_oxX.h:37 */
#define FFTLIB_FFT_DFTLARGE_IXX_CXX_OXX_NUMSHIFTS 1

/* reference: FFTLIB_FFT_dftLarge_ixX_cxX_oxX.h:42-64 (same fields and order) */
typedef struct {
    int8_t funcStyle;
    uint32_t fftSize;
    uint32_t batchSize;
    uint32_t interleave;
    uint32_t shiftVector[FFTLIB_FFT_DFTLARGE_IXX_CXX_OXX_NUMSHIFTS];
} FFTLIB_FFT_dftLarge_ixX_cxX_oxX_InitArgs;

/* reference: FFTLIB_FFT_dftLarge_ixX_cxX_oxX.h:76 */
int32_t FFTLIB_FFT_dftLarge_ixX_cxX_oxX_getHandleSize(FFTLIB_FFT_dftLarge_ixX_cxX_oxX_InitArgs *pKerInitArgs);
/* reference: FFTLIB_FFT_dftLarge_ixX_cxX_oxX.h:98-101 */
FFTLIB_STATUS FFTLIB_FFT_dftLarge_ixX_cxX_oxX_getSizes(const FFTLIB_FFT_dftLarge_ixX_cxX_oxX_InitArgs *pKerInitArgs,
                                                       FFTLIB_bufParams1D_t *bufParamsX,
                                                       FFTLIB_bufParams1D_t *bufParamsW,
                                                       FFTLIB_bufParams1D_t *bufParamsY);
/* reference: FFTLIB_FFT_dftLarge_ixX_cxX_oxX.h:119-121 */
FFTLIB_STATUS FFTLIB_FFT_dftLarge_ixX_cxX_oxX_twGen(const FFTLIB_FFT_dftLarge_ixX_cxX_oxX_InitArgs *pKerInitArgs,
                                                    void *pW, const FFTLIB_bufParams1D_t *bufParamsW);
/* reference: FFTLIB_FFT_dftLarge_ixX_cxX_oxX.h:145-149 */
FFTLIB_STATUS FFTLIB_FFT_dftLarge_ixX_cxX_oxX_init(FFTLIB_kernelHandle handle, const FFTLIB_bufParams1D_t *bufParamsX,
                                                   const FFTLIB_bufParams1D_t *bufParamsW,
                                                   const FFTLIB_bufParams1D_t *bufParamsY,
                                                   const FFTLIB_FFT_dftLarge_ixX_cxX_oxX_InitArgs *pKerInitArgs);
/* reference: FFTLIB_FFT_dftLarge_ixX_cxX_oxX.h:174-179 */
FFTLIB_STATUS FFTLIB_FFT_dftLarge_ixX_cxX_oxX_init_checkParams(
    FFTLIB_kernelHandle handle, const FFTLIB_bufParams1D_t *bufParamsX, const FFTLIB_bufParams1D_t *bufParamsW,
    const FFTLIB_bufParams1D_t *bufParamsY, const FFTLIB_FFT_dftLarge_ixX_cxX_oxX_InitArgs *pKerInitArgs);
/* reference: FFTLIB_FFT_dftLarge_ixX_cxX_oxX.h:210-213. The dense table of
 * fftSize above 152 (INT16) / 105 (INT32) does not fit in shared memory;
 * those sizes run the tiled multiply out of place (a pX == pY call is
 * staged through a temporary output). */
FFTLIB_STATUS FFTLIB_FFT_dftLarge_ixX_cxX_oxX_exec(FFTLIB_kernelHandle handle, const void *pX, const void *pW,
                                                   void *pY);
/* reference: FFTLIB_FFT_dftLarge_ixX_cxX_oxX.h:234-238 */
FFTLIB_STATUS FFTLIB_FFT_dftLarge_ixX_cxX_oxX_exec_checkParams(FFTLIB_kernelHandle handle, const void *pX,
                                                               const void *pW, const void *pY);

/* ---- highRadixDecompositions -------------------------------------------------- */

/* reference: FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX.h:45 */
#define FFTLIB_FFT_HIGHRADIXDECOMPOSITIONS_IXX_CXX_OXX_NUMSHIFTS 5

/* reference: FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX.h:50-72 (same fields and order) */
typedef struct {
    int8_t funcStyle;
    uint32_t fftSize;
    uint32_t batchSize;
    uint32_t interleave;
    uint32_t shiftVector[FFTLIB_FFT_HIGHRADIXDECOMPOSITIONS_IXX_CXX_OXX_NUMSHIFTS];
} FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_InitArgs;

/* reference: FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX.h:78. The
 * internal table (the d0-point and MMA/2-point DFTs): init writes the one of
 * its fftSize here, in the data type, as the reference's init does; the
 * kernels read a device copy. */
extern uint8_t FFTLIB_FFT_twData[32 * 32 * 3 * sizeof(int16_t)];

/* reference: FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX.h:88-89 */
int32_t FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_getHandleSize(
    FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_InitArgs *pKerInitArgs);
/* reference: FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX.h:114-118 */
FFTLIB_STATUS FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_getSizes(
    const FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_InitArgs *pKerInitArgs, FFTLIB_bufParams1D_t *bufParamsX,
    FFTLIB_bufParams1D_t *bufParamsW, FFTLIB_bufParams1D_t *bufParamsY);
/* reference: FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX.h:141-144 */
FFTLIB_STATUS FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_twGen(
    const FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_InitArgs *pKerInitArgs, void *pW,
    const FFTLIB_bufParams1D_t *bufParamsW);
/* reference: FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX.h:169-174 */
FFTLIB_STATUS FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_init(
    FFTLIB_kernelHandle handle, FFTLIB_bufParams1D_t *bufParamsX, FFTLIB_bufParams1D_t *bufParamsW,
    FFTLIB_bufParams1D_t *bufParamsY, FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_InitArgs *pKerInitArgs);
/* reference: FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX.h:199-204 */
FFTLIB_STATUS FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_init_checkParams(
    FFTLIB_kernelHandle handle, const FFTLIB_bufParams1D_t *bufParamsX, const FFTLIB_bufParams1D_t *bufParamsW,
    const FFTLIB_bufParams1D_t *bufParamsY,
    const FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_InitArgs *pKerInitArgs);
/* reference: FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX.h:234-238 */
FFTLIB_STATUS FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_exec(FFTLIB_kernelHandle handle, void *pX, void *pW,
                                                                  void *pY);
/* reference: FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX.h:259-262 */
FFTLIB_STATUS FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_exec_checkParams(FFTLIB_kernelHandle handle,
                                                                              const void *pX, const void *pW,
                                                                              const void *pY);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif
