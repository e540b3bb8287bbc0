// mma_ref_driver.cpp -- calls the reference's own natural-C integer DFT code
// (dftSmall _cn, LINALG matrixMatrixMultiply _cn used by dftLarge and called
// on its own, highRadixDecompositions _cn), compiled from its sources by
// oracle/Makefile, with the private-argument structures its optimized init
// would fill. TEST INFRASTRUCTURE ONLY (the checker of the integer oracle).
//
// The highRadix internal table (the reference keeps it in a global that its
// optimized twGen fills, c71/..._ci.cpp:2084-2112) comes from the caller.
#include <stdint.h>
#include <string.h>

#include "fft_c7xmma/FFTLIB_FFT_dftSmall_ixX_cxX_oxX/FFTLIB_FFT_dftSmall_ixX_cxX_oxX_priv.h"
#include "fft_c7xmma/FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX/FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_priv.h"
#include "linalg_c7xmma/FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX/FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_priv.h"

namespace {

template <class T, class A, uint32_t MMA>
int run(int variant, uint32_t n, uint32_t batch, uint32_t interleave, const uint32_t* shifts, const void* W,
        const void* W1, void* x, void* y)
{
    if (variant == 1) {
        FFTLIB_FFT_dftSmall_ixX_cxX_oxX_PrivArgs p;
        memset(&p, 0, sizeof(p));
        p.initArgs.fftSize = n;
        p.initArgs.batchSize = batch;
        p.initArgs.interleave = interleave;
        for (int i = 0; i < 5; ++i) p.initArgs.shiftVector[i] = shifts[i];
        return FFTLIB_FFT_dftSmall_ixX_cxX_oxX_exec_cn<T, A, MMA>(&p, x, W, y);
    }
    if (variant == 2) {
        FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_PrivArgs p;
        memset(&p, 0, sizeof(p));
        p.initArgs.shift = (int8_t)shifts[0];
        p.M = (int32_t)batch;
        p.K = (int32_t)(2 * n);
        p.N = (int32_t)(2 * n);
        p.strideAElements = p.strideBElements = p.strideCElements = (int32_t)(2 * n);
        return FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_exec_cn<T, A>(&p, x, W, y);
    }
    FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_PrivArgs p;
    memset(&p, 0, sizeof(p));
    p.initArgs.fftSize = n;
    p.initArgs.batchSize = batch;
    p.initArgs.interleave = interleave;
    for (int i = 0; i < 5; ++i) p.initArgs.shiftVector[i] = shifts[i];
    p.pW = (uint8_t*)W1;
    return FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_exec_cn<T, A, MMA>(&p, x, W, y);
}

} // namespace

extern "C" int ref_mma_exec(int bits, int variant, uint32_t n, uint32_t batch, uint32_t interleave,
                            const uint32_t* shifts, const void* W, const void* W1, void* x, void* y)
{
    if (bits == 16) return run<int16_t, int64_t, FFTLIB_MMA_SIZE_16_BIT>(variant, n, batch, interleave, shifts, W, W1, x, y);
    return run<int32_t, FFTLIB_int128_t, FFTLIB_MMA_SIZE_32_BIT>(variant, n, batch, interleave, shifts, W, W1, x, y);
}

// The LINALG multiply on its own: M x K by K x N, row strides in elements,
// INT8 / INT16 / INT32 as the reference's _cn instantiates it.
extern "C" int ref_linalg_exec(int bits, int32_t M, int32_t K, int32_t N, const void* A, int32_t lda, const void* B,
                               int32_t ldb, void* C, int32_t ldc, int32_t shift)
{
    FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_PrivArgs p;
    memset(&p, 0, sizeof(p));
    p.initArgs.shift = (int8_t)shift;
    p.M = M;
    p.K = K;
    p.N = N;
    p.strideAElements = lda;
    p.strideBElements = ldb;
    p.strideCElements = ldc;
    if (bits == 8) return FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_exec_cn<int8_t, int32_t>(&p, A, B, C);
    if (bits == 16) return FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_exec_cn<int16_t, int64_t>(&p, A, B, C);
    return FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_exec_cn<int32_t, FFTLIB_int128_t>(&p, A, B, C);
}
