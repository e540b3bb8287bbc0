// tables.h -- the reference's table generators on the GPU (internal; the
// exported forms are in fftlib_b200_ext.h). Bit-identical to the host
// generators; enqueued on `s`.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fftb200 {

// The stage-twiddle table of an n-point c2c transform (FP32), or the int16
// kernel's Q15 table (q15).
cudaError_t stage_twiddles_device(void* out, uint32_t n, bool q15, cudaStream_t s);
// The split factors of the n-point r2c (c2r = false) or c2r transform.
cudaError_t split_factors_device(float* sf, int32_t n, bool c2r, cudaStream_t s);
// The coordinator's dftLarge matrix (4 n^2 entries of INT16 / INT32).
cudaError_t dft_large_matrix_device(void* w, int bits, uint32_t n, uint32_t interleave, cudaStream_t s);

} // namespace fftb200
