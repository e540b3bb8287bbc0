// dft_int.h -- integer (INT16 / INT32) paths of the DFT coordinator
// FFTLIB_FFT_fft_ixX_cxX_oxX (internal to libfftlib_b200.so).
//
// Bit-exact with the reference's natural-C arithmetic:
//   dftSmall  (fftSize <= MMA/2)  Y = round_shift(X W), W the block-diagonal
//             real embedding with row stride MMA
//             (src/fft_c7xmma/FFTLIB_FFT_dftSmall_ixX_cxX_oxX/..._cn.cpp:18-46);
//   dftLarge  (fftSize == MMA, or 2 MMA with a large batch) the same product
//             with the dense 2N x 2N embedding, through the LINALG matrix
//             multiply (src/linalg_c7xmma/FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX/..._cn.cpp:27-62);
//   highRadix (larger) decimation stages of radix d0 then MMA/2, each an
//             exact complex DFT rounded by its shift, times a twiddle
//             rounded by bits - 1, then MMA/2-point DFTs stored in digit-
//             reversed order (..._highRadixDecompositions_ixX_cxX_oxX_cn.cpp:20-455).
// MMA = 32 for INT16 and 16 for INT32, the C7120 widths. Products and sums
// are exact (64-bit for INT16, 128-bit for INT32); results are saturated as
// the reference does, including its 128-bit saturation of non-negative
// values (FFTLIB_utility.h:546-566, only the low 64 bits are tested).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fftb200 {

enum IntVariant : int32_t { INT_DFT_SMALL = 1, INT_DFT_LARGE = 2, INT_HIGH_RADIX = 3 };

int int_mma_size(int bits);
// The reference's variant choice (FFTLIB_FFT_fft_ixX_cxX_oxX.cpp:13-50).
int int_dft_variant(int bits, uint32_t n, uint32_t batch, uint32_t interleave);
// Caller-table elements, as the reference's getSizes reports them.
uint32_t int_dft_w_size(int bits, uint32_t n, uint32_t batch, uint32_t interleave);
// highRadix lengths this path computes: n = d0 R^L with d0 <= R = MMA/2 the
// first-stage factor and at most four decimation stages (the reference's
// loop structure has no fifth).
bool int_high_radix_covered(int bits, uint32_t n);
// The caller's table (twGen) into host memory of the data type.
void int_dft_twgen_host(int bits, uint32_t n, uint32_t batch, uint32_t interleave, void* w);

// Enqueues the transform of `batch` rows on device buffers. highRadix works
// in place on x (overwritten, as in the reference) and needs x != y.
cudaError_t int_dft_launch(int bits, uint32_t n, uint32_t batch, uint32_t interleave, const uint32_t* shifts,
                           void* x, const void* w, void* y, cudaStream_t s);

// The same with the variant given (the public dftSmall / dftLarge /
// highRadixDecompositions entry points): dftSmall needs n <= MMA/2,
// dftLarge any n (its table is the dense 2n x 2n embedding; one that does
// not fit in shared memory runs the tiled multiply, which needs x != y),
// highRadix a covered length.
uint32_t int_dft_w_size_v(int bits, int variant, uint32_t n);
void int_dft_twgen_host_v(int bits, int variant, uint32_t n, uint32_t batch, uint32_t interleave, void* w);
cudaError_t int_dft_launch_v(int bits, int variant, uint32_t n, uint32_t batch, uint32_t interleave,
                             const uint32_t* shifts, void* x, const void* w, void* y, cudaStream_t s);
// The highRadix internal table of n (MMA x MMA entries of the data type).
void int_dft_w1_host(int bits, uint32_t n, void* out);

// The INT16 dftSmall / dftLarge product on the tensor cores (dft_int_tc.cu):
// rows of n2 = 2N values, n2 dividing 128; x 8-byte aligned.
bool int16_tc_supported(uint32_t n2, const void* x, const void* y);
cudaError_t launch_int16_tc(const int16_t* x, int16_t* y, const int16_t* w, uint32_t n2, uint32_t ld, uint32_t rows,
                            uint32_t shift, cudaStream_t s);
// The INT16 highRadix stages on the tensor cores (dft_int_hr_tc.cu):
// interleaved rows of n = 2^k >= 64 points, x 16-byte aligned, y and the
// twiddles 4-byte aligned. A decimation stage over blocks of s = 16^j points
// (j >= 2), in place, with its 16-point DFT F (the internal table's rows) and
// twiddles tw; the final stage of 16-point groups with the caller's last table
// block D into the digit-reversed positions of y (digits d0, mC, iC, hC).
bool int16_hr_tc_supported(uint32_t n, const void* x, const void* y, const void* tw);
cudaError_t launch_int16_hr_stage(int16_t* x, const int16_t* F, const int16_t* tw, uint32_t n, uint32_t s,
                                  uint32_t rows, uint32_t shift, cudaStream_t st);
cudaError_t launch_int16_hr_final(const int16_t* x, int16_t* y, const int16_t* D, uint32_t n, uint32_t d0,
                                  uint32_t mC, uint32_t iC, uint32_t hC, uint32_t rows, uint32_t shift,
                                  cudaStream_t st);
// The LINALG multiply on the tensor cores (int_mm_tc.cu): A and B rows
// 16-byte aligned; INT16 also K <= 16384. The same bits as the CUDA-core
// kernel.
bool int_mm_tc_supported(int bits, uint32_t M, uint32_t K, uint32_t N, const void* a, size_t lda, const void* b,
                         size_t ldb);
cudaError_t launch_int_mm_tc(int bits, uint32_t M, uint32_t K, uint32_t N, const void* a, size_t lda, const void* b,
                             size_t ldb, void* c, size_t ldc, uint32_t shift, cudaStream_t s);
// The INT8 multiply with its tiles copied by the Tensor Memory Accelerator
// (int_mm_tma.cu); cudaErrorNotSupported where its address and stride rules
// (16-byte aligned, non-overlapping rows) do not hold.
cudaError_t launch_int8_mm_tma(uint32_t M, uint32_t K, uint32_t N, const void* a, size_t lda, const void* b,
                               size_t ldb, void* c, size_t ldc, uint32_t shift, cudaStream_t s);
// The INT16 multiply with its raw tiles copied by the Tensor Memory
// Accelerator and converted to byte limbs in shared memory (K <= 16384).
cudaError_t launch_int16_mm_tma(uint32_t M, uint32_t K, uint32_t N, const void* a, size_t lda, const void* b,
                                size_t ldb, void* c, size_t ldc, uint32_t shift, cudaStream_t s);
// Whether the integer products use the tensor cores when they can (default
// on; the CUDA-core kernels give the same bits).
void int_set_tensor_cores(bool on);
bool int_tensor_cores();

// The LINALG matrix multiply C = round_shift(A B), A M x K, B K x N, C M x N,
// row strides in elements, bits 8 (int32 sums), 16 (int64) or 32 (128-bit)
// (src/linalg_c7xmma/FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX/..._cn.cpp:27-62).
// C must not overlap A or B.
cudaError_t int_matmul_launch(int bits, uint32_t M, uint32_t K, uint32_t N, const void* a, size_t lda, const void* b,
                              size_t ldb, void* c, size_t ldc, uint32_t shift, cudaStream_t s);

} // namespace fftb200
