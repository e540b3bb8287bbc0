// tc_dft.h -- split-precision tensor-core DFT (internal host API).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace fftb200 {

// Lengths with a tensor-core kernel: 8..64 as one DFT-GEMM, 128..4096
// (powers of two) as two DFT-GEMM stages with the twiddle fused between.
bool tc_dft_supported(uint32_t n);
// n = n1 * n2 (n2 == 1: one stage).
void tc_dft_factors(uint32_t n, uint32_t* n1, uint32_t* n2);

// FP32 computational matrix of the tensor-core path, in floats:
//   one stage:  the real embedding of the n-point DFT, (2n)^2 floats,
//               wr[(2j+c') * 2n + 2k+c] with [cos, -sin | sin, cos] blocks;
//   two stages: the n1- and n2-point embeddings, then n complex twiddles
//               W_n^j = (cos, -sin)(2 pi j / n), j < n.
size_t tc_dft_w_floats(uint32_t n);
// Generate it in FP64 with the angle reduced exactly (j k mod n), then
// round to FP32: on the device (w in device memory) or on the host.
cudaError_t tc_dft_gen_w_device(float* w, uint32_t n, cudaStream_t s);
void tc_dft_gen_w_host(float* w, uint32_t n);

// y[b] = DFT_n(x[b]) for b < batch, interleaved complex FP32, device
// pointers; w as above (device). err: error word (kErrTcTimeout on a wait
// that gave up).
cudaError_t launch_tc_dft(uint32_t n, const float2* x, float2* y, const float* w, uint32_t batch, uint32_t* err,
                          cudaStream_t s);

// Per-size launchers (tc_dft_one.cu / tc_dft_two.cu).
cudaError_t launch_tc_one(uint32_t n, const float2* x, float2* y, const float* w, uint32_t batch, uint32_t* err,
                          cudaStream_t s);
cudaError_t launch_tc_two(uint32_t n, const float2* x, float2* y, const float* w, uint32_t batch, uint32_t* err,
                          cudaStream_t s);

} // namespace fftb200
