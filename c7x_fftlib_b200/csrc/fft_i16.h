// fft_i16.h -- launcher of the bit-exact int16 FFT kernel (internal).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fftb200 {

// Number of radix-4 stages (= shift-vector entries read) for length n.
uint32_t i16_num_shifts(uint32_t n);

// x, y: batch x n interleaved int16 complex; w: the caller's Q15 radix-4
// table (2n int16); shifts: i16_num_shifts(n) entries. All device pointers.
// n must be a power of two, 1 <= n <= 16384.
cudaError_t launch_fft_i16(const int16_t* x, int16_t* y, const int16_t* w, const uint32_t* shifts,
                           uint32_t n, uint32_t batch, cudaStream_t s);

} // namespace fftb200
