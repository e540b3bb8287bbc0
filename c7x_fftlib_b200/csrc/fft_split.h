// fft_split.h -- stand-alone real-input split passes (internal).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fftb200 {

// y = split post-process of z (batch x h complex) into h+1 (outmode 0) or 2h
// (outmode 1) bins per transform; wsp[i] = W_{2h}^i, i < h.
cudaError_t launch_r2c_post(const float2* z, float2* y, const float2* wsp, uint32_t h, uint32_t batch,
                            int outmode, cudaStream_t s);

// z = split pre-process of x (batch x (h+1) or x 2h bins) into h complex.
cudaError_t launch_c2r_pre(const float2* x, float2* z, const float2* wsp, uint32_t h, uint32_t batch,
                           int inmode, cudaStream_t s);

} // namespace fftb200
