// capi_exec.h -- plan records and execution helpers shared by the exported
// FFTLIB entry points (internal to libfftlib_b200.so; defined in
// capi_fft_c7x.cu).
//
// Every helper accepts device or host buffers (host buffers are staged
// through pooled device memory by run_channels) and returns after the result
// is in the output buffer.
#pragma once

#include <stdint.h>

#include "capi_common.h"

namespace fftb200 {

// Writes the plan record of an _init into the caller's pBlock.
FFTLIB_STATUS write_record(void* pBlock, uint32_t kind, uint32_t n, uint32_t c, uint32_t mode, ComplexPlan* plan);
// Checks that pBlock holds a record of `kind` for length n; copies it out.
FFTLIB_STATUS read_record(void* pBlock, uint32_t kind, uint32_t n, PlanRecord* out);

// FP32 complex transforms of c channels of n points (inverse: scaled 1/n).
// plan may be null (looked up in the plan cache).
FFTLIB_STATUS exec_c2c(float* pX, float* pY, uint32_t n, uint32_t c, bool inverse, ComplexPlan* plan);
// FP32 real-input forward / real-output inverse over c channels of n reals
// (outmode / inmode 0: n/2+1 bins per channel, 1: n bins). pXFFT is the
// work buffer the global-pass lengths (n/2 > kMaxSingleN) need.
FFTLIB_STATUS exec_r2c(float* pX, float* pXFFT, float* pY, uint32_t n, uint32_t c, int outmode, ComplexPlan* plan);
FFTLIB_STATUS exec_c2r(float* pX, float* pXFFT, float* pY, uint32_t n, uint32_t c, int inmode, ComplexPlan* plan);
// int16 radix-4 transform with per-stage shifts (pW: the Q15 table of n).
// tg, gridCap, minBlocks: the int16 launch shape (0, 0, 3: the launcher's
// defaults).
FFTLIB_STATUS exec_i16(int16_t* pX, const int16_t* pW, int16_t* pY, const uint32_t* pShift, uint32_t numShifts,
                       uint32_t n, uint32_t c, uint32_t tg = 0, uint32_t gridCap = 0, uint32_t minBlocks = 3);

// Builds (or finds) the FP32 plan of an _init and records it in pBlock;
// real kinds plan the n/2-point complex transform with the split tables.
FFTLIB_STATUS init_fp32(void* pBlock, uint32_t kind, uint32_t n, uint32_t c, uint32_t mode, bool real);

} // namespace fftb200
