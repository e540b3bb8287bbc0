// fft_engine.h -- host-side entry points of the device kernels (internal to
// libfftlib_b200.so; the exported C ABI lives in capi_*.cpp).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "fft_args.h"

namespace fftb200 {

// Largest CTA size the engine instantiation with register capacity emax
// (complex values per thread) accepts; 0 if emax is not instantiated.
int engine_max_threads(int emax);

// Launch the FP32 Stockham engine described by a (grid = ceil(batch / M)):
// a fixed-size kernel when one is compiled for exactly this schedule, else
// the runtime-planned engine of width emax.
cudaError_t launch_fft(const FftArgs& a, int emax, cudaStream_t s);

// c2c rows of N contiguous values, one transform per thread (fft_small.cu),
// for the lengths small_fft_length accepts; launch_fft takes this path for
// every launch it fits.
bool small_fft_length(uint32_t n);
bool small_fft_eligible(const FftArgs& a);
cudaError_t launch_fft_small(const FftArgs& a, cudaStream_t s);

// A compiled fixed-size schedule.
struct StaticEntry {
    uint32_t n;
    int emax;
    uint32_t T;
    int P;
    int R[kMaxPasses];
    int maxThreads;
    cudaError_t (*launch)(const FftArgs&, cudaStream_t);
    // persistent bulk-copy pipelined variants (contiguous 16-byte aligned
    // rows), one per transform kind (indexed by IO_C2C, IO_R2C_SPLIT,
    // IO_C2R_SPLIT), or null
    cudaError_t (*launchPipelined[3])(const FftArgs&, cudaStream_t);
    // CTAs per SM of each variant on the current device, or null
    int (*residentPipelined[3])();
    // measured on B200 to beat the planner's heuristic schedule for this
    // length: plan_engine returns it instead
    bool preferred;
    // the pipelined variant splits c2r inputs in its first pass / r2c outputs
    // in its last pass in registers (two butterflies per thread, T = N/R/2)
    bool mirrorFirst;
    bool mirrorLast;
};
const std::vector<StaticEntry>& static_schedules();
// maxThreads of the compiled fixed-size kernel for this schedule, or 0.
int static_max_threads(uint32_t n, int emax, uint32_t T, int P, const int* R);
// CTAs per SM of its persistent pipelined variant on the current device, or
// 0 when the schedule has none.
int static_pipelined_resident(uint32_t n, int emax, uint32_t T, int P, const int* R);

// W[i] = exp(-2 pi i (i stride mod n) / n), i < count, computed in FP64.
cudaError_t launch_twiddle(float2* w, uint32_t n, uint32_t count, cudaStream_t s, uint32_t stride = 1);

// Per-pass twiddle blocks: pass j occupies entries off[j] .. off[j] +
// (R[j]-1)*Ns[j]; entry off + (q-1)*Ns + k = W_{Ns*R}^{q*k}, computed in FP64.
struct TwiddlePasses {
    uint32_t P;
    uint32_t R[kMaxPasses], Ns[kMaxPasses], off[kMaxPasses];
    uint32_t total;
};
cudaError_t launch_twiddle_passes(float2* w, const TwiddlePasses& tp, cudaStream_t s);

} // namespace fftb200
