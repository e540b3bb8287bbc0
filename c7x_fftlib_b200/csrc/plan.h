// plan.h -- planning, plan cache and device launch sequences of the FP32
// FFT kernels (internal to libfftlib_b200.so).
//
// A ComplexPlan describes one complex transform length n on one device:
// either a single-kernel Stockham schedule (n <= kMaxSingleN) or G global
// Stockham passes (one kernel each, every kernel a batch of R-point
// sub-transforms over strided columns with the pass twiddle fused into its
// loads). Its twiddle tables are generated once on the device in FP64 and
// stay resident in HBM.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "fft_args.h"

namespace fftb200 {

constexpr uint32_t kMaxSingleN = 16384;

struct EnginePlan {
    uint32_t n = 0;
    int emax = 0;        // register capacity of the engine instantiation
    uint32_t T = 0;      // threads per transform
    int P = 0;           // passes
    int R[kMaxPasses] = {};
    double score = 0.0;  // heuristic cost (lower is better)
};

bool is_235(uint32_t n);

// All feasible single-kernel schedules for n, best heuristic first
// (emaxOnly: restrict to one engine width; maxT: cap threads per transform).
std::vector<EnginePlan> engine_candidates(uint32_t n, int emaxOnly = 0, uint32_t maxT = 0);
bool plan_engine(uint32_t n, EnginePlan* out);

// Per-pass twiddle blocks of a schedule, allocated and filled on the device.
cudaError_t make_pass_table(float2** p, const EnginePlan& e, cudaStream_t s);

// Autotuner of the mixed-length kernel's schedules: times the heuristic's
// best candidates for (n, batch) and returns the fastest; results are cached
// per device, length, batch bucket and width constraints in memory and in a
// text file ($FFTLIB_B200_TUNE_CACHE, default $HOME/.cache/fftlib_b200_tune.txt).
// timer(e, x, y, batch, stream, &ok): average milliseconds of one launch of
// schedule e over `batch` transforms x -> y; the default times launch_fft.
using ScheduleTimer = float (*)(const EnginePlan&, float2*, float2*, uint32_t, cudaStream_t, bool*);
bool tune_schedule(uint32_t n, uint32_t batch, int emaxOnly, uint32_t maxT, EnginePlan* out,
                   ScheduleTimer timer = nullptr);
// True when $FFTLIB_B200_AUTOTUNE is set to a non-zero value.
bool autotune_enabled();
// Batch bucket of the tuning keys: the power of four at or above batch.
uint32_t tune_bucket(uint32_t batch);

// Transform kinds of the batched entry points, as tuning keys see them.
enum TuneKind : int { TUNE_C2C = 0, TUNE_IFFT = 1, TUNE_R2C = 2, TUNE_C2R = 3 };

// What the batched-path autotuner picks for one FP32 call shape: a radix
// schedule (its threads per transform included), transforms per CTA for the
// one-tile-per-CTA kernels (tileM, 0: the planner's), and for a fixed-size
// schedule whether its persistent pipelined kernel runs (noPipe false) and
// with how many CTAs (gridCap, 0: all that are resident).
struct BatchedChoice {
    EnginePlan eng;
    uint32_t gridCap = 0;
    uint32_t tileM = 0;
    bool noPipe = false;
};
std::string describe(const EnginePlan& e);
// Global Stockham passes for n > kMaxSingleN: n = R[0] R[1] ... R[G-1],
// each R <= kMaxGlobalRadix a single-kernel length, balanced and ordered so
// that every pass after the first can tile its columns in runs of 8 or more.
constexpr int kMaxGlobal = 4;
constexpr uint32_t kMaxGlobalRadix = 1024;
bool split_global(uint32_t n, int* G, uint32_t* R);

struct ComplexPlan {
    int device = 0;
    int sms = 0;                     // multiprocessors of the device
    uint32_t n = 0;
    EnginePlan eng;                  // single kernel
    float2* tw = nullptr;            //   its per-pass twiddle blocks
    bool multiPass = false;          // global Stockham passes
    int G = 0;
    uint32_t R[kMaxGlobal] = {};     //   their radices (sub-transform lengths)
    EnginePlan engG[kMaxGlobal];     //   the sub-transform schedules
    float2* twG[kMaxGlobal] = {};    //   and their per-pass blocks
    float2* twLo = nullptr;          //   W_n^r, r < 2^twLoBits
    float2* twHi = nullptr;          //   W_n^(2^twLoBits q), q < n / 2^twLoBits
    uint32_t twLoBits = 0;
    float2* twSplit = nullptr;       // W_{2n}^i, i < n (real-input kernels)
    // launch choices of the single kernel (the autotuner's; all 0 otherwise)
    uint32_t gridCap = 0;            //   CTAs of the persistent kernels (0: all resident)
    uint32_t tileM = 0;              //   transforms per CTA of the other kernels (0: planner's)
    bool noPipe = false;             //   one tile per CTA instead of the pipelined kernel
    bool tuned = false;              //   chosen by timing, for one kind and batch bucket
};

// Times the batched-path candidates of length base->n for `kind` (r2c / c2r
// with output / input mode `mode`) over a batch of about `batch` transforms
// through run_c2c / run_r2c / run_c2r, and returns the fastest: from the
// in-memory or on-disk cache when this (device, n, kind, dtype, mode, batch
// bucket) was timed before. base: the planner's plan of that length (its
// twSplit present for the real kinds). False if nothing could be timed.
bool tune_batched(const ComplexPlan* base, int kind, int mode, uint32_t batch, BatchedChoice* out);

// Host-visible error word of the current device (mapped pinned memory):
// kernels with bounded waits write a nonzero code there instead of hanging.
struct ErrorWord {
    volatile uint32_t* host = nullptr;
    uint32_t* dev = nullptr;
};
const ErrorWord& error_word();
// Returns the word's value and clears it.
uint32_t take_device_error();

// Cached per (current device, n). needSplit also creates twSplit.
// Returns nullptr (and sets *err) if n is not 2^a 3^b 5^c or on CUDA errors.
ComplexPlan* get_complex_plan(uint32_t n, bool needSplit, cudaError_t* err);
// Plan of a batched _init: get_complex_plan's, or with $FFTLIB_B200_AUTOTUNE
// set and n a single-kernel length, a plan with the autotuner's choice for
// (kind, mode, batch) (shared by every call shape that tunes to the same
// choice; the planner's when timing fails). Untuned r2c / c2r calls take a
// registered schedule of the same length whose pipelined kernel splits in
// registers when the planner's does not.
ComplexPlan* get_batched_plan(uint32_t n, bool needSplit, int kind, int mode, uint32_t batch, cudaError_t* err);
// "tuned" / "planner" plus the schedule and launch choices of p.
std::string describe_plan(const ComplexPlan* p);
void release_all_plans();

// Pick transforms-per-CTA and the staged-I/O mode for a launch.
void finalize_launch(FftArgs& a, const EnginePlan& e, bool contiguousIn, bool contiguousOut);
FftArgs engine_args(const EnginePlan& e, const float2* tw);

// Launch sequences (device pointers, stream s, no synchronization).
// run_c2c may overwrite `in` (work buffer of the passes when G > 2).
// gridCap: at most that many CTAs for the persistent kernels (0: all resident).
// overlapPrev: the launch may start while the stream's previous kernel runs
// (see FftArgs::overlapPrev; the caller guarantees that they are independent).
cudaError_t run_c2c(const ComplexPlan* p, float2* in, float2* out, uint32_t batch, bool inverse,
                    cudaStream_t s, uint32_t gridCap = 0, bool overlapPrev = false);
// h = p->n = numPoints / 2; x: batch x 2h reals; scratch: batch x h complex
// (needed only for global passes); y: batch x (h+1) or x 2h bins.
cudaError_t run_r2c(const ComplexPlan* p, float* x, float2* scratch, float2* y, uint32_t batch, int outmode,
                    cudaStream_t s);
// x: batch x (h+1) or x 2h bins; y: batch x 2h reals. scratch (batch x h
// complex) is needed when c2r_needs_scratch says so.
bool c2r_needs_scratch(const ComplexPlan* p, int inmode);
cudaError_t run_c2r(const ComplexPlan* p, const float2* x, float2* scratch, float* y, uint32_t batch,
                    int inmode, cudaStream_t s);

} // namespace fftb200
