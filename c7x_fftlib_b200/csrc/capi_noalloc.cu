// capi_noalloc.cu -- an FP32 c2c entry point that allocates no memory.
//
// The regular path (_init/_kernel) allocates device memory: the plan's
// twiddle tables (cudaMalloc), a mapped host error word (cudaHostAlloc) and,
// for host buffers, staging buffers. Some callers cannot allocate at call
// time -- code that runs under a fixed device-memory budget carved out at
// start-up, real-time loops that must not enter the allocator, or
// environments whose allocator is owned by another framework. This entry
// point serves them: its only scratch memory is the file-scope device array
// below, loaded with the module and held by every GPU that loads the library
// until the process exits.
#include <string.h>

#include "capi_common.h"
#include "fft_engine.h"
#include "fftlib_b200_ext.h"
#include "plan.h"

using namespace fftb200;

namespace {

// Scratch: 256 bytes of control words (word 0: error word of the pipelined
// kernel's bounded waits), then the per-pass twiddle table of the transform.
// A single-kernel schedule R[0] x R[1] x ... of N points has per-pass blocks
// of (R[i] - 1) * (R[0] ... R[i-1]) entries for i >= 1, N - R[0] in total, so
// kMaxSingleN slots hold the table of every length the planner accepts.
constexpr uint32_t kNoAllocControl = 32;                              // float2 slots (256 bytes)
constexpr uint32_t kNoAllocTable = kMaxSingleN;                       // float2 slots (128 KiB)
constexpr uint32_t kNoAllocScratch = kNoAllocControl + kNoAllocTable; // 128 KiB + 256 B
static_assert(kNoAllocTable >= kMaxSingleN - 2u, "the table must hold N - R[0] entries for N <= kMaxSingleN");

static __device__ __align__(256) float2 g_noalloc_scratch[kNoAllocScratch];

// Device address of g_noalloc_scratch on the current device. In host code the
// symbol name is only a host-side stand-in: the address comes from
// cudaGetSymbolAddress with the device current. It is looked up on every call
// (no allocation once the module is loaded), so a cudaDeviceReset, which
// reloads the module, never leaves a stale address behind.
float2* scratch_address(cudaError_t* err)
{
    void* p = nullptr;
    *err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    return *err == cudaSuccess ? (float2*)p : nullptr;
}

// Per-pass twiddle block layout of a schedule (the same as the planned path).
TwiddlePasses pass_layout(const EnginePlan& e)
{
    TwiddlePasses tp{};
    uint32_t ns = 1, off = 0;
    for (int i = 0; i < e.P; ++i) {
        const uint32_t r = (uint32_t)e.R[i];
        if (i > 0) {
            tp.R[tp.P] = r;
            tp.Ns[tp.P] = ns;
            tp.off[tp.P] = off;
            tp.P++;
            off += (r - 1u) * ns;
        }
        ns *= r;
    }
    tp.total = off;
    return tp;
}

} // namespace

extern "C" FFTLIB_STATUS FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelNoAlloc(FFTLIB_F32* pX, FFTLIB_F32* pY,
                                                                                  uint32_t numPoints,
                                                                                  uint32_t numChannels, void* stream)
{
    if (!pX || !pY) {
        set_error("pX and pY must be device buffers");
        return FFTLIB_ERR_NULL_POINTER;
    }
    EnginePlan e;
    if (!is_235(numPoints) || !plan_engine(numPoints, &e)) {
        set_error("numPoints %u: the allocation-free entry point takes 2^a 3^b 5^c lengths up to %u", numPoints,
                  kMaxSingleN);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    const TwiddlePasses tp = pass_layout(e);  // tp.total = N - R[0] < kNoAllocTable (static_assert above)
    if (!is_device_ptr(pX) || !is_device_ptr(pY)) {
        set_error("pX and pY must be device buffers (host buffers would need staging memory)");
        return FFTLIB_ERR_INVALID_VALUE;
    }
    cudaError_t err = cudaSuccess;
    float2* scratch = scratch_address(&err);
    if (!scratch) return cuda_fail(err, "cudaGetSymbolAddress");
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t* errWord = (uint32_t*)scratch;
    float2* table = scratch + kNoAllocControl;

    // the error word must start at zero; the table is rebuilt for this length
    if ((err = cudaMemsetAsync(errWord, 0, sizeof(uint32_t), s)) != cudaSuccess) return cuda_fail(err, "memset");
    if ((err = launch_twiddle_passes(table, tp, s)) != cudaSuccess) return cuda_fail(err, "twiddle table");
    FftArgs a = engine_args(e, table);
    a.err = errWord;
    a.in = (const float2*)pX;
    a.out = (float2*)pY;
    a.batch = numChannels;
    a.inBatch = numPoints;
    a.inElem = 1;
    a.outBatch = numPoints;
    a.outElem = 1;
    finalize_launch(a, e, true, true);
    if (numChannels && (err = launch_fft(a, e.emax, s)) != cudaSuccess) return cuda_fail(err, "fft launch");
    if ((err = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(err, "fft1dBatched c2c (no-alloc)");
    uint32_t word = 0;
    if ((err = cudaMemcpy(&word, errWord, sizeof(word), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(err, "error word");
    if (word) {
        set_error("device-side wait timed out (code %u)", word);
        return FFTLIB_ERR_FAILURE;
    }
    return FFTLIB_SUCCESS;
}
