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

#include <mutex>

#include "capi_common.h"
#include "fft_engine.h"
#include "fftlib_b200_ext.h"
#include "plan.h"

using namespace fftb200;

namespace {

// Scratch: 256 bytes of control words (word 0: error word of the pipelined
// kernel's bounded waits), then the per-pass twiddle table of the transform.
constexpr uint32_t kNoAllocControl = 32;                        // float2 slots (256 bytes)
constexpr uint32_t kNoAllocScratch = kNoAllocControl + 32768;   // float2 slots (256 KiB + 256 B)

static __device__ __align__(256) float2 g_noalloc_scratch[kNoAllocScratch];

// Device address of g_noalloc_scratch per device. In host code the symbol
// name is only a host-side stand-in: the address must come from
// cudaGetSymbolAddress with the device current.
float2* scratch_address(int dev, cudaError_t* err)
{
    static std::mutex mu;
    static float2* addr[64] = {};
    *err = cudaSuccess;
    if (dev < 0 || dev >= 64) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        *err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (*err != cudaSuccess) return nullptr;
        addr[dev] = (float2*)p;
    }
    return addr[dev];
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
    const TwiddlePasses tp = pass_layout(e);
    if (tp.total > kNoAllocScratch - kNoAllocControl) {
        set_error("numPoints %u needs %u twiddles, more than the %u the scratch array holds", numPoints, tp.total,
                  kNoAllocScratch - kNoAllocControl);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    if (!is_device_ptr(pX) || !is_device_ptr(pY)) {
        set_error("pX and pY must be device buffers (host buffers would need staging memory)");
        return FFTLIB_ERR_INVALID_VALUE;
    }
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return cuda_fail(err, "cudaGetDevice");
    float2* scratch = scratch_address(dev, &err);
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
