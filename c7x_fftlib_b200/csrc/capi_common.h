// capi_common.h -- shared helpers of the exported C ABI (internal).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <vector>

#include "FFTLIB_types.h"

namespace fftb200 {

struct ComplexPlan;

// Plan record kept at the start of the caller's pBlock by every _init.
constexpr uint32_t kRecordMagic = 0x42323030u; // "B200"
enum RecordKind : uint32_t {
    REC_C2C = 1, REC_IFFT = 2, REC_R2C = 3, REC_C2R = 4, REC_I16 = 5,  // batched kernels
    REC_1D_C2C = 6, REC_1D_IFFT = 7, REC_1D_R2C = 8, REC_1D_C2R = 9, REC_1D_I16 = 10,  // single-transform kernels
};

struct PlanRecord {
    uint32_t magic;
    uint32_t kind;
    uint32_t numPoints;
    uint32_t numChannels;
    uint32_t mode;       // r2c outmode / c2r inMode
    int32_t  device;
    ComplexPlan* plan;   // FP32 kinds
    uint32_t i16Tg;      // int16: threads per transform (0: the launcher's default)
    uint32_t i16GridCap; //   and CTA cap (0: all resident)
    uint32_t i16MinBlocks; // and register budget (CTAs per SM; 0: the default)
    uint32_t i16Tuned;   //   nonzero when the autotuner chose them
};
static_assert(sizeof(PlanRecord) <= 64, "plan record must fit the smallest pBlock");

// Thread-local description of the last failure, for FFTLIB_b200_lastError.
void set_error(const char* fmt, ...);
const char* last_error();

// FFTLIB status for a CUDA error (FFTLIB_ERR_FAILURE, message recorded).
FFTLIB_STATUS cuda_fail(cudaError_t e, const char* what);

// True if the device can address p as device (or managed) memory.
bool is_device_ptr(const void* p);

// Restores the current device on scope exit.
struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int dev);
    ~DeviceScope();
};

// One buffer argument of a batched call: per-channel byte size, direction,
// and where it lives.
struct ChannelBuf {
    void* ptr;
    size_t perChannel;
    bool input;
    bool output;
};

// Runs fn over the channels, giving it device pointers for each buffer.
// Buffers already in device memory are passed through (offset per chunk);
// host buffers are staged through pooled device memory in chunks on two
// streams, so host->device copy, compute and device->host copy of
// consecutive chunks overlap. Returns after all work completed.
using ChunkFn = std::function<cudaError_t(const std::vector<void*>& dptr, uint32_t c0, uint32_t count,
                                          cudaStream_t s)>;
cudaError_t run_channels(std::vector<ChannelBuf>& bufs, uint32_t channels, const ChunkFn& fn);

// Device copy of a small host table (twiddles, shift vector), copied
// synchronously and valid until the next call on this thread with the same
// slot (0 <= slot < kTableSlots); device pointers are returned unchanged.
constexpr int kTableSlots = 4;
cudaError_t device_table(const void* p, size_t bytes, int slot, const void** out);

} // namespace fftb200
