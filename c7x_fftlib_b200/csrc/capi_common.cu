// capi_common.cu -- error reporting, pointer classification and host-buffer
// staging for the exported C ABI.
#include "capi_common.h"
#include "plan.h"

#include <stdarg.h>
#include <stdio.h>

#include <algorithm>
#include <mutex>
#include <string>

namespace fftb200 {

namespace {
thread_local char t_error[512];
constexpr size_t kChunkBytes = 32u << 20; // staged bytes per chunk (all host buffers)
constexpr size_t kAlign = 256;
// Staging slots, each with its own stream running copy-in, compute and
// copy-out of one chunk: with three, the host-to-device copy of chunk k + 2
// never waits for the device-to-host copy of chunk k (one slot would be the
// copy-out's, one the compute's, one the copy-in's), so both copy directions
// stream back to back.
constexpr int kSlots = 3;

size_t round_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

struct Staging {
    std::mutex mu;
    void* buf[kSlots] = {};
    size_t cap[kSlots] = {};
    cudaStream_t st[kSlots] = {};
};

Staging* staging_for(int dev)
{
    static std::mutex mu;
    static Staging* pools[64] = {};
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[dev]) pools[dev] = new Staging();
    return pools[dev];
}

cudaError_t ensure(Staging& S, int slot, size_t bytes)
{
    if (!S.st[slot]) {
        cudaError_t e = cudaStreamCreateWithFlags(&S.st[slot], cudaStreamNonBlocking);
        if (e != cudaSuccess) return e;
    }
    if (S.cap[slot] >= bytes) return cudaSuccess;
    if (S.buf[slot]) {
        cudaStreamSynchronize(S.st[slot]);
        cudaFree(S.buf[slot]);
        S.buf[slot] = nullptr;
        S.cap[slot] = 0;
    }
    cudaError_t e = cudaMalloc(&S.buf[slot], bytes);
    if (e == cudaSuccess) S.cap[slot] = bytes;
    return e;
}
} // namespace

void set_error(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_error, sizeof(t_error), fmt, ap);
    va_end(ap);
}

const char* last_error() { return t_error; }

FFTLIB_STATUS cuda_fail(cudaError_t e, const char* what)
{
    set_error("%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
    return FFTLIB_ERR_FAILURE;
}

bool is_device_ptr(const void* p)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

DeviceScope::DeviceScope(int dev)
{
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
}

DeviceScope::~DeviceScope()
{
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
}

cudaError_t run_channels(std::vector<ChannelBuf>& bufs, uint32_t channels, const ChunkFn& fn)
{
    std::vector<bool> dev(bufs.size());
    bool allDev = true;
    size_t perCh = 0;
    for (size_t i = 0; i < bufs.size(); ++i) {
        dev[i] = bufs[i].ptr == nullptr || is_device_ptr(bufs[i].ptr);
        if (!dev[i]) {
            allDev = false;
            perCh += bufs[i].perChannel;
        }
    }
    std::vector<void*> dptr(bufs.size());
    if (allDev) {
        for (size_t i = 0; i < bufs.size(); ++i) dptr[i] = bufs[i].ptr;
        cudaStream_t s = cudaStreamPerThread;
        cudaError_t e = fn(dptr, 0, channels, s);
        if (e != cudaSuccess) return e;
        e = cudaStreamSynchronize(s);
        if (e == cudaSuccess && take_device_error()) return cudaErrorLaunchTimeout;
        return e;
    }
    int devId = 0;
    cudaError_t e = cudaGetDevice(&devId);
    if (e != cudaSuccess) return e;
    Staging* S = staging_for(devId);
    if (!S) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(S->mu);

    const uint32_t chunk = (uint32_t)std::max<size_t>(1, std::min<size_t>(channels, kChunkBytes / std::max<size_t>(perCh, 1)));
    size_t slotBytes = 0;
    for (size_t i = 0; i < bufs.size(); ++i)
        if (!dev[i]) slotBytes += round_up(bufs[i].perChannel * chunk);
    const uint32_t chunks = (channels + chunk - 1u) / chunk;
    const int slots = (int)std::min<uint32_t>((uint32_t)kSlots, chunks);
    for (int s = 0; s < slots; ++s)
        if ((e = ensure(*S, s, slotBytes)) != cudaSuccess) return e;

    for (uint32_t c0 = 0, it = 0; c0 < channels; c0 += chunk, ++it) {
        const int slot = (int)(it % (uint32_t)slots);
        cudaStream_t st = S->st[slot];
        const uint32_t cc = std::min(chunk, channels - c0);
        char* base = (char*)S->buf[slot];
        size_t off = 0;
        for (size_t i = 0; i < bufs.size(); ++i) {
            char* host = (char*)bufs[i].ptr;
            if (dev[i]) {
                dptr[i] = host ? host + (size_t)c0 * bufs[i].perChannel : nullptr;
                continue;
            }
            dptr[i] = base + off;
            off += round_up(bufs[i].perChannel * chunk);
            if (bufs[i].input) {
                e = cudaMemcpyAsync(dptr[i], host + (size_t)c0 * bufs[i].perChannel, (size_t)cc * bufs[i].perChannel,
                                    cudaMemcpyHostToDevice, st);
                if (e != cudaSuccess) return e;
            }
        }
        if ((e = fn(dptr, c0, cc, st)) != cudaSuccess) return e;
        for (size_t i = 0; i < bufs.size(); ++i) {
            if (dev[i] || !bufs[i].output) continue;
            e = cudaMemcpyAsync((char*)bufs[i].ptr + (size_t)c0 * bufs[i].perChannel, dptr[i],
                                (size_t)cc * bufs[i].perChannel, cudaMemcpyDeviceToHost, st);
            if (e != cudaSuccess) return e;
        }
    }
    cudaError_t first = cudaSuccess;
    for (int s = 0; s < slots; ++s) {
        const cudaError_t es = cudaStreamSynchronize(S->st[s]);
        if (first == cudaSuccess) first = es;
    }
    if (first == cudaSuccess && take_device_error()) return cudaErrorLaunchTimeout;
    return first;
}

cudaError_t device_table(const void* p, size_t bytes, int slot, const void** out)
{
    if (p == nullptr || is_device_ptr(p)) {
        *out = p;
        return cudaSuccess;
    }
    if (slot < 0 || slot >= kTableSlots) return cudaErrorInvalidValue;
    struct Tab {
        void* ptr[kTableSlots] = {};
        size_t cap[kTableSlots] = {};
        int dev = -1;
    };
    thread_local Tab tabs[8];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    Tab& t = tabs[dev & 7];
    if (t.dev != dev) {
        t = Tab();
        t.dev = dev;
    }
    if (t.cap[slot] < bytes) {
        if (t.ptr[slot]) {
            cudaDeviceSynchronize();
            cudaFree(t.ptr[slot]);
        }
        t.ptr[slot] = nullptr;
        t.cap[slot] = 0;
        if ((e = cudaMalloc(&t.ptr[slot], bytes)) != cudaSuccess) return e;
        t.cap[slot] = bytes;
    }
    e = cudaMemcpy(t.ptr[slot], p, bytes, cudaMemcpyHostToDevice);
    // a copy from pageable memory may return before its DMA lands, and the
    // kernel that reads the table may run on a stream that does not wait for
    // the legacy stream
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
    *out = t.ptr[slot];
    return e;
}

} // namespace fftb200
