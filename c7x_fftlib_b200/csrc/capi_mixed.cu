// capi_mixed.cu -- uneven-length FP32 c2c batches in one persistent launch
// (include/fftlib_b200/fftlib_b200_ext.h, FFTLIB_b200_fftMixed_*).
//
// create() groups the transforms by length, chooses a schedule per group
// (heuristic, or timed by the autotuner), builds the device tables (group
// schedules, tiles ordered by cost, per-transform offsets) and the group
// twiddle tables. exec() replays a CUDA graph holding the counter reset and
// the single persistent launch; execPerSize() launches the same kernel once
// per distinct length, for comparison.
#include <string.h>

#include <algorithm>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "capi_common.h"
#include "fft_mixed.h"
#include "fftlib_b200_ext.h"
#include "plan.h"

using namespace fftb200;

struct FFTLIB_b200_mixed {
    int device = 0;
    uint32_t count = 0;
    uint32_t flags = 0;
    std::vector<uint32_t> groupN;
    std::vector<EnginePlan> groupPlan;
    std::vector<uint32_t> groupM;
    std::vector<uint32_t> groupTileBegin, groupTileEnd; // ranges in dTilesByGroup
    std::vector<float2*> groupTw;
    MixedGroup* dGroups = nullptr;
    MixedTile* dTiles = nullptr;        // ordered by cost (persistent launch)
    MixedTile* dTilesByGroup = nullptr; // grouped (per-size launches)
    uint64_t* dOffsets = nullptr;
    uint32_t* dCounter = nullptr;
    uint32_t numTiles = 0;
    size_t smem = 0;
    uint32_t grid = 0;
    cudaStream_t capture = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* gx = nullptr;
    void* gy = nullptr;
};

namespace {

constexpr uint32_t kMixedMaxT = 256;

FftArgs group_args(const EnginePlan& e, const float2* tw, bool inverse)
{
    FftArgs a = engine_args(e, tw);
    a.inElem = a.outElem = 1; // rows are addressed through the offsets table
    a.conjIn = a.conjOut = inverse ? 1 : 0;
    a.scale = inverse ? 1.0f / (float)e.n : 1.0f;
    uint32_t M = std::max(1u, (uint32_t)mixed_block() / e.T);
    M = std::min(M, std::max(1u, (48u * 1024u) / (a.slen * 8u)));
    a.M = M;
    return a;
}

// Autotuner timer: one group of `batch` contiguous transforms through the
// mixed-batch kernel itself.
float time_mixed_group(const EnginePlan& e, float2* x, float2* y, uint32_t batch, cudaStream_t s, bool* ok)
{
    *ok = false;
    float2* tw = nullptr;
    MixedGroup* dg = nullptr;
    MixedTile* dt = nullptr;
    uint64_t* doff = nullptr;
    uint32_t* cnt = nullptr;
    float ms = 0.f;
    cudaError_t err = make_pass_table(&tw, e, s);
    const FftArgs a = group_args(e, tw, false);
    std::vector<MixedTile> tiles;
    for (uint32_t b = 0; b < batch; b += a.M) tiles.push_back(MixedTile{0, b, std::min(a.M, batch - b), 0});
    std::vector<uint64_t> offs(batch);
    for (uint32_t i = 0; i < batch; ++i) offs[i] = (uint64_t)i * e.n;
    const MixedGroup g{a};
    if (err == cudaSuccess) err = cudaMalloc(&dg, sizeof(g));
    if (err == cudaSuccess) err = cudaMalloc(&dt, tiles.size() * sizeof(MixedTile));
    if (err == cudaSuccess) err = cudaMalloc(&doff, offs.size() * sizeof(uint64_t));
    if (err == cudaSuccess) err = cudaMalloc(&cnt, sizeof(uint32_t));
    if (err == cudaSuccess) err = cudaMemcpy(dg, &g, sizeof(g), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(dt, tiles.data(), tiles.size() * sizeof(MixedTile), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(doff, offs.data(), offs.size() * sizeof(uint64_t), cudaMemcpyHostToDevice);
    int resident = 0, sms = 0;
    const size_t smem = (size_t)a.M * a.slen * 8u;
    int dev = 0;
    if (err == cudaSuccess) err = cudaGetDevice(&dev);
    if (err == cudaSuccess) err = mixed_configure(smem, &resident);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (err == cudaSuccess) {
        MixedLaunch L{};
        L.groups = dg;
        L.tiles = dt;
        L.numTiles = (uint32_t)tiles.size();
        L.offsets = doff;
        L.x = x;
        L.y = y;
        L.counter = cnt;
        L.grid = std::min<uint32_t>(L.numTiles, (uint32_t)std::max(1, resident * sms));
        L.smem = smem;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        err = launch_mixed(L, s);
        cudaEventRecord(e0, s);
        for (int r = 0; r < 5 && err == cudaSuccess; ++r) err = launch_mixed(L, s);
        cudaEventRecord(e1, s);
        if (err == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess) {
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= 5.f;
            *ok = true;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    if (err != cudaSuccess) cudaGetLastError();
    cudaStreamSynchronize(s);
    cudaFree(tw);
    cudaFree(dg);
    cudaFree(dt);
    cudaFree(doff);
    cudaFree(cnt);
    return ms;
}

bool mixed_schedule(uint32_t n, uint32_t batch, bool tune, EnginePlan* e)
{
    if (!is_235(n) || n > kMaxSingleN) return false;
    if (tune && tune_schedule(n, batch, mixed_emax(), kMixedMaxT, e, &time_mixed_group)) return true;
    std::vector<EnginePlan> c = engine_candidates(n, mixed_emax(), kMixedMaxT);
    if (c.empty()) return false;
    *e = c.front();
    return true;
}

void release(FFTLIB_b200_mixed* h)
{
    if (!h) return;
    DeviceScope scope(h->device);
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    if (h->capture) cudaStreamDestroy(h->capture);
    for (float2* t : h->groupTw) cudaFree(t);
    cudaFree(h->dGroups);
    cudaFree(h->dTiles);
    cudaFree(h->dTilesByGroup);
    cudaFree(h->dOffsets);
    cudaFree(h->dCounter);
    delete h;
}

MixedLaunch launch_desc(const FFTLIB_b200_mixed* h, const MixedTile* tiles, uint32_t numTiles, const float* x,
                        float* y)
{
    MixedLaunch L{};
    L.groups = h->dGroups;
    L.tiles = tiles;
    L.numTiles = numTiles;
    L.offsets = h->dOffsets;
    L.x = (const float2*)x;
    L.y = (float2*)y;
    L.counter = h->dCounter;
    L.grid = std::min(h->grid, numTiles);
    L.smem = h->smem;
    return L;
}

} // namespace

extern "C" {

FFTLIB_STATUS FFTLIB_b200_fftMixed_supported(uint32_t numPoints)
{
    EnginePlan e;
    return mixed_schedule(numPoints, 1, false, &e) ? FFTLIB_SUCCESS : FFTLIB_ERR_INVALID_DIMENSION;
}

FFTLIB_STATUS FFTLIB_b200_fftMixed_create(const uint32_t* numPoints, uint32_t count, uint32_t flags,
                                          FFTLIB_b200_mixedHandle* handle)
{
    if (!numPoints || !handle) return FFTLIB_ERR_NULL_POINTER;
    *handle = nullptr;
    const bool inverse = flags & FFTLIB_B200_MIXED_INVERSE;
    const bool tune = (flags & FFTLIB_B200_MIXED_AUTOTUNE) || autotune_enabled();
    // group the transforms by length, largest first
    std::map<uint32_t, std::vector<uint32_t>, std::greater<uint32_t>> byN;
    std::vector<uint64_t> offset(count);
    uint64_t off = 0;
    for (uint32_t i = 0; i < count; ++i) {
        byN[numPoints[i]].push_back(i);
        offset[i] = off;
        off += numPoints[i];
    }
    FFTLIB_b200_mixed* h = new FFTLIB_b200_mixed();
    h->count = count;
    h->flags = flags;
    cudaGetDevice(&h->device);
    std::vector<MixedGroup> groups;
    std::vector<MixedTile> tiles;
    std::vector<uint64_t> offsByGroup;
    cudaStream_t s = cudaStreamPerThread;
    for (auto& kv : byN) {
        const uint32_t n = kv.first;
        EnginePlan e;
        if (!mixed_schedule(n, (uint32_t)kv.second.size(), tune, &e)) {
            set_error("length %u is not 2^a 3^b 5^c up to %u threads per transform", n, kMixedMaxT);
            release(h);
            return FFTLIB_ERR_INVALID_DIMENSION;
        }
        float2* tw = nullptr;
        cudaError_t err = make_pass_table(&tw, e, s);
        if (err != cudaSuccess) {
            release(h);
            return cuda_fail(err, "mixed twiddle tables");
        }
        h->groupTw.push_back(tw);
        const FftArgs a = group_args(e, tw, inverse);
        const uint32_t M = a.M;
        h->smem = std::max(h->smem, (size_t)M * a.slen * 8u);
        const uint32_t g = (uint32_t)groups.size();
        groups.push_back(MixedGroup{a});
        h->groupN.push_back(n);
        h->groupPlan.push_back(e);
        h->groupM.push_back(M);
        h->groupTileBegin.push_back((uint32_t)tiles.size());
        const uint32_t first = (uint32_t)offsByGroup.size();
        for (uint32_t i : kv.second) offsByGroup.push_back(offset[i]);
        const uint32_t cnt = (uint32_t)kv.second.size();
        for (uint32_t b = 0; b < cnt; b += M) tiles.push_back(MixedTile{g, first + b, std::min(M, cnt - b), 0});
        h->groupTileEnd.push_back((uint32_t)tiles.size());
    }
    h->numTiles = (uint32_t)tiles.size();
    // persistent order: most expensive tiles first (groups are already in
    // decreasing length; within a group full tiles first)
    std::vector<MixedTile> lpt = tiles;
    std::stable_sort(lpt.begin(), lpt.end(), [&](const MixedTile& a, const MixedTile& b) {
        const double ca = (double)h->groupN[a.group] * a.count, cb = (double)h->groupN[b.group] * b.count;
        return ca > cb;
    });
    cudaError_t err = cudaSuccess;
    auto upload = [&](void** dst, const void* src, size_t bytes) {
        if (err != cudaSuccess) return;
        err = cudaMalloc(dst, std::max<size_t>(bytes, 16));
        if (err == cudaSuccess && bytes) err = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
    };
    upload((void**)&h->dGroups, groups.data(), groups.size() * sizeof(MixedGroup));
    upload((void**)&h->dTiles, lpt.data(), lpt.size() * sizeof(MixedTile));
    upload((void**)&h->dTilesByGroup, tiles.data(), tiles.size() * sizeof(MixedTile));
    upload((void**)&h->dOffsets, offsByGroup.data(), offsByGroup.size() * sizeof(uint64_t));
    if (err == cudaSuccess) err = cudaMalloc(&h->dCounter, sizeof(uint32_t));
    int resident = 0, sms = 0;
    if (err == cudaSuccess) err = mixed_configure(h->smem, &resident);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&h->capture, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) {
        release(h);
        return cuda_fail(err, "mixed plan");
    }
    h->grid = (uint32_t)std::max(1, resident * sms);
    *handle = h;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_b200_fftMixed_exec(FFTLIB_b200_mixedHandle h, const FFTLIB_F32* pX, FFTLIB_F32* pY,
                                        void* stream)
{
    if (!h || !pX || !pY) return FFTLIB_ERR_NULL_POINTER;
    if (h->numTiles == 0) return FFTLIB_SUCCESS;
    DeviceScope scope(h->device);
    cudaError_t err = cudaSuccess;
    if (!h->exec || h->gx != pX || h->gy != pY) {
        // capture the counter reset and the persistent launch for these buffers
        if (h->exec) cudaGraphExecDestroy(h->exec);
        if (h->graph) cudaGraphDestroy(h->graph);
        h->exec = nullptr;
        h->graph = nullptr;
        err = cudaStreamBeginCapture(h->capture, cudaStreamCaptureModeThreadLocal);
        if (err == cudaSuccess) {
            cudaError_t le = launch_mixed(launch_desc(h, h->dTiles, h->numTiles, pX, pY), h->capture);
            err = cudaStreamEndCapture(h->capture, &h->graph);
            if (err == cudaSuccess) err = le;
        }
        if (err == cudaSuccess) err = cudaGraphInstantiate(&h->exec, h->graph, 0);
        if (err != cudaSuccess) return cuda_fail(err, "mixed graph capture");
        h->gx = pX;
        h->gy = pY;
    }
    err = cudaGraphLaunch(h->exec, (cudaStream_t)stream);
    return err == cudaSuccess ? FFTLIB_SUCCESS : cuda_fail(err, "mixed graph launch");
}

FFTLIB_STATUS FFTLIB_b200_fftMixed_execPerSize(FFTLIB_b200_mixedHandle h, const FFTLIB_F32* pX, FFTLIB_F32* pY,
                                               void* stream)
{
    if (!h || !pX || !pY) return FFTLIB_ERR_NULL_POINTER;
    DeviceScope scope(h->device);
    for (size_t g = 0; g < h->groupN.size(); ++g) {
        const uint32_t b = h->groupTileBegin[g], e = h->groupTileEnd[g];
        cudaError_t err = launch_mixed(launch_desc(h, h->dTilesByGroup + b, e - b, pX, pY), (cudaStream_t)stream);
        if (err != cudaSuccess) return cuda_fail(err, "mixed per-size launch");
    }
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_b200_fftMixed_describe(FFTLIB_b200_mixedHandle h, char* buf, uint32_t len)
{
    if (!h || !buf || len == 0) return FFTLIB_ERR_NULL_POINTER;
    std::ostringstream os;
    os << h->count << " transforms, " << h->groupN.size() << " lengths, " << h->numTiles << " tiles, grid "
       << h->grid << ", smem " << h->smem;
    for (size_t g = 0; g < h->groupN.size(); ++g)
        os << "; " << describe(h->groupPlan[g]) << " M=" << h->groupM[g] << " tiles="
           << (h->groupTileEnd[g] - h->groupTileBegin[g]);
    const std::string s = os.str();
    strncpy(buf, s.c_str(), len - 1);
    buf[len - 1] = '\0';
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_b200_fftMixed_destroy(FFTLIB_b200_mixedHandle h)
{
    release(h);
    return FFTLIB_SUCCESS;
}

} // extern "C"
