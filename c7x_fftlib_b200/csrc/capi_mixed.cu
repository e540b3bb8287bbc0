// capi_mixed.cu -- uneven-length FP32 c2c batches in one persistent launch
// (include/fftlib_b200/fftlib_b200_ext.h, FFTLIB_b200_fftMixed_*).
//
// create() groups the transforms by length. A group whose transforms lie
// back to back and whose length has a persistent pipelined fixed-size kernel
// (every 2^a 3^b 5^c length from 8 to 4096) is a "fixed group": it runs that
// kernel, the fixed groups' launches back to back, each one starting while its
// predecessor drains (programmatic dependent launch), or spread over up to 8
// graph branches with grids proportional to their shares of the batch. Every
// other group gets a runtime-radix schedule (heuristic, or timed by the
// autotuner) in the persistent mixed kernel (fft_mixed.cu), which walks a
// device-resident tile table ordered by cost. exec() replays a CUDA graph of
// these launches, the persistent kernel's on a branch of its own;
// FFTLIB_B200_MIXED_PERSISTENT_ONLY puts every group in the persistent
// kernel. execPerSize() launches the persistent kernel once per distinct
// length, for comparison.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "capi_common.h"
#include "fft_engine.h"
#include "fft_mixed.h"
#include "fftlib_b200_ext.h"
#include "plan.h"

using namespace fftb200;

struct FFTLIB_b200_mixed {
    int device = 0;
    uint32_t count = 0;
    uint32_t flags = 0;
    std::vector<uint32_t> groupN;
    std::vector<int> groupCls;
    std::vector<EnginePlan> groupPlan;
    std::vector<uint32_t> groupM;
    std::vector<uint32_t> groupCount;
    std::vector<uint32_t> groupTileBegin, groupTileEnd; // ranges in dTilesByGroup
    std::vector<float2*> groupTw;
    MixedGroup* dGroups = nullptr;
    MixedTile* dTiles = nullptr;        // per class, most expensive first (persistent launches)
    MixedTile* dTilesByGroup = nullptr; // grouped (per-size launches)
    uint64_t* dOffsets = nullptr;
    uint32_t numTiles = 0;
    // per class: its tiles in dTiles, stage length, shared memory, grid
    uint32_t clsTileBegin[kMixedClasses] = {}, clsTiles[kMixedClasses] = {};
    uint32_t clsStage[kMixedClasses] = {};
    uint32_t groupStage = 0;            // largest stage of any group (per-size launches)
    uint32_t clsGrid[kMixedClasses] = {};
    uint32_t perSizeGrid[kMixedClasses] = {};  // resident CTAs of each class at groupStage
    // fixed groups: the regular plan's fixed-size kernel on a grid share
    struct Fixed {
        uint32_t n, count;
        uint64_t offset;       // complex elements
        ComplexPlan* plan;
        uint32_t grid;
        uint32_t branch;
    };
    std::vector<Fixed> fixed;           // ordered by branch
    uint64_t fixedPoints = 0;
    uint32_t fixedBranches = 0;
    // the fixed groups' graph branches, then one per class with tiles
    std::vector<cudaStream_t> branches;
    std::vector<cudaEvent_t> joins;
    cudaStream_t capture = nullptr;
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* gx = nullptr;
    void* gy = nullptr;
};

namespace {

constexpr uint32_t kMixedMaxT = 256;

// Transforms per tile: enough to give the CTA its 256 threads, as many as
// one shared-memory stage holds.
FftArgs group_args(const EnginePlan& e, const float2* tw, bool inverse)
{
    FftArgs a = engine_args(e, tw);
    a.inElem = a.outElem = 1; // rows are addressed through the offsets table
    a.conjIn = a.conjOut = inverse ? 1 : 0;
    a.scale = inverse ? 1.0f / (float)e.n : 1.0f;
    a.err = error_word().dev;
    uint32_t M = std::max(1u, mixed_block() / e.T);
    M = std::min(M, std::max(1u, mixed_stage_max_bytes() / (a.slen * 8u)));
    a.M = M;
    return a;
}

// Complex values of the stage a group's tiles need (even: stages start on
// 16-byte boundaries).
uint32_t stage_len(const FftArgs& a) { return (a.M * a.slen + 1u) & ~1u; }

// How a tile of `count` transforms whose offsets start at offs reaches
// shared memory (kTileBulk / kTileRows / plain loads).
uint32_t tile_flags(const uint64_t* offs, uint32_t count, uint32_t n)
{
    bool contiguous = (offs[0] % 2u) == 0 && ((uint64_t)count * n) % 2u == 0;
    bool rows = (n % 2u) == 0;
    for (uint32_t m = 0; m < count; ++m) {
        if (offs[m] != offs[0] + (uint64_t)m * n) contiguous = false;
        if (offs[m] % 2u) rows = false;
    }
    return contiguous ? kTileBulk : rows ? kTileRows : 0u;
}

int class_of(const EnginePlan& e) { return e.emax > 16 ? kMixedW20 : kMixedW16; }

MixedLaunch class_launch(int cls, const MixedGroup* groups, const MixedTile* tiles, uint32_t numTiles,
                         const uint64_t* offsets, const float* x, float* y, uint32_t stageLen, uint32_t grid)
{
    MixedLaunch L{};
    L.cls = cls;
    L.groups = groups;
    L.tiles = tiles;
    L.numTiles = numTiles;
    L.offsets = offsets;
    L.x = (const float2*)x;
    L.y = (float2*)y;
    L.err = error_word().dev;
    L.stageLen = stageLen;
    L.smem = mixed_smem(stageLen);
    L.grid = std::max(1u, std::min(grid, numTiles));
    return L;
}

// Resident CTAs of a class's kernel with this stage length, over the device.
cudaError_t class_grid(int cls, uint32_t stageLen, int device, uint32_t* grid)
{
    int resident = 0, sms = 0;
    cudaError_t err = mixed_configure(cls, mixed_smem(stageLen), &resident);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    *grid = (uint32_t)std::max(1, resident * sms);
    return err;
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
    float ms = 0.f;
    cudaError_t err = make_pass_table(&tw, e, s);
    const FftArgs a = group_args(e, tw, false);
    std::vector<uint64_t> offs(batch);
    for (uint32_t i = 0; i < batch; ++i) offs[i] = (uint64_t)i * e.n;
    std::vector<MixedTile> tiles;
    for (uint32_t b = 0; b < batch; b += a.M) {
        const uint32_t c = std::min(a.M, batch - b);
        tiles.push_back(MixedTile{0, b, c, tile_flags(&offs[b], c, e.n)});
    }
    const MixedGroup g{a};
    const int cls = class_of(e);
    if (err == cudaSuccess) err = cudaMalloc(&dg, sizeof(g));
    if (err == cudaSuccess) err = cudaMalloc(&dt, tiles.size() * sizeof(MixedTile));
    if (err == cudaSuccess) err = cudaMalloc(&doff, offs.size() * sizeof(uint64_t));
    // the descriptors go up on the timing stream itself: a synchronous copy
    // from pageable memory may return before its DMA lands, and this
    // non-blocking stream would not wait for it
    if (err == cudaSuccess) err = cudaMemcpyAsync(dg, &g, sizeof(g), cudaMemcpyHostToDevice, s);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(dt, tiles.data(), tiles.size() * sizeof(MixedTile), cudaMemcpyHostToDevice, s);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(doff, offs.data(), offs.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, s);
    int dev = 0;
    uint32_t grid = 1;
    if (err == cudaSuccess) err = cudaGetDevice(&dev);
    if (err == cudaSuccess) err = class_grid(cls, stage_len(a), dev, &grid);
    if (err == cudaSuccess) {
        const MixedLaunch L = class_launch(cls, dg, dt, (uint32_t)tiles.size(), doff, (const float*)x, (float*)y,
                                           stage_len(a), grid);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        err = launch_mixed(L, s);
        cudaEventRecord(e0, s);
        for (int r = 0; r < 5 && err == cudaSuccess; ++r) err = launch_mixed(L, s);
        cudaEventRecord(e1, s);
        if (err == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess && !take_device_error()) {
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
    return ms;
}

// The group's schedule: the 16-wide class when a schedule of at most 256
// threads per transform exists there, else the 20-wide class.
bool mixed_schedule(uint32_t n, uint32_t batch, bool tune, EnginePlan* e)
{
    if (!is_235(n) || n > kMaxSingleN) return false;
    for (int cls = 0; cls < kMixedClasses; ++cls) {
        const int emax = mixed_class_emax(cls);
        if (tune && tune_schedule(n, batch, emax, kMixedMaxT, e, &time_mixed_group)) return true;
        std::vector<EnginePlan> c = engine_candidates(n, emax, kMixedMaxT);
        if (!c.empty()) {
            *e = c.front();
            return true;
        }
    }
    return false;
}

void release(FFTLIB_b200_mixed* h)
{
    if (!h) return;
    DeviceScope scope(h->device);
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    if (h->capture) cudaStreamDestroy(h->capture);
    for (cudaStream_t b : h->branches) cudaStreamDestroy(b);
    for (cudaEvent_t e : h->joins) cudaEventDestroy(e);
    if (h->fork) cudaEventDestroy(h->fork);
    for (float2* t : h->groupTw) cudaFree(t);
    cudaFree(h->dGroups);
    cudaFree(h->dTiles);
    cudaFree(h->dTilesByGroup);
    cudaFree(h->dOffsets);
    delete h;
}

// Every launch of the batch on its own branch: the fixed groups' kernels
// and the persistent kernel of every class that has tiles, forked from and
// joined back into s.
cudaError_t enqueue_all(FFTLIB_b200_mixed* h, const float* x, float* y, cudaStream_t s)
{
    const bool inverse = h->flags & FFTLIB_B200_MIXED_INVERSE;
    cudaError_t err = cudaEventRecord(h->fork, s);
    for (cudaStream_t b : h->branches)
        if (err == cudaSuccess) err = cudaStreamWaitEvent(b, h->fork, 0);
    // the groups of a branch touch disjoint parts of x and y, so each launch
    // after a branch's first may start while its predecessor drains
    for (size_t i = 0; i < h->fixed.size() && err == cudaSuccess; ++i) {
        const auto& f = h->fixed[i];
        const bool follows = i > 0 && h->fixed[i - 1].branch == f.branch;
        float2* in = const_cast<float2*>(reinterpret_cast<const float2*>(x)) + f.offset;
        err = run_c2c(f.plan, in, reinterpret_cast<float2*>(y) + f.offset, f.count, inverse, h->branches[f.branch],
                      f.grid, follows);
    }
    size_t br = h->fixedBranches;
    for (int cls = kMixedClasses - 1; cls >= 0 && err == cudaSuccess; --cls) {
        if (!h->clsTiles[cls]) continue;
        err = launch_mixed(class_launch(cls, h->dGroups, h->dTiles + h->clsTileBegin[cls], h->clsTiles[cls],
                                        h->dOffsets, x, y, h->clsStage[cls], h->clsGrid[cls]),
                           h->branches[br++]);
    }
    for (size_t b = 0; b < h->branches.size() && err == cudaSuccess; ++b) {
        err = cudaEventRecord(h->joins[b], h->branches[b]);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(s, h->joins[b], 0);
    }
    return err;
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
    std::vector<char> groupFixed;
    cudaStream_t s = cudaStreamPerThread;
    for (auto& kv : byN) {
        const uint32_t n = kv.first;
        // a fixed group: its transforms back to back, its length with a
        // persistent pipelined fixed-size kernel
        // (moving the small groups into the persistent kernel measured slower:
        // on a reduced share it becomes the batch's tail)
        bool isFixed = !(flags & FFTLIB_B200_MIXED_PERSISTENT_ONLY);
        for (size_t k = 0; isFixed && k < kv.second.size(); ++k)
            isFixed = offset[kv.second[k]] == offset[kv.second[0]] + (uint64_t)k * n;
        if (isFixed) {
            cudaError_t perr = cudaSuccess;
            ComplexPlan* cp = get_complex_plan(n, false, &perr);
            isFixed = cp && !cp->multiPass &&
                      static_pipelined_resident(n, cp->eng.emax, cp->eng.T, cp->eng.P, cp->eng.R) > 0;
            if (isFixed)
                h->fixed.push_back(
                    FFTLIB_b200_mixed::Fixed{n, (uint32_t)kv.second.size(), offset[kv.second[0]], cp, 0, 0});
            if (perr != cudaSuccess) cudaGetLastError();
        }
        groupFixed.push_back(isFixed ? 1 : 0);
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
        const int cls = class_of(e);
        h->clsStage[cls] = std::max(h->clsStage[cls], stage_len(a));
        h->groupStage = std::max(h->groupStage, stage_len(a));
        const uint32_t g = (uint32_t)groups.size();
        groups.push_back(MixedGroup{a});
        h->groupN.push_back(n);
        h->groupCls.push_back(cls);
        h->groupPlan.push_back(e);
        h->groupM.push_back(M);
        h->groupCount.push_back((uint32_t)kv.second.size());
        h->groupTileBegin.push_back((uint32_t)tiles.size());
        const uint32_t first = (uint32_t)offsByGroup.size();
        for (uint32_t i : kv.second) offsByGroup.push_back(offset[i]);
        const uint32_t cnt = (uint32_t)kv.second.size();
        for (uint32_t b = 0; b < cnt; b += M) {
            const uint32_t c = std::min(M, cnt - b);
            tiles.push_back(MixedTile{g, first + b, c, tile_flags(&offsByGroup[first + b], c, n)});
        }
        h->groupTileEnd.push_back((uint32_t)tiles.size());
    }
    h->numTiles = (uint32_t)tiles.size();
    // persistent order, per class: most expensive tiles first (groups are
    // already in decreasing length; within a group full tiles first)
    std::vector<MixedTile> lpt;
    for (int cls = 0; cls < kMixedClasses; ++cls) {
        h->clsTileBegin[cls] = (uint32_t)lpt.size();
        for (const MixedTile& t : tiles)
            if (h->groupCls[t.group] == cls && !groupFixed[t.group]) lpt.push_back(t);
        std::stable_sort(lpt.begin() + h->clsTileBegin[cls], lpt.end(), [&](const MixedTile& a, const MixedTile& b) {
            const double ca = (double)h->groupN[a.group] * a.count, cb = (double)h->groupN[b.group] * b.count;
            return ca > cb;
        });
        h->clsTiles[cls] = (uint32_t)lpt.size() - h->clsTileBegin[cls];
    }
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
    // a copy from pageable memory may return before its DMA lands; the graph
    // replays on streams that do not wait for the legacy stream
    if (err == cudaSuccess) err = cudaDeviceSynchronize();
    for (int cls = 0; cls < kMixedClasses && err == cudaSuccess; ++cls) {
        if (h->clsTiles[cls]) err = class_grid(cls, h->clsStage[cls], h->device, &h->clsGrid[cls]);
    }
    // per-size launches use the largest stage of any group with both classes,
    // and every class that has a group (fixed groups included) on its full
    // resident grid
    for (int cls = 0; cls < kMixedClasses && err == cudaSuccess; ++cls) {
        const bool used = std::find(h->groupCls.begin(), h->groupCls.end(), cls) != h->groupCls.end();
        if (used) err = class_grid(cls, h->groupStage, h->device, &h->perSizeGrid[cls]);
    }
    // Branches: the fixed groups are packed into kMaxBranches branches,
    // largest work first onto the least loaded; each class with tiles takes a
    // branch of its own. Every branch gets the fraction of the device (SMs
    // times a kernel's CTAs per SM) that its work is of the batch's and runs
    // its launches back to back on it, each launch after the first starting
    // while its predecessor drains (programmatic dependent launch); the
    // runtime-radix passes of the persistent kernel count twice per byte.
    // One branch measured best on B200 (the launches then stream through the
    // device one after another: 0.093 ms for the 20,000-transform set against
    // 0.097-0.099 ms on 2 to 8 branches); $FFTLIB_B200_MIXED_BRANCHES (1-8)
    // sets another count (at most 8: the device's hardware work queues).
    size_t kMaxBranches = 1;
    if (const char* v = getenv("FFTLIB_B200_MIXED_BRANCHES")) {
        const long b = strtol(v, nullptr, 10);
        if (b >= 1 && b <= 8) kMaxBranches = (size_t)b;
    }
    size_t classBranches = 0;
    for (int cls = 0; cls < kMixedClasses; ++cls) classBranches += h->clsTiles[cls] ? 1 : 0;
    size_t fixedBranches = 0;
    if (err == cudaSuccess && !h->fixed.empty()) {
        int sms = 0;
        err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
        double total = 0.0, clsW[kMixedClasses] = {};
        for (const auto& f : h->fixed) total += (double)f.n * f.count;
        for (size_t g = 0; g < groupFixed.size(); ++g)
            if (!groupFixed[g]) clsW[h->groupCls[g]] += 2.0 * h->groupN[g] * h->groupCount[g];
        for (int cls = 0; cls < kMixedClasses; ++cls) total += clsW[cls];
        fixedBranches = std::max<size_t>(1, std::min(h->fixed.size(), kMaxBranches - std::min(classBranches, kMaxBranches - 1)));
        std::vector<double> load(fixedBranches, 0.0);
        std::vector<size_t> order(h->fixed.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
            return (double)h->fixed[a].n * h->fixed[a].count > (double)h->fixed[b].n * h->fixed[b].count;
        });
        for (size_t i : order) {
            const size_t b = (size_t)(std::min_element(load.begin(), load.end()) - load.begin());
            h->fixed[i].branch = (uint32_t)b;
            load[b] += (double)h->fixed[i].n * h->fixed[i].count;
        }
        for (auto& f : h->fixed) {
            const int res = static_pipelined_resident(f.n, f.plan->eng.emax, f.plan->eng.T, f.plan->eng.P,
                                                      f.plan->eng.R);
            f.grid = (uint32_t)std::max(1.0, std::round((double)sms * res * load[f.branch] / total));
            h->fixedPoints += (uint64_t)f.n * f.count;
        }
        // launches of a branch in its order: largest and smallest work in
        // turn, so the launch that follows a large one (and starts while it
        // drains) is a short one that fills its tail (20,000-transform set:
        // 90 us against 92.5-93.5 us for ascending or descending length)
        {
            using Fx = FFTLIB_b200_mixed::Fixed;
            std::stable_sort(h->fixed.begin(), h->fixed.end(), [](const Fx& a, const Fx& b) {
                return (uint64_t)a.n * a.count > (uint64_t)b.n * b.count;
            });
            std::vector<Fx> o;
            size_t lo = 0, hi = h->fixed.size();
            while (lo < hi) {
                o.push_back(h->fixed[lo++]);
                if (lo < hi) o.push_back(h->fixed[--hi]);
            }
            h->fixed = o;
        }
        std::stable_sort(h->fixed.begin(), h->fixed.end(), [](const FFTLIB_b200_mixed::Fixed& a,
                                                              const FFTLIB_b200_mixed::Fixed& b) {
            return a.branch < b.branch;
        });
        for (int cls = 0; cls < kMixedClasses; ++cls)
            if (h->clsTiles[cls])
                h->clsGrid[cls] =
                    std::max(1u, std::min(h->clsGrid[cls], (uint32_t)std::round(h->clsGrid[cls] * clsW[cls] / total)));
    }
    h->fixedBranches = (uint32_t)fixedBranches;
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&h->capture, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming);
    const size_t nb = fixedBranches + classBranches;
    for (size_t b = 0; b < nb && err == cudaSuccess; ++b) {
        cudaStream_t bs = nullptr;
        cudaEvent_t be = nullptr;
        err = cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking);
        if (err == cudaSuccess) h->branches.push_back(bs);
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&be, cudaEventDisableTiming);
        if (err == cudaSuccess) h->joins.push_back(be);
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) {
        release(h);
        return cuda_fail(err, "mixed plan");
    }
    *handle = h;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_b200_fftMixed_exec(FFTLIB_b200_mixedHandle h, const FFTLIB_F32* pX, FFTLIB_F32* pY,
                                        void* stream)
{
    if (!h || !pX || !pY) return FFTLIB_ERR_NULL_POINTER;
    if (h->numTiles == 0) return FFTLIB_SUCCESS;
    DeviceScope scope(h->device);
    if (take_device_error()) {
        set_error("a device-side wait of an earlier launch timed out");
        return FFTLIB_ERR_FAILURE;
    }
    cudaError_t err = cudaSuccess;
    if (!h->exec || h->gx != pX || h->gy != pY) {
        // capture the counter reset and the persistent launch for these buffers
        if (h->exec) cudaGraphExecDestroy(h->exec);
        if (h->graph) cudaGraphDestroy(h->graph);
        h->exec = nullptr;
        h->graph = nullptr;
        err = cudaStreamBeginCapture(h->capture, cudaStreamCaptureModeThreadLocal);
        if (err == cudaSuccess) {
            cudaError_t le = enqueue_all(h, pX, pY, h->capture);
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
        const int cls = h->groupCls[g];
        cudaError_t err = launch_mixed(class_launch(cls, h->dGroups, h->dTilesByGroup + b, e - b, h->dOffsets, pX, pY,
                                                    h->groupStage, h->perSizeGrid[cls]),
                                       (cudaStream_t)stream);
        if (err != cudaSuccess) return cuda_fail(err, "mixed per-size launch");
    }
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_b200_fftMixed_describe(FFTLIB_b200_mixedHandle h, char* buf, uint32_t len)
{
    if (!h || !buf || len == 0) return FFTLIB_ERR_NULL_POINTER;
    std::ostringstream os;
    os << h->count << " transforms, " << h->groupN.size() << " lengths, " << h->fixed.size()
       << " fixed-size groups (" << h->fixedPoints << " points, grids";
    for (const auto& f : h->fixed) os << " " << f.n << ":" << f.branch << "/" << f.grid;
    os << "), " << h->numTiles << " tiles";
    for (int cls = 0; cls < kMixedClasses; ++cls)
        if (h->clsTiles[cls])
            os << "; class E" << mixed_class_emax(cls) << ": " << h->clsTiles[cls] << " tiles, grid " << h->clsGrid[cls]
               << ", stage " << h->clsStage[cls] * 8u << " B";
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
