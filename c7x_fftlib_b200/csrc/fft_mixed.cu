// fft_mixed.cu -- persistent kernel for batches of FP32 c2c transforms of
// uneven lengths (K6).
//
// The host groups the transforms by length; every group has its own
// schedule (FftArgs: radices, threads per transform T, transforms per tile
// M, twiddle table) and its transforms are cut into tiles of M. Tiles are
// ordered by cost, largest first, and CTA b takes tiles b, b + grid, ... (a
// tile holds about 256 E complex values whatever its length, so the static
// round robin stays balanced and needs no atomic counter).
//
// Each CTA owns a ring of two shared-memory stages fed by bulk asynchronous
// copies (cp.async.bulk global -> shared, completion on an mbarrier): while
// the CTA runs the passes of tile i, the copy of tile i + 1 is in flight. A
// tile whose transforms lie back to back is one copy; otherwise one copy per
// transform; rows off a 16-byte boundary are copied in by the threads. The
// first pass reads its inputs from the stage, the passes in between exchange
// through the stage's padded layout, the last pass stores to HBM from
// registers. The group's schedule is copied into shared memory
// per tile (two buffers, so the next tile's copy never overwrites one still
// read) and the passes dispatch their radix at run time, every radix a
// compile-time codelet.
//
// Every wait is bounded (fft_pipeline.cuh): a wait that gives up sets the
// error word, drains the copies in flight (bounded) and ends the CTA.
#include <algorithm>
#include <mutex>

#include "fft_mixed.h"
#include "fft_pipeline.cuh"

namespace fftb200 {

namespace {
constexpr int kMixedBlock = 256;
constexpr int kMixedStages = 2;
// a stage holds one tile: M padded transforms (up to one N = 4096 transform)
constexpr uint32_t kMixedStageMaxBytes = 36u * 1024u;
constexpr uint32_t kArgsWords = (uint32_t)(sizeof(FftArgs) / 4);
static_assert(sizeof(FftArgs) % 4 == 0 && kArgsWords <= (uint32_t)kMixedBlock, "FftArgs copy");
} // namespace

template <int EMAX, int MINB>
__global__ void __launch_bounds__(kMixedBlock, MINB)
    k_fft_mixed(const MixedGroup* __restrict__ groups, const MixedTile* __restrict__ tiles, uint32_t numTiles,
                const uint64_t* __restrict__ offsets, const float2* x, float2* y, uint32_t stageLen, uint32_t bulkOk,
                uint32_t* err)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float2* stages = (float2*)smem_raw;
    uint64_t* bar = (uint64_t*)(stages + (size_t)kMixedStages * stageLen);
    __shared__ __align__(16) FftArgs s_args[2];
    __shared__ uint32_t s_fail;
    const uint32_t tid = threadIdx.x;
    const uint32_t G = gridDim.x;

    // which tiles bulk copies may bring in (none when x is off a 16-byte
    // boundary)
    const uint32_t bulkMask = bulkOk ? (kTileBulk | kTileRows) : 0u;
    // one thread issues the copies of a tile into stage s
    auto issue = [&](uint32_t tile, int s) {
        const MixedTile tl = tiles[tile];
        float2* dst = stages + (size_t)s * stageLen;
        const uint32_t n = groups[tl.group].args.N;
        const uint32_t flags = tl.flags & bulkMask;
        if (flags & kTileBulk) {
            const uint32_t bytes = tl.count * n * 8u;
            mbar_expect_tx(&bar[s], bytes);
            bulk_copy_g2s(dst, x + offsets[tl.first], bytes, &bar[s]);
        } else if (flags & kTileRows) {
            mbar_expect_tx(&bar[s], tl.count * n * 8u);
            for (uint32_t m = 0; m < tl.count; ++m)
                bulk_copy_g2s(dst + (size_t)m * n, x + offsets[tl.first + m], n * 8u, &bar[s]);
        } else {
            mbar_arrive(&bar[s]);
        }
    };

    if (tid == 0) {
        s_fail = 0;
        for (int s = 0; s < kMixedStages; ++s) mbar_init(&bar[s], 1);
        fence_mbarrier_init();
    }
    __syncthreads();
    if (tid == 0) {
        for (int s = 0; s < kMixedStages; ++s) {
            const uint32_t tile = blockIdx.x + (uint32_t)s * G;
            if (tile < numTiles) issue(tile, s);
        }
    }

    float2 v[EMAX];
    uint32_t it = 0;
    for (uint32_t tile = blockIdx.x; tile < numTiles; tile += G, ++it) {
        const int s = (int)(it % kMixedStages);
        const MixedTile tl = tiles[tile];
        // this tile's schedule; buffer it & 1 was last read two tiles ago,
        // before the barrier every thread passed at the previous tile
        FftArgs& a = s_args[it & 1u];
        if (tid < kArgsWords)
            reinterpret_cast<uint32_t*>(&a)[tid] = reinterpret_cast<const uint32_t*>(&groups[tl.group].args)[tid];
        if (tid == 0 && !mbar_wait_bounded(&bar[s], (it / kMixedStages) & 1u)) s_fail = 1u;
        __syncthreads();
        if (s_fail) break;
        // every thread has finished the previous tile: its stage takes the
        // tile kMixedStages - 1 steps ahead
        if (tid == 0 && it > 0) {
            fence_proxy_async_smem();
            const uint32_t next = tile + (uint32_t)(kMixedStages - 1) * G;
            if (next < numTiles) issue(next, (int)((it - 1) % kMixedStages));
        }

        float2* st = stages + (size_t)s * stageLen;
        const uint32_t T = a.T, used = T * a.M, N = a.N;
        if (!(tl.flags & bulkMask)) {
            // rows off a 16-byte boundary: the threads copy the tile in
            const uint32_t total = tl.count * N;
            for (uint32_t e = tid; e < total; e += kMixedBlock) {
                const uint32_t mm = fastdiv(e, N, a.nMagic);
                st[e] = x[offsets[tl.first + mm] + (e - mm * N)];
            }
            __syncthreads();
        }
        // threads beyond T*M get a lane index past every butterfly: they only
        // take part in the barriers
        uint32_t m = 0, t = 0xFFFFu;
        if (tid < used) {
            m = tid / T;
            t = tid - m * T;
        }
        const bool active = tid < used && m < tl.count;
        const uint64_t off = active ? offsets[tl.first + m] : 0;
        const float2* rowIn = x + off;
        float2* rowOut = y + off;
        float2* sm = st + m * a.slen;
        const float2* raw = st + (size_t)m * N;  // this transform's inputs in the stage
        const int P = (int)a.P;
        // an odd first radix scatters with an odd stride: the boundary after
        // pass 0 is unpadded (kNoPad, see run_pass)
        const bool noPad0 = P > 1 && (a.pass[0].R & 1);
        for (int p = 0; p < P; ++p) {
            dispatch_radix<EMAX>(a.pass[p].R, [&](auto r) {
                constexpr int RR = decltype(r)::value;
                if constexpr (RR % 2 == 1) {
                    if (p == 0 && noPad0) {
                        run_pass<EMAX, RR, NoHook, true, kPad16, kNoPad>(a, a.pass[p], true, false, T, v, sm, t,
                                                                         active, rowIn, rowOut, raw);
                        return;
                    }
                }
                if (p == 1 && noPad0) {
                    run_pass<EMAX, RR, NoHook, true, kNoPad, kPad16>(a, a.pass[p], false, p + 1 == P, T, v, sm, t,
                                                                     active, rowIn, rowOut, raw);
                    return;
                }
                run_pass<EMAX, RR, NoHook, true>(a, a.pass[p], p == 0, p + 1 == P, T, v, sm, t, active, rowIn,
                                                 rowOut, raw);
            });
        }
    }

    if (s_fail && tid == 0) {
        *(volatile uint32_t*)err = kErrPipelineTimeout;
        // drain every copy still in flight (bounded): the steps it ..
        // it + stages - 2 were issued (at it = 0 all initial stages were)
        const uint32_t last = it == 0 ? (uint32_t)kMixedStages - 1u : it + (uint32_t)kMixedStages - 2u;
        for (uint32_t itk = it; itk <= last; ++itk) {
            const uint32_t tile = blockIdx.x + itk * G;
            if (tile < numTiles) mbar_wait_bounded(&bar[itk % kMixedStages], (itk / kMixedStages) & 1u);
        }
    }
}

namespace {

template <int EMAX, int MINB>
cudaError_t configure_one(size_t smem, int* residentPerSm)
{
    auto k = k_fft_mixed<EMAX, MINB>;
    static std::mutex mu;
    static size_t configured[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    {
        // the limit only ever grows, so launches planned earlier stay valid
        std::lock_guard<std::mutex> lock(mu);
        if (dev >= 64 || configured[dev] < smem) {
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            if (dev < 64) configured[dev] = smem;
        }
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(residentPerSm, k, kMixedBlock, smem);
}

} // namespace

int mixed_class_emax(int cls) { return cls == kMixedW20 ? 20 : 16; }
uint32_t mixed_block() { return (uint32_t)kMixedBlock; }
uint32_t mixed_stage_max_bytes() { return kMixedStageMaxBytes; }
size_t mixed_smem(uint32_t stageLen) { return (size_t)kMixedStages * stageLen * 8u + 8u * kMixedStages; }

cudaError_t mixed_configure(int cls, size_t smem, int* residentPerSm)
{
    return cls == kMixedW20 ? configure_one<20, 2>(smem, residentPerSm) : configure_one<16, 3>(smem, residentPerSm);
}

cudaError_t launch_mixed(const MixedLaunch& L, cudaStream_t s)
{
    if (L.numTiles == 0) return cudaSuccess;
    // bulk copies need a 16-byte aligned source (tile flags assume x is)
    const uint32_t bulkOk = ((uintptr_t)L.x & 15u) == 0 ? 1u : 0u;
    if (L.cls == kMixedW20)
        k_fft_mixed<20, 2><<<L.grid, kMixedBlock, L.smem, s>>>(L.groups, L.tiles, L.numTiles, L.offsets, L.x, L.y,
                                                               L.stageLen, bulkOk, L.err);
    else
        k_fft_mixed<16, 3><<<L.grid, kMixedBlock, L.smem, s>>>(L.groups, L.tiles, L.numTiles, L.offsets, L.x, L.y,
                                                               L.stageLen, bulkOk, L.err);
    return cudaGetLastError();
}

} // namespace fftb200
