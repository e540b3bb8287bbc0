// fft_pipeline.cuh -- persistent, TMA-pipelined fixed-size FFT kernel.
//
// A CTA walks over tiles of M contiguous transforms (tile = blockIdx.x,
// blockIdx.x + gridDim.x, ...). A ring of STAGES shared-memory tiles is fed
// by bulk asynchronous copies (cp.async.bulk global->shared, completion on an
// mbarrier): while the CTA runs the passes of tile i out of one stage, the
// copies for the next tiles are already in flight, so HBM reads never wait
// for compute. The first pass reads its inputs straight from the stage, the
// intermediate passes exchange through a padded shared-memory buffer and the
// last pass stores to HBM from registers.
//
// Every wait is bounded (iteration and wall-clock limits). A wait that gives
// up sets bit kErrPipelineTimeout in the launch's error word, drains the
// copies still in flight (again bounded) and ends the CTA; the host reports
// the error word after synchronizing.
#pragma once

#include "fft_stockham.cuh"

namespace fftb200 {

constexpr uint32_t kErrPipelineTimeout = 1u;

FFT_DEV uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

FFT_DEV void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

FFT_DEV void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Plain arrival (no transaction bytes): completes a phase of count 1.
FFT_DEV void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

FFT_DEV bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n"
        "  .reg .pred p;\n"
        "  mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "  selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

FFT_DEV uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for phase `parity` of bar: gives up after 2^22 polls or one
// second, whichever comes first.
FFT_DEV bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    const uint64_t t0 = global_ns();
    for (uint32_t i = 0; i < (1u << 22); ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 255u) == 255u && global_ns() - t0 > 1000000000ull) return false;
    }
    return false;
}

FFT_DEV void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

FFT_DEV void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
FFT_DEV void fence_mbarrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Stage length in complex values: the padded exchange layout of one
// transform, rounded to an even count so every stage starts 16-byte aligned.
__host__ __device__ constexpr uint32_t pipe_stage_len(uint32_t n) { return (smem_len(n) + 1u) & ~1u; }

// Shared-memory bytes of the pipelined kernel (m transforms per tile).
__host__ __device__ constexpr size_t pipe_smem_bytes(uint32_t n, int stages, int m = 1)
{
    return (size_t)stages * (size_t)m * pipe_stage_len(n) * 8u + 8u * (size_t)stages + 16u;
}

// Transforms per tile: enough to give the CTA 256 threads for short
// transforms, one for transforms of 128 threads or more.
__host__ __device__ constexpr int pipe_tile(int t) { return t >= 128 ? 1 : (256 / t < 1 ? 1 : 256 / t); }

// CTAs per SM the kernel is compiled for: as many as the shared memory
// (228 KB per SM, 1 KB reserved per CTA) and 2048 threads allow, at most 8;
// with regFloor > 0 also few enough to leave every thread that many of the
// SM's 65,536 registers (schedules with radix-9/12 passes need about 100 and
// spill when the shared-memory bound alone caps them near 40).
__host__ __device__ constexpr int pipe_min_blocks(uint32_t n, int threads, int stages, int m = 1, int regFloor = 0)
{
    const int bySmem = (int)((228u * 1024u) / (pipe_smem_bytes(n, stages, m) + 1024u));
    const int byThreads = 2048 / threads;
    int b = bySmem < byThreads ? bySmem : byThreads;
    if (regFloor > 0) {
        const int byRegs = 65536 / (((threads + 31) / 32) * 32 * regFloor);
        b = b < byRegs ? b : byRegs;
    }
    return b < 1 ? 1 : (b > 8 ? 8 : b);
}

// Whether pass p of schedule S can run mirrored (two butterflies per thread,
// T = N / R / 2; see run_pass).
template <class S>
__host__ __device__ constexpr bool pipe_mirrorable(int p)
{
    return S::EMAX / S::R[p] == 2 && 2 * S::T == S::N / S::R[p];
}

// Input span of a tile of m transforms with input rows of ic complex values:
// the copy starts at the even element s0 at or below the tile's first value
// (shift = 0 or 1 elements before it) and covers ncopy (even) elements, all
// of the nelem the tile needs except, at the very end of the input, one.
struct TileSpan {
    uint64_t s0;
    uint32_t shift, ncopy, nelem;
};
FFT_DEV TileSpan tile_span(uint32_t tile, uint32_t m, uint32_t batch, uint64_t ic, uint64_t totalIn)
{
    const uint64_t first = (uint64_t)tile * m;
    const uint64_t count = min((uint64_t)m, (uint64_t)batch - first);
    const uint64_t b = first * ic;
    TileSpan t;
    t.s0 = b & ~1ull;
    t.shift = (uint32_t)(b - t.s0);
    t.nelem = t.shift + (uint32_t)(count * ic);
    const uint64_t want = ((uint64_t)t.nelem + 1u) & ~1ull;
    t.ncopy = (uint32_t)(min(want, totalIn - t.s0) & ~1ull);
    return t;
}

// A tile is M consecutive transforms (c2c; the half-length complex FFT of
// r2c with its split epilogue; or of c2r, inMode 0, with the split computed
// from the raw bins in pass 0). One bulk copy lands their inputs,
// unpadded and back to back, at the start of the stage; the first pass of
// transform m reads its input from there and (after the CTA-wide barrier
// inside the pass, when every input has been read) writes its outputs in the
// padded layout at m * SL, and so on; a stage is refilled as soon as the
// CTA has moved past the tile it held. IO (IO_C2C, IO_R2C_SPLIT or IO_C2R_SPLIT) is the one
// transform kind the instantiation serves, so that none of them carries the
// others' code (a.ioMode equals it).
template <class S, int STAGES, int M, int IO>
FFT_DEV void fft_pipeline(const FftArgs& a)
{
    static_assert(S::P >= 2, "the pipelined kernel needs at least two passes");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr uint32_t N = (uint32_t)S::N;
    constexpr uint32_t SL = pipe_stage_len(N);
    constexpr uint32_t STL = (uint32_t)M * SL;
    float2* stages = (float2*)smem_raw;
    uint64_t* bar = (uint64_t*)(stages + (size_t)STAGES * STL);
    __shared__ uint32_t s_fail;

    const uint32_t tid = threadIdx.x;
    const uint32_t m = tid / (uint32_t)S::T;
    const uint32_t t = tid - m * (uint32_t)S::T;
    const uint32_t tiles = (a.batch + (uint32_t)M - 1u) / (uint32_t)M;
    const uint32_t G = gridDim.x;
    // a kernel launched after this one with programmatic stream
    // serialization may start now (a no-op for every other launch)
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

    // a tile's inputs are count * IC contiguous complex values (IC = the
    // input row length: N, or N + 1 bins for c2r); see tile_span
    const uint64_t IC = (uint64_t)a.inBatch;
    const uint64_t totalIn = (uint64_t)a.batch * IC;
    auto issue = [&](uint32_t tile, int s) {
        const TileSpan sp = tile_span(tile, (uint32_t)M, a.batch, IC, totalIn);
        mbar_expect_tx(&bar[s], sp.ncopy * 8u);
        bulk_copy_g2s(stages + (size_t)s * STL, a.in + sp.s0, sp.ncopy * 8u, &bar[s]);
    };

    if (tid == 0) {
        s_fail = 0;
        for (int s = 0; s < STAGES; ++s) mbar_init(&bar[s], 1);
        fence_mbarrier_init();
    }
    __syncthreads();
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            const uint32_t tile = blockIdx.x + (uint32_t)s * G;
            if (tile < tiles) issue(tile, s);
        }
    }

    float2 v[S::EMAX];
    uint32_t it = 0;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += G, ++it) {
        const int s = (int)(it % STAGES);
        // one thread waits for the stage; the barrier passes the data (and
        // the outcome) on to the others
        float2* st = stages + (size_t)s * STL;
        const TileSpan sp = tile_span(tile, (uint32_t)M, a.batch, IC, totalIn);
        const uint32_t shift = sp.shift;
        if (tid == 0) {
            if (!mbar_wait_bounded(&bar[s], (it / STAGES) & 1u)) s_fail = 1u;
            else if (sp.nelem > sp.ncopy) st[sp.ncopy] = a.in[sp.s0 + sp.ncopy];  // odd element at the very end
        }
        __syncthreads();
        if (s_fail) break;
        // every thread is past the previous tile (its last pass, and the r2c
        // epilogue, read that tile's stage before this barrier): refill that
        // stage with the tile STAGES-1 iterations ahead right away
        if (tid == 0 && it > 0) {
            fence_proxy_async_smem();
            const uint32_t next = tile + (uint32_t)(STAGES - 1) * G;
            if (next < tiles) issue(next, (int)((it - 1) % STAGES));
        }

        const uint32_t gidx = tile * (uint32_t)M + m;
        const bool active = gidx < a.batch;
        float2* rowOut = a.out + (size_t)gidx * (size_t)a.outBatch;
        // a schedule whose first (last) pass can run mirrored splits the
        // c2r input (r2c output) there, in registers
        constexpr bool kC2RMirror = IO == IO_C2R_SPLIT && pipe_mirrorable<S>(0);
        constexpr bool kR2CMirror = IO == IO_R2C_SPLIT && pipe_mirrorable<S>(S::P - 1);
        if constexpr (IO == IO_C2R_SPLIT && !kC2RMirror) {
            // c2r (inMode 0): turn the h + 1 bins into the h-point input Z in
            // place, Z[i] = ((X[i] + y) + i conj(W) (X[i] - y)) / 2 with
            // y = conj(X[h - i]); each thread owns the pair (i, h - i)
            float2* row = st + shift + m * (uint32_t)IC;
            if (active) {
                for (uint32_t i = t; i <= N / 2u; i += (uint32_t)S::T) {
                    const uint32_t ip = N - i;
                    const float2 xi = row[i], xp = row[ip];
                    // W_{2h}^(h-i) = -conj(W_{2h}^i): one table load serves the
                    // pair, with the accuracy of the table's own entry
                    float2 zi, zp;
                    c2r_split_pair(xi, xp, __ldg(&a.twSplit[i]), zi, zp);
                    row[i] = zi;
                    if (i != 0u && ip != i) row[ip] = zp;
                }
            }
            __syncthreads();
        }
        static_for<S::P>([&](auto p) FFT_INL {
            constexpr int P = decltype(p)::value;
            constexpr PassInfo pi = S::pass(P);
            constexpr int L0 = first_boundary_layout(S::R[0]);
            const float2* raw = st + shift + m * (uint32_t)IC;
            if constexpr (P == 0) {
                if constexpr (kC2RMirror)
                    run_pass<S::EMAX, S::R[P], NoHook, false, kPad16, L0, true, kMirrorC2R>(
                        a, pi, true, P + 1 == S::P, (uint32_t)S::T, v, st + m * SL, t, active, nullptr, rowOut, raw);
                else
                    run_pass<S::EMAX, S::R[P], NoHook, false, kPad16, L0, true>(
                        a, pi, true, P + 1 == S::P, (uint32_t)S::T, v, st + m * SL, t, active, nullptr, rowOut, raw);
            } else if constexpr (P + 1 == S::P) {
                if constexpr (kR2CMirror)
                    run_pass<S::EMAX, S::R[P], NoHook, false, P == 1 ? L0 : kPad16, kPad16, true, kMirrorR2C>(
                        a, pi, false, true, (uint32_t)S::T, v, st + m * SL, t, active, nullptr, rowOut);
                else
                    run_pass<S::EMAX, S::R[P], NoHook, false, P == 1 ? L0 : kPad16, kPad16, true>(
                        a, pi, false, true, (uint32_t)S::T, v, st + m * SL, t, active, nullptr, rowOut);
            } else {
                run_pass<S::EMAX, S::R[P], NoHook, false, P == 1 ? L0 : kPad16, kPad16, true>(
                    a, pi, false, false, (uint32_t)S::T, v, st + m * SL, t, active, nullptr, rowOut);
            }
        });
        // r2c without the mirrored last pass: that pass left Z in natural
        // order in the padded layout; the split writes the h + 1 (or 2h)
        // bins. The stage is refilled only after the next iteration's first
        // barrier, when this has finished.
        if constexpr (IO == IO_R2C_SPLIT && !kR2CMirror) r2c_epilogue(a, st + m * SL, t, rowOut, active);
    }

    if (s_fail && tid == 0) {
        *(volatile uint32_t*)a.err = kErrPipelineTimeout;
        // drain every copy still in flight (bounded): the failed one and the
        // STAGES-2 issued after it, or at it = 0 every initial stage
        const uint32_t last = it == 0 ? (uint32_t)STAGES - 1u : it + (uint32_t)STAGES - 2u;
        for (uint32_t itk = it; itk <= last; ++itk) {
            const uint32_t tile = blockIdx.x + itk * G;
            if (tile < tiles) mbar_wait_bounded(&bar[itk % STAGES], (itk / STAGES) & 1u);
        }
    }
}

} // namespace fftb200
