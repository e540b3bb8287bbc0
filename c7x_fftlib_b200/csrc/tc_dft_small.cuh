// tc_dft_small.cuh -- one-stage split-FP16 tensor-core DFT for N = 8..64.
//
// Rows of 64 complex values ("super-rows": 64/N consecutive transforms) are
// transformed by one 128 x 128 real DFT-GEMM whose matrix is block-diagonal,
// 64/N copies of the 2N x 2N embedding of the N-point DFT (the reference's
// dftSmall layout, src/fft_c7xmma/FFTLIB_FFT_dftSmall_ixX_cxX_oxX/c71/
// FFTLIB_FFT_dftSmall_ixX_cxX_oxX_ci.cpp:119-212, restated for FP32). The
// matrix is the A operand and the data the B operand,
//     D[M = 128 output components][N = 64 super-rows] = W^T . X^T,
// so a warp of the epilogue owns 32 consecutive output components of every
// super-row in the tile and writes each super-row's 128-byte slice with one
// coalesced store. Because a diagonal block only feeds its own outputs, every
// transform keeps its own power-of-two scale.
//
// Roles per CTA (one persistent CTA per SM): 8 loader warps (HBM -> registers
// -> per-transform scale -> FP16 hi/lo -> K-major swizzled shared memory,
// next tile prefetched into L2), 8 epilogue warps (tensor memory -> unscale ->
// HBM) and one warp that allocates tensor memory and issues the MMAs (the
// two small cross products first, then hi.hi). Four tile buffers; every wait
// is bounded.
#pragma once

#include "tc_dft.cuh"

namespace fftb200 {

template <int V>
struct IntC {
    static constexpr int value = V;
};
template <bool V>
struct BoolC {
    static constexpr bool value = V;
};

template <int N_>
struct TcSmall {
    static constexpr int N = N_;
    static constexpr int G = 64 / N;   // transforms per super-row
    static constexpr int TS = 64;      // super-rows per tile = MMA N
    static constexpr int NB = 4;       // operand tile buffers
    static constexpr int LW = 8, EW = 8;
    static constexpr int MMA_WARP = LW + EW;
    static constexpr int THREADS = 32 * (MMA_WARP + 1);
    using LA = KMajor<128, 128>;  // W^T: rows = output component, K = input component
    using LB = KMajor<TS, 128>;   // data: rows = super-rows, K = input component
    static constexpr uint32_t W_HALF = LA::BYTES;  // 32 KB
    static constexpr uint32_t HALF_TILE = LB::BYTES;  // 16 KB
    static constexpr uint32_t TILE = 2 * HALF_TILE;
    static constexpr uint32_t OFF_W = NB * TILE;
    static constexpr uint32_t OFF_S = OFF_W + 2 * W_HALF;  // per-transform unscale factors, 2 NB slots
    static constexpr uint32_t OFF_BAR = (OFF_S + 4u * 2 * NB * TS * G + 7u) & ~7u;
    static constexpr int NBARS = 3 * NB + 1;
    static constexpr uint32_t OFF_MISC = OFF_BAR + 8u * NBARS;
    static constexpr uint32_t SMEM = OFF_MISC + 16u + 1024u;
    static constexpr uint32_t TMEM_COLS = NB * TS;  // 256
    static constexpr int A_FULL = 0, D_FULL = NB, D_FREE = 2 * NB, DRAIN = 3 * NB;
    static_assert(64 % N == 0 && N >= 8, "N = 8, 16, 32 or 64");
    static_assert(SMEM <= 227u * 1024u, "shared memory per CTA");
};

template <int N>
__global__ void __launch_bounds__(TcSmall<N>::THREADS, 1)
    k_tc_small(const float2* __restrict__ x, float2* __restrict__ y, const float* __restrict__ w, uint32_t batch,
               uint32_t* err)
{
    using S = TcSmall<N>;
    constexpr int G = S::G, TS = S::TS, NB = S::NB;
    extern __shared__ unsigned char tc_smem_raw[];
    unsigned char* sm = tc_smem_raw + ((1024u - (smem_addr(tc_smem_raw) & 1023u)) & 1023u);
    const uint32_t sbase = smem_addr(sm);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + S::OFF_BAR);
    uint32_t* misc = reinterpret_cast<uint32_t*>(sm + S::OFF_MISC);
    volatile uint32_t* abortFlag = misc + 1;
    float* unscale = reinterpret_cast<float*>(sm + S::OFF_S);  // 2^-(row shift + W shift) per transform

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rows = (batch + G - 1) / G;  // super-rows
    const uint32_t numTiles = (rows + TS - 1) / TS;

    if (threadIdx.x == 0) {
        for (int i = 0; i < S::NBARS; ++i) mbar_init(&bars[i], 1);
        misc[1] = 0;
        fence_mbarrier_init();
    }
    if (warp == S::MMA_WARP) {
        tmem_alloc(&misc[0], S::TMEM_COLS);
        tmem_relinquish();
    }
    // W^T operand, block-diagonal: row (k', c) of block j = k'/N, K index
    // (n', c') of the same block holds the N-point embedding entry
    // wr[(2 n + c') * 2N + 2 k + c] (n = n' mod N, k = k' mod N), zero elsewhere
    {
        unsigned char* hi = sm + S::OFF_W;
        unsigned char* lo = hi + S::W_HALF;
        const float sc = exp2i(kTcWShift);
        for (int it = threadIdx.x; it < 128 * 16; it += blockDim.x) {
            const int row = it >> 4, j = it & 15;  // 16-byte chunk j: K = 8 j .. 8 j + 7
            uint32_t h[4], l[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int k0 = 8 * j + 2 * e;
                float a = 0.f, b = 0.f;
                if (k0 / (2 * N) == row / (2 * N)) {
                    const int kk = k0 % (2 * N), rr = row % (2 * N);
                    a = __ldg(w + (size_t)kk * (2 * N) + rr) * sc;
                    b = __ldg(w + (size_t)(kk + 1) * (2 * N) + rr) * sc;
                }
                split2(a, b, h[e], l[e]);
            }
            const uint32_t off = S::LA::chunk(row, j);
            *reinterpret_cast<uint4*>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<uint4*>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
        }
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = misc[0];

    if (warp < S::LW) {
        // ================= loaders =================
        // lane l holds complex 2l, 2l+1 of a super-row; transform j of the
        // super-row spans lanes [j N/2, (j+1) N/2)
        constexpr int LPT = N / 2;          // lanes per transform
        constexpr int RPW = TS / S::LW;     // super-rows per warp per tile
        const int j = threadIdx.x;
        const int tj = lane / LPT;
        // the tile's rows are contiguous in HBM: the next tile of this CTA is
        // pulled into L2 while this one is converted
        auto prefetch = [&](uint32_t tl) {
            if (j != 0 || tl >= numTiles) return;
            const uint64_t first = (uint64_t)tl * TS * 64;  // first complex value of the tile
            const uint64_t cnt = min((uint64_t)TS * 64, (uint64_t)batch * N - first);
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(x + first), "r"((uint32_t)(cnt * 8u))
                         : "memory");
        };
        prefetch(blockIdx.x);
        uint32_t i = 0;
        for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++i) {
            prefetch(tile + gridDim.x);
            const int b = (int)(i % NB);
            const uint32_t u = i / NB, slot = i % (2 * NB);
            // super-row r is 32 contiguous float4; lane l loads float4 l of it
            const float4* xb = reinterpret_cast<const float4*>(x + (size_t)tile * TS * 64) + warp * RPW * 32 + lane;
            float4 v[RPW];
            if ((uint64_t)(tile + 1) * TS * G <= batch) {
#pragma unroll
                for (int k = 0; k < RPW; ++k) v[k] = __ldg(xb + k * 32);
            } else {
#pragma unroll
                for (int k = 0; k < RPW; ++k) {
                    const uint64_t gt = ((uint64_t)tile * TS + warp * RPW + k) * G + tj;  // this lane's transform
                    v[k] = gt < batch ? __ldg(xb + k * 32) : make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
            int sh[RPW];
#pragma unroll
            for (int k = 0; k < RPW; ++k) {
                float m = fmaxf(fmaxf(fabsf(v[k].x), fabsf(v[k].y)), fmaxf(fabsf(v[k].z), fabsf(v[k].w)));
#pragma unroll
                for (int o = LPT / 2; o >= 1; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
                sh[k] = row_shift(m);
            }
            bool bad = false;
            if (u >= 1 && j == 0) bad = !tc_wait(&bars[S::D_FULL + b], (u - 1) & 1u, abortFlag, err);
            if (group_sync_or(1, 32 * S::LW, bad)) break;
            unsigned char* hiB = sm + b * S::TILE;
            unsigned char* loB = hiB + S::HALF_TILE;
#pragma unroll
            for (int k = 0; k < RPW; ++k) {
                const int r = warp * RPW + k;
                const float sc = exp2i(sh[k]);
                uint32_t h0, h1, l0, l1;
                split2(v[k].x * sc, v[k].y * sc, h0, l0);
                split2(v[k].z * sc, v[k].w * sc, h1, l1);
                const uint32_t off = S::LB::chunk(r, lane >> 1) + (uint32_t)(lane & 1) * 8u;
                *reinterpret_cast<uint2*>(hiB + off) = make_uint2(h0, h1);
                *reinterpret_cast<uint2*>(loB + off) = make_uint2(l0, l1);
                if ((lane % LPT) == 0) unscale[slot * (TS * G) + r * G + tj] = exp2i(-(sh[k] + kTcWShift));
            }
            fence_proxy_async_smem();
            group_sync(1, 32 * S::LW);
            if (j == 0) mbar_arrive(&bars[S::A_FULL + b]);
        }
    } else if (warp == S::MMA_WARP) {
        // ================= MMA issue =================
        if (lane == 0) {
            constexpr uint32_t idesc = umma_idesc_f16(TS);
            constexpr int KS = 128 / 16;
            const uint32_t wHi = sbase + S::OFF_W, wLo = wHi + S::W_HALF;
            uint32_t i = 0;
            for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++i) {
                const int b = (int)(i % NB);
                const uint32_t u = i / NB;
                if (!tc_wait(&bars[S::A_FULL + b], u & 1u, abortFlag, err)) break;
                if (u >= 1 && !tc_wait(&bars[S::D_FREE + b], (u - 1) & 1u, abortFlag, err)) break;
                tc_fence_after();
                const uint32_t xHi = sbase + b * S::TILE, xLo = xHi + S::HALF_TILE;
                const uint32_t d = tmem + (uint32_t)(b * TS);
                // cross products first: only the final hi.hi updates round at
                // the accumulator's full magnitude
#pragma unroll
                for (int s = 0; s < KS; ++s)
                    tc_mma_f16(d, S::LA::desc(wHi, 0, s), S::LB::desc(xLo, 0, s), idesc, s > 0 ? 1u : 0u);
#pragma unroll
                for (int s = 0; s < KS; ++s)
                    tc_mma_f16(d, S::LA::desc(wLo, 0, s), S::LB::desc(xHi, 0, s), idesc, 1u);
#pragma unroll
                for (int s = 0; s < KS; ++s)
                    tc_mma_f16(d, S::LA::desc(wHi, 0, s), S::LB::desc(xHi, 0, s), idesc, 1u);
                tc_commit(&bars[S::D_FULL + b]);
            }
            tc_commit(&bars[S::DRAIN]);
            mbar_wait_bounded(&bars[S::DRAIN], 0);
        }
        __syncwarp();
    } else {
        // ================= epilogue =================
        // thread = output component l (bin l/2 of the super-row, re or im) of
        // half the super-rows of the tile; l belongs to transform l / (2N)
        const int et = threadIdx.x - 32 * S::LW;  // 0..255
        const int q = warp & 3, ch = (warp - S::LW) >> 2;
        const int l = 32 * q + lane;
        const int tj = l / (2 * N);
        const uint32_t laneBase = (uint32_t)(32 * q) << 16;
        float* yf = reinterpret_cast<float*>(y);
        uint32_t i = 0;
        for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++i) {
            const int b = (int)(i % NB);
            const uint32_t u = i / NB, slot = i % (2 * NB);
            bool bad = false;
            if (et == 0) bad = !tc_wait(&bars[S::D_FULL + b], u & 1u, abortFlag, err);
            if (group_sync_or(3, 32 * S::EW, bad)) break;
            tc_fence_after();
            // per super-row r of the tile: y[(tile TS + r) 128 + l] = D[l][r] * unscale;
            // addresses are a per-tile base plus compile-time offsets, and a
            // tile inside the batch needs no bounds checks
            const float* us = unscale + slot * (TS * G) + tj;
            float* ybase = yf + (size_t)tile * TS * 128 + l;
            const uint32_t dbase = tmem + laneBase + (uint32_t)(b * TS);
            const bool full = (uint64_t)(tile + 1) * TS * G <= batch;
            auto half = [&](auto chc, auto fullc) {
                constexpr int CH = decltype(chc)::value;
                constexpr bool FULL = decltype(fullc)::value;
#pragma unroll
                for (int cc = 0; cc < TS / 2; cc += 16) {
                    const int c0 = CH * (TS / 2) + cc;
                    float v[16];
                    tmem_ld16(dbase + (uint32_t)c0, v);
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        const int r = c0 + e;
                        if (FULL || ((uint64_t)tile * TS + r) * G + tj < batch) ybase[r * 128] = v[e] * us[r * G];
                    }
                }
            };
            if (ch == 0) {
                if (full) half(IntC<0>{}, BoolC<true>{}); else half(IntC<0>{}, BoolC<false>{});
            } else {
                if (full) half(IntC<1>{}, BoolC<true>{}); else half(IntC<1>{}, BoolC<false>{});
            }
            tc_fence_before();
            group_sync(3, 32 * S::EW);
            if (et == 0) mbar_arrive(&bars[S::D_FREE + b]);
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == S::MMA_WARP) {
        tc_fence_after();
        tmem_dealloc(tmem, S::TMEM_COLS);
    }
}

template <int N>
cudaError_t launch_tc_small(const float2* x, float2* y, const float* w, uint32_t batch, uint32_t* err, cudaStream_t s)
{
    using S = TcSmall<N>;
    if (batch == 0) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static bool configured[64] = {};
    static int sms[64] = {};
    {
        std::lock_guard<std::mutex> lock(mu);
        if (dev >= 64) return cudaErrorInvalidDevice;
        if (!configured[dev]) {
            e = cudaFuncSetAttribute(k_tc_small<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
            if (e != cudaSuccess) return e;
            e = cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return e;
            configured[dev] = true;
        }
    }
    const uint64_t rows = (batch + S::G - 1) / S::G;
    const uint64_t tiles = (rows + S::TS - 1) / S::TS;
    const uint32_t grid = (uint32_t)(tiles < (uint64_t)sms[dev] ? tiles : (uint64_t)sms[dev]);
    k_tc_small<N><<<grid, S::THREADS, S::SMEM, s>>>(x, y, w, batch, err);
    return cudaGetLastError();
}

} // namespace fftb200
