// tc_dft.cuh -- DFT as a split-precision tensor-core GEMM (tcgen05, sm_100a).
//
// FP32 complex rows are transformed as Y = X . W over the real 2N embedding
// (interleaved re/im along K; W holds [cos, -sin | sin, cos] 2x2 blocks, the
// layout of src/fft_c7xmma/FFTLIB_FFT_dftLarge_ixX_cxX_oxX/c71/
// FFTLIB_FFT_dftLarge_ixX_cxX_oxX_ci.cpp:122-138). Both operands are split
// into FP16 hi + lo parts, X after a per-row power-of-two scale, W after a
// fixed 2^12 scale; the three products hi.hi + hi.lo + lo.hi accumulate in
// FP32 in tensor memory. Their sum carries about 22 significant bits of
// every operand, so the result is within a few 1e-7 of the FP64 DFT.
//
// This file holds the shared tcgen05 helpers and the two-stage kernel
// (N = N1 * N2, the reference coordinator's highRadixDecompositions variant,
// src/fft_c7xmma/FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX/
// FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_cn.cpp:20-438, restated here
// as one Cooley-Tukey split); the one-stage kernel for N <= 64 (dftSmall /
// dftLarge) is in tc_dft_small.cuh. With n = N2 n1 + n2 and k = k1 + N1 k2:
//      stage 1 (rows (t, n2), K = n1):  Z[n2][k1] = sum_n1 x[N2 n1 + n2] W_N1^(n1 k1)
//      twiddle (fused into the stage-1 epilogue): Z'[n2][k1] = Z[n2][k1] W_N^(n2 k1)
//      stage 2 (rows (t, k1), K = n2): y[k1 + N1 k2] = sum_n2 Z'[n2][k1] W_N2^(n2 k2)
// The stage-1 epilogue reads the accumulator row of (t, n2) from tensor
// memory, rescales, twiddles, splits and writes it transposed into the
// K-major stage-2 operand in shared memory; the stage-2 epilogue writes
// natural-order output straight to HBM. One persistent CTA per SM walks
// tiles of T transforms (256 rows per stage up to N = 1024, 128 above).
//
// Warp roles: 8 loader warps (HBM -> registers -> scale/split -> swizzled
// shared-memory operand), 8 transposer warps, 4 epilogue warps, and one warp
// whose elected lane allocates tensor memory and issues every tcgen05.mma.
// Hand-offs use mbarriers over NB tile buffers (2 to 8, by shared and tensor
// memory); every wait is bounded and a wait that gives up sets kErrTcTimeout
// in the launch's error word and makes every role leave its loop.
#pragma once

#include <cuda_fp16.h>
#include <stdint.h>

#include "fft_pipeline.cuh"

namespace fftb200 {

constexpr uint32_t kErrTcTimeout = 2u;
constexpr int kTcWShift = 12;  // W is stored as hi/lo of W * 2^12

// ---- tcgen05 / barrier wrappers ----------------------------------------------

FFT_DEV void tmem_alloc(uint32_t* dst, uint32_t cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(cols)
                 : "memory");
}
FFT_DEV void tmem_relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory"); }
FFT_DEV void tmem_dealloc(uint32_t taddr, uint32_t cols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
FFT_DEV void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
FFT_DEV void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
FFT_DEV void tc_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}
// D (+)= A . B, A and B from shared memory, FP16 inputs, FP32 accumulator.
FFT_DEV void tc_mma_f16(uint32_t d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n"
        "  .reg .pred p;\n"
        "  setp.ne.b32 p, %4, 0;\n"
        "  tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n"
        "}\n" ::"r"(d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// 16 consecutive FP32 columns of this thread's tensor-memory lane. The wait
// takes the registers as operands so no use can be scheduled before it.
FFT_DEV void tmem_ld16(uint32_t taddr, float (&f)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])::"memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) f[i] = __uint_as_float(r[i]);
}

FFT_DEV void tmem_ld8(uint32_t taddr, float (&f)[8])
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
                   "+r"(r[7])::"memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = __uint_as_float(r[i]);
}

// Named barrier over `count` threads that also ORs a predicate across them:
// every participant returns the same value.
FFT_DEV bool group_sync_or(uint32_t id, uint32_t count, bool pred)
{
    uint32_t out;
    asm volatile(
        "{\n"
        "  .reg .pred p, q;\n"
        "  setp.ne.u32 q, %1, 0;\n"
        "  bar.red.or.pred p, %2, %3, q;\n"
        "  selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(out)
        : "r"((uint32_t)pred), "r"(id), "r"(count)
        : "memory");
    return out != 0;
}
FFT_DEV void group_sync(uint32_t id, uint32_t count)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Bounded wait that also gives up when another role has aborted. On timeout
// it raises the CTA's abort flag and the launch's error bit.
FFT_DEV bool tc_wait(uint64_t* bar, uint32_t parity, volatile uint32_t* abortFlag, uint32_t* err)
{
    const uint64_t t0 = global_ns();
    for (uint32_t i = 0; i < (1u << 24); ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 63u) == 63u) {
            if (*abortFlag) return false;
            if (global_ns() - t0 > 1000000000ull) break;
        }
    }
    *abortFlag = 1u;
    if (err) atomicOr(err, kErrTcTimeout);
    return false;
}

// ---- operand layouts ------------------------------------------------------------

// Shared-memory descriptor of a K-major, swizzled operand (tcgen05 matrix
// descriptor: start >> 4 at [0,14), leading byte offset >> 4 at [16,30),
// stride byte offset >> 4 at [32,46), version 1 at [46,48), layout type at
// [61,64): 2 = 128-byte swizzle, 4 = 64-byte, 6 = 32-byte).
FFT_DEV uint64_t umma_desc(uint32_t saddr, uint32_t sbo, uint32_t layout)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
           ((uint64_t)1u << 46) | ((uint64_t)layout << 61);
}

// Instruction descriptor: FP32 accumulator, FP16 A and B, both K-major,
// M = 128, N = n.
__host__ __device__ constexpr uint32_t umma_idesc_f16(int n)
{
    return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// R rows of K FP16 values, K-major. Rows are `W` bytes wide inside a swizzle
// atom (W = 128, 64 or 32 bytes; 8 rows form one atom, SBO = 8 W); a row
// wider than 128 bytes continues in further regions of R * 128 bytes. The
// 16-byte chunk j of row r sits at offset ^ (((offset >> 7) & mask) << 4),
// the swizzle the tensor core applies on the absolute address, so the
// operand base must be 1024-byte aligned.
template <int R, int K>
struct KMajor {
    static constexpr int ROWB = 2 * K;
    static constexpr int W = ROWB >= 128 ? 128 : ROWB;
    static_assert(W == 128 || W == 64 || W == 32, "row bytes must be 32, 64 or a multiple of 128");
    static_assert(R % 8 == 0, "rows must be a multiple of 8");
    static constexpr uint32_t REGION = (uint32_t)R * W;
    static constexpr uint32_t MASK = W == 128 ? 7u : (W == 64 ? 3u : 1u);
    static constexpr uint32_t LAYOUT = W == 128 ? 2u : (W == 64 ? 4u : 6u);
    static constexpr uint32_t BYTES = (uint32_t)R * ROWB;

    FFT_DEV static uint32_t chunk(int r, int j)
    {
        const uint32_t kb = (uint32_t)j * 16u;
        const uint32_t off = (kb / W) * REGION + (uint32_t)r * W + (kb % W);
        return off ^ (((off >> 7) & MASK) << 4);
    }
    // rows [128 m, 128 m + 128) (or all rows for a B operand, m = 0), K step s of 16
    FFT_DEV static uint64_t desc(uint32_t base, int m, int s)
    {
        const uint32_t kb = (uint32_t)s * 32u;
        return umma_desc(base + (kb / W) * REGION + (uint32_t)m * 128u * W + (kb % W), 8u * W, LAYOUT);
    }
};

// ---- kernel shape ----------------------------------------------------------------

template <int N1_, int N2_>
struct TcShape {
    static constexpr int N1 = N1_, N2 = N2_;
    static constexpr int N = N1 * N2;
    // transforms per tile: 256 rows per stage up to N = 1024 (short tiles
    // would spend their time in hand-offs), 128 above
    static constexpr int T = (N1 * N2 <= 1024 ? 256 : 128) / (N1 < N2 ? N1 : N2);
    static constexpr int R1 = T * N2;  // stage-1 rows
    static constexpr int R2 = T * N1;  // stage-2 rows
    static constexpr int MB1 = R1 / 128, MB2 = R2 / 128;
    static constexpr int K1 = 2 * N1, K2 = 2 * N2;  // GEMM K (= output columns) per stage
    static constexpr int LW = 8, XW = 8, EW = 4;
    static constexpr int MMA_WARP = LW + XW + EW;
    static constexpr int THREADS = 32 * (MMA_WARP + 1);
    using L1 = KMajor<R1, K1>;
    using L2 = KMajor<R2, K2>;
    using LW1 = KMajor<K1, K1>;
    using LW2 = KMajor<K2, K2>;
    static constexpr bool kSharedW = N1 == N2;
    static constexpr uint32_t HALF_TILE = L1::BYTES;  // one of hi / lo
    static constexpr uint32_t TILE = 2 * HALF_TILE;
    static constexpr uint32_t W1_HALF = LW1::BYTES;
    static constexpr uint32_t W2_HALF = kSharedW ? 0u : LW2::BYTES;
    static constexpr uint32_t D1_COLS = MB1 * K1, D2_COLS = MB2 * K2;
    // tile buffers: as many as shared memory (about 200 KB for tiles and
    // matrices) and tensor memory (512 columns) allow, between 2 and 8
    static constexpr int NB_SMEM = (int)((200u * 1024u - 2u * (W1_HALF + W2_HALF)) / TILE);
    static constexpr int NB_TMEM = (int)(512u / (D1_COLS + D2_COLS));
    static constexpr int NB_MAX = NB_SMEM < NB_TMEM ? NB_SMEM : NB_TMEM;
    static constexpr int NB = NB_MAX > 8 ? 8 : (NB_MAX < 2 ? 2 : NB_MAX);
    static constexpr int TABA = N / 64 + 1, TABB = 64;
    static constexpr uint32_t OFF_W1 = NB * TILE;
    static constexpr uint32_t OFF_W2 = OFF_W1 + 2 * W1_HALF;
    static constexpr uint32_t OFF_TAB = OFF_W2 + 2 * W2_HALF;
    static constexpr uint32_t OFF_S1 = OFF_TAB + 8u * (TABA + TABB);
    static constexpr uint32_t OFF_S2 = OFF_S1 + 4u * 2 * NB * R1;
    static constexpr uint32_t OFF_PART = OFF_S2 + 4u * 2 * NB * T;
    static constexpr uint32_t OFF_LMAX = OFF_PART + 4u * 2 * R1;
    static constexpr uint32_t OFF_BAR = (OFF_LMAX + 4u * 2 * R1 + 7u) & ~7u;
    static constexpr int NBARS = 6 * NB + 1;
    static constexpr uint32_t OFF_MISC = OFF_BAR + 8u * NBARS;
    static constexpr uint32_t SMEM = OFF_MISC + 16u + 1024u;  // + slack to align the base to 1024
    static constexpr uint32_t TMEM_USED = NB * (D1_COLS + D2_COLS);
    static constexpr uint32_t TMEM_COLS =
        TMEM_USED <= 32 ? 32 : TMEM_USED <= 64 ? 64 : TMEM_USED <= 128 ? 128 : TMEM_USED <= 256 ? 256 : 512;
    static_assert(TMEM_USED <= 512, "tensor memory holds 512 columns");
    static_assert(SMEM <= 227u * 1024u, "shared memory per CTA");
    static_assert(K1 >= 16 && K1 <= 256 && K2 >= 16 && K2 <= 256, "MMA N in [16, 256]");
    // the transposer's swizzle constants need the k1 of each half-row group
    // to start at a multiple of 8
    static_assert(N1 >= 16, "N1 >= 16");
    static_assert(R1 % 128 == 0 && R2 % 128 == 0 && R1 <= 256, "rows per stage");
    // barrier indices
    static constexpr int A_FULL = 0, D1_FULL = NB, D1_FREE = 2 * NB, S2_FULL = 3 * NB, D2_FULL = 4 * NB,
                         D2_FREE = 5 * NB, DRAIN = 6 * NB;
};

// ---- small numeric helpers --------------------------------------------------------

FFT_DEV float exp2i(int e) { return __int_as_float((e + 127) << 23); }  // e in [-126, 127]

FFT_DEV int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Power-of-two shift S with max|v| * 2^S in [2^14, 2^15) (clamped to
// [-100, 100]; 0 for an all-zero row).
FFT_DEV int row_shift(float m)
{
    const int e = (int)((__float_as_uint(m) >> 23) & 0xFFu);
    if (e == 0) return m == 0.f ? 0 : 100;
    return clampi(141 - e, -100, 100);
}

FFT_DEV uint32_t h2_bits(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }

// hi = fp16(a, b), lo = fp16(a - hi, b - hi): the differences are exact in FP32.
FFT_DEV void split2(float a, float b, uint32_t& hi, uint32_t& lo)
{
    const __half2 h = __floats2half2_rn(a, b);
    const float2 hf = __half22float2(h);
    hi = h2_bits(h);
    lo = h2_bits(__floats2half2_rn(a - hf.x, b - hf.y));
}

// ---- kernel -----------------------------------------------------------------------

template <class LA, class LB, int MB, int NCOL>
FFT_DEV void issue_split_gemm(uint32_t d, uint32_t aHi, uint32_t aLo, uint32_t bHi, uint32_t bLo)
{
    constexpr uint32_t idesc = umma_idesc_f16(NCOL);
    constexpr int KS = LB::ROWB / 32;  // K steps of 16 values
#pragma unroll
    for (int m = 0; m < MB; ++m) {
        const uint32_t dd = d + (uint32_t)(m * NCOL);
        // the two small cross products first: the accumulator rounds at
        // every update relative to its running value, so only the KS
        // hi.hi updates that come last round at full magnitude
#pragma unroll
        for (int s = 0; s < KS; ++s) tc_mma_f16(dd, LA::desc(aHi, m, s), LB::desc(bLo, 0, s), idesc, s > 0 ? 1u : 0u);
#pragma unroll
        for (int s = 0; s < KS; ++s) tc_mma_f16(dd, LA::desc(aLo, m, s), LB::desc(bHi, 0, s), idesc, 1u);
#pragma unroll
        for (int s = 0; s < KS; ++s) tc_mma_f16(dd, LA::desc(aHi, m, s), LB::desc(bHi, 0, s), idesc, 1u);
    }
}

// Fill the B operand (rows = output index (k, c), K = input index (n, c'))
// of an n-point DFT matrix from its FP32 real embedding wr[(2n+c') * 2n + 2k+c].
template <class LB>
FFT_DEV void fill_dft_operand(unsigned char* hi, unsigned char* lo, const float* __restrict__ wr, int n2x)
{
    const int chunks = n2x * (n2x / 8);
    const float sc = exp2i(kTcWShift);
    for (int it = threadIdx.x; it < chunks; it += blockDim.x) {
        const int row = it / (n2x / 8), j = it % (n2x / 8);
        uint32_t h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float a = __ldg(wr + (size_t)(8 * j + 2 * e) * n2x + row) * sc;
            const float b = __ldg(wr + (size_t)(8 * j + 2 * e + 1) * n2x + row) * sc;
            split2(a, b, h[e], l[e]);
        }
        const uint32_t off = LB::chunk(row, j);
        *reinterpret_cast<uint4*>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
}

template <int N1, int N2>
__global__ void __launch_bounds__(TcShape<N1, N2>::THREADS, 1)
    k_tc_dft(const float2* __restrict__ x, float2* __restrict__ y, const float* __restrict__ w, uint32_t batch,
             uint32_t* err)
{
    using S = TcShape<N1, N2>;
    constexpr int N = S::N, T = S::T, NB = S::NB;
    extern __shared__ unsigned char tc_smem_raw[];
    unsigned char* sm = tc_smem_raw + ((1024u - (smem_addr(tc_smem_raw) & 1023u)) & 1023u);
    const uint32_t sbase = smem_addr(sm);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + S::OFF_BAR);
    uint32_t* misc = reinterpret_cast<uint32_t*>(sm + S::OFF_MISC);  // [0] tensor memory base, [1] abort
    volatile uint32_t* abortFlag = misc + 1;
    int* s1ring = reinterpret_cast<int*>(sm + S::OFF_S1);
    int* s2ring = reinterpret_cast<int*>(sm + S::OFF_S2);
    int* part = reinterpret_cast<int*>(sm + S::OFF_PART);
    float* lmax = reinterpret_cast<float*>(sm + S::OFF_LMAX);
    float2* tabA = reinterpret_cast<float2*>(sm + S::OFF_TAB);
    float2* tabB = tabA + S::TABA;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t numTiles = (batch + T - 1) / T;

    // ---- set-up: barriers, tensor memory, DFT operands, twiddle tables
    if (threadIdx.x == 0) {
        for (int i = 0; i < S::NBARS; ++i) mbar_init(&bars[i], 1);
        misc[1] = 0;
        fence_mbarrier_init();
    }
    if (warp == S::MMA_WARP) {
        tmem_alloc(&misc[0], S::TMEM_COLS);
        tmem_relinquish();
    }
    fill_dft_operand<typename S::LW1>(sm + S::OFF_W1, sm + S::OFF_W1 + S::W1_HALF, w, S::K1);
    {
        const float* w2 = w + (size_t)S::K1 * S::K1;
        if constexpr (!S::kSharedW)
            fill_dft_operand<typename S::LW2>(sm + S::OFF_W2, sm + S::OFF_W2 + S::W2_HALF, w2, S::K2);
        const float2* tw = reinterpret_cast<const float2*>(w2 + (size_t)S::K2 * S::K2);
        for (int i = threadIdx.x; i < S::TABA + S::TABB; i += blockDim.x)
            tabA[i] = i < S::TABA ? tw[(64 * i) % N] : tw[i - S::TABA];
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = misc[0];

    if (warp < S::LW) {
        // ================= loaders: HBM -> scale -> hi/lo operand =================
        const int j = threadIdx.x;  // 0..255
        // the next tile's input (contiguous) is pulled into L2 while this one
        // is converted, so its loads do not wait a full HBM latency
        auto prefetch = [&](uint32_t tl) {
            if (j != 0 || tl >= numTiles) return;
            const uint32_t first = tl * (uint32_t)T;
            const uint32_t cnt = min((uint32_t)T, batch - first);
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(x + (size_t)first * N),
                         "r"(cnt * (uint32_t)N * 8u)
                         : "memory");
        };
        prefetch(blockIdx.x);
        uint32_t i = 0;
        for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++i) {
            prefetch(tile + gridDim.x);
            const int b = (int)(i % NB);
            const uint32_t u = i / NB, slot = i % (2 * NB);
            unsigned char* hiB = sm + b * S::TILE;
            unsigned char* loB = hiB + S::HALF_TILE;
            {
                constexpr int H = 256 / S::R1;  // threads per row
                constexpr int CPH = N1 / H;     // complex values per thread
                constexpr int NCH = CPH / 4;    // 16-byte chunks per thread
                // a warp covers 32 consecutive rows and one half of K, so its
                // loads are 256-byte runs and its stores hit distinct banks
                const int h = H == 2 ? (warp & 1) : 0;
                const int r = H == 2 ? (warp >> 1) * 32 + lane : j;
                const int t = r / N2, n2 = r % N2;
                const uint32_t gt = tile * (uint32_t)T + (uint32_t)t;
                float2 v[CPH];
                if (gt < batch) {
                    const float2* src = x + (size_t)gt * N + n2 + (size_t)N2 * h * CPH;
#pragma unroll
                    for (int s = 0; s < CPH; ++s) v[s] = __ldg(src + (size_t)s * N2);
                } else {
#pragma unroll
                    for (int s = 0; s < CPH; ++s) v[s] = make_float2(0.f, 0.f);
                }
                float m = 0.f;
#pragma unroll
                for (int s = 0; s < CPH; ++s) m = fmaxf(m, fmaxf(fabsf(v[s].x), fabsf(v[s].y)));
                if (H == 2) lmax[h * S::R1 + r] = m;
                bool bad = false;
                if (u >= 1 && j == 0) bad = !tc_wait(&bars[S::D2_FULL + b], (u - 1) & 1u, abortFlag, err);
                if (group_sync_or(1, 32 * S::LW, bad)) break;
                if (H == 2) m = fmaxf(m, lmax[(h ^ 1) * S::R1 + r]);
                const int sh = row_shift(m);
                const float sc = exp2i(sh);
#pragma unroll
                for (int c = 0; c < NCH; ++c) {
                    uint32_t hh[4], ll[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) split2(v[4 * c + e].x * sc, v[4 * c + e].y * sc, hh[e], ll[e]);
                    const uint32_t off = S::L1::chunk(r, (h * CPH) / 4 + c);
                    *reinterpret_cast<uint4*>(hiB + off) = make_uint4(hh[0], hh[1], hh[2], hh[3]);
                    *reinterpret_cast<uint4*>(loB + off) = make_uint4(ll[0], ll[1], ll[2], ll[3]);
                }
                if (h == 0) s1ring[slot * S::R1 + r] = sh;
            }
            fence_proxy_async_smem();
            group_sync(1, 32 * S::LW);
            if (j == 0) mbar_arrive(&bars[S::A_FULL + b]);
        }
    } else if (warp == S::MMA_WARP) {
        // ================= MMA issue (one lane) =================
        if (lane == 0) {
            uint32_t count = 0;
            for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x) ++count;
            auto stage1 = [&](uint32_t i) -> bool {
                const int b = (int)(i % NB);
                const uint32_t u = i / NB;
                if (!tc_wait(&bars[S::A_FULL + b], u & 1u, abortFlag, err)) return false;
                if (u >= 1 && !tc_wait(&bars[S::D1_FREE + b], (u - 1) & 1u, abortFlag, err)) return false;
                tc_fence_after();
                const uint32_t a = sbase + b * S::TILE;
                issue_split_gemm<typename S::L1, typename S::LW1, S::MB1, S::K1>(
                    tmem + b * S::D1_COLS, a, a + S::HALF_TILE, sbase + S::OFF_W1, sbase + S::OFF_W1 + S::W1_HALF);
                tc_commit(&bars[S::D1_FULL + b]);
                return true;
            };
            auto stage2 = [&](uint32_t i) -> bool {
                const int b = (int)(i % NB);
                const uint32_t u = i / NB;
                if (!tc_wait(&bars[S::S2_FULL + b], u & 1u, abortFlag, err)) return false;
                if (u >= 1 && !tc_wait(&bars[S::D2_FREE + b], (u - 1) & 1u, abortFlag, err)) return false;
                tc_fence_after();
                const uint32_t a = sbase + b * S::TILE;
                const uint32_t wb = S::kSharedW ? sbase + S::OFF_W1 : sbase + S::OFF_W2;
                const uint32_t wl = S::kSharedW ? wb + S::W1_HALF : wb + S::W2_HALF;
                issue_split_gemm<typename S::L2, typename S::LW2, S::MB2, S::K2>(
                    tmem + NB * S::D1_COLS + b * S::D2_COLS, a, a + S::HALF_TILE, wb, wl);
                tc_commit(&bars[S::D2_FULL + b]);
                return true;
            };
            bool ok = count == 0 || stage1(0);
            for (uint32_t i = 0; ok && i < count; ++i) {
                if (i + 1 < count) ok = stage1(i + 1);
                if (ok) ok = stage2(i);
            }
            // wait for every MMA issued above before tensor memory is released
            tc_commit(&bars[S::DRAIN]);
            mbar_wait_bounded(&bars[S::DRAIN], 0);
        }
        __syncwarp();
    } else if (warp < S::LW + S::XW) {
        // ================= transposers: D1 -> twiddle -> stage-2 operand =================
        {
            const int xt = threadIdx.x - 32 * S::LW;  // 0..255
            const int q = warp & 3, ch = (warp - S::LW) >> 2;
            constexpr int HC = S::K1 / 2;  // accumulator columns per half
            constexpr int CW = HC >= 16 ? 16 : 8;
            constexpr int SEG = N2 < 32 ? N2 : 32;
            const uint32_t laneBase = (uint32_t)(32 * q) << 16;
            uint32_t i = 0;
            for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++i) {
                const int b = (int)(i % NB);
                const uint32_t u = i / NB, slot = i % (2 * NB);
                bool bad = false;
                if (xt == 0) bad = !tc_wait(&bars[S::D1_FULL + b], u & 1u, abortFlag, err);
                if (group_sync_or(2, 32 * S::XW, bad)) break;
                tc_fence_after();
                const uint32_t dcol = tmem + laneBase + b * S::D1_COLS;
                // pass 1: per-row maxima -> per-transform stage-2 shift
#pragma unroll
                for (int m = 0; m < S::MB1; ++m) {
                    const int row = m * 128 + 32 * q + lane;
                    float pm = 0.f;
#pragma unroll
                    for (int c0 = 0; c0 < HC; c0 += CW) {
                        float f[CW];
                        if constexpr (CW == 16)
                            tmem_ld16(dcol + m * S::K1 + ch * HC + c0, f);
                        else
                            tmem_ld8(dcol + m * S::K1 + ch * HC + c0, f);
#pragma unroll
                        for (int e = 0; e < CW; ++e) pm = fmaxf(pm, fabsf(f[e]));
                    }
                    const int eRaw = (int)((__float_as_uint(pm) >> 23) & 0xFFu);
                    int ez = pm > 0.f ? eRaw - s1ring[slot * S::R1 + row] : -100000;
                    // rows of one transform are SEG-lane segments of the warp
#pragma unroll
                    for (int o = SEG / 2; o >= 1; o >>= 1) ez = max(ez, __shfl_xor_sync(0xffffffffu, ez, o));
                    if ((lane & (SEG - 1)) == 0) part[ch * (S::R1 / SEG) + row / SEG] = ez;
                }
                group_sync(2, 32 * S::XW);
                for (int tt = xt; tt < T; tt += 32 * S::XW) {
                    int E = -100000;
#pragma unroll
                    for (int sg = 0; sg < N2 / SEG; ++sg) {
                        const int id = tt * (N2 / SEG) + sg;
                        E = max(E, max(part[id], part[S::R1 / SEG + id]));
                    }
                    s2ring[slot * T + tt] = E < -50000 ? 0 : clampi(141 - E + kTcWShift, -100, 100);
                }
                group_sync(2, 32 * S::XW);
                // pass 2: rescale, twiddle, split, write transposed. Row r2 =
                // t N1 + k1 of the stage-2 operand gets (re, im) of Z' at K
                // position 2 n2. Within a group of 8 consecutive k1 (r2 = 8j+e)
                // the swizzle term is a constant of e, and the twiddles
                // W_N^(n2 k1) follow from one table product by the
                // recurrence w <- w W_N^n2 (the power-of-two rescale rides on
                // the first factor).
                using L2 = typename S::L2;
                unsigned char* hiB = sm + b * S::TILE;
                unsigned char* loB = hiB + S::HALF_TILE;
#pragma unroll
                for (int m = 0; m < S::MB1; ++m) {
                    const int row = m * 128 + 32 * q + lane;
                    const int t = row / N2, n2 = row % N2;
                    const int s2 = s2ring[slot * T + t];
                    const float f = exp2i(clampi(s2 - s1ring[slot * S::R1 + row] - kTcWShift, -126, 126));
                    const float2 step = tabB[n2];  // W_N^n2 (n2 < 64)
                    const uint32_t kbytes = (uint32_t)(n2 >> 2) * 16u;
                    const uint32_t colOff = kbytes % L2::W;
                    const uint32_t rowOff = (kbytes / L2::W) * L2::REGION + (uint32_t)(n2 & 3) * 4u;
#pragma unroll
                    for (int c0 = 0; c0 < HC; c0 += CW) {
                        float v[CW];
                        if constexpr (CW == 16)
                            tmem_ld16(dcol + m * S::K1 + ch * HC + c0, v);
                        else
                            tmem_ld8(dcol + m * S::K1 + ch * HC + c0, v);
                        const int kbase = (ch * HC + c0) / 2;  // multiple of 8
                        const uint32_t base = rowOff + (uint32_t)(t * N1 + kbase) * L2::W;
                        float wr = 0.f, wi = 0.f;
#pragma unroll
                        for (int e = 0; e < CW / 2; ++e) {
                            if ((e & 3) == 0) {  // re-anchor every 4: at most 3 recurrence steps
                                const int ex = n2 * (kbase + e);
                                const float2 ta = tabA[ex >> 6], tb = tabB[ex & 63];
                                wr = (ta.x * tb.x - ta.y * tb.y) * f;
                                wi = (ta.x * tb.y + ta.y * tb.x) * f;
                            } else {
                                const float nr = wr * step.x - wi * step.y;
                                wi = wr * step.y + wi * step.x;
                                wr = nr;
                            }
                            const float zr = v[2 * e], zi = v[2 * e + 1];
                            uint32_t hh, ll;
                            split2(zr * wr - zi * wi, zr * wi + zi * wr, hh, ll);
                            const uint32_t swz = ((((uint32_t)e * L2::W) >> 7) & L2::MASK) << 4;
                            const uint32_t off = base + (uint32_t)e * L2::W + (colOff ^ swz);
                            *reinterpret_cast<uint32_t*>(hiB + off) = hh;
                            *reinterpret_cast<uint32_t*>(loB + off) = ll;
                        }
                    }
                }
                fence_proxy_async_smem();
                tc_fence_before();
                group_sync(2, 32 * S::XW);
                if (xt == 0) {
                    mbar_arrive(&bars[S::D1_FREE + b]);
                    mbar_arrive(&bars[S::S2_FULL + b]);
                }
            }
        }
    } else {
        // ================= epilogue: accumulator -> unscale -> HBM =================
        const int et = threadIdx.x - 32 * (S::LW + S::XW);
        const int q = warp & 3;
        const uint32_t laneBase = (uint32_t)(32 * q) << 16;
        uint32_t i = 0;
        for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++i) {
            const int b = (int)(i % NB);
            const uint32_t u = i / NB, slot = i % (2 * NB);
            const int fullBar = S::D2_FULL;
            const int freeBar = S::D2_FREE;
            bool bad = false;
            if (et == 0) bad = !tc_wait(&bars[fullBar + b], u & 1u, abortFlag, err);
            if (group_sync_or(3, 32 * S::EW, bad)) break;
            tc_fence_after();
            {
                constexpr int CW = S::K2 >= 16 ? 16 : 8;
#pragma unroll
                for (int m = 0; m < S::MB2; ++m) {
                    const int row = m * 128 + 32 * q + lane;
                    const int t = row / N1, k1 = row % N1;
                    const uint32_t gt = tile * (uint32_t)T + (uint32_t)t;
                    const float f = exp2i(-(s2ring[slot * T + t] + kTcWShift));
                    const uint32_t dcol = tmem + laneBase + NB * S::D1_COLS + b * S::D2_COLS + m * S::K2;
#pragma unroll
                    for (int c0 = 0; c0 < S::K2; c0 += CW) {
                        float v[CW];
                        if constexpr (CW == 16)
                            tmem_ld16(dcol + c0, v);
                        else
                            tmem_ld8(dcol + c0, v);
                        if (gt < batch) {
                            float2* dst = y + (size_t)gt * N + k1 + (size_t)N1 * (c0 / 2);
#pragma unroll
                            for (int e = 0; e < CW / 2; ++e)
                                dst[(size_t)N1 * e] = make_float2(v[2 * e] * f, v[2 * e + 1] * f);
                        }
                    }
                }
            }
            tc_fence_before();
            group_sync(3, 32 * S::EW);
            if (et == 0) mbar_arrive(&bars[freeBar + b]);
        }
    }

    // ---- tear-down
    tc_fence_before();
    __syncthreads();
    if (warp == S::MMA_WARP) {
        tc_fence_after();
        tmem_dealloc(tmem, S::TMEM_COLS);
    }
}

}  // namespace fftb200
