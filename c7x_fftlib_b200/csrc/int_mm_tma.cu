// int_mm_tma.cu -- the LINALG INT8 and INT16 multiplies C = round_shift(A B)
// on the tensor cores with their operand tiles brought in by the Tensor
// Memory Accelerator, bit-exact with the reference's natural C
// (src/linalg_c7xmma/FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX/
// FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_cn.cpp:27-62).
//
// One thread issues, per chunk of 128 K values, two 2-D tiled bulk tensor
// copies with 128-byte swizzle into a ring of six shared-memory stages: the
// A tile (128 rows of C x 128 bytes of K, K-major) and the B tile (128 K rows
// x 128 bytes of N, MN-major, the layout B has in memory). Both land in the
// canonical swizzled layouts the MMA reads; the copies zero-fill outside the
// matrices, which adds nothing to the sums. One thread issues the MMAs
// (signed 8-bit, S32 accumulators), 4 epilogue warps turn the accumulators
// into shift-rounded, saturated bytes. Every wait is bounded; a wait that
// gives up sets kErrTcTimeout in the launch's error word, and the copy
// thread waits (bounded) for its copies in flight before the CTA ends.
#include <cuda.h>

#include <mutex>

#include "dft_int.h"
#include "int_arith.cuh"
#include "plan.h"
#include "tc_dft.cuh"

namespace fftb200 {

namespace {

struct MmTma {
    static constexpr int BN = 128;
    static constexpr int NS = 6;  // K-chunk stages
    static constexpr int NA = 2;  // accumulator buffers
    static constexpr int TMA_WARP = 0, MMA_WARP = 1, EPI0 = 2, EW = 4;
    static constexpr int THREADS = 32 * (EPI0 + EW);
    using LT = KMajor<128, 64>;  // 128 rows of 128 bytes, 128-byte swizzle
    static constexpr uint32_t TILE = LT::BYTES;  // 16 KB
    static constexpr uint32_t STAGE = 2 * TILE;  // A then B
    static constexpr uint32_t OFF_BAR = NS * STAGE;
    static constexpr int NBARS = 2 * NS + 2 * NA + 1;
    static constexpr uint32_t OFF_MISC = OFF_BAR + 8u * NBARS;
    static constexpr uint32_t SMEM = OFF_MISC + 16u + 1024u;
    static constexpr uint32_t TMEM_COLS = 256;
    static constexpr int FULL = 0, EMPTY = NS, AFULL = 2 * NS, AEMPTY = 2 * NS + NA, DRAIN = 2 * NS + 2 * NA;
    static_assert(NA * BN <= (int)TMEM_COLS, "tensor memory");
    static_assert(SMEM <= 227u * 1024u, "shared memory per CTA");
};

struct TmaArgs {
    void* c;
    size_t ldc;
    uint32_t M, K, N;
    uint32_t shift;
    uint32_t tilesN, numTiles, chunks;
    uint32_t* err;
};

FFT_DEV void tma_load_2d(void* dst, const CUtensorMap* map, int32_t x, int32_t y, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

FFT_DEV void tc_mma_s8(uint32_t d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n"
        "  .reg .pred p;\n"
        "  setp.ne.b32 p, %4, 0;\n"
        "  tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n"
        "}\n" ::"r"(d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

FFT_DEV void tmem_ld16_acc(uint32_t taddr, int32_t (&v)[16])
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
    for (int i = 0; i < 16; ++i) v[i] = (int32_t)r[i];
}

__global__ void __launch_bounds__(MmTma::THREADS, 1)
    k_int8_mm_tma(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, TmaArgs p)
{
    using S = MmTma;
    constexpr int NS = S::NS, NA = S::NA, BN = S::BN;
    extern __shared__ unsigned char mm_tma_smem_raw[];
    unsigned char* sm = mm_tma_smem_raw + ((1024u - (smem_addr(mm_tma_smem_raw) & 1023u)) & 1023u);
    const uint32_t sbase = smem_addr(sm);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + S::OFF_BAR);
    uint32_t* misc = reinterpret_cast<uint32_t*>(sm + S::OFF_MISC);
    volatile uint32_t* abortFlag = misc + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int8_t* Cm = static_cast<int8_t*>(p.c);

    if (threadIdx.x == 0) {
        for (int i = 0; i < S::NBARS; ++i) mbar_init(&bars[i], 1);
        misc[1] = 0;
        fence_mbarrier_init();
    }
    if (warp == S::MMA_WARP) {
        tmem_alloc(&misc[0], S::TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = misc[0];
    const uint32_t myTiles = blockIdx.x < p.numTiles ? (p.numTiles - 1u - blockIdx.x) / gridDim.x + 1u : 0u;
    const uint32_t total = myTiles * p.chunks;

    if (warp == S::TMA_WARP) {
        // ================= tile copies =================
        if (lane == 0) {
            uint32_t g = 0;
            for (; g < total; ++g) {
                const int st = (int)(g % NS);
                const uint32_t u = g / NS;
                if (u >= 1 && !tc_wait(&bars[S::EMPTY + st], (u - 1) & 1u, abortFlag, p.err)) break;
                const uint32_t ti = g / p.chunks, ch = g - ti * p.chunks;
                const uint32_t tile = blockIdx.x + ti * gridDim.x;
                const int32_t m0 = (int32_t)((tile / p.tilesN) * 128u), n0 = (int32_t)((tile % p.tilesN) * (uint32_t)BN);
                const int32_t k0 = (int32_t)(ch * 128u);
                unsigned char* a = sm + st * S::STAGE;
                mbar_expect_tx(&bars[S::FULL + st], S::STAGE);
                tma_load_2d(a, &tmA, k0, m0, &bars[S::FULL + st]);
                tma_load_2d(a + S::TILE, &tmB, n0, k0, &bars[S::FULL + st]);
            }
            // the copies still in flight land before the CTA ends: the last
            // phase armed on each stage (complete already on the normal path)
            for (int st = 0; st < NS; ++st) {
                const uint32_t armed = g > (uint32_t)st ? (g - 1u - (uint32_t)st) / NS + 1u : 0u;
                if (armed) mbar_wait_bounded(&bars[S::FULL + st], (armed - 1u) & 1u);
            }
        }
        __syncwarp();
    } else if (warp == S::MMA_WARP) {
        // ================= MMA issue =================
        if (lane == 0) {
            // signed 8-bit A and B, S32 accumulator, M = 128, N = 128, B MN-major
            constexpr uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | (1u << 16) |
                                       ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
            constexpr int KS = 128 / 32;
            uint32_t g = 0;
            bool stop = false;
            for (uint32_t ti = 0; ti < myTiles && !stop; ++ti) {
                const int a = (int)(ti % NA);
                const uint32_t ua = ti / NA;
                if (ua >= 1 && !tc_wait(&bars[S::AEMPTY + a], (ua - 1) & 1u, abortFlag, p.err)) break;
                const uint32_t d = tmem + (uint32_t)a * BN;
                for (uint32_t ch = 0; ch < p.chunks; ++ch, ++g) {
                    const int st = (int)(g % NS);
                    const uint32_t u = g / NS;
                    if (!tc_wait(&bars[S::FULL + st], u & 1u, abortFlag, p.err)) {
                        stop = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t aA = sbase + st * S::STAGE, aB = aA + S::TILE;
                    // K step of 32: 32 bytes along the K-major A rows, 4 atoms
                    // of 8 rows x 128 bytes of the MN-major B
#pragma unroll
                    for (int s = 0; s < KS; ++s)
                        tc_mma_s8(d, S::LT::desc(aA, 0, s), umma_desc(aB + 4096u * (uint32_t)s, 1024u, 2u), idesc,
                                  (ch > 0 || s > 0) ? 1u : 0u);
                    tc_commit(&bars[S::EMPTY + st]);
                }
                if (stop) break;
                tc_commit(&bars[S::AFULL + a]);
            }
            tc_commit(&bars[S::DRAIN]);
            mbar_wait_bounded(&bars[S::DRAIN], 0);
        }
        __syncwarp();
    } else {
        // ================= epilogue =================
        const int et = threadIdx.x - 32 * S::EPI0;  // 0..127
        const int q = warp & 3;
        const uint32_t laneBase = (uint32_t)(32 * q) << 16;
        for (uint32_t ti = 0; ti < myTiles; ++ti) {
            const int a = (int)(ti % NA);
            const uint32_t ua = ti / NA;
            bool bad = false;
            if (et == 0) bad = !tc_wait(&bars[S::AFULL + a], ua & 1u, abortFlag, p.err);
            if (group_sync_or(3, 32 * S::EW, bad)) break;
            tc_fence_after();
            const uint32_t tile = blockIdx.x + ti * gridDim.x;
            const uint32_t m0 = (tile / p.tilesN) * 128u, n0 = (tile % p.tilesN) * (uint32_t)BN;
            const uint32_t m = m0 + (uint32_t)(32 * q + lane);
            const uint32_t dbase = tmem + laneBase + (uint32_t)a * BN;
            int8_t* crow = Cm + (size_t)m * p.ldc + n0;
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 16) {
                int32_t acc[16];
                tmem_ld16_acc(dbase + (uint32_t)c0, acc);
                uint32_t wv[4] = {0u, 0u, 0u, 0u};
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    wv[e >> 2] |= (uint32_t)(uint8_t)shift_round<int8_t>(acc[e], p.shift) << (8 * (e & 3));
                if (m < p.M) {
                    int8_t* dst = crow + c0;
                    if (n0 + (uint32_t)c0 + 16u <= p.N && ((uintptr_t)dst & 15u) == 0) {
                        *reinterpret_cast<uint4*>(dst) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
                    } else {
#pragma unroll
                        for (int e = 0; e < 16; ++e)
                            if (n0 + (uint32_t)(c0 + e) < p.N) dst[e] = (int8_t)(wv[e >> 2] >> (8 * (e & 3)));
                    }
                }
            }
            tc_fence_before();
            group_sync(3, 32 * S::EW);
            if (et == 0) mbar_arrive(&bars[S::AEMPTY + a]);
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == S::MMA_WARP) {
        tc_fence_after();
        tmem_dealloc(tmem, S::TMEM_COLS);
    }
}

// INT16: the raw tiles (A 128 rows x 128 values, B 128 K rows x 64 values,
// no swizzle) land in a ring of raw stages; 8 converter warps turn each into
// the offset-binary byte limbs (A K-major, B MN-major, swizzled) of a ring of
// operand stages and form the row and column sums; the MMA and epilogue are
// those of k_int_mm_tc<true>.
struct Mm16Tma {
    static constexpr int BN = 64;
    static constexpr int NR = 2, NS = 2, NA = 2, RS = 8;
    static constexpr int TMA_WARP = 0, MMA_WARP = 1, CV0 = 2, CW = 8, EPI0 = CV0 + CW, EW = 4;
    static constexpr int THREADS = 32 * (EPI0 + EW);
    using LA = KMajor<128, 64>;   // A limb: 128 rows of 128 bytes (128-byte swizzle)
    using LBM = KMajor<128, 32>;  // B limb, MN-major: 128 K rows of 64 bytes (64-byte swizzle)
    static constexpr uint32_t RAW_A = 128u * 128u * 2u;  // 32 KB
    static constexpr uint32_t RAW_B = 128u * 64u * 2u;   // 16 KB
    static constexpr uint32_t RAW = RAW_A + RAW_B;
    static constexpr uint32_t A_LIMB = LA::BYTES, B_LIMB = LBM::BYTES;
    static constexpr uint32_t LIMB_PAIR = A_LIMB + B_LIMB;
    static constexpr uint32_t STAGE = 2 * LIMB_PAIR;  // A hi, B hi, A lo, B lo
    static constexpr uint32_t OFF_ST = NR * RAW;
    static constexpr uint32_t OFF_RS = OFF_ST + NS * STAGE;
    static constexpr uint32_t OFF_CP = OFF_RS + 4u * RS * 128u;
    static constexpr uint32_t OFF_CS = OFF_CP + 4u * CW * BN;
    static constexpr uint32_t OFF_BAR = (OFF_CS + 4u * RS * BN + 7u) & ~7u;
    static constexpr int NBARS = 2 * NR + 2 * NS + 2 * NA + 1;
    static constexpr uint32_t OFF_MISC = OFF_BAR + 8u * NBARS;
    static constexpr uint32_t SMEM = OFF_MISC + 16u + 1024u;
    static constexpr uint32_t ACC = 3u * BN;
    static constexpr uint32_t TMEM_COLS = 512;
    static constexpr int RFULL = 0, REMPTY = NR, FULL = 2 * NR, EMPTY = 2 * NR + NS, AFULL = 2 * NR + 2 * NS,
                         AEMPTY = AFULL + NA, DRAIN = AEMPTY + NA;
    static_assert(NA * ACC <= TMEM_COLS, "tensor memory");
    static_assert(NR + NS + NA <= RS, "sum slots");
    static_assert(SMEM <= 227u * 1024u, "shared memory per CTA");
    static_assert(RAW % 1024u == 0 && A_LIMB % 1024u == 0 && B_LIMB % 1024u == 0, "1024-byte aligned stages");
};

__global__ void __launch_bounds__(Mm16Tma::THREADS, 1)
    k_int16_mm_tma(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, TmaArgs p)
{
    using S = Mm16Tma;
    constexpr int NR = S::NR, NS = S::NS, NA = S::NA, RS = S::RS, BN = S::BN;
    extern __shared__ unsigned char mm16_tma_smem_raw[];
    unsigned char* sm = mm16_tma_smem_raw + ((1024u - (smem_addr(mm16_tma_smem_raw) & 1023u)) & 1023u);
    const uint32_t sbase = smem_addr(sm);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + S::OFF_BAR);
    uint32_t* misc = reinterpret_cast<uint32_t*>(sm + S::OFF_MISC);
    volatile uint32_t* abortFlag = misc + 1;
    int32_t* rowsum = reinterpret_cast<int32_t*>(sm + S::OFF_RS);
    int32_t* cpart = reinterpret_cast<int32_t*>(sm + S::OFF_CP);
    int32_t* colsum = reinterpret_cast<int32_t*>(sm + S::OFF_CS);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int16_t* Cm = static_cast<int16_t*>(p.c);

    if (threadIdx.x == 0) {
        for (int i = 0; i < S::NBARS; ++i) mbar_init(&bars[i], 1);
        misc[1] = 0;
        fence_mbarrier_init();
    }
    if (warp == S::MMA_WARP) {
        tmem_alloc(&misc[0], S::TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = misc[0];
    const uint32_t myTiles = blockIdx.x < p.numTiles ? (p.numTiles - 1u - blockIdx.x) / gridDim.x + 1u : 0u;
    const uint32_t total = myTiles * p.chunks;

    if (warp == S::TMA_WARP) {
        // ================= raw tile copies =================
        if (lane == 0) {
            uint32_t g = 0;
            for (; g < total; ++g) {
                const int r = (int)(g % NR);
                const uint32_t u = g / NR;
                if (u >= 1 && !tc_wait(&bars[S::REMPTY + r], (u - 1) & 1u, abortFlag, p.err)) break;
                const uint32_t ti = g / p.chunks, ch = g - ti * p.chunks;
                const uint32_t tile = blockIdx.x + ti * gridDim.x;
                const int32_t m0 = (int32_t)((tile / p.tilesN) * 128u), n0 = (int32_t)((tile % p.tilesN) * (uint32_t)BN);
                const int32_t k0 = (int32_t)(ch * 128u);
                unsigned char* raw = sm + r * S::RAW;
                mbar_expect_tx(&bars[S::RFULL + r], S::RAW);
                tma_load_2d(raw, &tmA, k0, m0, &bars[S::RFULL + r]);
                tma_load_2d(raw + S::RAW_A, &tmB, n0, k0, &bars[S::RFULL + r]);
            }
            for (int r = 0; r < NR; ++r) {
                const uint32_t armed = g > (uint32_t)r ? (g - 1u - (uint32_t)r) / NR + 1u : 0u;
                if (armed) mbar_wait_bounded(&bars[S::RFULL + r], (armed - 1u) & 1u);
            }
        }
        __syncwarp();
    } else if (warp >= S::CV0 && warp < S::EPI0) {
        // ================= conversion to offset-binary limbs =================
        const int tid = threadIdx.x - 32 * S::CV0;  // 0..255
        const int cw = warp - S::CV0;
        int32_t rs[8], cs[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) rs[e] = cs[e] = 0;
        for (uint32_t g = 0; g < total; ++g) {
            const int r = (int)(g % NR), st = (int)(g % NS);
            const uint32_t ur = g / NR, u = g / NS;
            const uint32_t ti = g / p.chunks, ch = g - ti * p.chunks;
            bool bad = false;
            if (tid == 0) {
                bad = !tc_wait(&bars[S::RFULL + r], ur & 1u, abortFlag, p.err);
                if (!bad && u >= 1) bad = !tc_wait(&bars[S::EMPTY + st], (u - 1) & 1u, abortFlag, p.err);
            }
            if (group_sync_or(1, 32 * S::CW, bad)) break;
            if (ch == 0u) {
#pragma unroll
                for (int e = 0; e < 8; ++e) rs[e] = cs[e] = 0;
            }
            const unsigned char* rawA = sm + r * S::RAW;
            const unsigned char* rawB = rawA + S::RAW_A;
            unsigned char* aHi = sm + S::OFF_ST + st * S::STAGE;
            unsigned char* bHi = aHi + S::A_LIMB;
            unsigned char* aLo = aHi + S::LIMB_PAIR;
            unsigned char* bLo = bHi + S::LIMB_PAIR;
            // A: 16 pieces of 8 values per 256-byte row; 16 lanes read a row
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int it = tid + 256 * q;
                const int row = it >> 4, j = it & 15;
                const uint4 v = *reinterpret_cast<const uint4*>(rawA + row * 256 + j * 16);
                const uint32_t a0 = v.x ^ 0x80008000u, a1 = v.y ^ 0x80008000u;
                const uint32_t a2 = v.z ^ 0x80008000u, a3 = v.w ^ 0x80008000u;
                const uint32_t h0 = __byte_perm(a0, a1, 0x7531u), h1 = __byte_perm(a2, a3, 0x7531u);
                const uint32_t l0 = __byte_perm(a0, a1, 0x6420u), l1 = __byte_perm(a2, a3, 0x6420u);
                rs[q] += (int32_t)(256u * (__dp4a(h0, 0x01010101u, 0u) + __dp4a(h1, 0x01010101u, 0u)) +
                                   __dp4a(l0, 0x01010101u, 0u) + __dp4a(l1, 0x01010101u, 0u));
                const uint32_t off = S::LA::chunk(row, j >> 1) + (uint32_t)(j & 1) * 8u;
                *reinterpret_cast<uint2*>(aHi + off) = make_uint2(h0, h1);
                *reinterpret_cast<uint2*>(aLo + off) = make_uint2(l0, l1);
            }
            // B: 8 pieces of 8 values per 128-byte K row; a thread's pieces are
            // always columns 8 (tid & 7) .. + 7
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int it = tid + 256 * q;
                const int row = it >> 3, j = it & 7;
                const uint4 v = *reinterpret_cast<const uint4*>(rawB + row * 128 + j * 16);
                const uint32_t w[4] = {v.x ^ 0x80008000u, v.y ^ 0x80008000u, v.z ^ 0x80008000u, v.w ^ 0x80008000u};
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    cs[2 * e] += (int32_t)(w[e] & 0xFFFFu);
                    cs[2 * e + 1] += (int32_t)(w[e] >> 16);
                }
                const uint32_t h0 = __byte_perm(w[0], w[1], 0x7531u), h1 = __byte_perm(w[2], w[3], 0x7531u);
                const uint32_t l0 = __byte_perm(w[0], w[1], 0x6420u), l1 = __byte_perm(w[2], w[3], 0x6420u);
                const uint32_t off = S::LBM::chunk(row, j >> 1) + (uint32_t)(j & 1) * 8u;
                *reinterpret_cast<uint2*>(bHi + off) = make_uint2(h0, h1);
                *reinterpret_cast<uint2*>(bLo + off) = make_uint2(l0, l1);
            }
            if (ch + 1u == p.chunks) {
                // the tile's sums: rows over the 16 lanes that read them, columns
                // over lanes l, l ^ 8, l ^ 16, l ^ 24 and then the 8 warps
                const int slot = (int)(ti % RS);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    int32_t t = rs[q];
                    t += __shfl_xor_sync(0xffffffffu, t, 1);
                    t += __shfl_xor_sync(0xffffffffu, t, 2);
                    t += __shfl_xor_sync(0xffffffffu, t, 4);
                    t += __shfl_xor_sync(0xffffffffu, t, 8);
                    if ((tid & 15) == 0) rowsum[slot * 128 + ((tid + 256 * q) >> 4)] = t;
                }
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    cs[e] += __shfl_xor_sync(0xffffffffu, cs[e], 8);
                    cs[e] += __shfl_xor_sync(0xffffffffu, cs[e], 16);
                }
                if (lane < 8) {
#pragma unroll
                    for (int e = 0; e < 8; ++e) cpart[cw * BN + 8 * lane + e] = cs[e];
                }
                group_sync(1, 32 * S::CW);
                if (tid < BN) {
                    int32_t sum = 0;
#pragma unroll
                    for (int w8 = 0; w8 < S::CW; ++w8) sum += cpart[w8 * BN + tid];
                    colsum[slot * BN + tid] = sum;
                }
            }
            fence_proxy_async_smem();
            group_sync(1, 32 * S::CW);
            if (tid == 0) {
                mbar_arrive(&bars[S::REMPTY + r]);
                mbar_arrive(&bars[S::FULL + st]);
            }
        }
    } else if (warp == S::MMA_WARP) {
        // ================= MMA issue =================
        if (lane == 0) {
            // unsigned 8-bit limbs, S32 accumulators, M = 128, N = 64, B MN-major
            constexpr uint32_t idesc = (2u << 4) | (1u << 16) | ((uint32_t)(BN >> 3) << 17) |
                                       ((uint32_t)(128 >> 4) << 24);
            constexpr int KS = 128 / 32;
            auto bdesc = [](uint32_t base, int s) { return umma_desc(base + 2048u * (uint32_t)s, 512u, 4u); };
            uint32_t g = 0;
            bool stop = false;
            for (uint32_t ti = 0; ti < myTiles && !stop; ++ti) {
                const int a = (int)(ti % NA);
                const uint32_t ua = ti / NA;
                if (ua >= 1 && !tc_wait(&bars[S::AEMPTY + a], (ua - 1) & 1u, abortFlag, p.err)) break;
                const uint32_t d = tmem + (uint32_t)a * S::ACC;
                for (uint32_t ch = 0; ch < p.chunks; ++ch, ++g) {
                    const int st = (int)(g % NS);
                    const uint32_t u = g / NS;
                    if (!tc_wait(&bars[S::FULL + st], u & 1u, abortFlag, p.err)) {
                        stop = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t aHi = sbase + S::OFF_ST + st * S::STAGE, bHi = aHi + S::A_LIMB;
                    const uint32_t aLo = aHi + S::LIMB_PAIR, bLo = bHi + S::LIMB_PAIR;
#pragma unroll
                    for (int s = 0; s < KS; ++s)
                        tc_mma_s8(d, S::LA::desc(aHi, 0, s), bdesc(bHi, s), idesc, (ch > 0 || s > 0) ? 1u : 0u);
#pragma unroll
                    for (int s = 0; s < KS; ++s)
                        tc_mma_s8(d + BN, S::LA::desc(aHi, 0, s), bdesc(bLo, s), idesc, (ch > 0 || s > 0) ? 1u : 0u);
#pragma unroll
                    for (int s = 0; s < KS; ++s)
                        tc_mma_s8(d + BN, S::LA::desc(aLo, 0, s), bdesc(bHi, s), idesc, 1u);
#pragma unroll
                    for (int s = 0; s < KS; ++s)
                        tc_mma_s8(d + 2 * BN, S::LA::desc(aLo, 0, s), bdesc(bLo, s), idesc,
                                  (ch > 0 || s > 0) ? 1u : 0u);
                    tc_commit(&bars[S::EMPTY + st]);
                }
                if (stop) break;
                tc_commit(&bars[S::AFULL + a]);
            }
            tc_commit(&bars[S::DRAIN]);
            mbar_wait_bounded(&bars[S::DRAIN], 0);
        }
        __syncwarp();
    } else {
        // ================= epilogue =================
        // sum a b = 2^16 hh + 2^8 mid + ll + Kp 2^30 - 2^15 (sum a' + sum b'),
        // |sum a b| <= K 2^30 <= 2^44: every shift of 46 or more gives 0, as
        // 46 does; (v + 2^(s-1)) >> s equals ((v >> (s-1)) + 1) >> 1
        const int et = threadIdx.x - 32 * S::EPI0;  // 0..127
        const int q = warp & 3;
        const uint32_t laneBase = (uint32_t)(32 * q) << 16;
        const uint32_t s8 = p.shift & 0xFFu;
        const uint32_t sh = s8 > 46u ? 46u : s8;
        const long long rnd = sh ? (1ll << (sh - 1u)) : 0ll;
        const long long kp = (long long)p.chunks * 128ll << 30;
        for (uint32_t ti = 0; ti < myTiles; ++ti) {
            const int a = (int)(ti % NA);
            const uint32_t ua = ti / NA;
            bool bad = false;
            if (et == 0) bad = !tc_wait(&bars[S::AFULL + a], ua & 1u, abortFlag, p.err);
            if (group_sync_or(3, 32 * S::EW, bad)) break;
            tc_fence_after();
            const uint32_t tile = blockIdx.x + ti * gridDim.x;
            const uint32_t m0 = (tile / p.tilesN) * 128u, n0 = (tile % p.tilesN) * (uint32_t)BN;
            const uint32_t m = m0 + (uint32_t)(32 * q + lane);
            const uint32_t dbase = tmem + laneBase + (uint32_t)a * S::ACC;
            const int slot = (int)(ti % RS);
            const long long rowc = kp - ((long long)rowsum[slot * 128 + 32 * q + lane] << 15);
            int16_t* crow = Cm + (size_t)m * p.ldc + n0;
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 16) {
                int32_t hh[16], mid[16], ll[16];
                tmem_ld16_acc(dbase + (uint32_t)c0, hh);
                tmem_ld16_acc(dbase + (uint32_t)(BN + c0), mid);
                tmem_ld16_acc(dbase + (uint32_t)(2 * BN + c0), ll);
                uint32_t wv[8];
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const long long v = ((long long)hh[e] << 16) + ((long long)mid[e] << 8) + (long long)ll[e] + rowc -
                                        ((long long)colsum[slot * BN + c0 + e] << 15);
                    const long long qv = (v + rnd) >> sh;
                    const int16_t o = qv > 32767ll ? (int16_t)32767 : (qv < -32768ll ? (int16_t)-32768 : (int16_t)qv);
                    if (e & 1) wv[e >> 1] |= (uint32_t)(uint16_t)o << 16;
                    else wv[e >> 1] = (uint32_t)(uint16_t)o;
                }
                if (m < p.M) {
                    int16_t* dst = crow + c0;
                    if (n0 + (uint32_t)c0 + 16u <= p.N && ((uintptr_t)dst & 15u) == 0) {
                        *reinterpret_cast<uint4*>(dst) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
                        *reinterpret_cast<uint4*>(dst + 8) = make_uint4(wv[4], wv[5], wv[6], wv[7]);
                    } else {
#pragma unroll
                        for (int e = 0; e < 16; ++e)
                            if (n0 + (uint32_t)(c0 + e) < p.N) dst[e] = (int16_t)(wv[e >> 1] >> (16 * (e & 1)));
                    }
                }
            }
            tc_fence_before();
            group_sync(3, 32 * S::EW);
            if (et == 0) mbar_arrive(&bars[S::AEMPTY + a]);
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == S::MMA_WARP) {
        tc_fence_after();
        tmem_dealloc(tmem, S::TMEM_COLS);
    }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_tiled()
{
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(f);
    });
    return fn;
}

// A 2-D matrix of `outer` rows of `inner` elements (1 or 2 bytes), row
// stride `stride` bytes, read in boxes of boxInner x boxOuter elements.
bool tile_map(CUtensorMap* map, const void* base, int bytes, uint64_t inner, uint64_t outer, uint64_t stride,
              uint32_t boxInner, uint32_t boxOuter, CUtensorMapSwizzle swizzle)
{
    EncodeTiled fn = encode_tiled();
    if (!fn) return false;
    const cuuint64_t dims[2] = {inner, outer};
    const cuuint64_t strides[1] = {stride};
    const cuuint32_t box[2] = {boxInner, boxOuter};
    const cuuint32_t es[2] = {1u, 1u};
    return fn(map, bytes == 1 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_UINT16, 2,
              const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Raises the kernel's shared-memory limit once per device (slot: which
// kernel) and returns the SM count.
template <class K>
cudaError_t configure(K kernel, int slot, uint32_t smem, int* smsOut)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static bool configured[2][64] = {};
    static int sms[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 64 || slot < 0 || slot > 1) return cudaErrorInvalidDevice;
    if (!configured[slot][dev]) {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        configured[slot][dev] = true;
    }
    *smsOut = sms[dev];
    return cudaSuccess;
}

} // namespace

cudaError_t launch_int8_mm_tma(uint32_t M, uint32_t K, uint32_t N, const void* a, size_t lda, const void* b,
                               size_t ldb, void* c, size_t ldc, uint32_t shift, cudaStream_t s)
{
    using S = MmTma;
    // whole rows of A and B, 16-byte aligned (the copies' address and stride rules)
    if (((uintptr_t)a & 15u) || ((uintptr_t)b & 15u) || lda % 16u || ldb % 16u || lda < K || ldb < N)
        return cudaErrorNotSupported;
    CUtensorMap ma, mb;
    if (!tile_map(&ma, a, 1, K, M, lda, 128u, 128u, CU_TENSOR_MAP_SWIZZLE_128B) ||
        !tile_map(&mb, b, 1, N, K, ldb, 128u, 128u, CU_TENSOR_MAP_SWIZZLE_128B))
        return cudaErrorNotSupported;
    int sms = 0;
    cudaError_t e = configure(k_int8_mm_tma, 0, S::SMEM, &sms);
    if (e != cudaSuccess) return e;
    TmaArgs p{};
    p.c = c;
    p.ldc = ldc;
    p.M = M;
    p.K = K;
    p.N = N;
    p.shift = shift;
    p.tilesN = (N + S::BN - 1) / S::BN;
    const uint64_t tiles = (uint64_t)((M + 127u) / 128u) * p.tilesN;
    if (tiles > 0xFFFFFFFFull) return cudaErrorNotSupported;
    p.numTiles = (uint32_t)tiles;
    p.chunks = (K + 127u) / 128u;
    p.err = error_word().dev;
    const uint32_t grid = (uint32_t)(tiles < (uint64_t)sms ? tiles : (uint64_t)sms);
    k_int8_mm_tma<<<grid, S::THREADS, S::SMEM, s>>>(ma, mb, p);
    return cudaGetLastError();
}

cudaError_t launch_int16_mm_tma(uint32_t M, uint32_t K, uint32_t N, const void* a, size_t lda, const void* b,
                                size_t ldb, void* c, size_t ldc, uint32_t shift, cudaStream_t s)
{
    using S = Mm16Tma;
    // whole rows of A and B, 16-byte aligned; K small enough for the
    // accumulators (2 K 255^2 < 2^31)
    if (((uintptr_t)a & 15u) || ((uintptr_t)b & 15u) || lda % 8u || ldb % 8u || lda < K || ldb < N ||
        K > 16384u)
        return cudaErrorNotSupported;
    CUtensorMap ma, mb;
    if (!tile_map(&ma, a, 2, K, M, lda * 2u, 128u, 128u, CU_TENSOR_MAP_SWIZZLE_NONE) ||
        !tile_map(&mb, b, 2, N, K, ldb * 2u, 64u, 128u, CU_TENSOR_MAP_SWIZZLE_NONE))
        return cudaErrorNotSupported;
    int sms = 0;
    cudaError_t e = configure(k_int16_mm_tma, 1, S::SMEM, &sms);
    if (e != cudaSuccess) return e;
    TmaArgs p{};
    p.c = c;
    p.ldc = ldc;
    p.M = M;
    p.K = K;
    p.N = N;
    p.shift = shift;
    p.tilesN = (N + S::BN - 1) / S::BN;
    const uint64_t tiles = (uint64_t)((M + 127u) / 128u) * p.tilesN;
    if (tiles > 0xFFFFFFFFull) return cudaErrorNotSupported;
    p.numTiles = (uint32_t)tiles;
    p.chunks = (K + 127u) / 128u;
    p.err = error_word().dev;
    const uint32_t grid = (uint32_t)(tiles < (uint64_t)sms ? tiles : (uint64_t)sms);
    k_int16_mm_tma<<<grid, S::THREADS, S::SMEM, s>>>(ma, mb, p);
    return cudaGetLastError();
}

} // namespace fftb200
