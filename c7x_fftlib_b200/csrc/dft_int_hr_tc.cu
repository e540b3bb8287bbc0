// dft_int_hr_tc.cu -- the INT16 highRadixDecompositions stages of radix 16
// (MMA / 2) on the tensor cores, bit-exact with the reference's natural C
// (src/fft_c7xmma/FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX/
// FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_cn.cpp) and with the
// CUDA-core kernels k_int_stage / k_int_final of dft_int.cu.
//
// A data row is the 16 complex inputs of one radix-16 DFT: butterfly q of a
// decimation stage (points q + m s/16 of a block of s points) or one group of
// the final stage (16 consecutive points). 128 data rows form the A operand
// of a tile (M = 128, K = 32 values: point m's real and imaginary parts at
// k = 2m, 2m + 1); the 32 x 32 real embedding of the 16-point DFT is the B
// operand (N = 64: output n = 2l + part, a column of ones at n = 32 and zero
// columns). Thread = data row in the epilogue, so the 16 outputs of a row sit
// in one thread: the stage's twiddle multiply needs no exchange, and a warp's
// stores of one output l are 32 consecutive points (stages) or the
// digit-reversed positions of 32 consecutive groups (final).
//
// Exactness as in dft_int_tc.cu: values in offset binary v' = v + 32768 =
// 256 h + l, three u8 x u8 products summed exactly in S32 accumulators,
//   sum x W = 2^16 hh + 2^8 mid + ll - 2^15 (sum x' + sum W') + 32 2^30
//           = 256 T + ll,  T = 256 hh + mid + 128 (2^20 - sum x' - sum W'),
// where the ones column gives sum x' = 256 mid + ll of that column. With
// K = 32, hh < 2^21, mid < 2^22 and |128 (2^20 - ...)| < 2^29, so T is a
// 32-bit value and the epilogue rounds and saturates 256 T + ll without
// 64-bit arithmetic (hr_round). The internal table's entries lie in
// [-32767, 32767], so the negated ones of a stage's matrix are INT16 values
// too.
//
// The reference forms a stage's real part with the saturating negation of the
// imaginary inputs, c1 neg(ai); neg(-32768) = 32767 = -(-32768) - 1, so the
// real part is the plain complex product minus c1(l, m) for every input m
// whose imaginary part is -32768. The converters record those m per row (a
// 16-bit mask); the epilogue subtracts the correction where the mask is not 0.
//
// Raw tiles arrive by bulk copies: a stage whose butterflies are 128 or more
// apart (s/16 >= 128) copies 16 runs of 128 points, the other stages and the
// final stage one contiguous run of 16 points per data row.
//
// Roles per CTA (one persistent CTA per SM): 4 converter warps (raw values ->
// offset bytes -> swizzled K-major shared memory, one data row per thread),
// 8 epilogue warps (three accumulators -> 32-bit T -> shift, round,
// saturate, twiddle -> HBM), one warp that owns tensor memory and issues the
// 4 MMAs of a tile, one copy thread. Every wait is bounded; a wait that gives
// up sets kErrTcTimeout in the launch's error word.
#include <mutex>

#include "dft_int.h"
#include "int_arith.cuh"
#include "plan.h"
#include "tc_dft.cuh"

namespace fftb200 {

namespace {

struct HrTc {
    static constexpr int TM = 128;  // data rows per tile = MMA M
    static constexpr int NO = 64;   // MMA N: 32 outputs, the ones column, zero columns
    static constexpr int NB = 4;    // operand tile buffers (shared memory)
    static constexpr int NA = 2;    // accumulator buffers (tensor memory)
    static constexpr int NR = 3;    // raw tile stages
    static constexpr int RS = 8;    // negation-mask slots: a slot is rewritten NB + NA tiles after its epilogue
    static constexpr int CW = 4, EW = 8;
    static constexpr int MMA_WARP = CW + EW, COPY_WARP = MMA_WARP + 1;
    static constexpr int THREADS = 32 * (COPY_WARP + 1);
    using LA = KMajor<TM, 16>;  // data limb: 128 rows x 32 bytes
    using LB = KMajor<NO, 16>;  // matrix limb: 64 columns x 32 bytes
    static constexpr uint32_t A_LIMB = LA::BYTES;  // 4 KB
    static constexpr uint32_t B_LIMB = LB::BYTES;  // 2 KB
    static constexpr uint32_t TILE = 2 * A_LIMB;
    static constexpr uint32_t RAWB = (uint32_t)TM * 16u * 4u;  // 8 KB: 16 complex INT16 points per row
    static constexpr uint32_t OFF_B = NB * TILE;
    static constexpr uint32_t OFF_RAW = OFF_B + 2 * B_LIMB;
    static constexpr uint32_t OFF_CW = OFF_RAW + NR * RAWB;  // 32 column terms 128 (2^20 - sum W')
    static constexpr uint32_t OFF_MK = OFF_CW + 4u * 32u;    // RS x TM masks (uint16)
    static constexpr uint32_t OFF_BAR = (OFF_MK + 2u * RS * TM + 7u) & ~7u;
    static constexpr int NBARS = 2 * NB + 2 * NA + 1 + 2 * NR;
    static constexpr uint32_t OFF_MISC = OFF_BAR + 8u * NBARS;
    static constexpr uint32_t SMEM = OFF_MISC + 16u + 1024u;
    static constexpr uint32_t ACC = 3 * NO;  // hh, mid, ll columns of one buffer
    static constexpr uint32_t TMEM_COLS = 512;
    static constexpr int A_FULL = 0, S_FREE = NB, D_FULL = 2 * NB, D_FREE = 2 * NB + NA, DRAIN = 2 * NB + 2 * NA,
                         R_FULL = DRAIN + 1, R_EMPTY = R_FULL + NR;
    static_assert(NA * ACC <= TMEM_COLS, "tensor memory");
    static_assert(RS >= NB + NA, "mask slots");
    static_assert(CW * 32 == TM, "one converter thread per data row");
    static_assert(EW == 8, "two epilogue warps per lane quarter, 8 outputs l each");
    static_assert(OFF_B % 1024u == 0 && B_LIMB % 1024u == 0 && OFF_RAW % 16u == 0, "operand alignment");
    static_assert(SMEM <= 227u * 1024u, "shared memory per CTA");
};

struct HrArgs {
    const int16_t* x;   // rows of n interleaved points (stage: transformed in place)
    int16_t* y;         // where the outputs go (stage: x)
    const int16_t* F;   // stage: the 16-point DFT, row l of 32 entries ((cos, -sin) pairs)
    const int16_t* tw;  // stage: its twiddle pairs at [q / 16][l][q mod 16]
    const int16_t* D;   // final: the caller's last table block (32 rows of 32)
    uint32_t n;         // points per row
    uint32_t lgPer;     // log2 of the data rows per row (n / 16)
    uint32_t lgStride;  // stage: log2 of s / 16, the distance of a butterfly's points
    uint32_t lgD0, lgM, lgI, lgH;  // final: log2 of the digits d0, mC, iC, hC of a group index
    uint32_t shift;
    uint64_t total;  // data rows of the launch
    uint32_t* err;
};

// Instruction descriptor: S32 accumulator, unsigned 8-bit A and B, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t hr_idesc(int n)
{
    return (2u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

FFT_DEV void hr_mma(uint32_t d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
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

// 16 consecutive 32-bit columns of this thread's tensor-memory lane.
FFT_DEV void hr_ld16(uint32_t taddr, int32_t (&v)[16])
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

// Entry (k, n) of the real embedding, n < 32: input k = 2m + kind (kind 0 the
// real, 1 the imaginary part of point m), output n = 2l + part.
template <bool FINAL>
__device__ __forceinline__ int32_t hr_entry(const HrArgs& a, int k, int n)
{
    if (FINAL) return a.D[n * 32 + (k ^ 1)];  // xr = d[2m] ai + d[2m+1] ar, row 2l (real) or 2l + 1
    const int m = k >> 1, kind = k & 1, l = n >> 1, part = n & 1;
    const int32_t c0 = a.F[l * 32 + 2 * m], c1 = a.F[l * 32 + 2 * m + 1];
    if (part == 0) return kind == 0 ? c0 : -c1;  // yr = c0 ar - c1 ai (then the saturation correction)
    return kind == 0 ? c1 : c0;                  // yi = c1 ar + c0 ai
}

// The limbs of matrix column n: offset binary for the outputs, the ones
// column (h = 0, l = 1) at n = 32, zeros above.
template <bool FINAL>
__device__ __forceinline__ uint32_t hr_limb_entry(const HrArgs& a, int k, int n)
{
    if (n < 32) return (uint32_t)(hr_entry<FINAL>(a, k, n) + 32768);
    return n == 32 ? 1u : 0u;
}

// floor((256 T + L + 2^(s-1)) / 2^s) saturated to INT16 (the reference's
// shiftAndRound of the exact sum 256 T + L, |256 T + L| < 2^36), in 32-bit
// integers. s = the shift's low byte, capped at 37: every larger shift gives 0
// for such sums, as 37 does. For s >= 8 the low byte L folds into T, for
// s < 8 T is first clamped to +-2^22, beyond which the result saturates either
// way.
struct HrRound {
    bool big;
    int sE, sh, r1, r2;
};

__device__ __forceinline__ HrRound hr_round_of(uint32_t shift)
{
    HrRound R;
    const uint32_t s8 = shift & 0xFFu;
    R.sE = s8 > 37u ? 37 : (int)s8;
    R.big = R.sE >= 8;
    R.sh = R.big ? R.sE - 8 : 8 - R.sE;
    R.r1 = R.sE == 8 ? 128 : (R.sE > 0 && R.sE < 8 ? (1 << (R.sE - 1)) : 0);
    R.r2 = R.sE > 8 ? (1 << (R.sE - 9)) : 0;
    return R;
}

// The rounded value before saturation (|q| < 2^31).
__device__ __forceinline__ int32_t hr_round_q(const HrRound& R, int32_t T, int32_t L)
{
    if (R.big) return (T + ((L + R.r1) >> 8) + R.r2) >> R.sh;
    const int32_t A = min(max(T, -(1 << 22)), 1 << 22);
    return A * (1 << R.sh) + ((L + R.r1) >> R.sE);
}

__device__ __forceinline__ int32_t hr_round(const HrRound& R, int32_t T, int32_t L)
{
    return min(max(hr_round_q(R, T, L), -32768), 32767);
}

// One complex INT16 point from two 32-bit values, each saturated: the real
// part in the low half, the imaginary part in the high half.
__device__ __forceinline__ uint32_t hr_pack_sat(int32_t re, int32_t im)
{
    uint32_t d;
    asm("cvt.pack.sat.s16.s32 %0, %1, %2;" : "=r"(d) : "r"(im), "r"(re));
    return d;
}

// First point of data row r (global index) of a decimation stage; q is its
// butterfly index inside the block.
__device__ __forceinline__ uint64_t hr_stage_point(const HrArgs& a, uint64_t r, uint32_t* q)
{
    const uint64_t row = r >> a.lgPer;
    const uint32_t g = (uint32_t)(r & ((1ull << a.lgPer) - 1u));
    const uint32_t blk = g >> a.lgStride;
    *q = g & ((1u << a.lgStride) - 1u);
    return row * a.n + ((uint64_t)blk << (a.lgStride + 4u)) + *q;
}

template <bool FINAL>
__global__ void __launch_bounds__(HrTc::THREADS, 1) k_int16_hr_tc(const HrArgs a)
{
    using S = HrTc;
    constexpr int TM = S::TM, NB = S::NB, NA = S::NA, RS = S::RS, NO = S::NO;
    extern __shared__ unsigned char hr_smem_raw[];
    unsigned char* sm = hr_smem_raw + ((1024u - (smem_addr(hr_smem_raw) & 1023u)) & 1023u);
    const uint32_t sbase = smem_addr(sm);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + S::OFF_BAR);
    uint32_t* misc = reinterpret_cast<uint32_t*>(sm + S::OFF_MISC);
    volatile uint32_t* abortFlag = misc + 1;
    int32_t* colE = reinterpret_cast<int32_t*>(sm + S::OFF_CW);
    uint16_t* masks = reinterpret_cast<uint16_t*>(sm + S::OFF_MK);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t numTiles = (uint32_t)((a.total + TM - 1) / TM);
    // butterflies 128 or more apart: 16 runs of 128 points per tile
    const bool runs = !FINAL && a.lgStride >= 7u;

    if (threadIdx.x == 0) {
        for (int i = 0; i < S::NBARS; ++i) mbar_init(&bars[i], 1);
        misc[1] = 0;
        fence_mbarrier_init();
    }
    if (warp == S::MMA_WARP) {
        tmem_alloc(&misc[0], S::TMEM_COLS);
        tmem_relinquish();
    }
    // the matrix operand: column n, 16-byte chunk j = inputs 16 j .. 16 j + 15
    {
        unsigned char* hi = sm + S::OFF_B;
        unsigned char* lo = hi + S::B_LIMB;
        for (int it = threadIdx.x; it < NO * 2; it += blockDim.x) {
            const int n = it >> 1, j = it & 1;
            uint32_t h[4] = {0u, 0u, 0u, 0u}, q[4] = {0u, 0u, 0u, 0u};
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                const uint32_t u = hr_limb_entry<FINAL>(a, 16 * j + e, n);
                h[e >> 2] |= (u >> 8) << (8 * (e & 3));
                q[e >> 2] |= (u & 255u) << (8 * (e & 3));
            }
            const uint32_t off = S::LB::chunk(n, j);
            *reinterpret_cast<uint4*>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<uint4*>(lo + off) = make_uint4(q[0], q[1], q[2], q[3]);
        }
        // per output column: 128 (2^20 - sum W')
        for (int n = threadIdx.x; n < 32; n += blockDim.x) {
            int32_t s = 0;
            for (int k = 0; k < 32; ++k) s += hr_entry<FINAL>(a, k, n) + 32768;
            colE[n] = 128 * ((1 << 20) - s);
        }
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = misc[0];

    if (warp < S::CW) {
        // ================= converters: thread = data row =================
        const int r = threadIdx.x;
        // position (in points) of the row's point m in the raw stage
        const uint32_t lgS = runs ? 7u : (FINAL ? 0u : a.lgStride);
        const uint32_t rowPos = FINAL ? 16u * (uint32_t)r
                                      : (((uint32_t)r >> lgS) << (lgS + 4u)) + ((uint32_t)r & ((1u << lgS) - 1u));
        const uint32_t mStep = FINAL ? 1u : (1u << lgS);
        uint32_t i = 0;
        for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++i) {
            const int b = (int)(i % NB), rr = (int)(i % S::NR);
            const uint32_t u = i / NB, ur = i / S::NR, slot = i % RS;
            bool badr = false;
            if (r == 0) badr = !tc_wait(&bars[S::R_FULL + rr], ur & 1u, abortFlag, a.err);
            if (group_sync_or(1, 32 * S::CW, badr)) break;
            const unsigned char* raw = sm + S::OFF_RAW + rr * S::RAWB;
            uint32_t w[16];
            if (FINAL) {
                // 64 contiguous bytes
#pragma unroll
                for (int z = 0; z < 4; ++z) {
                    const uint4 v = *reinterpret_cast<const uint4*>(raw + 4u * rowPos + 16u * (uint32_t)z);
                    w[4 * z] = v.x;
                    w[4 * z + 1] = v.y;
                    w[4 * z + 2] = v.z;
                    w[4 * z + 3] = v.w;
                }
            } else {
#pragma unroll
                for (int m = 0; m < 16; ++m)
                    w[m] = *reinterpret_cast<const uint32_t*>(raw + 4u * (rowPos + (uint32_t)m * mStep));
            }
            uint32_t mask = 0;
            if (!FINAL) {
#pragma unroll
                for (int m = 0; m < 16; ++m) mask |= ((w[m] >> 16) == 0x8000u ? 1u : 0u) << m;
            }
            uint32_t hw[8], lw[8];
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                // offset binary flips each value's sign bit; point 2p's real and
                // imaginary parts, then point 2p + 1's
                const uint32_t a0 = w[2 * p] ^ 0x80008000u, a1 = w[2 * p + 1] ^ 0x80008000u;
                hw[p] = __byte_perm(a0, a1, 0x7531u);
                lw[p] = __byte_perm(a0, a1, 0x6420u);
            }
            bool bad = false;
            if (u >= 1 && r == 0) bad = !tc_wait(&bars[S::S_FREE + b], (u - 1) & 1u, abortFlag, a.err);
            // every converter has read its raw values: the stage can be refilled
            if (group_sync_or(1, 32 * S::CW, bad)) break;
            if (r == 0) mbar_arrive(&bars[S::R_EMPTY + rr]);
            unsigned char* hiA = sm + b * S::TILE;
            unsigned char* loA = hiA + S::A_LIMB;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const uint32_t off = S::LA::chunk(r, j);
                *reinterpret_cast<uint4*>(hiA + off) = make_uint4(hw[4 * j], hw[4 * j + 1], hw[4 * j + 2], hw[4 * j + 3]);
                *reinterpret_cast<uint4*>(loA + off) = make_uint4(lw[4 * j], lw[4 * j + 1], lw[4 * j + 2], lw[4 * j + 3]);
            }
            if (!FINAL) masks[slot * TM + r] = (uint16_t)mask;
            fence_proxy_async_smem();
            group_sync(1, 32 * S::CW);
            if (r == 0) mbar_arrive(&bars[S::A_FULL + b]);
        }
    } else if (warp == S::COPY_WARP) {
        // ================= raw tile copies =================
        if (lane == 0) {
            uint32_t i = 0;
            for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++i) {
                const int rr = (int)(i % S::NR);
                const uint32_t ur = i / S::NR;
                if (ur >= 1 && !tc_wait(&bars[S::R_EMPTY + rr], (ur - 1) & 1u, abortFlag, a.err)) break;
                const uint64_t base = (uint64_t)tile * TM;
                unsigned char* raw = sm + S::OFF_RAW + rr * S::RAWB;
                if (runs) {
                    // a full tile inside one block: 16 runs of 128 points, s/16 apart
                    uint32_t q;
                    const uint64_t p0 = hr_stage_point(a, base, &q);
                    mbar_expect_tx(&bars[S::R_FULL + rr], S::RAWB);
                    for (int m = 0; m < 16; ++m)
                        bulk_copy_g2s(raw + (uint32_t)m * 512u, a.x + 2u * (p0 + ((uint64_t)m << a.lgStride)), 512u,
                                      &bars[S::R_FULL + rr]);
                } else {
                    // whole blocks (or groups) of 16 points each: one run
                    const uint64_t rows = min((uint64_t)TM, a.total - base);
                    const uint32_t bytes = (uint32_t)rows * 64u;
                    mbar_expect_tx(&bars[S::R_FULL + rr], bytes);
                    bulk_copy_g2s(raw, a.x + 32u * base, bytes, &bars[S::R_FULL + rr]);
                }
            }
            // the copies still in flight land before the CTA ends
            for (int rr = 0; rr < S::NR; ++rr) {
                const uint32_t armed = i > (uint32_t)rr ? (i - 1u - (uint32_t)rr) / S::NR + 1u : 0u;
                if (armed) mbar_wait_bounded(&bars[S::R_FULL + rr], (armed - 1u) & 1u);
            }
        }
        __syncwarp();
    } else if (warp == S::MMA_WARP) {
        // ================= MMA issue =================
        if (lane == 0) {
            constexpr uint32_t idesc = hr_idesc(NO);
            const uint32_t bHi = sbase + S::OFF_B, bLo = bHi + S::B_LIMB;
            uint32_t i = 0;
            for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++i) {
                const int b = (int)(i % NB), ac = (int)(i % NA);
                const uint32_t u = i / NB, ua = i / NA;
                if (!tc_wait(&bars[S::A_FULL + b], u & 1u, abortFlag, a.err)) break;
                if (ua >= 1 && !tc_wait(&bars[S::D_FREE + ac], (ua - 1) & 1u, abortFlag, a.err)) break;
                tc_fence_after();
                const uint32_t aHi = sbase + b * S::TILE, aLo = aHi + S::A_LIMB;
                const uint32_t d = tmem + (uint32_t)ac * S::ACC;
                hr_mma(d, S::LA::desc(aHi, 0, 0), S::LB::desc(bHi, 0, 0), idesc, 0u);
                hr_mma(d + NO, S::LA::desc(aHi, 0, 0), S::LB::desc(bLo, 0, 0), idesc, 0u);
                hr_mma(d + NO, S::LA::desc(aLo, 0, 0), S::LB::desc(bHi, 0, 0), idesc, 1u);
                hr_mma(d + 2 * NO, S::LA::desc(aLo, 0, 0), S::LB::desc(bLo, 0, 0), idesc, 0u);
                tc_commit(&bars[S::S_FREE + b]);
                tc_commit(&bars[S::D_FULL + ac]);
            }
            tc_commit(&bars[S::DRAIN]);
            mbar_wait_bounded(&bars[S::DRAIN], 0);
        }
        __syncwarp();
    } else {
        // ================= epilogue: thread = data row, 8 outputs l =================
        const int et = threadIdx.x - 32 * S::CW;  // 0 .. 32 EW - 1
        const int qd = warp & 3, hf = (warp - S::CW) >> 2;
        const int r = 32 * qd + lane;
        const uint32_t laneBase = (uint32_t)(32 * qd) << 16;
        const HrRound R = hr_round_of(a.shift);
        uint32_t i = 0;
        for (uint32_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x, ++i) {
            const int ac = (int)(i % NA);
            const uint32_t ua = i / NA, slot = i % RS;
            bool bad = false;
            if (et == 0) bad = !tc_wait(&bars[S::D_FULL + ac], ua & 1u, abortFlag, a.err);
            if (group_sync_or(3, 32 * S::EW, bad)) break;
            tc_fence_after();
            const uint32_t dbase = tmem + laneBase + (uint32_t)ac * S::ACC;
            int32_t hh[16], mid[16], ll[16];
            // the ones column first: sum x' of the row
            hr_ld16(dbase + (uint32_t)(NO + 32), mid);
            int32_t sx = mid[0] * 256;
            hr_ld16(dbase + (uint32_t)(2 * NO + 32), ll);
            sx += ll[0];
            hr_ld16(dbase + (uint32_t)(16 * hf), hh);
            hr_ld16(dbase + (uint32_t)(NO + 16 * hf), mid);
            hr_ld16(dbase + (uint32_t)(2 * NO + 16 * hf), ll);
            const uint32_t mask = FINAL ? 0u : (uint32_t)masks[slot * TM + r];
            // the accumulators are in registers: the next tile's MMAs may start
            tc_fence_before();
            group_sync(3, 32 * S::EW);
            if (et == 0) mbar_arrive(&bars[S::D_FREE + ac]);

            const uint64_t row = (uint64_t)tile * TM + (uint64_t)r;
            if (row >= a.total) continue;
            // T of each output: sum x W = 256 T + ll
            const int32_t sx128 = 128 * sx;
            int32_t T[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) T[c] = hh[c] * 256 + mid[c] + (colE[16 * hf + c] - sx128);
            if (!FINAL) {
                uint32_t q;
                const uint64_t p0 = hr_stage_point(a, row, &q);
                const int16_t* twq = a.tw + (q >> 4) * 512u + 2u * (q & 15u);
                uint32_t* out = reinterpret_cast<uint32_t*>(a.y) + p0;
#pragma unroll
                for (int c2 = 0; c2 < 8; ++c2) {
                    const int l = 8 * hf + c2;
                    int32_t lr = ll[2 * c2];
                    if (mask) {
                        for (uint32_t mm = mask; mm; mm &= mm - 1u) lr -= a.F[l * 32 + 2 * (__ffs((int)mm) - 1) + 1];
                    }
                    const int32_t tr = hr_round(R, T[2 * c2], lr);
                    const int32_t ti = hr_round(R, T[2 * c2 + 1], ll[2 * c2 + 1]);
                    const uint32_t e = *reinterpret_cast<const uint32_t*>(twq + l * 32);
                    const int32_t e0 = (int16_t)(e & 0xFFFFu), e1 = (int16_t)(e >> 16);
                    const int32_t ne0 = e0 == -32768 ? 32767 : -e0;  // the reference's saturating negation
                    // |e1 tr + ne0 ti| < 2^31; e0 tr + e1 ti reaches 2^31 (and wraps
                    // to INT32_MIN) only for four values of -32768, a result of 32767
                    const int32_t sr = e1 * tr + ne0 * ti;
                    const int32_t si = (int32_t)((uint32_t)(e0 * tr) + (uint32_t)(e1 * ti));
                    const int32_t im = si == INT32_MIN ? 32767 : (si + 16384) >> 15;
                    out[(uint64_t)l << a.lgStride] = hr_pack_sat((sr + 16384) >> 15, im);
                }
            } else {
                const uint64_t rw = row >> a.lgPer;
                uint32_t g = (uint32_t)(row & ((1ull << a.lgPer) - 1u));
                // digits of the group index (powers of two): h fastest, then i, m, k
                const uint32_t h = g & ((1u << a.lgH) - 1u);
                g >>= a.lgH;
                const uint32_t ii = g & ((1u << a.lgI) - 1u);
                g >>= a.lgI;
                const uint32_t mm = g & ((1u << a.lgM) - 1u);
                const uint32_t k = g >> a.lgM;
                const uint32_t dst0 =
                    (h << (a.lgD0 + a.lgM + a.lgI)) + (ii << (a.lgD0 + a.lgM)) + (mm << a.lgD0) + k;
                uint32_t* out = reinterpret_cast<uint32_t*>(a.y) + rw * a.n + dst0;
#pragma unroll
                for (int c2 = 0; c2 < 8; ++c2) {
                    const int l = 8 * hf + c2;
                    out[(uint64_t)l << a.lgPer] =
                        hr_pack_sat(hr_round_q(R, T[2 * c2], ll[2 * c2]), hr_round_q(R, T[2 * c2 + 1], ll[2 * c2 + 1]));
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == S::MMA_WARP) {
        tc_fence_after();
        tmem_dealloc(tmem, S::TMEM_COLS);
    }
}

template <bool FINAL>
cudaError_t launch_hr(const HrArgs& a, cudaStream_t s)
{
    using S = HrTc;
    if (a.total == 0) return cudaSuccess;
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
            e = cudaFuncSetAttribute(k_int16_hr_tc<FINAL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
            if (e != cudaSuccess) return e;
            e = cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return e;
            configured[dev] = true;
        }
    }
    const uint64_t tiles = (a.total + S::TM - 1) / S::TM;
    const uint32_t grid = (uint32_t)(tiles < (uint64_t)sms[dev] ? tiles : (uint64_t)sms[dev]);
    k_int16_hr_tc<FINAL><<<grid, S::THREADS, S::SMEM, s>>>(a);
    return cudaGetLastError();
}

uint32_t hr_lg2(uint32_t v) { return (uint32_t)(31 - __builtin_clz(v)); }

} // namespace

bool int16_hr_tc_supported(uint32_t n, const void* x, const void* y, const void* tw)
{
    return n >= 64 && (n & (n - 1u)) == 0 && ((uintptr_t)x & 15u) == 0 && ((uintptr_t)y & 3u) == 0 &&
           ((uintptr_t)tw & 3u) == 0;
}

cudaError_t launch_int16_hr_stage(int16_t* x, const int16_t* F, const int16_t* tw, uint32_t n, uint32_t s,
                                  uint32_t rows, uint32_t shift, cudaStream_t st)
{
    // blocks of s = 16^j points (j >= 2), butterflies s / 16 apart
    if (s < 256 || (s & (s - 1u)) || n % s || (hr_lg2(s) & 3u)) return cudaErrorInvalidValue;
    HrArgs a{};
    a.x = x;
    a.y = x;
    a.F = F;
    a.tw = tw;
    a.n = n;
    a.lgPer = hr_lg2(n) - 4u;
    a.lgStride = hr_lg2(s) - 4u;
    a.shift = shift;
    a.total = (uint64_t)rows << a.lgPer;
    a.err = error_word().dev;
    return launch_hr<false>(a, st);
}

cudaError_t launch_int16_hr_final(const int16_t* x, int16_t* y, const int16_t* D, uint32_t n, uint32_t d0,
                                  uint32_t mC, uint32_t iC, uint32_t hC, uint32_t rows, uint32_t shift,
                                  cudaStream_t st)
{
    const auto pow2 = [](uint32_t v) { return v != 0 && (v & (v - 1u)) == 0; };
    if (n < 64 || !pow2(n) || !pow2(d0) || !pow2(mC) || !pow2(iC) || !pow2(hC) ||
        (uint64_t)d0 * mC * iC * hC * 16u != n)
        return cudaErrorInvalidValue;
    HrArgs a{};
    a.x = x;
    a.y = y;
    a.D = D;
    a.n = n;
    a.lgPer = hr_lg2(n) - 4u;
    a.lgD0 = hr_lg2(d0);
    a.lgM = hr_lg2(mC);
    a.lgI = hr_lg2(iC);
    a.lgH = hr_lg2(hC);
    a.shift = shift;
    a.total = (uint64_t)rows << a.lgPer;
    a.err = error_word().dev;
    return launch_hr<true>(a, st);
}

} // namespace fftb200
