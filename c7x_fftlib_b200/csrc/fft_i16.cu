// fft_i16.cu -- batched int16 complex FFT with per-stage shift (K5),
// bit-exact with FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_cn
// (src/fft_c7x/FFTLIB_fft1dBatched_i16sc_c16sc_o16sc/..._cn.c:191-338).
//
// The result of the reference is defined by its exact integer sequence:
// radix-4 decimation-in-frequency stages with int16 two's-complement
// intermediates, the VCROT90H-style multiply by j, Q15 twiddle products
// rounded and saturated like VCMPYR1HH, a rounding right shift per stage,
// the 8-point stage special case and a final bit reversal. Butterflies within
// a stage are independent, so a CTA keeps one transform (as packed short2) in
// shared memory and runs each stage's butterflies across its threads; every
// butterfly performs exactly the reference's operations, so the output is
// identical bit for bit.
//
// Register-resident fusion: two consecutive radix-4 stages touch 16 points
// {k0 + i*M/16} of one length-M block, so a thread loads those 16 points,
// runs both stages in registers and stores once, halving shared-memory
// traffic and barriers.
#include <cuda_runtime.h>
#include <algorithm>
#include <map>
#include <mutex>
#include <utility>
#include <stdint.h>

#include "fft_i16.h"

namespace fftb200 {

__device__ __forceinline__ int16_t wrap16(int v) { return (int16_t)(uint16_t)(unsigned)v; }

// Right shift rounding by the last bit shifted out; the mask is formed as
// the reference forms it on x86 (32-bit shift by shift-1 with the count
// taken mod 32, narrowed to int16), which makes shift 0 a no-op.
__device__ __forceinline__ int16_t shift_round(int16_t v, uint32_t shift)
{
    const int16_t mask = (int16_t)(uint16_t)(1u << ((shift - 1u) & 31u));
    const int vi = v;
    const int s = (int)(shift & 31u);
    return wrap16(((vi & (int)mask) != 0) ? ((vi >> s) + 1) : (vi >> s));
}

// The same rounding shift with the per-stage constants precomputed. When
// the reference's mask is non-zero (shift in 1..16) it adds bit s - 1 back
// after the shift; (v >> s) + bit_{s-1}(v) = (v + 2^(s-1)) >> s for an int16 v
// (floor division), so one add and one shift do it; otherwise it is v >> s.
// apply = false: the stage is not followed by a shift (the 8-point stage).
//
// A Q15 product is rounded before that shift. With
// f(v) = floor((v + add) / 2^s), non-decreasing, f(clamp(u)) =
// clamp(f(u), f(-32768), f(32767)), and nested floor divisions compose:
// f(floor((x + 2^14) / 2^15)) = floor((x + K) / 2^(15+s)), K = 2^14 + add 2^15.
// K is even, so that is floor((floor(x / 2) + K / 2) / 2^(14+s)), which stays
// in 32 bits for a difference of products (|x| <= 2^31 - 2^15; a sum is
// offset first, cmul_q15); for 14 + s >= 31 every such quotient is 0 or -1
// and a shift by 31 gives it.
struct ShiftRound {
    int s, add;
    int k2, sh, lo, hi;  // the product path: K / 2, 14 + s (at most 31), f(-32768), f(32767)
    int k2u;             // (K - C) / 2 for a sum offset by C = 2^31 - 2^16 (cmul_q15)
    uint32_t lo2, hi2;   // f(-32768), f(32767) in both halfwords
    __device__ __forceinline__ explicit ShiftRound(uint32_t shift, bool apply = true)
    {
        if (!apply) shift = 0;
        s = (int)(shift & 31u);
        const uint32_t rb = (shift - 1u) & 31u;
        add = rb < 16u ? (int)(1u << rb) : 0;  // the mask narrowed to int16 is non-zero
        k2 = 0x2000 + add * 16384;
        k2u = k2 - 0x3FFF8000;
        sh = min(14 + s, 31);
        lo = (-32768 + add) >> s;
        hi = (32767 + add) >> s;
        lo2 = ((uint32_t)lo & 0xFFFFu) * 0x10001u;
        hi2 = ((uint32_t)hi & 0xFFFFu) * 0x10001u;
    }
    // the result always fits in int16 (for s = 0 nothing is added), so no
    // wrap is needed
    __device__ __forceinline__ int16_t operator()(int16_t v) const { return (int16_t)(((int)v + add) >> s); }
};

struct C16 {
    int16_t re, im;
};

__device__ __forceinline__ C16 ld(const short2* p) { short2 v = *p; return C16{v.x, v.y}; }
__device__ __forceinline__ void st(short2* p, C16 c) { *p = make_short2(c.re, c.im); }

// (re, im) halves of a packed pair (re low) and the packing
__device__ __forceinline__ int lo16(uint32_t v) { return (int)(int16_t)(uint16_t)v; }
__device__ __forceinline__ int hi16(uint32_t v) { return (int)v >> 16; }
__device__ __forceinline__ uint32_t pack16(int re, int im)
{
    return (uint32_t)(uint16_t)re | ((uint32_t)im << 16);
}

// Two 32-bit values packed as int16 halves (re low, im high) with signed
// saturation (cvt.pack.sat: its first source goes to the upper half).
__device__ __forceinline__ uint32_t pack_sat16(int re, int im)
{
    uint32_t d;
    asm("cvt.pack.sat.s16.s32 %0, %1, %2;" : "=r"(d) : "r"(im), "r"(re));
    return d;
}

// Q15 complex product with the reference's rounding and saturation, then the
// stage shift: for each component x = a*b +/- c*d formed exactly,
// ((x + 0x4000) << 1) clamped to [-2^31, 0x7FFF0000] and shifted right by 16
// equals clamp((x + 0x4000) >> 15) to [-32768, 32767] ((2u) >> 16 == u >> 15
// with floor semantics, and the clamp bounds map onto each other); that and
// the shift are one step (ShiftRound). Products of int16 values lie in
// [-(2^30 - 2^15), 2^30], and 2^30 only for (-32768)^2, so the difference
// (re = x.re*w.x - x.im*w.y) always fits in int32 (|x| <= 2^31 - 2^15, so
// halving and adding K/2 cannot overflow), and the sum (im = x.re*w.y +
// x.im*w.x) lies in [-(2^31 - 2^16), 2^31]: offset by C = 2^31 - 2^16 it is
// exact as an unsigned word u, and floor(x / 2) + K / 2 = (u >> 1) + (K - C) / 2
// stays within int32 (add <= 2^15); the one sum beyond int32, 2^31 with all
// four factors -32768, then rounds and saturates to 32767 like every other
// sum. Both components are clamped to [f(-32768), f(32767)] at once on the
// packed pair: saturating to int16 first changes nothing, since those bounds
// lie within int16.
__device__ __forceinline__ uint32_t cmul_q15(uint32_t xv, int2 w, const ShiftRound& sr)
{
    const int re = lo16(xv), im = hi16(xv);
    const int vr = (((re * w.x - im * w.y) >> 1) + sr.k2) >> sr.sh;
    const int vi = ((int)(((uint32_t)(re * w.y) + (uint32_t)(im * w.x) + 0x7FFF0000u) >> 1) + sr.k2u) >> sr.sh;
    return __vmaxs2(__vmins2(pack_sat16(vr, vi), sr.hi2), sr.lo2);
}

// One 4-point butterfly on p0..p3 (stride q apart in the stage), each an
// (re, im) pair packed in 32 bits (re low); outputs written back as bins
// 0, 2, 1, 3 (the reference's slot order), each followed by the stage's
// shift sr (the identity for the 8-point stage); tw: the three Q15 twiddles
// (of bins 1, 2, 3) unless notw. The sums and differences run in
// per-halfword SIMD: __vadd2 / __vsub2 wrap each 16-bit half exactly as the
// reference's int16 arithmetic does, and __vnegss2 saturates -(-32768) to
// 32767 as its j-rotation does (only the imaginary half of that result is
// used: j = (sat(-d2.im), d2.re)). Bin 0's Q15 product with 32767+1 (the
// reference's 0x7FFF0000 >> 16 scale by 2^15) rounds back to itself exactly,
// so only the shift applies to it; the shift and the Q15 products work on
// the unpacked halves (cmul_q15).

__device__ __forceinline__ void bfly4_packed(uint32_t& p0, uint32_t& p1, uint32_t& p2, uint32_t& p3, bool notw,
                                             const int2* tw, uint32_t k, uint32_t q, const ShiftRound& sr)
{
    const uint32_t s1 = __vadd2(p0, p2), s2 = __vadd2(p1, p3);
    const uint32_t d1 = __vsub2(p0, p2), d2 = __vsub2(p1, p3);
    const uint32_t j = __byte_perm(__vnegss2(d2), d2, 0x5432u);
    const uint32_t x0 = __vadd2(s1, s2), x2 = __vsub2(s1, s2);
    const uint32_t x1 = __vsub2(d1, j), x3 = __vadd2(d1, j);
    p0 = pack16(sr((int16_t)lo16(x0)), sr((int16_t)hi16(x0)));
    if (!notw) {
        const int2 w1 = tw[k], w2 = tw[q + k], w3 = tw[2 * q + k];
        p2 = cmul_q15(x1, w1, sr);
        p1 = cmul_q15(x2, w2, sr);
        p3 = cmul_q15(x3, w3, sr);
    } else {
        p2 = pack16(sr((int16_t)lo16(x1)), sr((int16_t)hi16(x1)));
        p1 = pack16(sr((int16_t)lo16(x2)), sr((int16_t)hi16(x2)));
        p3 = pack16(sr((int16_t)lo16(x3)), sr((int16_t)hi16(x3)));
    }
}

// Shared-memory index with one pad word per 16: the 16-point gathers of the
// fused stages and the bit-reversed final gather hit distinct banks.
// For an m-point block (m a multiple of 16) and k0 < s16 = m / 16,
// pad16(blk*m + k0 + i*s16) = pad16(blk*m + k0) + pad16(i*s16): the points
// of a fused group sit at fixed offsets from its padded base (for s16 >= 16
// i*s16 is a multiple of 16; below, k0 + i*s16 crosses a multiple of 16
// exactly where i*s16 does).
__device__ __forceinline__ uint32_t pad16(uint32_t i) { return i + (i >> 4); }

// 16-byte asynchronous copy global -> shared (both addresses 16-byte aligned),
// completed by cp_async_wait_all in the issuing thread.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Two radix-4 stages on one m-point block per 16-point group: block m with
// shift shiftA, then the four m/4 sub-blocks with shiftB (m a power of two
// >= 16; the 8-point special case where m or m/4 is 8). FLAT: the points are
// read from flat (unpadded) src instead of su, for the first stage (m = n,
// where a warp's 16-point groups are consecutive columns, conflict-free).
template <bool FLAT = false>
__device__ __forceinline__ void fused_pair(uint32_t* su, const int2* tw, uint32_t m, uint32_t n, uint32_t t,
                                           uint32_t tg, uint32_t shiftA, uint32_t shiftB,
                                           const uint32_t* src = nullptr)
{
    const uint32_t m2 = m / 4u;
    const ShiftRound srA(shiftA, m != 8u), srB(shiftB, m2 != 8u);
    const int2* tw2 = tw + 3u * (m / 4u);
    const uint32_t s16 = m / 16u;
    const uint32_t ls16 = 31u - __clz(s16);  // m is a power of two: shifts, not divisions
    const uint32_t groups = n / 16u;         // (block, k0) pairs
    const uint32_t qA = m / 4u, qB = m2 / 4u;
    for (uint32_t gi = t; gi < groups; gi += tg) {
        const uint32_t blk = gi >> ls16, k0 = gi & (s16 - 1u);
        const uint32_t pb = pad16(blk * m + k0);
        uint32_t p[16];
#pragma unroll
        for (int i = 0; i < 16; ++i)
            p[i] = FLAT ? src[blk * m + k0 + (uint32_t)i * s16] : su[pb + pad16((uint32_t)i * s16)];
        // stage A (block m): butterflies k = k0 + i*s16, points i, i+4, i+8, i+12
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t kA = k0 + (uint32_t)i * s16;
            const bool notwA = (m == 4u) || (m == 8u && kA == 0u);
            bfly4_packed(p[i], p[i + 4], p[i + 8], p[i + 12], notwA, tw, kA, qA, srA);
        }
        // stage B (block m/4): sub-block s (points 4s..4s+3), butterfly k0
        const bool notwB = (m2 == 4u) || (m2 == 8u && k0 == 0u);
#pragma unroll
        for (int s = 0; s < 4; ++s)
            bfly4_packed(p[4 * s], p[4 * s + 1], p[4 * s + 2], p[4 * s + 3], notwB, tw2, k0, qB, srB);
#pragma unroll
        for (int i = 0; i < 16; ++i) su[pb + pad16((uint32_t)i * s16)] = p[i];
    }
}

__host__ __device__ constexpr uint32_t i16_log2(uint32_t n) { return n > 1u ? 1u + i16_log2(n / 2u) : 0u; }

// Persistent CTAs of G groups; a group of tg threads owns one transform at a
// time (its own padded shared-memory region) and the CTA walks the batch G
// transforms at a step. The caller's twiddle table and the shift vector are
// copied into shared memory once per CTA.
// MINB: CTAs per SM the registers are budgeted for (3: 80 registers; 4: 64,
// with a few spilled values), a launch-shape choice of the autotuner.
// NC: the transform length when fixed at compile time (every stage's block
// size, stride and special case then fold into constants and the stage loop
// unrolls), 0 for the kernel that takes it at run time.
// vecIn / vecOut: 16-byte loads of x / stores of y (aligned buffers, n % 4 == 0).
// MAXT: the largest block: 256 (groups of up to 256 threads), or 1024 for the
// longest lengths, where one transform per CTA takes up to 1024 threads.
// TG: the threads per transform when fixed at compile time (the default
// launch of a fixed length: every loop's trip count becomes a constant), 0
// when taken from tgArg.
// PF: the next transform's input is copied (cp.async, 16 bytes) into a flat
// shared-memory buffer of the group while the current one is transformed;
// the first stage reads it from there. Needs vecIn and n >= 64.
template <int MINB, uint32_t NC, int MAXT = 256, uint32_t TG = 0, bool PF = false>
__global__ void __launch_bounds__(MAXT, MINB) k_fft_i16(const short2* __restrict__ x, short2* __restrict__ y,
                                                 const short2* __restrict__ w,
                                                 const uint32_t* __restrict__ shifts, uint32_t nsh, uint32_t nArg,
                                                 uint32_t lognArg, uint32_t batch, uint32_t tgArg, bool vecIn,
                                                 bool vecOut)
{
    static_assert(!PF || NC >= 64u, "the prefetching build needs a fixed length of at least 64");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint32_t s_shift[8];
    const uint32_t n = NC ? NC : nArg;
    const uint32_t logn = NC ? i16_log2(NC) : lognArg;
    const uint32_t padn = n + (n >> 4);
    const uint32_t tg = TG ? TG : tgArg;
    const uint32_t nthreads = TG ? (TG > 256u ? TG : 256u) : blockDim.x;
    const uint32_t G = nthreads / tg;
    const uint32_t g = threadIdx.x / tg, t = threadIdx.x - g * tg;
    // the caller's Q15 table as 32-bit pairs (one load per twiddle, no
    // extraction), then the transforms' padded regions
    int2* stw = reinterpret_cast<int2*>(smem_raw);
    short2* smem = reinterpret_cast<short2*>(stw + n);
    short2* sx = smem + g * padn;
    uint32_t* su = reinterpret_cast<uint32_t*>(sx);
    // PF: the flat input buffers follow the G padded regions (16-byte aligned:
    // padn * 4 bytes is a multiple of 16 for n >= 64)
    uint32_t* inb = reinterpret_cast<uint32_t*>(smem + G * padn) + g * n;
    const auto prefetch = [&](uint32_t bb) {
        const int4* s4 = reinterpret_cast<const int4*>(x + (size_t)bb * n);
        for (uint32_t i4 = t; i4 < n / 4u; i4 += tg) cp_async16(inb + 4u * i4, s4 + i4);
    };
    for (uint32_t i = threadIdx.x; i < n; i += nthreads) {
        const short2 v = w[i];
        stw[i] = make_int2(v.x, v.y);
    }
    if (threadIdx.x < nsh && threadIdx.x < 8u) s_shift[threadIdx.x] = shifts[threadIdx.x];
    if constexpr (PF) {
        if (blockIdx.x * G + g < batch) prefetch(blockIdx.x * G + g);
        cp_async_commit();
    }
    __syncthreads();

    for (uint32_t b0 = blockIdx.x * G; b0 < batch; b0 += gridDim.x * G) {
        const uint32_t b = b0 + g;
        const bool active = b < batch;
        if constexpr (PF) {
            cp_async_wait_all();  // this thread's copies of transform b
        } else if (active) {
            const short2* src = x + (size_t)b * n;
            if (vecIn) {  // 16-byte loads: four points each
                const int4* s4 = reinterpret_cast<const int4*>(src);
                for (uint32_t i4 = t; i4 < n / 4u; i4 += tg) {
                    const int4 v = __ldg(s4 + i4);
                    const uint32_t i = 4u * i4;
                    sx[pad16(i)] = *reinterpret_cast<const short2*>(&v.x);
                    sx[pad16(i + 1)] = *reinterpret_cast<const short2*>(&v.y);
                    sx[pad16(i + 2)] = *reinterpret_cast<const short2*>(&v.z);
                    sx[pad16(i + 3)] = *reinterpret_cast<const short2*>(&v.w);
                }
            } else {
                for (uint32_t i = t; i < n; i += tg) sx[pad16(i)] = src[i];
            }
        }
        __syncthreads();

        uint32_t m = n, stage = 0, shift = 0;
        const int2* tw = stw;
        // An odd number of radix-4 stages (logn / 2 of them, the 8-point stage
        // included) leaves one stage outside the fused pairs; it runs first, at
        // m = n, where its butterflies read consecutive points (conflict-free)
        // — run last, at m = 4 or 8, its four loads per thread collide in banks.
        // The stages run in the same order either way, each butterfly the same.
        const uint32_t nst = logn / 2u;
        if (nst & 1u) {
            shift = s_shift[0];
            const uint32_t q = m / 4u, lq = logn - 2u;  // q = n / 4: blk = 0, k = j
            if (active) {
                const ShiftRound sr(shift, m != 8u);
                for (uint32_t j = t; j < n / 4u; j += tg) {
                    const uint32_t blk = j >> lq, k = j & (q - 1u);
                    const uint32_t base = blk * m + k;
                    uint32_t u0, u1, u2, u3;
                    if (PF) {
                        u0 = inb[base], u1 = inb[base + q], u2 = inb[base + 2 * q], u3 = inb[base + 3 * q];
                    } else {
                        u0 = su[pad16(base)], u1 = su[pad16(base + q)], u2 = su[pad16(base + 2 * q)],
                        u3 = su[pad16(base + 3 * q)];
                    }
                    bfly4_packed(u0, u1, u2, u3, (m == 4u) || (m == 8u && k == 0u), tw, k, q, sr);
                    su[pad16(base)] = u0;
                    su[pad16(base + q)] = u1;
                    su[pad16(base + 2 * q)] = u2;
                    su[pad16(base + 3 * q)] = u3;
                }
            }
            __syncthreads();
            if constexpr (PF) {  // the input buffer is free: fetch the group's next transform
                if (b + gridDim.x * G < batch) prefetch(b + gridDim.x * G);
                cp_async_commit();
            }
            tw += 3u * q;
            m = q;
            stage = 1;
        }
        // pairs of radix-4 stages fused in registers: 16 points per thread
        if constexpr (NC != 0u) {
#pragma unroll
            for (uint32_t pair = 0; pair < i16_log2(NC) / 4u; ++pair) {
                const bool first = PF && pair == 0u && !(nst & 1u);
                if (active) {
                    if (first)
                        fused_pair<true>(su, tw, m, n, t, tg, s_shift[stage], s_shift[stage + 1], inb);
                    else
                        fused_pair(su, tw, m, n, t, tg, s_shift[stage], s_shift[stage + 1]);
                }
                __syncthreads();
                if (first) {
                    if (b + gridDim.x * G < batch) prefetch(b + gridDim.x * G);
                    cp_async_commit();
                }
                shift = s_shift[stage + 1];
                tw += 3u * (m / 4u) + 3u * (m / 16u);
                m /= 16u;
                stage += 2;
            }
        } else {
            for (uint32_t pair = 0; pair < nst / 2u; ++pair) {
                if (active) fused_pair(su, tw, m, n, t, tg, s_shift[stage], s_shift[stage + 1]);
                __syncthreads();
                shift = s_shift[stage + 1];
                tw += 3u * (m / 4u) + 3u * (m / 16u);
                m /= 16u;
                stage += 2;
            }
        }
        // trailing radix-2 shares the shift of the 8-point stage
        if (m == 2u) {
            if (active) {
                for (uint32_t j = t; j < n / 2u; j += tg) {
                    const C16 a = ld(sx + pad16(2 * j)), c = ld(sx + pad16(2 * j + 1));
                    st(sx + pad16(2 * j),
                       C16{shift_round(wrap16(a.re + c.re), shift), shift_round(wrap16(a.im + c.im), shift)});
                    st(sx + pad16(2 * j + 1),
                       C16{shift_round(wrap16(a.re - c.re), shift), shift_round(wrap16(a.im - c.im), shift)});
                }
            }
            __syncthreads();
        }
        // bit-reversed gather into natural order
        if (active) {
            short2* dst = y + (size_t)b * n;
            if (vecOut && n >= 64u) {
                // outputs 4j..4j+3 come from r(4j) + {0, n/2, n/4, 3n/4} (the
                // reversed low bits are disjoint from r(4j)'s), each a multiple
                // of 16, so their padded indices are pad16(r(4j)) + pad16(offset)
                const uint32_t o1 = pad16(n / 2u), o2 = pad16(n / 4u), o3 = pad16(3u * (n / 4u));
                int4* d4 = reinterpret_cast<int4*>(dst);
                for (uint32_t j = t; j < n / 4u; j += tg) {
                    const uint32_t r = pad16(__brev(4u * j) >> (32u - logn));
                    d4[j] = make_int4((int)su[r], (int)su[r + o1], (int)su[r + o2], (int)su[r + o3]);
                }
            } else {
                for (uint32_t k = t; k < n; k += tg) {
                    const uint32_t r = logn ? (__brev(k) >> (32u - logn)) : 0u;
                    dst[k] = sx[pad16(r)];
                }
            }
        }
        __syncthreads();  // the region is reloaded next iteration
    }
}

uint32_t i16_num_shifts(uint32_t n)
{
    uint32_t s = 0;
    for (uint32_t m = n; m > 2u; m /= 4u) ++s;
    return s;
}

// The fixed-length kernels (at most 64 registers, four CTAs per SM): n / 16, timed
// faster than n / 32 at N = 256 and 4096 (20.6 / 53.3 us against 21.5 /
// 55.6 us on 16,384 / 4,096 transforms) and level at 1024 (26.7 us). The
// run-time-length kernel (80 registers, three CTAs): n / 32, timed faster
// than n / 16 at N = 256, 1024 and 4096 (27.8 / 30.8 / 74.1 us against
// 28.8 / 32.9 / 77.2 us on 16,384 / 4,096 / 2,048 transforms).
// N = 8192 and 16384: n / 16 threads (512 / 1024) on one transform per CTA;
// with 256 threads per transform one CTA per SM (shared memory) leaves 8
// warps to the SM.
uint32_t i16_default_tg(uint32_t n)
{
    return std::max(1u, std::min(i16_max_tg(n), i16_fixed_length(n, n / 16u) ? n / 16u : n / 32u));
}

uint32_t i16_max_tg(uint32_t n) { return (n == 8192u || n == 16384u) ? 1024u : 256u; }

uint32_t i16_block_threads(uint32_t tg) { return std::max(256u, tg); }

bool i16_prefetch(uint32_t n, uint32_t tg, uint32_t minBlocks)
{
    return minBlocks != 4u && n >= 64u && n <= 2048u && (n & (n - 1u)) == 0 && tg == n / 16u;
}

size_t i16_smem_bytes(uint32_t n, uint32_t tg, bool prefetch)
{
    const uint32_t G = i16_block_threads(tg) / tg;
    return (size_t)n * sizeof(int2) + (size_t)G * (n + (n >> 4)) * sizeof(short2) +
           (prefetch ? (size_t)G * n * sizeof(short2) : 0u);
}

namespace {

using I16Kernel = void (*)(const short2*, short2*, const short2*, const uint32_t*, uint32_t, uint32_t, uint32_t,
                           uint32_t, uint32_t, bool, bool);

// a length with a compile-time kernel: the default launch (n / 16 threads per
// transform) has its thread count built in too
template <uint32_t NC>
I16Kernel fixed_kernel(uint32_t minBlocks, uint32_t tg, bool prefetch)
{
    if (minBlocks == 4u) return &k_fft_i16<4, NC>;
    if (tg != NC / 16u) return &k_fft_i16<3, NC>;
    if constexpr (NC <= 2048u) {
        if (prefetch) return &k_fft_i16<3, NC, 256, NC / 16u, true>;
    }
    return &k_fft_i16<3, NC, 256, NC / 16u>;
}

// tg > 256: the 1024-thread kernels of the longest lengths (one transform per
// CTA); nullptr for other lengths. Lengths without a compile-time kernel take
// the run-time one. prefetch: the cp.async build where i16_prefetch allows it.
I16Kernel i16_kernel(uint32_t n, uint32_t minBlocks, uint32_t tg, bool prefetch)
{
    prefetch = prefetch && i16_prefetch(n, tg, minBlocks);
    if (tg > 256u) {
        if (n == 8192u) return tg == 512u ? &k_fft_i16<1, 8192u, 1024, 512u> : &k_fft_i16<1, 8192u, 1024>;
        if (n == 16384u) return tg == 1024u ? &k_fft_i16<1, 16384u, 1024, 1024u> : &k_fft_i16<1, 16384u, 1024>;
        return nullptr;
    }
    switch (n) {
    case 64u: return fixed_kernel<64u>(minBlocks, tg, prefetch);
    case 128u: return fixed_kernel<128u>(minBlocks, tg, prefetch);
    case 256u: return fixed_kernel<256u>(minBlocks, tg, prefetch);
    case 512u: return fixed_kernel<512u>(minBlocks, tg, prefetch);
    case 1024u: return fixed_kernel<1024u>(minBlocks, tg, prefetch);
    case 2048u: return fixed_kernel<2048u>(minBlocks, tg, prefetch);
    case 4096u: return fixed_kernel<4096u>(minBlocks, tg, prefetch);
    default: return minBlocks == 4u ? &k_fft_i16<4, 0u> : &k_fft_i16<3, 0u>;
    }
}

cudaError_t i16_configure(I16Kernel kern, size_t smem)
{
    static std::mutex mu;
    static std::map<std::pair<int, I16Kernel>, size_t> configured;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (smem <= 48u * 1024u) return cudaSuccess;
    std::lock_guard<std::mutex> lock(mu);
    size_t& done = configured[std::make_pair(dev, kern)];
    if (done >= smem) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) done = smem;
    return e;
}

} // namespace

bool i16_fixed_length(uint32_t n, uint32_t tg)
{
    const I16Kernel k = i16_kernel(n, 3u, tg, false);
    return k != nullptr && k != &k_fft_i16<3, 0u>;
}

int i16_resident(uint32_t n, uint32_t tg, uint32_t minBlocks)
{
    // as launched on aligned buffers
    const bool pf = i16_prefetch(n, tg, minBlocks);
    const size_t smem = i16_smem_bytes(n, tg, pf);
    const I16Kernel kern = i16_kernel(n, minBlocks, tg, pf);
    int perSm = 0;
    if (!kern || i16_configure(kern, smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, (int)i16_block_threads(tg), smem) !=
            cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return perSm;
}

cudaError_t launch_fft_i16(const int16_t* x, int16_t* y, const int16_t* w, const uint32_t* shifts,
                           uint32_t n, uint32_t batch, cudaStream_t s, uint32_t tg, uint32_t gridCap,
                           uint32_t minBlocks)
{
    if (batch == 0) return cudaSuccess;
    uint32_t logn = 0;
    while ((1u << logn) < n) ++logn;
    if (tg == 0) tg = i16_default_tg(n);
    if (tg > i16_max_tg(n) || (tg & (tg - 1u))) return cudaErrorInvalidValue;
    const bool vecIn = (((uintptr_t)x & 15u) == 0) && (n % 4u) == 0;
    const bool vecOut = (((uintptr_t)y & 15u) == 0) && (n % 4u) == 0;
    const bool pf = vecIn && i16_prefetch(n, tg, minBlocks);
    const I16Kernel kern = i16_kernel(n, minBlocks, tg, pf);
    if (!kern) return cudaErrorInvalidValue;
    const uint32_t threads = i16_block_threads(tg);
    const uint32_t G = threads / tg;
    const size_t smem = i16_smem_bytes(n, tg, pf);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = i16_configure(kern, smem);
    if (e != cudaSuccess) return e;
    int perSm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, (int)threads, smem);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const uint64_t steps = (batch + G - 1u) / G;
    uint32_t grid = (uint32_t)std::min<uint64_t>(steps, (uint64_t)std::max(1, perSm) * (uint64_t)sms);
    if (gridCap) grid = std::max(1u, std::min(grid, gridCap));
    kern<<<grid, threads, smem, s>>>((const short2*)x, (short2*)y, (const short2*)w, shifts, i16_num_shifts(n), n,
                                     logn, batch, tg, vecIn, vecOut);
    return cudaGetLastError();
}

} // namespace fftb200
