// fft_i16_arith.cuh -- the int16 FFT's butterfly arithmetic in 32-bit
// registers, bit-exact with FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_cn
// (src/fft_c7x/FFTLIB_fft1dBatched_i16sc_c16sc_o16sc/..._cn.c: satAndScale
// :13-25, crot90H :27-34, shiftRightAndRound :36-45, butterflyNoTw :47-91,
// butterfly :93-169). Host and device code (the CPU checks run it too).
//
// Values live as int32 (re, im) pairs holding int16 values; the reference's
// int16 wrap-around is applied (sign extension of the low 16 bits) only
// where a value is used non-linearly, since wrapping commutes with sums and
// differences. Two identities cut the per-output work:
//
// * shiftRightAndRound: (v >> s) + bit_{s-1}(v) = (v + 2^(s-1)) >> s for an
//   int16 v (floor division); when the reference's int16 mask
//   (1 << (shift-1)) is zero (shift 0 and shifts of 17 and up, counts taken
//   mod 32 as on x86) it is v >> s.
// * satAndScale followed by that shift: with f(v) = floor((v + add) / 2^s),
//   f(clamp(floor((x + 2^14) / 2^15))) = clamp(floor((x + K) / 2^(15+s)),
//   f(-32768), f(32767)) with K = 2^14 + add 2^15, because f is
//   non-decreasing and nested floor divisions compose. x, the exact Q15
//   product sum, is formed in 64 bits, so the reference's int64 arithmetic
//   (including the 2^31 sum of four -32768 factors) needs no special case.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define I16_HD __host__ __device__ __forceinline__
#else
#define I16_HD inline
#endif

namespace fftb200 {

struct CI {
    int32_t re, im;
};

// int16 wrap-around of a 32-bit value (sign extension of its low half)
I16_HD int32_t sx16(int32_t v) { return (int32_t)(int16_t)(uint16_t)(uint32_t)v; }

I16_HD int32_t imin(int32_t a, int32_t b) { return a < b ? a : b; }
I16_HD int32_t imax(int32_t a, int32_t b) { return a > b ? a : b; }

// Low 32 bits of v >> sh (arithmetic), 0 <= sh < 64.
I16_HD int32_t shr64_lo(int64_t v, int32_t sh)
{
#if defined(__CUDA_ARCH__)
    const uint32_t lo = (uint32_t)(uint64_t)v;
    const int32_t hi = (int32_t)(v >> 32);
    return sh < 32 ? (int32_t)__funnelshift_r(lo, (uint32_t)hi, (uint32_t)sh) : hi >> (sh - 32);
#else
    return (int32_t)(v >> sh);
#endif
}

// Per-stage constants of the shift applied after a radix-4 stage.
struct I16Shift {
    int32_t add;    // 2^(s-1) when the reference rounds, else 0
    int32_t s;      // shift & 31
    int32_t sh;     // 15 + s
    int64_t K;      // 2^14 + add 2^15
    int32_t lo, hi; // f(-32768), f(32767)
};

// apply = false: the stage is not followed by a shift (the 8-point stage).
I16_HD I16Shift i16_shift(uint32_t shift, bool apply)
{
    I16Shift c;
    if (!apply) shift = 0;
    const uint32_t rb = (shift - 1u) & 31u;
    c.s = (int32_t)(shift & 31u);
    c.add = rb < 16u ? (int32_t)(1u << rb) : 0;
    c.sh = 15 + c.s;
    c.K = (int64_t)16384 + (int64_t)c.add * 32768;
    c.lo = (-32768 + c.add) >> c.s;
    c.hi = (32767 + c.add) >> c.s;
    return c;
}

// shiftRightAndRound of an int16 value
I16_HD int32_t i16_round(int32_t v, const I16Shift& c) { return (v + c.add) >> c.s; }

// satAndScale of the exact Q15 sum x, then the stage shift
I16_HD int32_t i16_q15(int64_t x, const I16Shift& c) { return imin(imax(shr64_lo(x + c.K, c.sh), c.lo), c.hi); }

// (xr + i xi) (wr + i wi) rounded like VCMPYR1HH, then shifted
I16_HD CI i16_cmul(int32_t xr, int32_t xi, CI w, const I16Shift& c)
{
    const int64_t re = (int64_t)xr * w.re - (int64_t)xi * w.im;
    const int64_t im = (int64_t)xr * w.im + (int64_t)xi * w.re;
    return CI{i16_q15(re, c), i16_q15(im, c)};
}

// The reference's radix-4 butterfly on p0..p3 (points q apart), its outputs
// in the reference's slot order (bin 0, 2, 1, 3), each followed by the
// stage shift. notw: the twiddle-free butterfly (butterflyNoTw).
I16_HD void i16_bfly4(CI& p0, CI& p1, CI& p2, CI& p3, bool notw, CI w1, CI w2, CI w3, const I16Shift& c)
{
    const int32_t s1r = p0.re + p2.re, s1i = p0.im + p2.im;
    const int32_t s2r = p1.re + p3.re, s2i = p1.im + p3.im;
    const int32_t d1r = p0.re - p2.re, d1i = p0.im - p2.im;
    const int32_t d2r = p1.re - p3.re;
    // crot90H: j d2 = (-d2.im, d2.re), with -(-32768) saturated to 32767
    const int32_t jr = imin(-sx16(p1.im - p3.im), 32767), ji = d2r;
    const CI x0{i16_round(sx16(s1r + s2r), c), i16_round(sx16(s1i + s2i), c)};
    const int32_t x1r = sx16(d1r - jr), x1i = sx16(d1i - ji);
    const int32_t x2r = sx16(s1r - s2r), x2i = sx16(s1i - s2i);
    const int32_t x3r = sx16(d1r + jr), x3i = sx16(d1i + ji);
    CI y1, y2, y3;
    if (notw) {
        y1 = CI{i16_round(x1r, c), i16_round(x1i, c)};
        y2 = CI{i16_round(x2r, c), i16_round(x2i, c)};
        y3 = CI{i16_round(x3r, c), i16_round(x3i, c)};
    } else {
        // x0's own product with 2^15 rounds back to x0 (satAndScale of x0 << 15)
        y1 = i16_cmul(x1r, x1i, w1, c);
        y2 = i16_cmul(x2r, x2i, w2, c);
        y3 = i16_cmul(x3r, x3i, w3, c);
    }
    p0 = x0;
    p1 = y2;
    p2 = y1;
    p3 = y3;
}

} // namespace fftb200
