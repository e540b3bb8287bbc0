// fft_stockham.cuh -- the FP32 batched FFT engine (device side).
//
// One CTA holds M transforms of length N in shared memory. T threads work on
// one transform; in each Stockham pass a thread gathers its butterflies'
// inputs into registers (up to EMAX complex values), applies the pass
// twiddles, runs the in-register DFT codelet and scatters the outputs.
// The first pass reads straight from HBM (or from a shared-memory tile for
// short transforms) and the last pass writes straight to HBM in natural
// order, so the reference's separate bit/digit-reversal copy
// (FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_cn.c:412-491) disappears into the
// pass index arithmetic: each transform costs one HBM read and one HBM write.
//
// The inverse transform is conj(FFT(conj(x))) * scale, applied on load and
// store (FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_cn.c:209-227, 432-506).
// Real-input variants fuse the reference's split post-process
// (FFTLIB_fft1dBatched_i32f_c32fc_o32fc_cn.c:40-121) into an epilogue and
// its split pre-process (FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_cn.c:35-83)
// into the first pass.
#pragma once

#include "fft_args.h"
#include "fft_device.cuh"

namespace fftb200 {

// Smallest radix an engine instantiation carries: the widest one leaves the
// short radices (many butterflies per thread, large unrolled code) to the
// narrower instantiations.
__host__ __device__ constexpr int engine_min_radix(int emax) { return emax >= 32 ? 8 : 1; }

// Calls f(integral_constant<R>) for the runtime radix r; radices are the
// 2^a 3^b 5^c values in [engine_min_radix(EMAX), EMAX] (1 is the trivial
// one-point transform).
template <int EMAX, class F>
FFT_DEV void dispatch_radix(int r, F&& f)
{
    static_for<EMAX + 1>([&](auto d) FFT_INL {
        constexpr int D = decltype(d)::value;
        constexpr bool ok235 = [] {
            int x = D;
            if (x < 1 || x < engine_min_radix(EMAX)) return false;
            while (x % 2 == 0) x /= 2;
            while (x % 3 == 0) x /= 3;
            while (x % 5 == 0) x /= 5;
            return x == 1;
        }();
        if constexpr (ok235) {
            if (r == D) f(d);
        }
    });
}

// Pass-0 input element idx of transform b (complex index into the pass's
// length-N sequence), with the c2r split pre-process when requested.
FFT_DEV float2 load_in(const FftArgs& a, const float2* rowIn, uint32_t idx, const float2* tile)
{
    float2 z;
    if (a.ioMode == IO_C2R_SPLIT) {
        // Z = X A' + y B' = 0.5 [(X + y) + i conj(W) (X - y)], W = W_{2h}^idx,
        // y = conj(X[h - idx]) (inMode 0) or X[idx + h] (inMode 1).
        const uint32_t h = a.N;
        const uint32_t ip = a.realMode ? idx + h : h - idx;
        float2 x, y;
        if (a.staged) {
            x = tile[smem_swz(idx)];
            y = tile[smem_swz(ip)];
        } else {
            x = rowIn[(int64_t)idx * a.inElem];
            y = rowIn[(int64_t)ip * a.inElem];
        }
        if (!a.realMode) y = cconj(y);
        const float2 w = __ldg(&a.twSplit[idx]);
        const float2 s = cadd(x, y), d = csub(x, y);
        const float2 icw = make_float2(w.y, w.x); // i * conj(w)
        z = cscale(cadd(s, cmul(icw, d)), 0.5f);
    } else if (a.staged) {
        z = tile[smem_swz(idx)];
    } else {
        z = rowIn[(int64_t)idx * a.inElem];
    }
    return a.conjIn ? cconj(z) : z;
}

FFT_DEV float2 finish(const FftArgs& a, float2 z)
{
    if (a.conjOut) z = cconj(z);
    return cscale(z, a.scale);
}

// One pass. pi, first, last and T are either runtime values (the generic
// engine) or compile-time constants (the fixed-size kernels), in which case
// all index arithmetic folds away after inlining.
struct NoHook {
    FFT_DEV void operator()() const {}
};

// Padded index of idx0 + q*step for q < R: when step is a multiple of 16 the
// pad of every element equals the pad of idx0 plus q*step/16, so one padded
// base serves the whole butterfly.
FFT_DEV uint32_t swz_step(uint32_t swzBase, uint32_t idx0, uint32_t q, uint32_t step)
{
    return (step & 15u) == 0u ? swzBase + q * (step + (step >> 4)) : smem_swz(idx0 + q * step);
}

// Exchange layouts between two passes: kPad16, one pad slot per 16 values
// (smem_swz; conflict-free for the power-of-two strides of radix-2^k
// scatters), or kNoPad, the plain index: a first pass of odd radix R
// scatters with stride R (Ns = 1), which is conflict-free unpadded but
// collides in banks with the pad, and the next pass gathers consecutive
// values either way.
constexpr int kPad16 = 0, kNoPad = 1;

template <int L>
FFT_DEV uint32_t lay(uint32_t idx)
{
    return L == kNoPad ? idx : smem_swz(idx);
}
// lay<L>(idx0 + q * step) from base = lay<L>(idx0)
template <int L>
FFT_DEV uint32_t lay_step(uint32_t base, uint32_t idx0, uint32_t q, uint32_t step)
{
    return L == kNoPad ? base + q * step : swz_step(base, idx0, q, step);
}

// The layout of the boundary after pass 0 of a compile-time schedule whose
// first radix is R0 (the boundaries after later passes keep kPad16).
__host__ __device__ constexpr int first_boundary_layout(int r0) { return (r0 % 2) ? kNoPad : kPad16; }

// raw: when not null, the first pass reads its input from this unpadded
// shared-memory copy of the transform (filled by a bulk async copy);
// RAW_FIRST: raw is never null (only that path is compiled).
// LIN / LOUT: the exchange layout this pass gathers from (when it is not the
// first) and scatters to.
// afterGather runs right after the barrier that ends the pass's reads.
// rowIn / rowOut: this lane's transform in HBM (first / last pass).
// UNIT: the caller guarantees outElem == 1 (rows of contiguous values), so
// the last pass's stores take constant offsets from rowOut.
// MIRROR (kMirrorC2R on a first pass, kMirrorR2C on a last pass; the caller
// guarantees two butterflies per thread and T = nb / 2): thread t takes the
// butterflies t and nb - t (thread 0: 0 and nb / 2), whose values are the
// mirror images h - i of each other, so the real-signal split runs in
// registers: kMirrorC2R turns the raw h + 1 bins into the half-length input
// Z before the butterflies, kMirrorR2C writes the h + 1 (or 2h) bins from the
// butterfly outputs instead of scattering them.
constexpr int kMirrorNone = 0, kMirrorC2R = 1, kMirrorR2C = 2;

FFT_DEV uint32_t mirror_j(uint32_t t, int i, uint32_t nb) { return i == 0 ? t : (t == 0 ? nb / 2u : nb - t); }

FFT_DEV float2 r2c_split(float2 z, float2 zp, float2 w);
FFT_DEV void r2c_split_pair(float2 z, float2 zm, float2 w, float2& y, float2& ym);
FFT_DEV float2 c2r_split(float2 x, float2 xm, float2 w);
FFT_DEV void c2r_split_pair(float2 x, float2 xm, float2 w, float2& z, float2& zm);
template <int R>
FFT_DEV void c2r_mirror_split(const FftArgs& a, float2* v, uint32_t t, uint32_t nb, const float2* raw,
                              const float2 (&w)[R + 1]);
template <int R>
FFT_DEV void r2c_mirror_store(const FftArgs& a, const float2* v, uint32_t t, uint32_t nb, float2* row,
                              const float2 (&w)[R + 1]);

// Split-table index of slot q (0..R) of a mirrored pass: t + q nb for
// thread t != 0 (slot R repeats slot 0); for thread 0, q nb (q <= R/2), then
// nb/2 + (q - R/2 - 1) nb. The loads are issued before the pass's gather.
template <int R>
FFT_DEV uint32_t mirror_tw_index(uint32_t t, int q, uint32_t nb)
{
    const uint32_t q0 = (uint32_t)(q <= R / 2 ? q : q - R / 2 - 1);
    const uint32_t t0 = q <= R / 2 ? 0u : nb / 2u;
    return t != 0u ? t + (uint32_t)(q < R ? q : 0) * nb : t0 + q0 * nb;
}

template <int EMAX, int R, class Hook = NoHook, bool RAW_FIRST = false, int LIN = kPad16, int LOUT = kPad16,
          bool UNIT = false, int MIRROR = kMirrorNone>
FFT_DEV void run_pass(const FftArgs& a, const PassInfo pi, const bool first, const bool last,
                      const uint32_t T, float2 (&v)[EMAX], float2* sm, uint32_t t, bool active,
                      const float2* rowIn, float2* rowOut, const float2* raw = nullptr,
                      Hook afterGather = Hook())
{
    constexpr int BMAX = EMAX / R;
    static_assert(MIRROR == kMirrorNone || BMAX == 2, "the mirrored passes hold two butterflies per thread");
    const uint32_t nb = pi.stride; // butterflies in this pass: N / R
    auto bfly = [&](int i) FFT_INL { return MIRROR ? mirror_j(t, i, nb) : t + (uint32_t)i * T; };
    // the mirrored split's table entries, in flight during the gather
    [[maybe_unused]] float2 wsplit[MIRROR ? R + 1 : 1];
    if constexpr (MIRROR != kMirrorNone) {
        static_for<R + 1>([&](auto q) FFT_INL {
            wsplit[q] = __ldg(&a.twSplit[mirror_tw_index<R>(t, decltype(q)::value, nb)]);
        });
    }

    // gather
    static_for<BMAX>([&](auto i) FFT_INL {
        const uint32_t j = bfly(i);
        if (j < nb) {
            const uint32_t sj = lay<LIN>(j);
            static_for<R>([&](auto q) FFT_INL {
                const uint32_t idx = j + (uint32_t)q * nb;
                float2 z;
                if (first && (RAW_FIRST || raw)) {
                    z = raw[idx];  // conjugated below, once for the whole gather
                } else if (first && !RAW_FIRST) {
                    z = (active || a.staged) ? load_in(a, rowIn, idx, sm) : make_float2(0.f, 0.f);
                } else {
                    z = sm[lay_step<LIN>(sj, j, (uint32_t)q, nb)];
                }
                v[i * R + q] = z;
            });
        }
    });
    if constexpr (MIRROR == kMirrorC2R) c2r_mirror_split<R>(a, v, t, nb, raw, wsplit);
    // one uniform branch around the input conjugation of the inverse
    if (first && (RAW_FIRST || raw) && a.conjIn) {
        static_for<BMAX * R>([&](auto e) FFT_INL { v[e] = cconj(v[e]); });
    }

    // twiddle and butterfly
    static_for<BMAX>([&](auto i) FFT_INL {
        const uint32_t j = bfly(i);
        if (j < nb) {
            if (!first) {
                const uint32_t g = fastdiv(j, pi.Ns, pi.nsMagic);
                const uint32_t k = j - g * pi.Ns;
                // lanes of a warp read consecutive k: coalesced twiddle loads
                const float2* tw = a.tw + pi.twOffset + k;
                static_for<R - 1>([&](auto q1) FFT_INL {
                    constexpr int q = decltype(q1)::value + 1;
                    v[i * R + q] = cmul(v[i * R + q], __ldg(&tw[(q - 1) * pi.Ns]));
                });
            }
            dft<R>(&v[i * R]);
        }
    });

    if constexpr (MIRROR == kMirrorR2C) {
        if (active) r2c_mirror_store<R>(a, v, t, nb, rowOut, wsplit);
        return;
    }

    // scatter
    const bool direct = last && !a.staged && a.ioMode != IO_R2C_SPLIT;
    if (direct) {
        if (active) {
            float2* row = rowOut;
            // conjugation and scale of the inverse in one uniform branch (the
            // forward transform stores the butterfly outputs as they are)
            if (a.conjOut || a.scale != 1.0f) {
                static_for<BMAX * R>([&](auto e) FFT_INL { v[e] = finish(a, v[e]); });
            }
            static_for<BMAX>([&](auto i) FFT_INL {
                const uint32_t j = bfly(i);
                if (j < nb) {
                    static_for<R>([&](auto q) FFT_INL {
                        const uint32_t idx = j + (uint32_t)q * nb;
                        if constexpr (UNIT) row[idx] = v[i * R + q];
                        else row[(int64_t)idx * a.outElem] = v[i * R + q];
                    });
                }
            });
        }
        return;
    }
    if (!first || a.staged || RAW_FIRST || raw) {
        __syncthreads(); // every read of this pass is done
        afterGather();
    }
    static_for<BMAX>([&](auto i) FFT_INL {
        const uint32_t j = bfly(i);
        if (j < nb) {
            const uint32_t g = fastdiv(j, pi.Ns, pi.nsMagic);
            const uint32_t k = j - g * pi.Ns;
            const uint32_t base = g * pi.Ns * (uint32_t)R + k;
            const uint32_t sb = lay<LOUT>(base);
            // Ns = 1 with R = 16: base is a multiple of 16 and q < 16 share its pad
            const bool contiguous16 = LOUT == kPad16 && pi.Ns == 1u && R == 16;
            static_for<R>([&](auto q) FFT_INL {
                const uint32_t d = contiguous16 ? sb + (uint32_t)q : lay_step<LOUT>(sb, base, (uint32_t)q, pi.Ns);
                sm[d] = v[i * R + q];
            });
        }
    });
    __syncthreads();
}

// Y[i] = E + (-i W) O, E = (Z[i] + conj Z[h-i]) / 2, O = (Z[i] - conj Z[h-i]) / 2,
// W = W_{2h}^i: the reference's A[i] Z[i] + B[i] conj(Z[h-i]).
FFT_DEV float2 r2c_split(float2 z, float2 zp, float2 w)
{
    const float2 zc = cconj(zp);
    const float2 e = cscale(cadd(z, zc), 0.5f);
    const float2 o = cscale(csub(z, zc), 0.5f);
    const float2 miw = make_float2(w.y, -w.x); // -i * w
    return cadd(e, cmul(miw, o));
}

// Both bins of the pair (i, h - i) at once: y = e + q and ym = conj(e - q),
// q = -i w o, the mirrored bin's twiddle W_{2h}^(h-i) = -conj(w) folded into
// the conjugate (16 floating-point operations for the two).
FFT_DEV void r2c_split_pair(float2 z, float2 zm, float2 w, float2& y, float2& ym)
{
    const float2 e = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
    const float2 o = make_float2(0.5f * (z.x - zm.x), 0.5f * (z.y + zm.y));
    const float2 q = make_float2(fmaf(w.x, o.y, w.y * o.x), fmaf(w.y, o.y, -w.x * o.x));
    y = make_float2(e.x + q.x, e.y + q.y);
    ym = make_float2(e.x - q.x, q.y - e.y);
}

// Z[i] = ((X[i] + y) + i conj(W) (X[i] - y)) / 2, y = conj(X[h - i]), W = W_{2h}^i:
// the reference's X[i] A'[i] + conj(X[h - i]) B'[i].
FFT_DEV float2 c2r_split(float2 x, float2 xm, float2 w)
{
    const float2 y = cconj(xm);
    const float2 sum = cadd(x, y), d = csub(x, y);
    const float2 icw = make_float2(w.y, w.x);  // i * conj(w)
    return cscale(cadd(sum, cmul(icw, d)), 0.5f);
}

// Both Z of the pair (i, h - i): z = (s + p) / 2 and zm = conj(s - p) / 2 with
// s = x + conj(xm), p = i conj(w) (x - conj(xm)).
FFT_DEV void c2r_split_pair(float2 x, float2 xm, float2 w, float2& z, float2& zm)
{
    const float2 s = make_float2(x.x + xm.x, x.y - xm.y);
    const float2 d = make_float2(x.x - xm.x, x.y + xm.y);
    const float2 p = make_float2(fmaf(w.y, d.x, -w.x * d.y), fmaf(w.y, d.y, w.x * d.x));
    z = make_float2(0.5f * (s.x + p.x), 0.5f * (s.y + p.y));
    zm = make_float2(0.5f * (s.x - p.x), 0.5f * (p.y - s.y));
}

// c2r (inMode 0) split of the first pass's raw bins in registers. v[q] is
// X[j0 + q nb], v[R + q] is X[j1 + q nb] with (j0, j1) = (t, nb - t), or
// (0, nb / 2) for thread 0; the mirror h - i of j0 + q nb is j1 + (R-1-q) nb,
// of q nb (thread 0) (R - q) nb, and of bin 0 the Nyquist bin X[h] (raw[h]).
// W_{2h}^(h-i) = -conj(W_{2h}^i): one table load serves each pair.
template <int R>
FFT_DEV void c2r_mirror_split(const FftArgs& a, float2* v, uint32_t t, uint32_t nb, const float2* raw,
                              const float2 (&w)[R + 1])
{
    if (t != 0u) {
        static_for<R>([&](auto q) FFT_INL {
            constexpr int qq = decltype(q)::value;
            c2r_split_pair(v[qq], v[2 * R - 1 - qq], w[qq], v[qq], v[2 * R - 1 - qq]);
        });
        return;
    }
    const float2 xh = raw[a.N];
    v[0] = c2r_split(v[0], xh, w[0]);
    static_for<R / 2>([&](auto q1) FFT_INL {
        constexpr int q = decltype(q1)::value + 1;  // pairs (q, R - q), q = R/2 alone
        if constexpr (q != R - q) c2r_split_pair(v[q], v[R - q], w[q], v[q], v[R - q]);
        else v[q] = c2r_split(v[q], v[q], w[q]);
    });
    static_for<R / 2>([&](auto q1) FFT_INL {
        constexpr int q = decltype(q1)::value;  // pairs (q, R-1-q) of butterfly nb / 2
        c2r_split_pair(v[R + q], v[2 * R - 1 - q], w[R / 2 + 1 + q], v[R + q], v[2 * R - 1 - q]);
    });
}

// r2c split of the last pass's outputs in registers (the pairing of
// c2r_mirror_split), written as bins i and h - i of row (and, with
// realMode, their conjugates at 2h - i).
template <int R>
FFT_DEV void r2c_mirror_store(const FftArgs& a, const float2* v, uint32_t t, uint32_t nb, float2* row,
                              const float2 (&w)[R + 1])
{
    const uint32_t h = a.N;
    const bool full = a.realMode != 0;
    auto put = [&](uint32_t i, float2 y) FFT_INL {
        row[i] = y;
        if (full) row[2u * h - i] = cconj(y);
    };
    if (t != 0u) {
        static_for<R>([&](auto q) FFT_INL {
            constexpr int qq = decltype(q)::value;
            const uint32_t i = t + (uint32_t)qq * nb;
            float2 y, ym;
            r2c_split_pair(v[qq], v[2 * R - 1 - qq], w[qq], y, ym);
            put(i, y);
            put(h - i, ym);
        });
        return;
    }
    const float2 z0 = v[0];
    row[0] = make_float2(z0.x + z0.y, 0.f);
    row[h] = make_float2(z0.x - z0.y, 0.f);  // Nyquist bin
    static_for<R / 2>([&](auto q1) FFT_INL {
        constexpr int q = decltype(q1)::value + 1;
        const uint32_t i = (uint32_t)q * nb;
        if constexpr (q != R - q) {
            float2 y, ym;
            r2c_split_pair(v[q], v[R - q], w[q], y, ym);
            put(i, y);
            put(h - i, ym);
        } else {
            put(i, r2c_split(v[q], v[q], w[q]));
        }
    });
    static_for<R / 2>([&](auto q1) FFT_INL {
        constexpr int q = decltype(q1)::value;
        const uint32_t i = nb / 2u + (uint32_t)q * nb;
        float2 y, ym;
        r2c_split_pair(v[R + q], v[2 * R - 1 - q], w[R / 2 + 1 + q], y, ym);
        put(i, y);
        put(h - i, ym);
    });
}

FFT_DEV void r2c_epilogue(const FftArgs& a, const float2* sm, uint32_t t, float2* row, bool active)
{
    if (!active) return;
    const uint32_t h = a.N;
    for (uint32_t i = t; i <= h / 2; i += a.T) {
        if (i == 0) {
            const float2 z0 = sm[smem_swz(0)];
            row[0] = make_float2(z0.x + z0.y, 0.f);
            row[h] = make_float2(z0.x - z0.y, 0.f); // Nyquist bin
            continue;
        }
        const uint32_t ip = h - i;
        const float2 zi = sm[smem_swz(i)], zp = sm[smem_swz(ip)];
        // W_{2h}^(h-i) = -conj(W_{2h}^i): one table load serves the pair,
        // with the accuracy of the table's own entry (FP64 rounded to FP32)
        const float2 w = __ldg(&a.twSplit[i]);
        float2 yi, yp;
        r2c_split_pair(zi, zp, w, yi, yp);
        row[i] = yi;
        if (a.realMode) row[2 * h - i] = cconj(yi);
        if (ip != i) {
            row[ip] = yp;
            if (a.realMode) row[2 * h - ip] = cconj(yp);
        }
    }
}

// Offset (complex elements) of transform b's first input / output element.
FFT_DEV int64_t row_in(const FftArgs& a, uint32_t b)
{
    if (a.perCh == 0u) return (int64_t)b * a.inBatch;
    const uint32_t c = b / a.perCh;
    return (int64_t)c * a.inChStride + (int64_t)(b - c * a.perCh) * a.inBatch;
}

FFT_DEV int64_t row_out(const FftArgs& a, uint32_t b)
{
    if (a.perCh == 0u) return (int64_t)b * a.outBatch;
    const uint32_t c = b / a.perCh;
    const uint32_t j = b - c * a.perCh;
    int64_t off = (int64_t)c * a.outChStride;
    if (a.outGroup) {
        const uint32_t g = j / a.outGroup;
        off += (int64_t)g * a.outGroupStride + (int64_t)(j - g * a.outGroup) * a.outBatch;
    } else {
        off += (int64_t)j * a.outBatch;
    }
    return off;
}

// Cooperative, coalesced copy of the CTA's input into the per-transform
// shared-memory regions. Rows (inElem 1): the tile's transforms lie back to
// back. Columns (inElem != 1, a full tile of M transforms inside one
// channel, and inside one twNs block when the input twiddle is on):
// element i of the tile's transforms is a run of M adjacent values.
// U: column loads in flight per thread before their shared-memory stores.
// 4 by default; 8 for the 1024-point pass kernel, whose large column tiles
// hold few CTAs per SM anyway (4 transforms of 2^20 points as 1024 x 1024
// passes: 83 -> 75 us),
// while at 256 points the extra registers cost a CTA per SM (2^24: 0.308 ->
// 0.339 ms with 8).
template <int U = 4>
FFT_DEV void stage_in(const FftArgs& a, float2* smem, uint32_t b0)
{
    const uint32_t inCount = a.inCount, slen = a.slen;
    const uint32_t nm = min(a.M, a.batch - b0);
    const uint32_t total = nm * inCount;
    const float2* src = a.in + row_in(a, b0);
    if (a.inElem != 1) {
        const uint32_t j0 = a.twLo ? (b0 % a.perCh) % a.twNs : 0u;
        const uint32_t step = blockDim.x;
        for (uint32_t e0 = threadIdx.x; e0 < total; e0 += U * step) {
            float2 z[U], wl[U], wh[U];
            static_for<U>([&](auto u) FFT_INL {
                const uint32_t e = e0 + (uint32_t)u * step;
                if (e < total) {
                    const uint32_t i = fastdiv(e, a.M, a.mMagic);
                    const uint32_t mm = e - i * a.M;
                    z[u] = src[(int64_t)i * a.inElem + (int64_t)mm * a.inBatch];
                    if (a.twLo) {
                        const uint32_t p = i * (j0 + mm) * a.twStep;
                        wl[u] = __ldg(&a.twLo[p & ((1u << a.twLoBits) - 1u)]);
                        wh[u] = __ldg(&a.twHi[p >> a.twLoBits]);
                    }
                }
            });
            static_for<U>([&](auto u) FFT_INL {
                const uint32_t e = e0 + (uint32_t)u * step;
                if (e < total) {
                    const uint32_t i = fastdiv(e, a.M, a.mMagic);
                    const uint32_t mm = e - i * a.M;
                    // (conjIn is applied when the first pass reads the tile;
                    // passes with an input twiddle have conjIn 0)
                    float2 v = z[u];
                    if (a.twLo) v = cmul(v, cmul(wl[u], wh[u]));
                    smem[mm * slen + smem_swz(i)] = v;
                }
            });
        }
        return;
    }
    const uint32_t inMagic = a.inMagic;
    for (uint32_t e = threadIdx.x; e < total; e += blockDim.x) {
        const uint32_t mm = fastdiv(e, inCount, inMagic);
        const uint32_t i = e - mm * inCount;
        smem[mm * slen + smem_swz(i)] = src[e];
    }
}

// Counterpart of stage_in for the outputs (columns: a full tile inside one
// outGroup block).
FFT_DEV void stage_out(const FftArgs& a, const float2* smem, uint32_t b0)
{
    const uint32_t slen = a.slen;
    const uint32_t nm = min(a.M, a.batch - b0);
    const uint32_t total = nm * a.N;
    float2* dst = a.out + row_out(a, b0);
    if (a.outElem != 1) {
        for (uint32_t e = threadIdx.x; e < total; e += blockDim.x) {
            const uint32_t i = fastdiv(e, a.M, a.mMagic);
            const uint32_t mm = e - i * a.M;
            dst[(int64_t)i * a.outElem + (int64_t)mm * a.outBatch] = finish(a, smem[mm * slen + smem_swz(i)]);
        }
        return;
    }
    for (uint32_t e = threadIdx.x; e < total; e += blockDim.x) {
        const uint32_t mm = fastdiv(e, a.N, a.nMagic);
        const uint32_t i = e - mm * a.N;
        dst[e] = finish(a, smem[mm * slen + smem_swz(i)]);
    }
}

// Thread -> (transform m, lane t) mapping of a CTA.
FFT_DEV void lane_of(const FftArgs& a, uint32_t T, uint32_t* m, uint32_t* t)
{
    const uint32_t tid = threadIdx.x;
    if (a.batchMinor) {
        *t = tid / a.M;
        *m = tid - *t * a.M;
    } else {
        *m = tid / T;
        *t = tid - *m * T;
    }
}

// Whole-transform body for the CTA's transforms b0 .. b0+M-1 (schedule read
// from a.pass at run time).
// A staged tile of M transforms is computed in groups of Mc (a uniform loop:
// every thread takes part in every group's barriers).
FFT_DEV uint32_t tile_groups(const FftArgs& a) { return a.M / tile_group(a); }

template <int EMAX>
FFT_DEV void fft_tile(const FftArgs& a, float2* smem, uint32_t b0)
{
    uint32_t m0, t;
    lane_of(a, a.T, &m0, &t);
    if (a.staged) {
        stage_in(a, smem, b0);
        __syncthreads();
    }
    const uint32_t groups = tile_groups(a), mc = tile_group(a);
    for (uint32_t g = 0; g < groups; ++g) {
        const uint32_t m = g * mc + m0;
        const uint32_t b = b0 + m;
        const bool active = b < a.batch;
        float2* sm = smem + m * a.slen;
        const float2* rowIn = a.in + row_in(a, b);
        float2* rowOut = a.out + row_out(a, b);
        float2 v[EMAX];
        for (int p = 0; p < (int)a.P; ++p) {
            dispatch_radix<EMAX>(a.pass[p].R, [&](auto r) {
                run_pass<EMAX, decltype(r)::value>(a, a.pass[p], p == 0, p + 1 == (int)a.P, a.T, v, sm, t, active,
                                                   rowIn, rowOut);
            });
        }
        if (a.ioMode == IO_R2C_SPLIT) r2c_epilogue(a, sm, t, rowOut, active);
    }
    if (a.staged && a.ioMode != IO_R2C_SPLIT) stage_out(a, smem, b0);
}

// Compile-time schedule: length N, register capacity EMAX, T threads per
// transform, pass radices Rs... (the same pass layout and twiddle-table
// layout as the runtime planner produces).
template <int N_, int EMAX_, int T_, int... Rs>
struct StaticSchedule {
    static constexpr int N = N_, EMAX = EMAX_, T = T_, P = sizeof...(Rs);
    static constexpr int R[P] = {Rs...};
    static constexpr PassInfo pass(int p)
    {
        uint32_t ns = 1, off = 0;
        for (int i = 0; i < p; ++i) {
            if (i > 0) off += (uint32_t)(R[i] - 1) * ns;
            ns *= (uint32_t)R[i];
        }
        PassInfo pi{};
        pi.R = R[p];
        pi.Ns = ns;
        pi.nsMagic = fastdiv_magic(ns);
        pi.stride = (uint32_t)(N / R[p]);
        pi.twOffset = off;
        return pi;
    }
};

template <class S>
FFT_DEV void fft_tile_static(const FftArgs& a, float2* smem, uint32_t b0)
{
    uint32_t m0, t;
    lane_of(a, (uint32_t)S::T, &m0, &t);
    if (a.staged) {
        stage_in<S::N == 1024 ? 8 : 4>(a, smem, b0);
        __syncthreads();
    }
    const uint32_t groups = tile_groups(a), mc = tile_group(a);
    for (uint32_t g = 0; g < groups; ++g) {
        const uint32_t m = g * mc + m0;
        const uint32_t b = b0 + m;
        const bool active = b < a.batch;
        float2* sm = smem + m * a.slen;
        const float2* rowIn = a.in + row_in(a, b);
        float2* rowOut = a.out + row_out(a, b);
        float2 v[S::EMAX];
        static_for<S::P>([&](auto p) FFT_INL {
            constexpr int P = decltype(p)::value;
            constexpr PassInfo pi = S::pass(P);
            // (a one-pass schedule's only boundary is read by the r2c
            // epilogue or the staged store, in the padded layout)
            constexpr int L0 = S::P > 1 ? first_boundary_layout(S::R[0]) : kPad16;
            run_pass<S::EMAX, S::R[P], NoHook, false, P == 1 ? L0 : kPad16, P == 0 ? L0 : kPad16>(
                a, pi, P == 0, P + 1 == S::P, (uint32_t)S::T, v, sm, t, active, rowIn, rowOut);
        });
        if (a.ioMode == IO_R2C_SPLIT) r2c_epilogue(a, sm, t, rowOut, active);
    }
    if (a.staged && a.ioMode != IO_R2C_SPLIT) stage_out(a, smem, b0);
}

} // namespace fftb200
