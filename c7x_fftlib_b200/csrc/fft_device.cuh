// fft_device.cuh -- register-level building blocks of the B200 FFT kernels.
//
// * complex helpers on float2 (x = re, y = im),
// * compile-time sin/cos of 2*pi*k/r (own Taylor-series evaluation in
//   double, used only for the constants of the small in-register DFTs),
// * dft<R>(v): an R-point forward DFT on R values held in registers, for any
//   R whose prime factors are 2, 3 and 5; composite R is split recursively
//   (radix-4 first, else the smallest prime) with the inner twiddles folded
//   to constants, so every index and constant is resolved at compile time.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <utility>

#include "fft_args.h"

#define FFT_DEV __device__ __forceinline__
// For the lambdas of static_for in the hot paths: a lambda's call operator
// is only implicitly inline, and when many instantiations of one pass share
// it the compiler may emit it as a function of its own (a call with a stack
// frame per butterfly); this keeps every body inlined.
#define FFT_INL __attribute__((always_inline))

namespace fftb200 {

// ---------------------------------------------------------------------------
// compile-time helpers
// ---------------------------------------------------------------------------

template <int... Is, class F>
FFT_DEV void static_for_impl(std::integer_sequence<int, Is...>, F&& f)
{
    (f(std::integral_constant<int, Is>{}), ...);
}

// Calls f(std::integral_constant<int, i>{}) for i = 0 .. N-1.
template <int N, class F>
FFT_DEV void static_for(F&& f)
{
    static_for_impl(std::make_integer_sequence<int, N>{}, f);
}

// sin and cos of (pi/2) * (num/den) for 0 <= num < den, by Taylor series in
// double (the argument is at most pi/2, 30 terms reach full double accuracy).
__host__ __device__ constexpr double cx_sin_quarter(long num, long den)
{
    const double x = 1.5707963267948966 * (double)num / (double)den;
    double term = x, sum = x;
    for (int n = 1; n < 30; ++n) {
        term *= -x * x / (double)((2 * n) * (2 * n + 1));
        sum += term;
    }
    return sum;
}

__host__ __device__ constexpr double cx_cos_quarter(long num, long den)
{
    const double x = 1.5707963267948966 * (double)num / (double)den;
    double term = 1.0, sum = 1.0;
    for (int n = 1; n < 30; ++n) {
        term *= -x * x / (double)((2 * n - 1) * (2 * n));
        sum += term;
    }
    return sum;
}

// cos(2*pi*k/r) and sin(2*pi*k/r) for integer k, r > 0, with the angle
// reduced exactly in integers to a quadrant.
__host__ __device__ constexpr double cx_cos2pi(long k, long r)
{
    k = ((k % r) + r) % r;
    const long a = 4 * k;          // angle = (pi/2) * a / r
    const long q = a / r;          // quadrant 0..3
    const long rem = a - q * r;    // angle within quadrant = (pi/2) * rem / r
    const double s = cx_sin_quarter(rem, r), c = cx_cos_quarter(rem, r);
    return q == 0 ? c : q == 1 ? -s : q == 2 ? -c : s;
}

__host__ __device__ constexpr double cx_sin2pi(long k, long r)
{
    k = ((k % r) + r) % r;
    const long a = 4 * k;
    const long q = a / r;
    const long rem = a - q * r;
    const double s = cx_sin_quarter(rem, r), c = cx_cos_quarter(rem, r);
    return q == 0 ? s : q == 1 ? c : q == 2 ? -s : -c;
}

// ---------------------------------------------------------------------------
// complex arithmetic
// ---------------------------------------------------------------------------

FFT_DEV float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
FFT_DEV float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
FFT_DEV float2 cmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
FFT_DEV float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
FFT_DEV float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// a * (-i)
FFT_DEV float2 cmul_negi(float2 a) { return make_float2(a.y, -a.x); }
// a * (+i)
FFT_DEV float2 cmul_posi(float2 a) { return make_float2(-a.y, a.x); }

// a * W_R^K with W_R = exp(-2*pi*i/R), K and R compile-time.
template <int R, int K>
FFT_DEV float2 cmul_w(float2 a)
{
    constexpr int k = ((K % R) + R) % R;
    if constexpr (k == 0) {
        return a;
    } else if constexpr (4 * k == R) {
        return cmul_negi(a);
    } else if constexpr (2 * k == R) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (4 * k == 3 * R) {
        return cmul_posi(a);
    } else if constexpr (8 * k == R) {          // (1 - i)/sqrt2
        constexpr float h = 0.70710678118654752f;
        return make_float2((a.x + a.y) * h, (a.y - a.x) * h);
    } else if constexpr (8 * k == 3 * R) {      // (-1 - i)/sqrt2
        constexpr float h = 0.70710678118654752f;
        return make_float2((a.y - a.x) * h, -(a.x + a.y) * h);
    } else if constexpr (8 * k == 5 * R) {      // (-1 + i)/sqrt2
        constexpr float h = 0.70710678118654752f;
        return make_float2(-(a.x + a.y) * h, (a.x - a.y) * h);
    } else if constexpr (8 * k == 7 * R) {      // (1 + i)/sqrt2
        constexpr float h = 0.70710678118654752f;
        return make_float2((a.x - a.y) * h, (a.x + a.y) * h);
    } else {
        constexpr float c = (float)cx_cos2pi(k, R);
        constexpr float s = (float)cx_sin2pi(k, R);
        // (a.x + i a.y)(c - i s)
        return make_float2(fmaf(a.x, c, a.y * s), fmaf(a.y, c, -a.x * s));
    }
}

// ---------------------------------------------------------------------------
// in-register DFT codelets (forward, natural order in and out)
// ---------------------------------------------------------------------------

__host__ __device__ constexpr int dft_split(int r)
{
    return (r % 4 == 0 && r > 4) ? 4 : (r % 2 == 0) ? 2 : (r % 3 == 0) ? 3 : 5;
}

template <int R>
FFT_DEV void dft(float2* v);

template <>
FFT_DEV void dft<1>(float2*) {}

template <>
FFT_DEV void dft<2>(float2* v)
{
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

template <>
FFT_DEV void dft<3>(float2* v)
{
    constexpr float s3 = 0.86602540378443865f; // sin(2pi/3)
    const float2 t1 = cadd(v[1], v[2]);
    const float2 t2 = csub(v[1], v[2]);
    const float2 x0 = v[0];
    const float2 m = make_float2(fmaf(-0.5f, t1.x, x0.x), fmaf(-0.5f, t1.y, x0.y));
    v[0] = cadd(x0, t1);
    // X1 = m - i s3 t2, X2 = m + i s3 t2
    v[1] = make_float2(fmaf(s3, t2.y, m.x), fmaf(-s3, t2.x, m.y));
    v[2] = make_float2(fmaf(-s3, t2.y, m.x), fmaf(s3, t2.x, m.y));
}

template <>
FFT_DEV void dft<4>(float2* v)
{
    const float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const float2 t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = make_float2(t1.x + t3.y, t1.y - t3.x); // t1 - i t3
    v[3] = make_float2(t1.x - t3.y, t1.y + t3.x); // t1 + i t3
}

template <>
FFT_DEV void dft<5>(float2* v)
{
    constexpr float c1 = 0.30901699437494742f;  // cos(2pi/5)
    constexpr float c2 = -0.80901699437494742f; // cos(4pi/5)
    constexpr float s1 = 0.95105651629515357f;  // sin(2pi/5)
    constexpr float s2 = 0.58778525229247313f;  // sin(4pi/5)
    const float2 x0 = v[0];
    const float2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    const float2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    const float2 m1 = make_float2(fmaf(c2, a2.x, fmaf(c1, a1.x, x0.x)), fmaf(c2, a2.y, fmaf(c1, a1.y, x0.y)));
    const float2 m2 = make_float2(fmaf(c1, a2.x, fmaf(c2, a1.x, x0.x)), fmaf(c1, a2.y, fmaf(c2, a1.y, x0.y)));
    const float2 n1 = make_float2(fmaf(s2, b2.x, s1 * b1.x), fmaf(s2, b2.y, s1 * b1.y));
    const float2 n2 = make_float2(fmaf(-s1, b2.x, s2 * b1.x), fmaf(-s1, b2.y, s2 * b1.y));
    v[0] = make_float2(x0.x + a1.x + a2.x, x0.y + a1.y + a2.y);
    v[1] = make_float2(m1.x + n1.y, m1.y - n1.x); // m1 - i n1
    v[4] = make_float2(m1.x - n1.y, m1.y + n1.x); // m1 + i n1
    v[2] = make_float2(m2.x + n2.y, m2.y - n2.x);
    v[3] = make_float2(m2.x - n2.y, m2.y + n2.x);
}

// Composite R = P*Q: with n = Q*n1 + n2 and k = k1 + P*k2,
//   X[k1 + P k2] = sum_n2 W_Q^{n2 k2} W_R^{n2 k1} sum_n1 x[Q n1 + n2] W_P^{n1 k1}.
template <int R>
FFT_DEV void dft(float2* v)
{
    constexpr int P = dft_split(R);
    constexpr int Q = R / P;
    static_assert(P * Q == R && Q > 1, "dft<R>: R must be 2^a 3^b 5^c");
    float2 t[R];
    static_for<Q>([&](auto n2) FFT_INL {
        float2 a[P];
        static_for<P>([&](auto n1) FFT_INL { a[n1] = v[Q * n1 + n2]; });
        dft<P>(a);
        static_for<P>([&](auto k1) FFT_INL { t[k1 * Q + n2] = cmul_w<R, decltype(n2)::value * decltype(k1)::value>(a[k1]); });
    });
    static_for<P>([&](auto k1) FFT_INL {
        float2 b[Q];
        static_for<Q>([&](auto n2) FFT_INL { b[n2] = t[k1 * Q + n2]; });
        dft<Q>(b);
        static_for<Q>([&](auto k2) FFT_INL { v[k1 + P * k2] = b[k2]; });
    });
}

// ---------------------------------------------------------------------------
// fast division (magic from fastdiv_magic in fft_args.h) and the padded
// shared-memory index
// ---------------------------------------------------------------------------

FFT_DEV uint32_t fastdiv(uint32_t j, uint32_t d, uint32_t magic)
{
    return d == 1u ? j : __umulhi(j, magic);
}

// One pad slot per 16 complex values: strided writes of radix-2^k
// butterflies then land in distinct banks.
FFT_DEV uint32_t smem_swz(uint32_t idx) { return idx + (idx >> 4); }

} // namespace fftb200
