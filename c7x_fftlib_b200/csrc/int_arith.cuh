// int_arith.cuh -- exact integer arithmetic of the reference's natural C
// (FFTLIB_utility.h): accumulator types, saturation, shift-and-round and
// multiply-adds, shared by the integer DFT and matrix-multiply kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fftb200 {

template <class T> struct IntT;
template <> struct IntT<int8_t> {  // the LINALG multiply's INT8 data, int32 sums
    using Acc = int32_t;
    static constexpr int kBits = 8;
    static constexpr uint32_t kMma = 64;
};
template <> struct IntT<int16_t> {
    using Acc = long long;
    static constexpr int kBits = 16;
    static constexpr uint32_t kMma = 32;
};
template <> struct IntT<int32_t> {
    using Acc = __int128;
    static constexpr int kBits = 32;
    static constexpr uint32_t kMma = 16;
};

// ---- integer helpers (FFTLIB_utility.h) --------------------------------------

template <class T>
__device__ __forceinline__ T sat_to(typename IntT<T>::Acc x)
{
    using Acc = typename IntT<T>::Acc;
    constexpr long long mx = (1ll << (IntT<T>::kBits - 1)) - 1;
    if (x < 0) return x < (Acc)(-mx - 1) ? (T)(-mx - 1) : (T)(long long)x;
    if constexpr (IntT<T>::kBits == 32) {
        // the reference tests only the low 64 bits of a non-negative value
        const unsigned long long lo = (unsigned long long)x;
        return (lo & 0xFFFFFFFF80000000ull) ? (T)mx : (T)(long long)lo;
    } else {
        return x > (Acc)mx ? (T)mx : (T)x;
    }
}

// Arithmetic right shift; counts at or past the accumulator width give the
// sign (the reference's behaviour there is undefined).
template <class Acc>
__device__ __forceinline__ Acc sra(Acc x, uint32_t k)
{
    constexpr uint32_t w = sizeof(Acc) * 8u;
    if (k >= w) return x < 0 ? (Acc)-1 : (Acc)0;
    return x >> k;
}

// Round half up after a right shift by `shift` (its low byte, the
// reference's uint8_t parameter; 0: saturate only).
template <class T>
__device__ __forceinline__ T shift_round(typename IntT<T>::Acc x, uint32_t shift)
{
    const uint32_t s = shift & 0xFFu;
    if (s == 0) return sat_to<T>(x);
    return sat_to<T>(sra(sra(x, s - 1) + 1, 1u));
}

template <class T>
__device__ __forceinline__ T neg_sat(T a)
{
    constexpr long long mx = (1ll << (IntT<T>::kBits - 1)) - 1;
    return (long long)a == -mx - 1 ? (T)mx : (T)-a;
}

template <class T>
__device__ __forceinline__ typename IntT<T>::Acc mul(T a, T b)
{
    return (typename IntT<T>::Acc)((long long)a * (long long)b);
}

// acc + a b, exact: one 32 x 32 -> 64-bit multiply-add for INT16 data, a
// 64-bit product added into the 128-bit sum for INT32. INT8 products are
// summed in 32 bits, wrapping where the reference's int32 sum would overflow
// (undefined behaviour in its C).
__device__ __forceinline__ int32_t mac(int32_t acc, int8_t a, int8_t b)
{
    return (int32_t)((uint32_t)acc + (uint32_t)((int32_t)a * (int32_t)b));
}
__device__ __forceinline__ long long mac(long long acc, int16_t a, int16_t b)
{
    long long d;
    asm("mad.wide.s32 %0, %1, %2, %3;" : "=l"(d) : "r"((int)a), "r"((int)b), "l"(acc));
    return d;
}
__device__ __forceinline__ __int128 mac(__int128 acc, int32_t a, int32_t b)
{
    long long p;
    asm("mul.wide.s32 %0, %1, %2;" : "=l"(p) : "r"(a), "r"(b));
    return acc + (__int128)p;
}

} // namespace fftb200
