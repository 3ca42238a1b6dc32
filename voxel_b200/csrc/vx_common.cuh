// Device-side helpers shared by every kernel of the VoxelVM B200 backend.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "vx_types.h"

namespace vx {

// ---- element-type traits ---------------------------------------------------

template <typename T> struct Traits;
template <> struct Traits<double> { static constexpr int kId = F64; static constexpr bool kFloat = true; };
template <> struct Traits<float> { static constexpr int kId = F32; static constexpr bool kFloat = true; };
template <> struct Traits<int64_t> { static constexpr int kId = I64; static constexpr bool kFloat = false; };
template <> struct Traits<int32_t> { static constexpr int kId = I32; static constexpr bool kFloat = false; };
template <> struct Traits<uint64_t> { static constexpr int kId = U64; static constexpr bool kFloat = false; };
template <> struct Traits<uint32_t> { static constexpr int kId = U32; static constexpr bool kFloat = false; };

template <typename T>
__device__ __forceinline__ T from_bits(uint64_t b) {
    if constexpr (sizeof(T) == 8) return __builtin_bit_cast(T, b);
    else return __builtin_bit_cast(T, static_cast<uint32_t>(b));
}
template <typename T>
__device__ __forceinline__ uint64_t to_bits(T v) {
    if constexpr (sizeof(T) == 8) return __builtin_bit_cast(uint64_t, v);
    else return static_cast<uint64_t>(__builtin_bit_cast(uint32_t, v));
}

// Engine<T>::SetScalarT: the register image of a T result.  f32 results are
// widened to f64 (the backend's f32 register convention); signed 32-bit values
// are sign-extended, unsigned zero-extended.
template <typename T>
__device__ __forceinline__ uint64_t set_scalar(T v) {
    if constexpr (std::is_same<T, float>::value) return __builtin_bit_cast(uint64_t, static_cast<double>(v));
    else if constexpr (std::is_same<T, double>::value) return __builtin_bit_cast(uint64_t, v);
    else if constexpr (std::is_same<T, int32_t>::value) return static_cast<uint64_t>(static_cast<int64_t>(v));
    else return static_cast<uint64_t>(v);
}

// Addition in T with the rounding the CPU uses (no contraction, wraps for ints).
template <typename T>
__device__ __forceinline__ T t_add(T a, T b) {
    if constexpr (std::is_same<T, double>::value) return __dadd_rn(a, b);
    else if constexpr (std::is_same<T, float>::value) return __fadd_rn(a, b);
    else {
        using U = typename std::make_unsigned<T>::type;
        return static_cast<T>(static_cast<U>(a) + static_cast<U>(b));
    }
}

template <typename T>
__device__ __forceinline__ bool t_isnan(T v) {
    if constexpr (Traits<T>::kFloat) return v != v;
    else return false;
}

// C++ comparison operators on T (op codes EQ NE LT LE GT GE = 0..5).
template <typename T>
__device__ __forceinline__ bool t_cmp(T v, T t, int op) {
    switch (op) {
    case 0: return v == t;
    case 1: return v != t;
    case 2: return v < t;
    case 3: return v <= t;
    case 4: return v > t;
    default: return v >= t;
    }
}

// ---- compensated FP64 accumulation (Neumaier) --------------------------------

struct KSum {
    double s, c;
};

__device__ __forceinline__ void ksum_add(KSum& k, double x) {
    double t = __dadd_rn(k.s, x);
    double e = fabs(k.s) >= fabs(x) ? __dadd_rn(__dsub_rn(k.s, t), x) : __dadd_rn(__dsub_rn(x, t), k.s);
    k.s = t;
    // an infinite (or NaN) running sum has no rounding error to carry: its
    // error term would be inf - inf = NaN and turn an overflowed sum into NaN
    if (isfinite(t)) k.c = __dadd_rn(k.c, e);
}

__device__ __forceinline__ KSum ksum_merge(KSum a, KSum b) {
    KSum r = a;
    ksum_add(r, b.s);
    r.c = __dadd_rn(r.c, b.c);
    return r;
}

__device__ __forceinline__ double ksum_value(KSum k) { return __dadd_rn(k.s, k.c); }

// ---- warp helpers -----------------------------------------------------------

__device__ __forceinline__ uint64_t shfl_down_u64(uint64_t v, int d) {
    return __shfl_down_sync(0xffffffffu, v, d);
}
__device__ __forceinline__ double shfl_down_f64(double v, int d) {
    return __shfl_down_sync(0xffffffffu, v, d);
}

// Bounded wait helper: spin on a predicate with a cycle budget.  Returns false
// when the budget ran out so the caller can flag an error and return.
__device__ __forceinline__ bool budget_left(long long start, long long budget) {
    return (clock64() - start) < budget;
}

// End of the run of keys equal to keys[i] in an ascending array: the first
// index e > i with keys[e] != keys[i], or n.  Galloping (steps 1, 2, 4, ...)
// then bisection, so a run of length L costs O(log L) loads -- one load for
// the common run of one -- rather than a walk of L rows by one thread.
template <typename K>
__device__ __forceinline__ uint64_t sorted_run_end(const K* __restrict__ keys, uint64_t i, uint64_t n) {
    const K k = keys[i];
    uint64_t good = i, bad = n, step = 1;  // keys[good] == k; bad == n or keys[bad] != k
    for (;;) {
        const uint64_t probe = good + step;
        if (probe >= n) break;
        if (keys[probe] != k) {
            bad = probe;
            break;
        }
        good = probe;
        step <<= 1;
    }
    while (bad - good > 1) {
        const uint64_t mid = good + (bad - good) / 2;
        if (keys[mid] == k) good = mid; else bad = mid;
    }
    return bad;
}

}  // namespace vx
