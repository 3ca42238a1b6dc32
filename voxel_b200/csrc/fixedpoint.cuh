// Exact FP64 summation through a 192-bit two's-complement fixed-point
// accumulator (LSB weight 2^-96).
//
// Every finite double with 2^-96 <= |x| < 2^63 converts exactly (smaller
// magnitudes are truncated, an error below 2^-96 each); integer additions are
// associative, so concurrent atomic accumulation gives the exact sum no matter
// the order, and one correctly rounded conversion back to double finishes it.
// Sums are therefore deterministic across runs and grid shapes, and never less
// accurate than the reference's sequential row-order FP64 sum.
#pragma once

#include <stdint.h>

namespace vx {

struct Fix3 {
    uint64_t w0, w1, w2;
};

// x -> 192-bit fixed point.  Sets *bad for NaN / inf / |x| >= 2^63.
__device__ __forceinline__ Fix3 fix_from_double(double x, bool* bad) {
    uint64_t b = static_cast<uint64_t>(__double_as_longlong(x));
    int ex = static_cast<int>((b >> 52) & 0x7FF);
    Fix3 r{0, 0, 0};
    if (ex == 0x7FF) { *bad = true; return r; }
    if (ex == 0) return r;  // zero or subnormal (< 2^-1022): below the window
    uint64_t m = (b & ((1ull << 52) - 1)) | (1ull << 52);
    int s = ex - 1075 + 96;  // |x| * 2^96 = m * 2^s
    if (s >= 107) { *bad = true; return r; }  // |x| >= 2^63
    if (s < 0) {
        if (s > -64) r.w0 = m >> (-s);
    } else if (s < 64) {
        r.w0 = m << s;
        r.w1 = s ? (m >> (64 - s)) : 0;
    } else if (s < 128) {
        int t = s - 64;
        r.w1 = m << t;
        r.w2 = t ? (m >> (64 - t)) : 0;
    } else {
        r.w2 = m << (s - 128);
    }
    if (b >> 63) {  // two's complement negate
        r.w0 = ~r.w0; r.w1 = ~r.w1; r.w2 = ~r.w2;
        r.w0 += 1;
        if (r.w0 == 0) { r.w1 += 1; if (r.w1 == 0) r.w2 += 1; }
    }
    return r;
}

// Atomic 192-bit add into w[0..2] (shared or global memory).  Carries are
// taken from each word's returned old value, so concurrent adds compose.
__device__ __forceinline__ void fix_atomic_add(unsigned long long* w, const Fix3& a) {
    unsigned long long old0 = atomicAdd(&w[0], static_cast<unsigned long long>(a.w0));
    uint64_t c0 = (old0 + a.w0) < old0 ? 1 : 0;
    uint64_t add1 = a.w1 + c0;
    uint64_t c1 = (add1 < a.w1) ? 1 : 0;  // the addend itself wrapped
    if (add1) {
        unsigned long long old1 = atomicAdd(&w[1], static_cast<unsigned long long>(add1));
        c1 += (old1 + add1) < old1 ? 1 : 0;
    }
    uint64_t add2 = a.w2 + c1;
    if (add2) atomicAdd(&w[2], static_cast<unsigned long long>(add2));
}

// Non-atomic 192-bit add.
__device__ __forceinline__ void fix_add(Fix3& acc, const Fix3& a) {
    uint64_t s0 = acc.w0 + a.w0;
    uint64_t c0 = s0 < acc.w0 ? 1 : 0;
    uint64_t s1 = acc.w1 + a.w1;
    uint64_t c1 = s1 < acc.w1 ? 1 : 0;
    uint64_t s1c = s1 + c0;
    c1 += s1c < s1 ? 1 : 0;
    acc.w0 = s0;
    acc.w1 = s1c;
    acc.w2 = acc.w2 + a.w2 + c1;
}

// Correctly rounded conversion of the 192-bit value (LSB 2^-S) to double.
template <int S>
__device__ __forceinline__ double fix_to_double_s(Fix3 v) {
    bool neg = (v.w2 >> 63) != 0;
    if (neg) {
        v.w0 = ~v.w0; v.w1 = ~v.w1; v.w2 = ~v.w2;
        v.w0 += 1;
        if (v.w0 == 0) { v.w1 += 1; if (v.w1 == 0) v.w2 += 1; }
    }
    int top;
    if (v.w2) top = 191 - __clzll(static_cast<long long>(v.w2));
    else if (v.w1) top = 127 - __clzll(static_cast<long long>(v.w1));
    else if (v.w0) top = 63 - __clzll(static_cast<long long>(v.w0));
    else return 0.0;
    // top = sh + 63: shift right by sh (0..128) keeping the top 64 bits;
    // the shifted-out bits only matter as a sticky bit for rounding
    uint64_t chunk, sticky;
    int sh = top > 63 ? top - 63 : 0;
    if (sh == 0) {
        chunk = v.w0;
        sticky = 0;
    } else if (sh < 64) {
        chunk = (v.w0 >> sh) | (v.w1 << (64 - sh));
        sticky = (v.w0 << (64 - sh)) != 0;
    } else if (sh == 64) {
        chunk = v.w1;
        sticky = v.w0 != 0;
    } else if (sh < 128) {
        int t = sh - 64;
        chunk = (v.w1 >> t) | (v.w2 << (64 - t));
        sticky = (v.w0 != 0) || ((v.w1 << (64 - t)) != 0);
    } else {
        chunk = v.w2;
        sticky = (v.w0 | v.w1) != 0;
    }
    double d = __ull2double_rn(chunk | sticky);
    // scale by 2^(sh - S), a normal power of two for every reachable shift
    int e = sh - S;
    double p = __longlong_as_double(static_cast<long long>(static_cast<uint64_t>(e + 1023) << 52));
    d = __dmul_rn(d, p);
    return neg ? -d : d;
}

__device__ __forceinline__ double fix_to_double(Fix3 v) { return fix_to_double_s<96>(v); }

// f64 <-> unsigned key whose integer order is the numeric order (non-NaN).
__device__ __forceinline__ uint64_t f64_order_key(double x) {
    uint64_t b = static_cast<uint64_t>(__double_as_longlong(x));
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double f64_from_order_key(uint64_t k) {
    uint64_t b = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
    return __longlong_as_double(static_cast<long long>(b));
}

}  // namespace vx
