// Device core of the fused filter/compare/aggregate scan, shared by the
// single-program kernel (scan.cu) and the batched persistent executor
// (batch.cu).
//
// A "group" is iteration j of the lowered loop: the kLanes rows
// [off0 + j*kLanes, ...) of each column (VLOAD, include/voxel/exec/engine.hpp:
// 1947-1968, zero-padded past each column's count).  Predicate atoms are
// evaluated per lane; each reduction forms its lane values (F ? A : B) and
// reduces them over the group in T exactly like VSUM / VCOUNT / VRED_MIN /
// VRED_MAX (engine.hpp:2980-3110); the group result (a register image) is
// folded into its accumulator (ADD / SUB / ADDF / MIN / MAX, 1286-1400).
#pragma once

#include "vx_common.cuh"
#include "vx_types.h"

namespace vx {

struct Acc {
    uint64_t u;
    KSum k;
};

struct ScanPartial {
    uint64_t u[kMaxRed];
    double s[kMaxRed];
    double c[kMaxRed];
};

template <typename T>
__device__ __forceinline__ bool acc_is_float(uint8_t op) {
    return op == kAccAddF || (op == kAccTAdd && Traits<T>::kFloat);
}

__device__ __forceinline__ uint64_t acc_identity(uint8_t op) {
    if (op == kAccMin) return 0x7FFFFFFFFFFFFFFFull;
    if (op == kAccMax) return 0x8000000000000000ull;
    return 0;
}

template <typename T>
__device__ __forceinline__ void acc_fold(Acc& a, uint8_t op, uint64_t r) {
    switch (op) {
    case kAccAdd:
    case kAccSub: a.u += r; break;
    case kAccAddF: ksum_add(a.k, __longlong_as_double(static_cast<long long>(r))); break;
    case kAccTAdd:
        if constexpr (Traits<T>::kFloat) ksum_add(a.k, __longlong_as_double(static_cast<long long>(r)));
        else a.u += r;
        break;
    case kAccMin: if (static_cast<int64_t>(r) < static_cast<int64_t>(a.u)) a.u = r; break;
    case kAccMax: if (static_cast<int64_t>(r) > static_cast<int64_t>(a.u)) a.u = r; break;
    default: break;
    }
}

template <typename T>
__device__ __forceinline__ void acc_merge(Acc& a, uint8_t op, const Acc& b) {
    if (acc_is_float<T>(op)) {
        a.k = ksum_merge(a.k, b.k);
    } else if (op == kAccMin) {
        if (static_cast<int64_t>(b.u) < static_cast<int64_t>(a.u)) a.u = b.u;
    } else if (op == kAccMax) {
        if (static_cast<int64_t>(b.u) > static_cast<int64_t>(a.u)) a.u = b.u;
    } else {
        a.u += b.u;
    }
}

template <typename T, int NC>
__device__ __forceinline__ T col_val(const T (&v)[NC][32 / sizeof(T)], int c, int l) {
    T x = v[0][l];
#pragma unroll
    for (int k = 1; k < NC; ++k)
        if (c == k) x = v[k][l];
    return x;
}

template <typename T, int NC>
__device__ __forceinline__ T opnd_val(const Opnd& o, const T (&v)[NC][32 / sizeof(T)], int l) {
    if (o.kind == kOpCol) return col_val<T, NC>(v, o.col, l);
    if (o.kind == kOpConst) return from_bits<T>(o.bits);
    return T(0);
}

// All lanes of an operand (column lane values, a splatted constant, or zero):
// the kind is decided once per group, not per lane.
template <typename T, int NC>
__device__ __forceinline__ void opnd_lanes(const Opnd& o, const T (&v)[NC][32 / sizeof(T)],
                                           T (&out)[32 / sizeof(T)]) {
    constexpr int KL = 32 / sizeof(T);
    if (o.kind == kOpCol) {
#pragma unroll
        for (int l = 0; l < KL; ++l) out[l] = col_val<T, NC>(v, o.col, l);
    } else {
        const T c = o.kind == kOpConst ? from_bits<T>(o.bits) : T(0);
#pragma unroll
        for (int l = 0; l < KL; ++l) out[l] = c;
    }
}

// per-lane bitmask of the atoms that hold (compare op decided once per atom)
template <typename T, int NC>
__device__ __forceinline__ void eval_atoms(const ScanParams& p, const T (&v)[NC][32 / sizeof(T)],
                                           uint32_t (&ab)[32 / sizeof(T)]) {
    constexpr int KL = 32 / sizeof(T);
#pragma unroll
    for (int l = 0; l < KL; ++l) ab[l] = 0;
#pragma unroll
    for (int a = 0; a < kMaxAtoms; ++a) {
        if (a >= p.natoms) break;
        const Atom& at = p.atom[a];
        const T t = from_bits<T>(at.thr);
        const uint32_t bit = 1u << a;
        T x[KL];
#pragma unroll
        for (int l = 0; l < KL; ++l) x[l] = col_val<T, NC>(v, at.col, l);
        switch (at.op) {
        case 0:
#pragma unroll
            for (int l = 0; l < KL; ++l) ab[l] |= x[l] == t ? bit : 0u;
            break;
        case 1:
#pragma unroll
            for (int l = 0; l < KL; ++l) ab[l] |= x[l] != t ? bit : 0u;
            break;
        case 2:
#pragma unroll
            for (int l = 0; l < KL; ++l) ab[l] |= x[l] < t ? bit : 0u;
            break;
        case 3:
#pragma unroll
            for (int l = 0; l < KL; ++l) ab[l] |= x[l] <= t ? bit : 0u;
            break;
        case 4:
#pragma unroll
            for (int l = 0; l < KL; ++l) ab[l] |= x[l] > t ? bit : 0u;
            break;
        default:
#pragma unroll
            for (int l = 0; l < KL; ++l) ab[l] |= x[l] >= t ? bit : 0u;
            break;
        }
    }
}

// One group's lane values reduced like VSUM / VCOUNT / VRED_MIN / VRED_MAX
// (engine.hpp:2980-3110); returns the register image.
template <typename T>
__device__ __forceinline__ uint64_t reduce_group(uint8_t kind, const T (&x)[32 / sizeof(T)]) {
    constexpr int KL = 32 / sizeof(T);
    switch (kind) {
    case kRedSum: {
        T s = T(0);
#pragma unroll
        for (int l = 0; l < KL; ++l) s = t_add<T>(s, x[l]);
        return set_scalar<T>(s);
    }
    case kRedCount: {
        uint64_t c = 0;
#pragma unroll
        for (int l = 0; l < KL; ++l) c += (!t_isnan<T>(x[l]) && x[l] != T(0)) ? 1 : 0;
        return c;
    }
    case kRedMin: {
        T m = x[0];
#pragma unroll
        for (int l = 1; l < KL; ++l)
            if (x[l] < m || t_isnan<T>(x[l])) m = x[l];
        return set_scalar<T>(m);
    }
    default: {
        T m = x[0];
#pragma unroll
        for (int l = 1; l < KL; ++l)
            if (x[l] > m || t_isnan<T>(m)) m = x[l];
        return set_scalar<T>(m);
    }
    }
}

// Evaluate every reduction of one group; res[r] is the register image.
template <typename T, int NC, int NR>
__device__ __forceinline__ void eval_reds(const ScanParams& p, const T (&v)[NC][32 / sizeof(T)],
                                          const uint32_t (&ab)[32 / sizeof(T)], uint64_t (&res)[NR]) {
    constexpr int KL = 32 / sizeof(T);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        if (r >= p.nred) break;
        const Red& rd = p.red[r];
        T A[KL], B[KL], x[KL];
        opnd_lanes<T, NC>(rd.a, v, A);
        opnd_lanes<T, NC>(rd.b, v, B);
        const uint32_t pm = rd.pmask;
        const bool never = (pm & kMaskFalse) != 0;
#pragma unroll
        for (int l = 0; l < KL; ++l) x[l] = (!never && (ab[l] & pm) == pm) ? A[l] : B[l];
        res[r] = reduce_group<T>(rd.kind, x);
    }
}

template <typename T, int NC, int NR>
__device__ __forceinline__ void eval_group(const ScanParams& p, const T (&v)[NC][32 / sizeof(T)],
                                           uint64_t (&res)[NR]) {
    uint32_t ab[32 / sizeof(T)];
    eval_atoms<T, NC>(p, v, ab);
    eval_reds<T, NC, NR>(p, v, ab, res);
}

template <typename T, int NC>
__device__ __forceinline__ void load_group(const ScanParams& p, uint64_t j, bool vec,
                                           T (&v)[NC][32 / sizeof(T)]) {
    constexpr int KL = 32 / sizeof(T);
    uint64_t r0 = p.off0 + j * KL;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        if (c >= p.ncols) {
#pragma unroll
            for (int l = 0; l < KL; ++l) v[c][l] = T(0);
            continue;
        }
        const T* base = static_cast<const T*>(p.col[c]);
        if (vec && r0 + KL <= p.count[c]) {
            const uint4* q = reinterpret_cast<const uint4*>(base + r0);
            uint4 a = __ldcs(q);
            uint4 b = __ldcs(q + 1);
            T tmp[KL];
            *reinterpret_cast<uint4*>(&tmp[0]) = a;
            *reinterpret_cast<uint4*>(&tmp[KL / 2]) = b;
#pragma unroll
            for (int l = 0; l < KL; ++l) v[c][l] = tmp[l];
        } else {
#pragma unroll
            for (int l = 0; l < KL; ++l) {
                uint64_t idx = r0 + l;
                v[c][l] = (idx >= r0 && idx < p.count[c]) ? base[idx] : T(0);
            }
        }
    }
}

// warp + block reduction of per-thread accumulators into out[r] (all threads call)
template <typename T, int NR, int THREADS>
__device__ void block_reduce(const ScanParams& p, Acc (&acc)[NR], Acc* out) {
    __shared__ Acc sh[THREADS / 32][NR];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        if (r >= p.nred) break;
        uint8_t op = p.red[r].acc;
        for (int d = 16; d > 0; d >>= 1) {
            Acc o;
            o.u = shfl_down_u64(acc[r].u, d);
            o.k.s = shfl_down_f64(acc[r].k.s, d);
            o.k.c = shfl_down_f64(acc[r].k.c, d);
            acc_merge<T>(acc[r], op, o);
        }
        if (lane == 0) sh[warp][r] = acc[r];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            if (r >= p.nred) break;
            uint8_t op = p.red[r].acc;
            Acc a;
            a.u = acc_identity(op);
            a.k = {0.0, 0.0};
            if (lane < THREADS / 32) a = sh[lane][r];
            for (int d = 16; d > 0; d >>= 1) {
                Acc o;
                o.u = shfl_down_u64(a.u, d);
                o.k.s = shfl_down_f64(a.k.s, d);
                o.k.c = shfl_down_f64(a.k.c, d);
                acc_merge<T>(a, op, o);
            }
            if (lane == 0) out[r] = a;
        }
    }
    __syncthreads();
}

// Final register values from the merged accumulators: adds the all-zero
// padding groups [ndata, ngroups) and combines with the registers' values
// before the loop.  Run by one thread.
template <typename T, int NC, int NR>
__device__ void finalize_scan(const ScanParams& p, const Acc (&blk)[NR], ScanResult* out) {
    constexpr int KL = 32 / sizeof(T);
    uint64_t npad = p.ngroups - p.ndata;
    uint64_t res0[NR];
    if (npad) {
        T z[NC][KL];
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int l = 0; l < KL; ++l) z[c][l] = T(0);
        eval_group<T, NC, NR>(p, z, res0);
    }
    for (int r = 0; r < p.nred && r < NR; ++r) {
        uint8_t op = p.red[r].acc;
        Acc a = blk[r];
        if (npad) {
            out->last[r] = res0[r];
            if (acc_is_float<T>(op)) {
                double g = __longlong_as_double(static_cast<long long>(res0[r]));
                double hi = __dmul_rn(static_cast<double>(npad), g);
                double lo = fma(static_cast<double>(npad), g, -hi);
                ksum_add(a.k, hi);
                a.k.c = __dadd_rn(a.k.c, lo);
            } else if (op == kAccMin || op == kAccMax) {
                Acc o;
                o.u = res0[r];
                acc_merge<T>(a, op, o);
            } else {
                a.u += npad * res0[r];
            }
        }
        uint64_t a0 = p.acc0[r];
        uint64_t fin = a0;
        switch (op) {
        case kAccAdd: fin = a0 + a.u; break;
        case kAccSub: fin = a0 - a.u; break;
        case kAccAddF: {
            KSum k{__longlong_as_double(static_cast<long long>(a0)), 0.0};
            k = ksum_merge(k, a.k);
            fin = static_cast<uint64_t>(__double_as_longlong(ksum_value(k)));
            break;
        }
        case kAccTAdd:
            if constexpr (Traits<T>::kFloat) {
                KSum k{__longlong_as_double(static_cast<long long>(a0)), 0.0};
                k = ksum_merge(k, a.k);
                fin = static_cast<uint64_t>(__double_as_longlong(ksum_value(k)));
            } else {
                fin = set_scalar<T>(static_cast<T>(a0 + a.u));
            }
            break;
        case kAccMin: fin = static_cast<int64_t>(a.u) < static_cast<int64_t>(a0) ? a.u : a0; break;
        case kAccMax: fin = static_cast<int64_t>(a.u) > static_cast<int64_t>(a0) ? a.u : a0; break;
        default: break;
        }
        out->acc[r] = fin;
    }
    out->status = kOk;
}

}  // namespace vx
