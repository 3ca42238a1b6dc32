// Fused filter/compare/aggregate scan kernel (one lowered bytecode loop).
//
// One launch runs every iteration of a lowered loop (see scan_core.cuh for the
// per-group semantics).  Groups are independent, so threads take them
// grid-stride with 128-bit loads; integer / min / max folds are exact in any
// order, f64 folds use Neumaier compensation, and blocks combine in a fixed
// order in the last block to finish, so results are deterministic for a given
// grid.
#include <cstdio>

#include "rangeform.h"
#include "scan.h"
#include "scan_core.cuh"
#include "vx_runtime.h"

namespace vx {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 148 * 8;

template <typename T, int NC, int NR, int UNROLL>
__global__ void __launch_bounds__(kThreads) scan_kernel(const __grid_constant__ ScanParams p, int vec,
                                                        ScanPartial* part, unsigned int* done,
                                                        ScanResult* out) {
    constexpr int KL = 32 / sizeof(T);
    Acc acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        acc[r].u = r < p.nred ? acc_identity(p.red[r].acc) : 0;
        acc[r].k = {0.0, 0.0};
    }
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t lastj = p.ngroups - 1;
    for (uint64_t j0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j0 < p.ndata;
         j0 += stride * UNROLL) {
        T v[UNROLL][NC][KL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            uint64_t j = j0 + u * stride;
            if (j < p.ndata) load_group<T, NC>(p, j, vec != 0, v[u]);
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            uint64_t j = j0 + u * stride;
            if (j < p.ndata) {
                uint64_t res[NR];
                eval_group<T, NC, NR>(p, v[u], res);
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    if (r >= p.nred) break;
                    acc_fold<T>(acc[r], p.red[r].acc, res[r]);
                    if (j == lastj) out->last[r] = res[r];
                }
            }
        }
    }

    __shared__ Acc blk[NR];
    block_reduce<T, NR, kThreads>(p, acc, blk);
    if (threadIdx.x < NR && threadIdx.x < p.nred) {
        int r = threadIdx.x;
        part[blockIdx.x].u[r] = blk[r].u;
        part[blockIdx.x].s[r] = blk[r].k.s;
        part[blockIdx.x].c[r] = blk[r].k.c;
    }
    __threadfence();
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();

    // last block: fold the per-block partials in block order
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        acc[r].u = r < p.nred ? acc_identity(p.red[r].acc) : 0;
        acc[r].k = {0.0, 0.0};
    }
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            if (r >= p.nred) break;
            Acc o;
            o.u = __ldcg(&part[b].u[r]);
            o.k.s = __ldcg(&part[b].s[r]);
            o.k.c = __ldcg(&part[b].c[r]);
            acc_merge<T>(acc[r], p.red[r].acc, o);
        }
    }
    block_reduce<T, NR, kThreads>(p, acc, blk);
    if (threadIdx.x == 0) {
        *done = 0;
        finalize_scan<T, NC, NR>(p, blk, out);
    }
}

// Specialised kernel for the dominant shape, the reference's fast path and the
// Tier-0 loops of the same form: one column, one comparison atom, SUM of the
// lanes that pass (failing lanes are zero, as VFILTER writes them), folded into
// one accumulator.  The compare is a template parameter, so a group costs a
// few instructions instead of the generic per-lane interpretation; the fold,
// block partials and finalisation are the generic ones, so results are the
// same bits.
template <int OP, typename T>
__device__ __forceinline__ bool cmp_op(T v, T t) {
    if constexpr (OP == 6) return true;  // no predicate: every lane keeps its value
    else if constexpr (OP == 0) return v == t;
    else if constexpr (OP == 1) return v != t;
    else if constexpr (OP == 2) return v < t;
    else if constexpr (OP == 3) return v <= t;
    else if constexpr (OP == 4) return v > t;
    else return v >= t;
}

constexpr int kFsUnroll = 2;  // 2 groups in flight per thread, 6 blocks per SM (measured best)

// CNT = 1: a second reduction counts the same mask's passing lanes (VCOUNT of
// the VFILTER output: a passing lane counts when its value is nonzero and not
// NaN) into its own accumulator, as the config-1 program `filter x > t;
// SUM(x); COUNT` does.  cnt_all: the host proved that every passing value is
// nonzero and not NaN (x > t with t >= 0, and so on), so the count is the
// popcount of the mask.
template <typename T, int OP, int CNT>
__global__ void __launch_bounds__(kThreads, 6) fsum_kernel(const __grid_constant__ ScanParams p, int vec,
                                                          int cnt_all, ScanPartial* part, unsigned int* done,
                                                          ScanResult* out) {
    constexpr int KL = 32 / sizeof(T);
    constexpr int NR = 1 + CNT;
    const T thr = from_bits<T>(p.atom[0].thr);
    const uint8_t op = p.red[0].acc;
    Acc acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        acc[r].u = 0;
        acc[r].k = {0.0, 0.0};
    }
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t lastj = p.ngroups - 1;
    for (uint64_t j0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j0 < p.ndata;
         j0 += stride * kFsUnroll) {
        T v[kFsUnroll][1][KL];
#pragma unroll
        for (int u = 0; u < kFsUnroll; ++u) {
            uint64_t j = j0 + u * stride;
            if (j < p.ndata) load_group<T, 1>(p, j, vec != 0, v[u]);
        }
#pragma unroll
        for (int u = 0; u < kFsUnroll; ++u) {
            uint64_t j = j0 + u * stride;
            if (j < p.ndata) {
                T sum = T(0);  // left to right in T, like VSUM
                uint32_t c = 0;
#pragma unroll
                for (int l = 0; l < KL; ++l) {
                    const T y = v[u][0][l];
                    const bool pass = cmp_op<OP>(y, thr);
                    sum = t_add<T>(sum, pass ? y : T(0));
                    if constexpr (CNT) c += (pass && (cnt_all || (y != T(0) && !t_isnan<T>(y)))) ? 1u : 0u;
                }
                const uint64_t r = set_scalar<T>(sum);
                acc_fold<T>(acc[0], op, r);
                if constexpr (CNT) acc[NR - 1].u += c;
                if (j == lastj) {
                    out->last[0] = r;
                    if constexpr (CNT) out->last[NR - 1] = c;
                }
            }
        }
    }
    __shared__ Acc blk[NR];
    block_reduce<T, NR, kThreads>(p, acc, blk);
    if (threadIdx.x < NR) {
        const int r = threadIdx.x;
        part[blockIdx.x].u[r] = blk[r].u;
        part[blockIdx.x].s[r] = blk[r].k.s;
        part[blockIdx.x].c[r] = blk[r].k.c;
    }
    __threadfence();
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        acc[r].u = 0;
        acc[r].k = {0.0, 0.0};
    }
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            Acc o;
            o.u = __ldcg(&part[b].u[r]);
            o.k.s = __ldcg(&part[b].s[r]);
            o.k.c = __ldcg(&part[b].c[r]);
            acc_merge<T>(acc[r], p.red[r].acc, o);
        }
    }
    block_reduce<T, NR, kThreads>(p, acc, blk);
    if (threadIdx.x == 0) {
        *done = 0;
        finalize_scan<T, 1, NR>(p, blk, out);
    }
}

bool fsum_sum_red(const Red& r, uint32_t pmask) {
    if (r.kind != kRedSum || r.pmask != pmask || r.a.kind != kOpCol || r.a.col != 0) return false;
    if (!(r.b.kind == kOpZero || (r.b.kind == kOpConst && r.b.bits == 0))) return false;
    return r.acc == kAccAdd || r.acc == kAccSub || r.acc == kAccAddF || r.acc == kAccTAdd;
}

// one column, one compare atom, a masked SUM of the column (failing lanes are
// zero), and optionally the COUNT of the same VFILTER output
bool fsum_shape(const ScanParams& p) {
    // one compare atom, or none (every lane kept: SUM / COUNT of the column)
    if (p.ncols != 1 || p.natoms > 1 || p.nred < 1 || p.nred > 2) return false;
    if (p.natoms == 1 && (p.atom[0].col != 0 || p.atom[0].op > 5)) return false;
    const uint32_t pm = p.natoms ? 1u : 0u;
    if (!fsum_sum_red(p.red[0], pm)) return false;
    if (p.nred == 1) return true;
    const Red& c = p.red[1];
    if (c.kind != kRedCount || c.pmask != pm || c.acc != kAccAdd || c.a.kind != kOpCol || c.a.col != 0) return false;
    return c.b.kind == kOpZero || (c.b.kind == kOpConst && c.b.bits == 0);
}

// every value that passes `x OP thr` is nonzero and not NaN
template <typename T>
bool pass_implies_nonzero(int op, uint64_t thr_bits) {
    const T t = host_from_bits<T>(thr_bits);
    if (t != t) return false;  // NaN threshold: NE passes NaN
    switch (op) {
    case 0: return t != T(0);   // EQ
    case 2: return t <= T(0);   // LT
    case 3: return t < T(0);    // LE
    case 4: return t >= T(0);   // GT
    case 5: return t > T(0);    // GE
    default: return false;      // NE
    }
}

bool pass_implies_nonzero_of(const ScanParams& p) {
    if (p.natoms == 0) return false;
    switch (p.dtype) {
    case F64: return pass_implies_nonzero<double>(p.atom[0].op, p.atom[0].thr);
    case F32: return pass_implies_nonzero<float>(p.atom[0].op, p.atom[0].thr);
    case I64: return pass_implies_nonzero<int64_t>(p.atom[0].op, p.atom[0].thr);
    case I32: return pass_implies_nonzero<int32_t>(p.atom[0].op, p.atom[0].thr);
    case U64: return pass_implies_nonzero<uint64_t>(p.atom[0].op, p.atom[0].thr);
    default: return pass_implies_nonzero<uint32_t>(p.atom[0].op, p.atom[0].thr);
    }
}

int fsum_grid(uint64_t ndata) {
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t need = (ndata + static_cast<uint64_t>(kThreads) * kFsUnroll - 1) / (static_cast<uint64_t>(kThreads) * kFsUnroll);
    uint64_t cap = static_cast<uint64_t>(sms) * 6;  // one wave of resident blocks
    uint64_t g = need < cap ? need : cap;
    return g < 1 ? 1 : static_cast<int>(g);
}

// Range form (rangeform.h) of a one-column, one-reduction program: the atoms'
// conjunction as lo <= x <= hi (and x != ne[0], x != ne[1] when NE) with the
// reduction kind RK and its canonical fold fixed per instance.  Per group the
// lane values, the group result, the fold, the block partials and the
// finalisation are the generic kernel's, so results are the same bits.
template <typename T, int RK, bool NE>
__global__ void __launch_bounds__(kThreads, 6) range_scan_kernel(const __grid_constant__ ScanParams p,
                                                                const RangeForm rf, int vec, ScanPartial* part,
                                                                unsigned int* done, ScanResult* out) {
    constexpr int KL = 32 / sizeof(T);
    constexpr uint8_t accop = range_acc(RK, Traits<T>::kFloat);
    const T lo = from_bits<T>(rf.lo), hi = from_bits<T>(rf.hi);
    const T n0 = from_bits<T>(rf.ne[0]), n1 = from_bits<T>(rf.ne[1]);
    const T ac = p.red[0].a.kind == kOpConst ? from_bits<T>(p.red[0].a.bits) : T(0);
    const T bc = p.red[0].b.kind == kOpConst ? from_bits<T>(p.red[0].b.bits) : T(0);
    // COUNT of the constants: passing lanes count when ac is nonzero (and not
    // NaN), the others when bc is
    const uint32_t cnt_pass = (!t_isnan<T>(ac) && ac != T(0)) ? 1u : 0u;
    const uint32_t cnt_fail = (!t_isnan<T>(bc) && bc != T(0)) ? 1u : 0u;
    const bool cnt_col = RK == kRedCount && p.red[0].a.kind == kOpCol;  // VCOUNT of the column's passing lanes
    Acc acc[1];
    acc[0].u = acc_identity(accop);
    acc[0].k = {0.0, 0.0};
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t lastj = p.ngroups - 1;
    for (uint64_t j0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j0 < p.ndata;
         j0 += stride * kFsUnroll) {
        T v[kFsUnroll][1][KL];
#pragma unroll
        for (int u = 0; u < kFsUnroll; ++u) {
            const uint64_t j = j0 + u * stride;
            if (j < p.ndata) load_group<T, 1>(p, j, vec != 0, v[u]);
        }
#pragma unroll
        for (int u = 0; u < kFsUnroll; ++u) {
            const uint64_t j = j0 + u * stride;
            if (j >= p.ndata) continue;
            uint32_t pm = 0, nz = 0;
            T x[KL];
#pragma unroll
            for (int l = 0; l < KL; ++l) {
                const T y = v[u][0][l];
                bool pass = y >= lo && y <= hi;
                if constexpr (NE) pass = pass && y != n0 && y != n1;
                pm |= pass ? 1u << l : 0u;
                if constexpr (RK == kRedCount) nz |= (pass && y != T(0)) ? 1u << l : 0u;  // NaN never passes
                if constexpr (RK != kRedCount) x[l] = pass ? y : bc;
            }
            uint64_t r;
            if constexpr (RK == kRedCount) {
                const uint32_t np = __popc(pm);
                r = (cnt_col ? __popc(nz) : cnt_pass * np) + cnt_fail * (KL - np);
            } else {
                r = reduce_group<T>(RK, x);
            }
            acc_fold<T>(acc[0], accop, r);
            if (j == lastj) out->last[0] = r;
        }
    }
    __shared__ Acc blk[1];
    block_reduce<T, 1, kThreads>(p, acc, blk);
    if (threadIdx.x == 0) {
        part[blockIdx.x].u[0] = blk[0].u;
        part[blockIdx.x].s[0] = blk[0].k.s;
        part[blockIdx.x].c[0] = blk[0].k.c;
    }
    __threadfence();
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    acc[0].u = acc_identity(accop);
    acc[0].k = {0.0, 0.0};
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        Acc o;
        o.u = __ldcg(&part[b].u[0]);
        o.k.s = __ldcg(&part[b].s[0]);
        o.k.c = __ldcg(&part[b].c[0]);
        acc_merge<T>(acc[0], accop, o);
    }
    block_reduce<T, 1, kThreads>(p, acc, blk);
    if (threadIdx.x == 0) {
        *done = 0;
        finalize_scan<T, 1, 1>(p, blk, out);
    }
}

// Reduction codes of a multi-reduction range form: the kind, plus 4 for a
// COUNT of the column's lanes (VCOUNT of a VFILTER output) rather than of a
// constant.  A signature packs one code per reduction, 4 bits each, reduction
// 0 lowest; kSigRuntime reads the kinds from the parameters instead.
constexpr uint32_t kCodeCountCol = 4;
constexpr uint32_t kSigRuntime = 0xFFFFFFFFu;

__host__ __device__ constexpr uint32_t range_code(uint8_t kind, bool acol) {
    return kind == kRedCount && acol ? (kRedCount | kCodeCountCol) : kind;
}

// One reduction of a multi-reduction range form over a group whose passing
// lanes are the bits of pm: lane value = pass ? (column | constant a) : b,
// reduced like VSUM / VCOUNT / VRED_MIN / VRED_MAX.  CODE is the reduction's
// code, or kSigRuntime to read it from rd (warp-uniform branches).
template <typename T, uint32_t CODE>
__device__ __forceinline__ uint64_t range_group(const Red& rd, const T (&y)[32 / sizeof(T)], uint32_t pm) {
    constexpr int KL = 32 / sizeof(T);
    const T bc = rd.b.kind == kOpConst ? from_bits<T>(rd.b.bits) : T(0);
    const bool acol = CODE == kSigRuntime ? rd.a.kind == kOpCol
                                          : (CODE & 3u) != kRedCount || (CODE & kCodeCountCol) != 0;
    const uint8_t kind = CODE == kSigRuntime ? rd.kind : static_cast<uint8_t>(CODE & 3u);
    if (CODE != kSigRuntime && kind == kRedCount) {
        // passing lanes count when their value is nonzero (and not NaN: a NaN
        // never passes an interval); failing lanes when b is
        const bool bcnt = !t_isnan<T>(bc) && bc != T(0);
        uint32_t nz = pm;
        if (acol) {
            nz = 0;
#pragma unroll
            for (int l = 0; l < KL; ++l) nz |= ((pm >> l) & 1u) && y[l] != T(0) ? 1u << l : 0u;
        } else {
            const T ac = rd.a.kind == kOpConst ? from_bits<T>(rd.a.bits) : T(0);
            if (t_isnan<T>(ac) || ac == T(0)) nz = 0;
        }
        const uint32_t np = __popc(pm);
        return static_cast<uint64_t>(__popc(nz)) + (bcnt ? static_cast<uint64_t>(KL - np) : 0ull);
    }
    T x[KL];
    if (acol) {
#pragma unroll
        for (int l = 0; l < KL; ++l) x[l] = (pm >> l) & 1u ? y[l] : bc;
    } else {
        const T ac = rd.a.kind == kOpConst ? from_bits<T>(rd.a.bits) : T(0);
#pragma unroll
        for (int l = 0; l < KL; ++l) x[l] = (pm >> l) & 1u ? ac : bc;
    }
    return reduce_group<T>(kind, x);
}

template <uint32_t SIG, int R>
__host__ __device__ constexpr uint32_t sig_code() {
    return SIG == kSigRuntime ? kSigRuntime : (SIG >> (4 * R)) & 0xFu;
}

template <typename T, uint32_t SIG, int R, int NR>
__device__ __forceinline__ void fold_reds(const ScanParams& p, Acc (&acc)[NR], const T (&y)[32 / sizeof(T)],
                                          uint32_t pm, bool last, ScanResult* out) {
    if constexpr (R < NR) {
        const uint64_t res = range_group<T, sig_code<SIG, R>()>(p.red[R], y, pm);
        acc_fold<T>(acc[R], p.red[R].acc, res);
        if (last) out->last[R] = res;
        fold_reds<T, SIG, R + 1, NR>(p, acc, y, pm, last, out);
    }
}

constexpr int kMrUnroll = 2;  // 2 groups in flight per thread, 5 blocks per SM (4 unrolled groups at 3 blocks measured slower)

// Multi-reduction range form (rangeform.h): NR reductions of one column that
// share one predicate, e.g. `filter x > t; SUM(x); COUNT`.  The interval test
// runs once per lane; each reduction then forms and reduces its lane values
// and folds them with its canonical accumulator.  Group results, folds, block
// partials and the finalisation are the generic kernel's, so results are the
// same bits.  SIG fixes the reduction codes of the common shapes at compile
// time (kSigRuntime: any shape).
template <typename T, int NR, bool NE, uint32_t SIG>
__global__ void __launch_bounds__(kThreads, NR <= 2 ? 5 : 4) mrange_scan_kernel(
    const __grid_constant__ ScanParams p, const RangeForm rf, int vec, ScanPartial* part, unsigned int* done,
    ScanResult* out) {
    constexpr int KL = 32 / sizeof(T);
    const T lo = from_bits<T>(rf.lo), hi = from_bits<T>(rf.hi);
    const T n0 = from_bits<T>(rf.ne[0]), n1 = from_bits<T>(rf.ne[1]);
    Acc acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        acc[r].u = acc_identity(p.red[r].acc);
        acc[r].k = {0.0, 0.0};
    }
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t lastj = p.ngroups - 1;
    for (uint64_t j0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j0 < p.ndata;
         j0 += stride * kMrUnroll) {
        T v[kMrUnroll][1][KL];
#pragma unroll
        for (int u = 0; u < kMrUnroll; ++u) {
            const uint64_t j = j0 + u * stride;
            if (j < p.ndata) load_group<T, 1>(p, j, vec != 0, v[u]);
        }
#pragma unroll
        for (int u = 0; u < kMrUnroll; ++u) {
            const uint64_t j = j0 + u * stride;
            if (j >= p.ndata) continue;
            uint32_t pm = 0;
#pragma unroll
            for (int l = 0; l < KL; ++l) {
                const T y = v[u][0][l];
                bool pass = y >= lo && y <= hi;
                if constexpr (NE) pass = pass && y != n0 && y != n1;
                pm |= pass ? 1u << l : 0u;
            }
            fold_reds<T, SIG, 0, NR>(p, acc, v[u][0], pm, j == lastj, out);
        }
    }
    __shared__ Acc blk[NR];
    block_reduce<T, NR, kThreads>(p, acc, blk);
    if (threadIdx.x < NR) {
        const int r = threadIdx.x;
        part[blockIdx.x].u[r] = blk[r].u;
        part[blockIdx.x].s[r] = blk[r].k.s;
        part[blockIdx.x].c[r] = blk[r].k.c;
    }
    __threadfence();
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        acc[r].u = acc_identity(p.red[r].acc);
        acc[r].k = {0.0, 0.0};
    }
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            Acc o;
            o.u = __ldcg(&part[b].u[r]);
            o.k.s = __ldcg(&part[b].s[r]);
            o.k.c = __ldcg(&part[b].c[r]);
            acc_merge<T>(acc[r], p.red[r].acc, o);
        }
    }
    block_reduce<T, NR, kThreads>(p, acc, blk);
    if (threadIdx.x == 0) {
        *done = 0;
        finalize_scan<T, 1, NR>(p, blk, out);
    }
}

int mrange_grid(uint64_t ndata, int nred) {
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t need = (ndata + static_cast<uint64_t>(kThreads) * kMrUnroll - 1) / (static_cast<uint64_t>(kThreads) * kMrUnroll);
    uint64_t cap = static_cast<uint64_t>(sms) * (nred <= 2 ? 5 : 4);  // one wave of resident blocks
    uint64_t g = need < cap ? need : cap;
    return g < 1 ? 1 : static_cast<int>(g);
}

// the signature of p's reductions (4 bits each, reduction 0 lowest)
uint32_t range_signature(const ScanParams& p) {
    uint32_t sig = 0;
    for (int r = 0; r < p.nred; ++r)
        sig |= range_code(p.red[r].kind, p.red[r].a.kind == kOpCol) << (4 * r);
    return sig;
}

// compile-time signatures: SUM + COUNT of the filtered column (the config-1
// program), SUM + COUNT of a constant, and those with MIN and MAX after them
constexpr uint32_t kSigSumCountCol = kRedSum | ((kRedCount | kCodeCountCol) << 4);
constexpr uint32_t kSigSumCount = kRedSum | (kRedCount << 4);
constexpr uint32_t kSigSumCountMinMax = kSigSumCount | (kRedMin << 8) | (kRedMax << 12);
constexpr uint32_t kSigSumCountColMinMax = kSigSumCountCol | (kRedMin << 8) | (kRedMax << 12);

template <typename T>
int launch_mrange(const ScanParams& p, const RangeForm& rf, ScanResult* d_out, void* scratch, cudaStream_t s) {
    ScanPartial* part = static_cast<ScanPartial*>(scratch);
    unsigned int* done = reinterpret_cast<unsigned int*>(static_cast<char*>(scratch) + kMaxBlocks * sizeof(ScanPartial));
    const int vec = (reinterpret_cast<uintptr_t>(p.col[0]) + p.off0 * sizeof(T)) % 16 == 0 ? 1 : 0;
    const int grid = mrange_grid(p.ndata, p.nred);
    const bool ne = rf.fast == 2;
    const uint32_t sig = range_signature(p);
#define VX_MRS(NR, SIG)                                                                                        \
    (ne ? mrange_scan_kernel<T, NR, true, SIG><<<grid, kThreads, 0, s>>>(p, rf, vec, part, done, d_out)       \
        : mrange_scan_kernel<T, NR, false, SIG><<<grid, kThreads, 0, s>>>(p, rf, vec, part, done, d_out))
    if (p.nred == 2 && sig == kSigSumCountCol) VX_MRS(2, kSigSumCountCol);
    else if (p.nred == 2 && sig == kSigSumCount) VX_MRS(2, kSigSumCount);
    else if (p.nred == 4 && sig == kSigSumCountMinMax) VX_MRS(4, kSigSumCountMinMax);
    else if (p.nred == 4 && sig == kSigSumCountColMinMax) VX_MRS(4, kSigSumCountColMinMax);
    else if (p.nred == 2) VX_MRS(2, kSigRuntime);
    else if (p.nred == 3) VX_MRS(3, kSigRuntime);
    else VX_MRS(4, kSigRuntime);
#undef VX_MRS
    VX_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int launch_range(const ScanParams& p, const RangeForm& rf, ScanResult* d_out, void* scratch, cudaStream_t s) {
    ScanPartial* part = static_cast<ScanPartial*>(scratch);
    unsigned int* done = reinterpret_cast<unsigned int*>(static_cast<char*>(scratch) + kMaxBlocks * sizeof(ScanPartial));
    const int vec = (reinterpret_cast<uintptr_t>(p.col[0]) + p.off0 * sizeof(T)) % 16 == 0 ? 1 : 0;
    const int grid = fsum_grid(p.ndata);
#define VX_RS(RK, NE) range_scan_kernel<T, RK, NE><<<grid, kThreads, 0, s>>>(p, rf, vec, part, done, d_out)
    switch (rf.fast) {
    case 1: VX_RS(kRedSum, false); break;
    case 2: VX_RS(kRedSum, true); break;
    case 3: VX_RS(kRedCount, false); break;
    case 4: VX_RS(kRedCount, true); break;
    case 5: VX_RS(kRedMin, false); break;
    case 6: VX_RS(kRedMin, true); break;
    case 7: VX_RS(kRedMax, false); break;
    default: VX_RS(kRedMax, true); break;
    }
#undef VX_RS
    VX_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int launch_fsum(const ScanParams& p, ScanResult* d_out, void* scratch, cudaStream_t s) {
    ScanPartial* part = static_cast<ScanPartial*>(scratch);
    unsigned int* done = reinterpret_cast<unsigned int*>(static_cast<char*>(scratch) + kMaxBlocks * sizeof(ScanPartial));
    const int vec = (reinterpret_cast<uintptr_t>(p.col[0]) + p.off0 * sizeof(T)) % 16 == 0 ? 1 : 0;
    const int grid = fsum_grid(p.ndata);
    const int cnt_all = p.nred == 2 && pass_implies_nonzero_of(p) ? 1 : 0;
#define VX_FS(OP)                                                                                        \
    (p.nred == 2 ? fsum_kernel<T, OP, 1><<<grid, kThreads, 0, s>>>(p, vec, cnt_all, part, done, d_out)  \
                 : fsum_kernel<T, OP, 0><<<grid, kThreads, 0, s>>>(p, vec, cnt_all, part, done, d_out))
    switch (p.natoms ? p.atom[0].op : 6) {
    case 0: VX_FS(0); break;
    case 1: VX_FS(1); break;
    case 2: VX_FS(2); break;
    case 3: VX_FS(3); break;
    case 4: VX_FS(4); break;
    case 5: VX_FS(5); break;
    default: VX_FS(6); break;
    }
#undef VX_FS
    VX_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T, int NC, int NR, int UNROLL>
int launch_t(const ScanParams& p, int grid, ScanResult* d_out, void* scratch, cudaStream_t s) {
    ScanPartial* part = static_cast<ScanPartial*>(scratch);
    unsigned int* done = reinterpret_cast<unsigned int*>(static_cast<char*>(scratch) + kMaxBlocks * sizeof(ScanPartial));
    bool vec = true;
    for (int c = 0; c < p.ncols; ++c) {
        uintptr_t a = reinterpret_cast<uintptr_t>(p.col[c]) + p.off0 * sizeof(T);
        if (a % 16) vec = false;
    }
    scan_kernel<T, NC, NR, UNROLL><<<grid, kThreads, 0, s>>>(p, vec ? 1 : 0, part, done, d_out);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int dispatch(const ScanParams& p, int grid, ScanResult* d_out, void* scratch, cudaStream_t s) {
    if (fsum_shape(p)) return launch_fsum<T>(p, d_out, scratch, s);
    RangeForm rf;
    if (range_form_of(p, &rf, true)) return launch_range<T>(p, rf, d_out, scratch, s);
    if (multi_range_form_of(p, &rf)) return launch_mrange<T>(p, rf, d_out, scratch, s);
    if (p.ncols <= 1 && p.nred <= 2) return launch_t<T, 1, 2, 4>(p, grid, d_out, scratch, s);
    if (p.ncols <= 1) return launch_t<T, 1, kMaxRed, 2>(p, grid, d_out, scratch, s);
    return launch_t<T, kMaxCols, kMaxRed, 1>(p, grid, d_out, scratch, s);
}

// ---- segment aggregates (AGG_* opcodes) -------------------------------------

template <typename T>
__global__ void __launch_bounds__(kThreads) seg_agg_kernel(const T* col, uint64_t begin, uint64_t end,
                                                          int kind, uint64_t init_bits, ScanPartial* part,
                                                          unsigned int* done, uint64_t* out3) {
    // kind 0: count nonzero; 1: sum (ints widened to i64, floats in f64);
    // 3: min, 4: max, folded with < and > from the slot's current value, as
    // HandleAggregate does (NaN never replaces the running value).
    uint64_t cnt = 0, isum = 0;
    KSum k{0.0, 0.0};
    T m = from_bits<T>(init_bits);
    for (uint64_t i = begin + static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < end;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        T x = col[i];
        if (kind == 0) cnt += (x != T(0)) ? 1 : 0;
        else if (kind == 1) {
            if constexpr (Traits<T>::kFloat) ksum_add(k, static_cast<double>(x));
            else isum += static_cast<uint64_t>(static_cast<int64_t>(x));
        } else if (kind == 3) {
            if (x < m) m = x;
        } else {
            if (x > m) m = x;
        }
    }
    __shared__ uint64_t su[kThreads];
    __shared__ double ss[kThreads], sc[kThreads];
    __shared__ T sm[kThreads];
    int t = threadIdx.x;
    su[t] = kind == 0 ? cnt : isum;
    ss[t] = k.s;
    sc[t] = k.c;
    sm[t] = m;
    __syncthreads();
    for (int d = kThreads / 2; d > 0; d >>= 1) {
        if (t < d) {
            su[t] += su[t + d];
            KSum a{ss[t], sc[t]}, b{ss[t + d], sc[t + d]};
            a = ksum_merge(a, b);
            ss[t] = a.s;
            sc[t] = a.c;
            if (kind == 3 ? (sm[t + d] < sm[t]) : (sm[t + d] > sm[t])) sm[t] = sm[t + d];
        }
        __syncthreads();
    }
    if (t == 0) {
        part[blockIdx.x].u[0] = su[0];
        part[blockIdx.x].s[0] = ss[0];
        part[blockIdx.x].c[0] = sc[0];
        part[blockIdx.x].u[1] = to_bits<T>(sm[0]);
    }
    __threadfence();
    __shared__ bool is_last;
    __syncthreads();
    if (t == 0) is_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last || t != 0) return;
    __threadfence();
    uint64_t u = 0;
    KSum a{0.0, 0.0};
    T mm = from_bits<T>(init_bits);
    for (unsigned b = 0; b < gridDim.x; ++b) {
        u += __ldcg(&part[b].u[0]);
        KSum o{__ldcg(&part[b].s[0]), __ldcg(&part[b].c[0])};
        a = ksum_merge(a, o);
        T bm = from_bits<T>(__ldcg(&part[b].u[1]));
        if (kind == 3 ? (bm < mm) : (bm > mm)) mm = bm;
    }
    *done = 0;
    out3[0] = kind >= 3 ? to_bits<T>(mm) : u;
    out3[1] = static_cast<uint64_t>(__double_as_longlong(a.s));
    out3[2] = static_cast<uint64_t>(__double_as_longlong(a.c));
}

}  // namespace

const char* scan_kernel_name(const ScanParams& p) {
    RangeForm rf;
    if (fsum_shape(p)) return "fsum";
    if (range_form_of(p, &rf, true)) return "range";
    if (multi_range_form_of(p, &rf)) return "mrange";
    return "generic";
}

size_t scan_scratch_bytes() { return kMaxBlocks * sizeof(ScanPartial) + 256; }

int scan_scratch_init(void* scratch, cudaStream_t s) {
    VX_CUDA(cudaMemsetAsync(static_cast<char*>(scratch) + kMaxBlocks * sizeof(ScanPartial), 0, 256, s));
    return kOk;
}

int scan_grid(int dtype, uint64_t ndata, int ncols, int nred) {
    int sms = sm_count();
    if (sms <= 0) sms = 148;
    int unroll = (ncols <= 1 && nred <= 2) ? 4 : (ncols <= 1 ? 2 : 1);
    uint64_t need = (ndata + static_cast<uint64_t>(kThreads) * unroll - 1) / (static_cast<uint64_t>(kThreads) * unroll);
    int per_sm = 8;
    uint64_t cap = static_cast<uint64_t>(sms) * per_sm;
    if (cap > kMaxBlocks) cap = kMaxBlocks;
    uint64_t g = need < cap ? need : cap;
    (void)dtype;
    return g < 1 ? 1 : static_cast<int>(g);
}

int launch_scan(const ScanParams& p, ScanResult* d_out, void* scratch, cudaStream_t s) {
    int grid = scan_grid(p.dtype, p.ndata, p.ncols, p.nred);
    switch (p.dtype) {
    case F64: return dispatch<double>(p, grid, d_out, scratch, s);
    case F32: return dispatch<float>(p, grid, d_out, scratch, s);
    case I64: return dispatch<int64_t>(p, grid, d_out, scratch, s);
    case I32: return dispatch<int32_t>(p, grid, d_out, scratch, s);
    case U64: return dispatch<uint64_t>(p, grid, d_out, scratch, s);
    case U32: return dispatch<uint32_t>(p, grid, d_out, scratch, s);
    default: set_error(kErrInvalidArg, "unknown element type %d", p.dtype); return kErrInvalidArg;
    }
}

int launch_segment_agg(int dtype, const void* col, uint64_t begin, uint64_t end, int kind,
                       uint64_t init_bits, uint64_t* d_out3, void* scratch, cudaStream_t s) {
    ScanPartial* part = static_cast<ScanPartial*>(scratch);
    unsigned int* done = reinterpret_cast<unsigned int*>(static_cast<char*>(scratch) + kMaxBlocks * sizeof(ScanPartial));
    uint64_t n = end > begin ? end - begin : 0;
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t need = (n + kThreads * 4 - 1) / (kThreads * 4);
    uint64_t cap = static_cast<uint64_t>(sms) * 4;
    int grid = static_cast<int>(need < 1 ? 1 : (need < cap ? need : cap));
    switch (dtype) {
    case F64: seg_agg_kernel<double><<<grid, kThreads, 0, s>>>(static_cast<const double*>(col), begin, end, kind, init_bits, part, done, d_out3); break;
    case F32: seg_agg_kernel<float><<<grid, kThreads, 0, s>>>(static_cast<const float*>(col), begin, end, kind, init_bits, part, done, d_out3); break;
    case I64: seg_agg_kernel<int64_t><<<grid, kThreads, 0, s>>>(static_cast<const int64_t*>(col), begin, end, kind, init_bits, part, done, d_out3); break;
    case I32: seg_agg_kernel<int32_t><<<grid, kThreads, 0, s>>>(static_cast<const int32_t*>(col), begin, end, kind, init_bits, part, done, d_out3); break;
    case U64: seg_agg_kernel<uint64_t><<<grid, kThreads, 0, s>>>(static_cast<const uint64_t*>(col), begin, end, kind, init_bits, part, done, d_out3); break;
    case U32: seg_agg_kernel<uint32_t><<<grid, kThreads, 0, s>>>(static_cast<const uint32_t*>(col), begin, end, kind, init_bits, part, done, d_out3); break;
    default: set_error(kErrInvalidArg, "unknown element type %d", dtype); return kErrInvalidArg;
    }
    VX_CUDA(cudaGetLastError());
    return kOk;
}

}  // namespace vx
