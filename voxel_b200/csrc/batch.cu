// Batched persistent executor: many lowered programs in one launch.
//
// Replaces a loop of per-program Engine<T>::Run calls (include/voxel/exec/
// engine.hpp:70-81) for single-column filter/aggregate programs.  The host
// lowers every program (lower.cpp) to a ScanParams and splits its data groups
// into work items of kItemGroups groups; items of a program are contiguous in
// a global item list.  One persistent kernel takes items from a device work
// queue (an atomic counter), so big and small columns interleave across the
// SMs; per item a block:
//   - evaluates the program's groups exactly as the single-program kernel does
//     (scan_core.cuh) and writes a per-item partial of every reduction,
//   - counts the rows that satisfy all of the program's predicate atoms, gets
//     the item's output offset from a decoupled look-back over the program's
//     earlier items, and writes those row ids (ascending) into the program's
//     selection buffer while they fit its capacity (else flags overflow),
//   - and, if it is the program's last item to finish, folds the partials in
//     item order and writes the program's final registers and exact count.
// Every wait is bounded.  The launch (with its memsets) is captured into a
// CUDA graph once per batch and replayed.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <type_traits>
#include <vector>

#include "batch.h"
#include "engine.h"
#include "rangeform.h"
#include "scan_core.cuh"
#include "voxel_c.h"
#include "vx_runtime.h"
#include "vx_scan.cuh"

namespace vx {

namespace {

constexpr int kBThreads = 256;
constexpr int kBU = 2;          // groups per thread per pass
constexpr int kBW = 8;          // passes per item
constexpr int kBNR = 4;         // reductions per batched program
constexpr uint64_t kItemGroups = static_cast<uint64_t>(kBThreads) * kBU * kBW;
constexpr int kRangeBlocks = 4;  // resident blocks per SM of the range-form kernels

// shared memory of one block's current item (one copy for every element type)
struct ItemShared {
    uint32_t mask[kBW][kBThreads];  // selected lanes per pass (bit u*KL+l)
    uint32_t pw[kBW][kBThreads / 32];  // selected rows per (pass, warp), then their exclusive prefix
    Acc blk[kBNR];
    Acc wacc[kBThreads / 32][kBNR];  // per-warp reduction partials
    uint32_t stage[kBThreads / 32][32 * 8 * kBU];  // one warp's row ids of one pass (8 lanes per group at most)
    uint64_t item_base;
    uint64_t spill_a0, spill_p0;  // this item's arena range starts at output position p0 (rows past capacity)
    int spill_ok;
};

struct ItemPartial {
    uint64_t u[kBNR];
    double s[kBNR];
    double c[kBNR];
};

// Atom comparison of all lanes against one threshold (op decided per group).
template <typename T>
__device__ __forceinline__ void atom_lanes(uint8_t op, T t, uint32_t bit, const T (&x)[32 / sizeof(T)],
                                           uint32_t (&ab)[32 / sizeof(T)]) {
    constexpr int KL = 32 / sizeof(T);
    switch (op) {
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

// The evaluators read an item one pass at a time; ask L2 for the whole item
// up front (one bulk prefetch per pass, 16-byte aligned, inside the column) so
// HBM streams it while the passes compute.
template <typename T>
__device__ __forceinline__ void prefetch_item(const ScanParams& p, uint64_t g0) {
    constexpr int KL = 32 / sizeof(T);
    if (threadIdx.x < kBW && p.ncols >= 1) {
        const uint64_t jb = g0 + static_cast<uint64_t>(threadIdx.x) * kBThreads * kBU;
        const uint64_t je = min(jb + static_cast<uint64_t>(kBThreads) * kBU, p.ndata);
        const uint64_t r0 = p.off0 + jb * KL;
        const uint64_t r1 = min(p.off0 + je * KL, p.count[0]);
        if (jb < je && r0 < r1) {
            const uintptr_t base = reinterpret_cast<uintptr_t>(p.col[0]);
            const uintptr_t a = (base + r0 * sizeof(T) + 15) & ~uintptr_t(15);
            const uintptr_t b = (base + r1 * sizeof(T)) & ~uintptr_t(15);
            if (b > a)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(static_cast<uint32_t>(b - a))
                             : "memory");
        }
    }
}

// Second half of every item, shared by the evaluators: the item's reduction
// partial, its selected-row offset (per-pass / per-warp counts, one warp's
// prefix, the decoupled look-back over the program's earlier items) and the
// ascending row ids of its selection.  s_mask holds the evaluator's per-pass
// lane masks (bit u*KL+l of thread x = lane l of its u-th group).
template <typename T, int NR>
__device__ __forceinline__ void item_epilogue(const BatchProg& bp, uint64_t t, Acc (&acc)[NR], ItemPartial* part_item,
                                              BatchOut* out, unsigned long long* status_prog, int* err,
                                              ItemShared& sh, const SpillArgs& sp, uint32_t pid) {
    constexpr int KL = 32 / sizeof(T);
    const ScanParams& p = bp.p;
    uint32_t (*s_mask)[kBThreads] = sh.mask;
    const uint64_t g0 = t * kItemGroups;
    // Per warp: its reduction partials and its selected rows per pass; after
    // one barrier warp 0 merges the partials into the item's partial, takes
    // the exclusive prefix of the (pass, warp) counts in pass-major order
    // (= ascending row order), and gets the item's offset from the look-back.
    constexpr int kWarps = kBThreads / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        if (r >= p.nred) break;
        const uint8_t op = p.red[r].acc;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            Acc o;
            o.u = shfl_down_u64(acc[r].u, d);
            o.k.s = shfl_down_f64(acc[r].k.s, d);
            o.k.c = shfl_down_f64(acc[r].k.c, d);
            acc_merge<T>(acc[r], op, o);
        }
        if (lane == 0) sh.wacc[warp][r] = acc[r];
    }
#pragma unroll 1
    for (int w = 0; w < kBW; ++w) {
        const unsigned c = __reduce_add_sync(0xffffffffu, static_cast<unsigned>(__popc(s_mask[w][threadIdx.x])));
        if (lane == 0) sh.pw[w][warp] = c;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            if (r >= p.nred) break;
            const uint8_t op = p.red[r].acc;
            Acc a;
            a.u = acc_identity(op);
            a.k = {0.0, 0.0};
            if (lane < kWarps) a = sh.wacc[lane][r];
#pragma unroll
            for (int d = kWarps / 2; d > 0; d >>= 1) {
                Acc o;
                o.u = shfl_down_u64(a.u, d);
                o.k.s = shfl_down_f64(a.k.s, d);
                o.k.c = shfl_down_f64(a.k.c, d);
                acc_merge<T>(a, op, o);
            }
            if (lane == 0) {
                part_item->u[r] = a.u;
                part_item->s[r] = a.k.s;
                part_item->c[r] = a.k.c;
            }
        }
        constexpr int kPer = kBW * kWarps / 32;  // entries per lane
        uint32_t* flat = &sh.pw[0][0];
        uint32_t loc[kPer], sum = 0;
#pragma unroll
        for (int e = 0; e < kPer; ++e) {
            loc[e] = flat[lane * kPer + e];
            sum += loc[e];
        }
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        uint32_t run = incl - sum;
#pragma unroll
        for (int e = 0; e < kPer; ++e) {
            flat[lane * kPer + e] = run;
            run += loc[e];
        }
        const uint32_t total_item = __shfl_sync(0xffffffffu, incl, 31);
        const uint64_t e = lookback_exclusive_warp(status_prog, t, total_item, err);
        if (lane == 0) {
            sh.item_base = e;
            if (t == bp.nitems - 1) out->sel_count = e + total_item;
            // rows past the capacity: one arena range for the item, recorded as a fragment
            uint64_t a0 = 0, p0 = 0;
            int ok = 1;
            if (bp.sel_mask && bp.want_sel && e + total_item > bp.sel_cap) {
                p0 = e > bp.sel_cap ? e : bp.sel_cap;
                const uint64_t nov = e + total_item - p0;
                a0 = atomicAdd(sp.cursor, static_cast<unsigned long long>(nov));
                if (a0 + nov <= sp.cap) {
                    const unsigned int f = atomicAdd(sp.nfrags, 1u);  // < items: one per item at most
                    sp.frags[f] = SpillFrag{pid, static_cast<uint32_t>(nov), p0, a0};
                } else {
                    ok = 0;
                }
            }
            sh.spill_a0 = a0;
            sh.spill_p0 = p0;
            sh.spill_ok = ok;
        }
    }
    __syncthreads();
    if (!(bp.sel_mask && bp.want_sel)) return;
    // Row ids in ascending order: pass-major, then warp, then lane.  Each warp
    // gathers its rows of a pass in shared memory and stores them as one
    // contiguous run (whole sectors instead of one scattered word per lane).
    // Row ids are 32-bit, so the item's first row is taken mod 2^32.
    const uint64_t ibase = sh.item_base;
    const uint32_t row_item = static_cast<uint32_t>(p.off0 + g0 * KL);
    uint32_t* const sel_out = bp.sel_out;
    const uint64_t sel_cap = bp.sel_cap;
    uint32_t* const stage = sh.stage[warp];
    bool ovf = false;
#pragma unroll 1
    for (int w = 0; w < kBW; ++w) {
        uint32_t m = s_mask[w][threadIdx.x];
        const uint32_t c = __popc(m);
        uint32_t incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t wtot = __shfl_sync(0xffffffffu, incl, 31);
        if (wtot == 0) continue;  // uniform over the warp
        uint32_t k = incl - c;
        const uint32_t row0 = row_item + (static_cast<uint32_t>(w) * kBThreads * kBU + threadIdx.x * kBU) * KL;
        while (m) {
            const int b = __ffs(m) - 1;  // bit u*KL+l = row (jb+u)*KL+l of the item
            m &= m - 1;
            stage[k++] = row0 + static_cast<uint32_t>(b);
        }
        __syncwarp();
        const uint64_t gpos = ibase + sh.pw[w][warp];
        if (gpos + wtot <= sel_cap) {
            for (uint32_t i = lane; i < wtot; i += 32) sel_out[gpos + i] = stage[i];
        } else {
            ovf = true;
            for (uint32_t i = lane; i < wtot; i += 32) {
                const uint64_t pos = gpos + i;
                if (pos < sel_cap) sel_out[pos] = stage[i];
                else if (sh.spill_ok) sp.rows[sh.spill_a0 + (pos - sh.spill_p0)] = stage[i];
            }
        }
        __syncwarp();
    }
    if (ovf && lane == 0) {
        out->overflow = 1;
        if (!sh.spill_ok) out->spill_lost = 1;
    }
}

// Range form (BatchProg::fast != 0): one column, one reduction whose predicate
// is the conjunction of all atoms, rewritten on the host as lo <= x <= hi and
// (NE) x != ne[0] and x != ne[1].  RK is the reduction kind.  Same results as
// the atom-by-atom evaluation: every ordered atom is a closed interval in T's
// order, and NaN fails every interval test as it fails every ordered atom.
template <typename T, int RK, bool NE>
__device__ __forceinline__ void process_range(const BatchProg& bp, uint64_t t, ItemPartial* part_item, BatchOut* out,
                                           unsigned long long* status_prog, int* err, ItemShared& sh,
                                           const SpillArgs& sp, uint32_t pid) {
    constexpr int KL = 32 / sizeof(T);
    const ScanParams& p = bp.p;
    constexpr uint8_t accop = range_acc(RK, Traits<T>::kFloat);
    Acc acc[1];
    acc[0].u = acc_identity(accop);
    acc[0].k = {0.0, 0.0};
    const uint64_t g0 = t * kItemGroups;
    prefetch_item<T>(p, g0);
    // Everything the loop needs, in registers, in item-relative 32-bit units
    // (the descriptor lives in shared memory; reading it per group costs as
    // much as the evaluation).
    const uint64_t ibeg = p.off0 + g0 * KL;  // first row of the item
    const uint64_t cnt = p.count[0];
    const uint32_t ngi = static_cast<uint32_t>(min(static_cast<uint64_t>(kItemGroups), p.ndata - min(p.ndata, g0)));
    const uint32_t rleft = static_cast<uint32_t>(min(cnt - min(cnt, ibeg), kItemGroups * KL));
    const uint64_t lastj = p.ngroups - 1;
    const uint32_t llast = (lastj >= g0 && lastj - g0 < kItemGroups) ? static_cast<uint32_t>(lastj - g0) : 0xFFFFFFFFu;
    const T* __restrict__ ip = static_cast<const T*>(p.col[0]) + ibeg;  // dereferenced below rleft only
    const bool vec = bp.vec != 0;
    const T lo = from_bits<T>(bp.lo), hi = from_bits<T>(bp.hi);
    const T n0 = from_bits<T>(bp.ne[0]), n1 = from_bits<T>(bp.ne[1]);
    const Red& r0 = p.red[0];
    const T ac = r0.a.kind == kOpConst ? from_bits<T>(r0.a.bits) : T(0);
    const T bc = r0.b.kind == kOpConst ? from_bits<T>(r0.b.bits) : T(0);
    // COUNT of the constants: lanes that pass count when ac is nonzero (and
    // not NaN), the others when bc is
    const uint32_t cnt_pass = (!t_isnan<T>(ac) && ac != T(0)) ? 1u : 0u;
    const uint32_t cnt_fail = (!t_isnan<T>(bc) && bc != T(0)) ? 1u : 0u;
    uint64_t last_res = 0;
    bool has_last = false;
#pragma unroll 1
    for (int w = 0; w < kBW; ++w) {
        uint32_t mask = 0;
        const uint32_t jb = static_cast<uint32_t>(w) * kBThreads * kBU + threadIdx.x * kBU;
        T v[kBU][KL];
#pragma unroll
        for (int u = 0; u < kBU; ++u) {
            const uint32_t r = (jb + u) * KL;
            if (jb + u >= ngi) continue;
            if (vec && r + KL <= rleft) {
                const uint4* q = reinterpret_cast<const uint4*>(ip + r);
                const uint4 a = __ldcs(q), b = __ldcs(q + 1);
                *reinterpret_cast<uint4*>(&v[u][0]) = a;
                *reinterpret_cast<uint4*>(&v[u][KL / 2]) = b;
            } else {
#pragma unroll
                for (int l = 0; l < KL; ++l) v[u][l] = r + l < rleft ? ip[r + l] : T(0);
            }
        }
#pragma unroll
        for (int u = 0; u < kBU; ++u) {
            const uint32_t lj = jb + u;
            if (lj >= ngi) continue;
            uint32_t pm = 0;
            T x[KL];
#pragma unroll
            for (int l = 0; l < KL; ++l) {
                const T y = v[u][l];
                bool pass = y >= lo && y <= hi;
                if constexpr (NE) pass = pass && y != n0 && y != n1;
                pm |= pass ? 1u << l : 0u;
                if constexpr (RK != kRedCount) x[l] = pass ? y : bc;
            }
            uint64_t res;
            if constexpr (RK == kRedCount) {
                const uint32_t np = __popc(pm);
                res = cnt_pass * np + cnt_fail * (KL - np);
            } else {
                res = reduce_group<T>(RK, x);
            }
            acc_fold<T>(acc[0], accop, res);
            if (lj == llast) {
                last_res = res;
                has_last = true;
            }
            const uint32_t r = lj * KL;
            if (r + KL > rleft) pm &= r < rleft ? (1u << (rleft - r)) - 1u : 0u;
            mask |= pm << (u * KL);
        }
        sh.mask[w][threadIdx.x] = mask;
    }
    if (has_last) out->res.last[0] = last_res;
    item_epilogue<T, 1>(bp, t, acc, part_item, out, status_prog, err, sh, sp, pid);
}

// NA = 0: the generic evaluator (scan_core.cuh) for any program shape;
// NA = 1..4 (one column, one reduction, NA atoms): the same evaluation with the
// program's fields held in registers for the whole item.
template <typename T, int NR, int NA>
__device__ __forceinline__ void process_item(const BatchProg& bp, uint64_t t, ItemPartial* part_item, BatchOut* out,
                                          unsigned long long* status_prog, int* err, ItemShared& sh,
                                          const SpillArgs& sp, uint32_t pid) {
    constexpr int KL = 32 / sizeof(T);
    const ScanParams& p = bp.p;
    uint32_t (*s_mask)[kBThreads] = sh.mask;
    Acc acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        acc[r].u = r < p.nred ? acc_identity(p.red[r].acc) : 0;
        acc[r].k = {0.0, 0.0};
    }
    const uint64_t g0 = t * kItemGroups;
    prefetch_item<T>(p, g0);
    const uint64_t lastj = p.ngroups - 1;
    const bool vec = bp.vec != 0;
    // fast path: the program in registers
    T f_thr[NA > 0 ? NA : 1];
    uint8_t f_op[NA > 0 ? NA : 1];
    uint8_t f_kind = 0, f_acc = 0;
    uint32_t f_pm = 0, f_sel = 0;
    bool f_never = false, f_acol = false, f_bcol = false;
    T f_ac = T(0), f_bc = T(0);
    uint64_t f_cnt = 0, f_off = 0, f_ndata = 0;
    if constexpr (NA > 0) {
#pragma unroll
        for (int a = 0; a < NA; ++a) {
            f_thr[a] = from_bits<T>(p.atom[a].thr);
            f_op[a] = p.atom[a].op;
        }
        const Red& r0 = p.red[0];
        f_kind = r0.kind;
        f_acc = r0.acc;
        f_pm = r0.pmask;
        f_never = (r0.pmask & kMaskFalse) != 0;
        f_acol = r0.a.kind == kOpCol;
        f_bcol = r0.b.kind == kOpCol;
        f_ac = r0.a.kind == kOpConst ? from_bits<T>(r0.a.bits) : T(0);
        f_bc = r0.b.kind == kOpConst ? from_bits<T>(r0.b.bits) : T(0);
        f_sel = bp.sel_mask;
        f_cnt = p.count[0];
        f_off = p.off0;
        f_ndata = p.ndata;
    }
    // phase 1: evaluate every pass, fold the reductions, keep the selection masks
#pragma unroll 1
    for (int w = 0; w < kBW; ++w) {
        uint32_t mask = 0;
        // this thread's kBU contiguous groups of pass w
        const uint64_t jb = g0 + static_cast<uint64_t>(w) * kBThreads * kBU + static_cast<uint64_t>(threadIdx.x) * kBU;
        T v[kBU][1][KL];
#pragma unroll
        for (int u = 0; u < kBU; ++u)
            if (jb + u < (NA > 0 ? f_ndata : p.ndata)) load_group<T, 1>(p, jb + u, vec, v[u]);
        if constexpr (NA > 0) {
#pragma unroll
            for (int u = 0; u < kBU; ++u) {
                const uint64_t j = jb + u;
                if (j >= f_ndata) continue;
                uint32_t ab[KL];
#pragma unroll
                for (int l = 0; l < KL; ++l) ab[l] = 0;
#pragma unroll
                for (int a = 0; a < NA; ++a) atom_lanes<T>(f_op[a], f_thr[a], 1u << a, v[u][0], ab);
                T x[KL];
#pragma unroll
                for (int l = 0; l < KL; ++l) {
                    const bool pass = !f_never && (ab[l] & f_pm) == f_pm;
                    x[l] = pass ? (f_acol ? v[u][0][l] : f_ac) : (f_bcol ? v[u][0][l] : f_bc);
                }
                const uint64_t res = reduce_group<T>(f_kind, x);
                acc_fold<T>(acc[0], f_acc, res);
                if (j == lastj) out->res.last[0] = res;
                if (f_sel) {
                    const uint64_t row0 = f_off + j * KL;
                    const bool full = row0 + KL <= f_cnt;
#pragma unroll
                    for (int l = 0; l < KL; ++l)
                        if ((ab[l] & f_sel) == f_sel && (full || row0 + l < f_cnt)) mask |= 1u << (u * KL + l);
                }
            }
        } else {
#pragma unroll
        for (int u = 0; u < kBU; ++u) {
            uint64_t j = jb + u;
            if (j >= p.ndata) continue;
            uint32_t ab[KL];
            eval_atoms<T, 1>(p, v[u], ab);
            uint64_t res[NR];
            eval_reds<T, 1, NR>(p, v[u], ab, res);
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                if (r >= p.nred) break;
                acc_fold<T>(acc[r], p.red[r].acc, res[r]);
                if (j == lastj) out->res.last[r] = res[r];
            }
            if (bp.sel_mask) {
                uint64_t row0 = p.off0 + j * KL;
#pragma unroll
                for (int l = 0; l < KL; ++l)
                    if ((ab[l] & bp.sel_mask) == bp.sel_mask && row0 + l < p.count[0]) mask |= 1u << (u * KL + l);
            }
        }
        }
        s_mask[w][threadIdx.x] = mask;
    }
    item_epilogue<T, NR>(bp, t, acc, part_item, out, status_prog, err, sh, sp, pid);
}

template <typename T, int NR>
__device__ __forceinline__ void finalize_program(const BatchProg& bp, const ItemPartial* parts, BatchOut* out,
                                              ItemShared& sh) {
    const ScanParams& p = bp.p;
    Acc acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        acc[r].u = r < p.nred ? acc_identity(p.red[r].acc) : 0;
        acc[r].k = {0.0, 0.0};
    }
    for (uint32_t i = threadIdx.x; i < bp.nitems; i += blockDim.x) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            if (r >= p.nred) break;
            Acc o;
            o.u = __ldcg(&parts[i].u[r]);
            o.k.s = __ldcg(&parts[i].s[r]);
            o.k.c = __ldcg(&parts[i].c[r]);
            acc_merge<T>(acc[r], p.red[r].acc, o);
        }
    }
    Acc (&blk)[NR] = *reinterpret_cast<Acc (*)[NR]>(sh.blk);
    block_reduce<T, NR, kBThreads>(p, acc, blk);
    if (threadIdx.x == 0) finalize_scan<T, 1, NR>(p, blk, &out->res);
}

// One persistent kernel per program class (element type x one / several
// reductions): blocks take the class's items from its own device work queue
// (an atomic counter), so each kernel is compiled for one element type.
// pids: the class's programs; cstart[k]: first class-local item of pids[k].
template <typename T, int NR, int FAST>
__global__ void __launch_bounds__(kBThreads, FAST ? kRangeBlocks : 2) batch_kernel(const BatchProg* __restrict__ progs,
                                                          const uint32_t* __restrict__ pids, uint32_t npc,
                                                          const uint64_t* __restrict__ cstart, uint64_t citems,
                                                          ItemPartial* parts, unsigned long long* status,
                                                          unsigned int* pdone, unsigned int* item_ctr,
                                                          BatchOut* outs, int* err, const SpillArgs sp) {
    __shared__ uint64_t s_item, s_kbeg, s_kend;
    __shared__ uint32_t s_k;
    __shared__ __align__(16) BatchProg s_bp;
    __shared__ bool s_last;
    __shared__ ItemShared sh;
    uint32_t cached = 0xFFFFFFFFu;
    // Thread 0 claims an item only when the block is about to start it (an
    // item must never wait behind an item a block holds but has not started:
    // the look-back relies on claimed items making progress; finalising a
    // program waits on nothing).  The owning program is looked up only when
    // an item falls outside the block's current program.
    auto claim = [&]() {
        const uint64_t ci = atomicAdd(item_ctr, 1u);
        s_item = ci;
        if (ci < citems && (ci < s_kbeg || ci >= s_kend)) {
            // class program owning item ci: last start <= ci
            uint32_t lo = 0, hi = npc;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (cstart[mid] <= ci) lo = mid;
                else hi = mid;
            }
            s_k = lo;
            s_kbeg = cstart[lo];
            s_kend = cstart[lo + 1];
        }
    };
    if (threadIdx.x == 0) {
        s_kbeg = 1;
        s_kend = 0;
        claim();
    }
    __syncthreads();
    for (;;) {
        const uint64_t ci = s_item;
        if (ci >= citems) break;
        const uint32_t pid = pids[s_k];
        if (pid != cached) {  // uniform: every thread holds the same pid and cache
            const int4* src = reinterpret_cast<const int4*>(progs + pid);
            int4* dst = reinterpret_cast<int4*>(&s_bp);
            for (uint32_t i = threadIdx.x; i < sizeof(BatchProg) / 16; i += blockDim.x) dst[i] = src[i];
            cached = pid;
            __syncthreads();
        }
        const uint64_t t = ci - s_kbeg;
        const uint64_t it = s_bp.item0 + t;  // global item index
        if constexpr (FAST) {
            process_range<T, (FAST - 1) / 2, ((FAST - 1) & 1) != 0>(s_bp, t, parts + it, outs + pid,
                                                                   status + s_bp.item0, err, sh, sp, pid);
        } else if constexpr (NR == 1) {
            switch (s_bp.p.ncols == 1 ? s_bp.p.natoms : 0) {
            case 1: process_item<T, 1, 1>(s_bp, t, parts + it, outs + pid, status + s_bp.item0, err, sh, sp, pid); break;
            case 2: process_item<T, 1, 2>(s_bp, t, parts + it, outs + pid, status + s_bp.item0, err, sh, sp, pid); break;
            case 3: process_item<T, 1, 3>(s_bp, t, parts + it, outs + pid, status + s_bp.item0, err, sh, sp, pid); break;
            case 4: process_item<T, 1, 4>(s_bp, t, parts + it, outs + pid, status + s_bp.item0, err, sh, sp, pid); break;
            default: process_item<T, 1, 0>(s_bp, t, parts + it, outs + pid, status + s_bp.item0, err, sh, sp, pid); break;
            }
        } else {
            process_item<T, NR, 0>(s_bp, t, parts + it, outs + pid, status + s_bp.item0, err, sh, sp, pid);
        }
        // the item's partial and row ids are written: count it done, and take
        // the next item in the same step
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            s_last = atomicAdd(&pdone[pid], 1u) == s_bp.nitems - 1;
            claim();
        }
        __syncthreads();
        if (s_last) {  // uniform
            __threadfence();
            finalize_program<T, NR>(s_bp, parts + s_bp.item0, outs + pid, sh);
            if (threadIdx.x == 0) pdone[pid] = 0;
            __syncthreads();
        }
    }
}

// Program classes: element type x {8 range forms (reduction kind x excluded
// values), one interpreted reduction, several}; each class has its own item
// queue and kernel (one range form per kernel keeps its registers low).
constexpr int kKinds = 10;
constexpr int kClasses = 6 * kKinds;
static_assert(kClasses == Batch::kClasses, "class count");

int class_of(const BatchProg& bp) {
    return bp.p.dtype * kKinds + (bp.fast ? static_cast<int>(bp.fast) - 1 : bp.p.nred <= 1 ? 8 : 9);
}

template <typename T, int NR, int FAST>
int launch_class_t(const BatchProg* progs, const uint32_t* pids, uint32_t npc, const uint64_t* cstart,
                   uint64_t citems, ItemPartial* parts, unsigned long long* status, unsigned int* pdone,
                   unsigned int* ctr, BatchOut* outs, int* err, const SpillArgs& sp, cudaStream_t s) {
    static int per_sm = 0;
    if (!per_sm) {
        VX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<T, NR, FAST>, kBThreads, 0));
        if (per_sm < 1) per_sm = 1;
    }
    uint64_t grid = static_cast<uint64_t>(sm_count() > 0 ? sm_count() : 148) * per_sm;
    if (grid > citems) grid = citems;
    batch_kernel<T, NR, FAST><<<static_cast<unsigned>(grid), kBThreads, 0, s>>>(progs, pids, npc, cstart, citems,
                                                                              parts, status, pdone, ctr, outs, err, sp);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int launch_kind(int kind, const BatchProg* progs, const uint32_t* pids, uint32_t npc, const uint64_t* cstart,
                uint64_t citems, ItemPartial* parts, unsigned long long* status, unsigned int* pdone,
                unsigned int* ctr, BatchOut* outs, int* err, const SpillArgs& sp, cudaStream_t s) {
#define VX_K(NR, F) launch_class_t<T, NR, F>(progs, pids, npc, cstart, citems, parts, status, pdone, ctr, outs, err, sp, s)
    switch (kind) {
    case 0: return VX_K(1, 1);
    case 1: return VX_K(1, 2);
    case 2: return VX_K(1, 3);
    case 3: return VX_K(1, 4);
    case 4: return VX_K(1, 5);
    case 5: return VX_K(1, 6);
    case 6: return VX_K(1, 7);
    case 7: return VX_K(1, 8);
    case 8: return VX_K(1, 0);
    default: return VX_K(kBNR, 0);
    }
#undef VX_K
}

int launch_class(int cls, const BatchProg* progs, const uint32_t* pids, uint32_t npc, const uint64_t* cstart,
                 uint64_t citems, ItemPartial* parts, unsigned long long* status, unsigned int* pdone,
                 unsigned int* ctr, BatchOut* outs, int* err, const SpillArgs& sp, cudaStream_t s) {
#define VX_KIND(TT) \
    launch_kind<TT>(cls % kKinds, progs, pids, npc, cstart, citems, parts, status, pdone, ctr, outs, err, sp, s)
    switch (cls / kKinds) {
    case F64: return VX_KIND(double);
    case F32: return VX_KIND(float);
    case I64: return VX_KIND(int64_t);
    case I32: return VX_KIND(int32_t);
    case U64: return VX_KIND(uint64_t);
    default: return VX_KIND(uint32_t);
    }
#undef VX_KIND
}

bool set_range_form(BatchProg& bp) {
    RangeForm rf;
    const uint32_t all = bp.p.natoms ? (1u << bp.p.natoms) - 1u : 0u;
    if (bp.sel_mask != all || !range_form_of(bp.p, &rf)) return false;
    bp.fast = rf.fast;
    bp.lo = rf.lo;
    bp.hi = rf.hi;
    bp.ne[0] = rf.ne[0];
    bp.ne[1] = rf.ne[1];
    return true;
}

// Exact selections of overflowed programs: blocks [0, nlist) copy program k's
// rows that fit its buffer to d_pool + off[k]; the other blocks copy the
// spilled fragments of listed programs (offmap[pid] = its pool offset, or ~0).
struct GatherItem {
    const uint32_t* sel;
    uint64_t cap;  // rows in the buffer (min of capacity and count)
    uint64_t off;
};

__global__ void gather_overflow_kernel(const GatherItem* __restrict__ list, uint32_t nlist,
                                       const uint64_t* __restrict__ offmap, const SpillFrag* __restrict__ frags,
                                       const unsigned int* nfrags, const uint32_t* __restrict__ spill,
                                       uint32_t* __restrict__ pool) {
    if (blockIdx.x < nlist) {
        const GatherItem g = list[blockIdx.x];
        for (uint64_t r = threadIdx.x; r < g.cap; r += blockDim.x) pool[g.off + r] = __ldg(g.sel + r);
        return;
    }
    const unsigned int nf = *nfrags;
    for (unsigned int f = blockIdx.x - nlist; f < nf; f += gridDim.x - nlist) {
        const SpillFrag fr = frags[f];
        const uint64_t off = offmap[fr.pid];
        if (off == ~0ull) continue;
        for (uint32_t r = threadIdx.x; r < fr.n; r += blockDim.x) pool[off + fr.dst + r] = __ldg(spill + fr.src + r);
    }
}

__global__ void clear_outs_kernel(BatchOut* outs, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        outs[i].overflow = 0;
        outs[i].spill_lost = 0;
        outs[i].sel_count = 0;
    }
}

}  // namespace

Batch::~Batch() {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    if (capture_) cudaStreamDestroy(capture_);
    for (int b = 0; b < kBranches; ++b) {
        if (branch_[b]) cudaStreamDestroy(branch_[b]);
        if (join_[b]) cudaEventDestroy(join_[b]);
    }
    if (fork_) cudaEventDestroy(fork_);
}

int Batch::add(int dtype, const uint32_t* code, size_t len, const uint64_t* regs, const void* d_col, uint64_t count,
               bool want_sel, uint64_t sel_cap, uint32_t* d_sel) {
    Engine e(dtype);
    e.add_segment_device(d_col, count);
    for (int r = 0; r < 64; ++r) e.reg(r) = regs[r];
    e.load_program(code, len);
    std::vector<LoweredRegion> regions;
    int st = e.lower_regions(regions);
    if (st) return st;
    if (regions.size() != 1 || regions[0].params.ncols > 1 || regions[0].params.nred > kBNR) {
        set_error(kErrUnsupportedProgram, "batched programs need exactly one single-column loop with <= %d reductions",
                  kBNR);
        return kErrUnsupportedProgram;
    }
    BatchProg bp{};
    bp.p = regions[0].params;
    bp.p.col[0] = d_col;
    bp.sel_mask = bp.p.natoms ? ((1u << bp.p.natoms) - 1) : 0;
    bp.want_sel = want_sel ? 1 : 0;
    bp.sel_cap = sel_cap;
    bp.sel_out = d_sel;
    uintptr_t a = reinterpret_cast<uintptr_t>(d_col) + bp.p.off0 * dtype_size(dtype);
    bp.vec = (a % 16) == 0;
    set_range_form(bp);
    host_.push_back(bp);
    writes_.push_back(regions[0].writes);
    regs_.emplace_back(regs, regs + 64);
    dirty_ = true;
    return kOk;
}

void Batch::set_capacity(size_t i, uint64_t cap, uint32_t* d_sel) {
    host_[i].sel_cap = cap;
    host_[i].sel_out = d_sel;
    dirty_ = true;
}

int Batch::upload(cudaStream_t s) {
    const uint32_t np = static_cast<uint32_t>(host_.size());
    uint64_t items = 0;
    for (uint32_t i = 0; i < np; ++i) {
        uint64_t ni = (host_[i].p.ndata + kItemGroups - 1) / kItemGroups;
        if (ni == 0) ni = 1;  // every program finalises, even with no data groups
        host_[i].item0 = items;
        host_[i].nitems = static_cast<uint32_t>(ni);
        items += ni;
    }
    nitems_ = items;
    // programs by class (element type x one / several reductions), each class
    // with its own item queue: pids grouped by class, class-local item starts
    std::vector<uint32_t> pids;
    std::vector<uint64_t> cstart;
    pids.reserve(np);
    cstart.reserve(np + kClasses);
    for (int c = 0; c < kClasses; ++c) {
        cls_[c] = ClassQueue{};
        cls_[c].pid_off = static_cast<uint32_t>(pids.size());
        cls_[c].cs_off = static_cast<uint32_t>(cstart.size());
        uint64_t ci = 0;
        for (uint32_t i = 0; i < np; ++i) {
            const int ic = class_of(host_[i]);
            if (ic != c) continue;
            pids.push_back(i);
            cstart.push_back(ci);
            ci += host_[i].nitems;
        }
        cls_[c].np = static_cast<uint32_t>(pids.size()) - cls_[c].pid_off;
        cls_[c].items = ci;
        cstart.push_back(ci);
    }
    if (d_progs_.n < np * sizeof(BatchProg)) d_progs_ = DevBuf(np * sizeof(BatchProg) + 16);
    if (d_start_.n < cstart.size() * 8) d_start_ = DevBuf(cstart.size() * 8 + 8);
    if (d_pids_.n < np * 4 + 4) d_pids_ = DevBuf(np * 4 + 4);
    if (d_outs_.n < np * sizeof(BatchOut)) d_outs_ = DevBuf(np * sizeof(BatchOut) + 16);
    if (d_parts_.n < items * sizeof(ItemPartial)) d_parts_ = DevBuf(items * sizeof(ItemPartial) + 16);
    if (d_status_.n < items * 8 + 8 * kClasses) d_status_ = DevBuf(items * 8 + 8 * kClasses);
    if (d_pdone_.n < np * 4 + 16) {
        d_pdone_ = DevBuf(np * 4 + 16);
        if (d_pdone_.p) VX_CUDA(cudaMemsetAsync(d_pdone_.p, 0, d_pdone_.n, s));
    }
    if (!d_err_.p) {
        d_err_ = DevBuf(16);
        if (d_err_.p) VX_CUDA(cudaMemsetAsync(d_err_.p, 0, 16, s));
    }
    if (d_spill_.n < spill_cap_ * 4 + 16) d_spill_ = DevBuf(spill_cap_ * 4 + 16);
    if (d_frags_.n < items * sizeof(SpillFrag) + 16) d_frags_ = DevBuf(items * sizeof(SpillFrag) + 16);
    if (!d_spill_ctr_.p) d_spill_ctr_ = DevBuf(16);
    if (!d_progs_.p || !d_start_.p || !d_pids_.p || !d_outs_.p || !d_parts_.p || !d_status_.p || !d_pdone_.p ||
        !d_err_.p || !d_spill_.p || !d_frags_.p || !d_spill_ctr_.p)
        return kErrOutOfMemory;
    if (int st = h2d(d_progs_.p, host_.data(), np * sizeof(BatchProg), s)) return st;
    if (int st = h2d(d_start_.p, cstart.data(), cstart.size() * 8, s)) return st;
    if (int st = h2d(d_pids_.p, pids.data(), np * 4, s)) return st;
    if (int st = sync(s)) return st;
    if (graph_exec_) {
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
    }
    if (graph_) {
        cudaGraphDestroy(graph_);
        graph_ = nullptr;
    }
    dirty_ = false;
    return kOk;
}

int Batch::enqueue(cudaStream_t s, bool branches) {
    const uint32_t np = static_cast<uint32_t>(host_.size());
    VX_CUDA(cudaMemsetAsync(d_status_.p, 0, nitems_ * 8 + 8 * kClasses, s));
    clear_outs_kernel<<<(np + 255) / 256, 256, 0, s>>>(d_outs_.as<BatchOut>(), np);
    VX_CUDA(cudaGetLastError());
    VX_CUDA(cudaMemsetAsync(d_spill_ctr_.p, 0, 16, s));
    const SpillArgs sp{d_spill_.as<uint32_t>(), d_spill_.n / 4, d_spill_ctr_.as<unsigned long long>(),
                       d_frags_.as<SpillFrag>(), reinterpret_cast<unsigned int*>(d_spill_ctr_.as<unsigned long long>() + 1)};
    // The class kernels are independent: when recording, spread them over
    // parallel branches (largest class first, each to the least-loaded
    // branch), so one kernel's tail overlaps the next one's start.
    if (branches) {  // streams and events made before the recording began
        VX_CUDA(cudaEventRecord(fork_, s));
        for (int b = 0; b < kBranches; ++b) VX_CUDA(cudaStreamWaitEvent(branch_[b], fork_, 0));
    }
    std::vector<int> order;
    for (int c = 0; c < kClasses; ++c)
        if (cls_[c].np) order.push_back(c);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cls_[x].items > cls_[y].items; });
    // one item counter per class after the look-back status words
    unsigned int* ctr = reinterpret_cast<unsigned int*>(d_status_.as<unsigned long long>() + nitems_);
    uint64_t load[kBranches] = {};
    int st = kOk;
    for (int c : order) {
        int b = 0;
        if (branches)
            for (int k = 1; k < kBranches; ++k)
                if (load[k] < load[b]) b = k;
        load[b] += cls_[c].items;
        st = launch_class(c, d_progs_.as<BatchProg>(), d_pids_.as<uint32_t>() + cls_[c].pid_off, cls_[c].np,
                          d_start_.as<uint64_t>() + cls_[c].cs_off, cls_[c].items, d_parts_.as<ItemPartial>(),
                          d_status_.as<unsigned long long>(), d_pdone_.as<unsigned int>(), ctr + c,
                          d_outs_.as<BatchOut>(), d_err_.as<int>(), sp, branches ? branch_[b] : s);
        if (st) break;
    }
    if (branches) {  // join every branch, also after a failed launch, so the recording can end
        for (int b = 0; b < kBranches; ++b) {
            cudaEventRecord(join_[b], branch_[b]);
            cudaStreamWaitEvent(s, join_[b], 0);
        }
    }
    return st;
}

int Batch::launch(cudaStream_t s, bool use_graph) {
    if (host_.empty()) return kOk;
    if (dirty_) {
        if (int st = upload(s)) return st;
    }
    if (!use_graph) return enqueue(s, false);
    if (!graph_exec_) {
        // Recorded on a private stream: the caller's stream may be the legacy
        // default stream, which cannot be captured.  Recording runs nothing.
        if (!capture_) VX_CUDA(cudaStreamCreateWithFlags(&capture_, cudaStreamNonBlocking));
        for (int b = 0; b < kBranches; ++b) {
            if (!branch_[b]) VX_CUDA(cudaStreamCreateWithFlags(&branch_[b], cudaStreamNonBlocking));
            if (!join_[b]) VX_CUDA(cudaEventCreateWithFlags(&join_[b], cudaEventDisableTiming));
        }
        if (!fork_) VX_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
        VX_CUDA(cudaStreamBeginCapture(capture_, cudaStreamCaptureModeThreadLocal));
        int st = enqueue(capture_, true);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(capture_, &g);
        if (st) return st;
        VX_CUDA(e);
        graph_ = g;
        VX_CUDA(cudaGraphInstantiate(&graph_exec_, graph_, 0));
    }
    VX_CUDA(cudaGraphLaunch(graph_exec_, s));
    return kOk;
}

int Batch::fetch(cudaStream_t s) {
    const size_t np = host_.size();
    outs_.resize(np);
    if (!np) return kOk;
    if (int st = d2h(outs_.data(), d_outs_.p, np * sizeof(BatchOut), s)) return st;
    int h = 0;
    if (int st = d2h(&h, d_err_.p, 4, s)) return st;
    if (int st = sync(s)) return st;
    if (h) {
        cudaMemsetAsync(d_err_.p, 0, 4, s);
        set_error(kErrDeviceTimeout, "batched executor: a look-back wait ran out of budget");
        return kErrDeviceTimeout;
    }
    return kOk;
}

int Batch::gather_overflow(size_t n, const size_t* idx, uint32_t* d_pool, cudaStream_t s) {
    if (outs_.size() != host_.size()) {
        set_error(kErrInvalidArg, "batch gather before fetch");
        return kErrInvalidArg;
    }
    if (!n) return kOk;
    const size_t np = host_.size();
    std::vector<uint64_t> offmap(np, ~0ull);
    std::vector<GatherItem> list(n);
    uint64_t off = 0;
    bool lost = false;
    for (size_t k = 0; k < n; ++k) {
        if (idx[k] >= np) {
            set_error(kErrInvalidArg, "batch gather: program %zu out of range", idx[k]);
            return kErrInvalidArg;
        }
        const BatchOut& o = outs_[idx[k]];
        if (o.spill_lost) lost = true;
        const uint64_t cnt = o.sel_count;
        list[k] = GatherItem{host_[idx[k]].sel_out, cnt < host_[idx[k]].sel_cap ? cnt : host_[idx[k]].sel_cap, off};
        offmap[idx[k]] = off;
        off += cnt;
    }
    if (lost) {
        set_error(kErrCapacity, "batch gather: a listed program's overflow did not fit the spill arena; re-run it");
        return kErrCapacity;
    }
    if (d_offmap_.n < np * 8) d_offmap_ = DevBuf(np * 8 + 8);
    if (d_glist_.n < n * sizeof(GatherItem)) d_glist_ = DevBuf(n * sizeof(GatherItem) + 16);
    if (!d_offmap_.p || !d_glist_.p) return kErrOutOfMemory;
    if (int st = h2d(d_offmap_.p, offmap.data(), np * 8, s)) return st;
    if (int st = h2d(d_glist_.p, list.data(), n * sizeof(GatherItem), s)) return st;
    const unsigned grid = static_cast<unsigned>(n) + 4u * static_cast<unsigned>(sm_count() > 0 ? sm_count() : 148);
    gather_overflow_kernel<<<grid, 256, 0, s>>>(d_glist_.as<GatherItem>(), static_cast<uint32_t>(n),
                                               d_offmap_.as<uint64_t>(), d_frags_.as<SpillFrag>(),
                                               reinterpret_cast<unsigned int*>(d_spill_ctr_.as<unsigned long long>() + 1),
                                               d_spill_.as<uint32_t>(), d_pool);
    VX_CUDA(cudaGetLastError());
    return sync(s);
}

int Batch::rerun(size_t n, const size_t* idx, const size_t* caps, uint32_t* d_pool, cudaStream_t s) {
    if (outs_.size() != host_.size()) {
        set_error(kErrInvalidArg, "batch re-run before fetch");
        return kErrInvalidArg;
    }
    if (!n) return kOk;
    if (!sub_) {
        sub_.reset(new Batch());
        sub_->spill_cap_ = 1024;  // exact capacities: nothing spills
    }
    Batch& b = *sub_;
    b.host_.clear();
    b.writes_.clear();
    b.regs_.clear();
    uint64_t off = 0;
    for (size_t k = 0; k < n; ++k) {
        if (idx[k] >= host_.size()) {
            set_error(kErrInvalidArg, "batch re-run: program %zu out of range", idx[k]);
            return kErrInvalidArg;
        }
        BatchProg bp = host_[idx[k]];
        bp.want_sel = 1;
        bp.sel_cap = caps[k];
        bp.sel_out = d_pool + off;
        off += caps[k];
        b.host_.push_back(bp);
        b.writes_.push_back(writes_[idx[k]]);
        b.regs_.push_back(regs_[idx[k]]);
    }
    b.dirty_ = true;
    if (int st = b.launch(s, false)) return st;
    if (int st = b.fetch(s)) return st;
    for (size_t k = 0; k < n; ++k) outs_[idx[k]] = b.outs_[k];
    return kOk;
}

void Batch::registers(size_t i, uint64_t* regs) const {
    std::memcpy(regs, regs_[i].data(), 64 * 8);
    const BatchOut& o = outs_[i];
    for (const RegWrite& w : writes_[i]) {
        switch (w.kind) {
        case RegWrite::kAcc: regs[w.reg] = o.res.acc[w.red]; break;
        case RegWrite::kLast: if (host_[i].p.ngroups) regs[w.reg] = o.res.last[w.red]; break;
        case RegWrite::kValue: regs[w.reg] = w.value; break;
        }
    }
}

}  // namespace vx

using namespace vx;

extern "C" {

void* voxel_batch_create(void) { return new Batch(); }
void voxel_batch_destroy(void* b) { delete static_cast<Batch*>(b); }
size_t voxel_batch_size(const void* b) { return static_cast<const Batch*>(b)->size(); }

int voxel_batch_add(void* b, int dtype, const uint32_t* code, size_t len, const uint64_t* regs64, const void* d_col,
                    size_t count, int want_selection, size_t sel_capacity, uint32_t* d_sel) {
    clear_error();
    return static_cast<Batch*>(b)->add(dtype, code, len, regs64, d_col, count, want_selection != 0, sel_capacity,
                                       d_sel);
}

int voxel_batch_set_capacity(void* b, size_t prog, size_t capacity, uint32_t* d_sel) {
    Batch* B = static_cast<Batch*>(b);
    if (prog >= B->size()) return kErrInvalidArg;
    B->set_capacity(prog, capacity, d_sel);
    return kOk;
}

int voxel_batch_launch(void* b, int use_graph, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    return static_cast<Batch*>(b)->launch(static_cast<cudaStream_t>(stream), use_graph != 0);
}

int voxel_batch_fetch(void* b, void* stream) {
    clear_error();
    return static_cast<Batch*>(b)->fetch(static_cast<cudaStream_t>(stream));
}

int voxel_batch_results_all(const void* b, uint64_t* regs64, uint64_t* sel_counts, int* overflows) {
    const Batch* B = static_cast<const Batch*>(b);
    if (B->fetched() != B->size()) return kErrInvalidArg;
    for (size_t i = 0; i < B->size(); ++i) {
        if (regs64) B->registers(i, regs64 + 64 * i);
        if (sel_counts) sel_counts[i] = B->out(i).sel_count;
        if (overflows) overflows[i] = B->out(i).overflow + B->out(i).spill_lost;
    }
    return kOk;
}

int voxel_batch_gather_overflow(void* b, size_t n, const size_t* progs, uint32_t* d_pool, void* stream) {
    clear_error();
    return static_cast<Batch*>(b)->gather_overflow(n, progs, d_pool, static_cast<cudaStream_t>(stream));
}

int voxel_batch_set_spill_capacity(void* b, size_t rows) {
    static_cast<Batch*>(b)->set_spill_capacity(rows);
    return kOk;
}

int voxel_batch_rerun(void* b, size_t n, const size_t* progs, const size_t* capacities, uint32_t* d_pool,
                      void* stream) {
    clear_error();
    return static_cast<Batch*>(b)->rerun(n, progs, capacities, d_pool, static_cast<cudaStream_t>(stream));
}

int voxel_batch_form(const void* b, size_t prog) {
    const Batch* B = static_cast<const Batch*>(b);
    if (prog >= B->size()) return -1;
    return static_cast<int>(B->prog(prog).fast);
}

int voxel_batch_result(const void* b, size_t prog, uint64_t* regs64, uint64_t* sel_count, int* overflow) {
    const Batch* B = static_cast<const Batch*>(b);
    if (prog >= B->size() || prog >= B->fetched()) return kErrInvalidArg;
    if (regs64) B->registers(prog, regs64);
    if (sel_count) *sel_count = B->out(prog).sel_count;
    if (overflow) *overflow = B->out(prog).overflow + B->out(prog).spill_lost;
    return kOk;
}

}  // extern "C"
