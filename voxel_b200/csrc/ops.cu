// Remaining reference operators behind the C ABI, on the GPU:
//
//   HashAggregator<u32,f64> (include/voxel/ops/aggregate.hpp:159-301) as the
//     voxel_agg_* object and the one-shot voxel_groupby_*: a device
//     open-addressing table keyed by 64-bit slot words (key << 32 | 1, claimed
//     with one CAS, so a key is published atomically), grown by doubling when a
//     batch would push the load past 0.75 (the reference's limit); per-group
//     state is an exact fixed-point SUM, COUNT, MIN/MAX.  A batch first inserts
//     its keys (idempotent, retried after a grow), then accumulates its values.
//   GroupedAggregator::AccumulateSorted / FinalizeGroups (aggregate.hpp:665-706):
//     runs of equal keys are reduced with a warp segmented scan and one set of
//     atomics per warp segment.
//   SortOperator::SortAscending / SortDescending (sort.hpp:504-541, a stable
//     merge sort on f64 returning indices) and TopKSelect (490-502): the radix
//     sort on order-preserving u64 images of the values (-0.0 folded into +0.0 so
//     equal values keep their input order).
//   DictionaryEncoding<f64>::Build / DecodeBatch (encoding.hpp:113-167).
#include <algorithm>
#include <cstring>
#include <vector>

#include "fixedpoint.cuh"
#include "radix.h"
#include "voxel_c.h"
#include "vx_common.cuh"
#include "vx_runtime.h"
#include "vx_scan.cuh"

namespace vx {

namespace {

constexpr int kOThreads = 256;

int ogrid(uint64_t n, int per_sm = 8) {
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t b = (n + kOThreads - 1) / kOThreads;
    uint64_t cap = static_cast<uint64_t>(sms) * per_sm;
    if (b > cap) b = cap;
    return b < 1 ? 1 : static_cast<int>(b);
}

// Home slot of a key: Fibonacci (multiplicative) hashing, the top log2(cap)
// bits of k * 2^32/phi (two instructions).  The slot layout is internal: every
// result leaves the table sorted by key, so it need not follow the reference's
// murmur3 mixer (ops/hash.hpp:334-339), whose two 64-bit multiplies and
// shifts per row made both table kernels ALU-bound.
__device__ __forceinline__ uint32_t home_slot(uint32_t k, uint32_t shift) {
    return (k * 0x9E3779B1u) >> shift;
}

struct Table {
    unsigned long long* slot;  // 0 = empty, else (key << 32) | 1
    unsigned long long* sum;   // 3 words per slot
    unsigned long long* cnt;
    unsigned long long* mn;
    unsigned long long* mx;
    uint64_t mask;
    uint32_t shift;  // 32 - log2(mask + 1)
};

__global__ void table_init_kernel(Table t) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= t.mask;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        t.slot[i] = 0;
        t.sum[3 * i] = 0;
        t.sum[3 * i + 1] = 0;
        t.sum[3 * i + 2] = 0;
        t.cnt[i] = 0;
        t.mn[i] = ~0ull;
        t.mx[i] = 0;
    }
}

// Phase 1 bookkeeping, once per warp and row batch: the new groups the warp
// inserted are added to the table's group count at once, and a count past the
// load limit raises the overflow flag.  `seen` is lane 0's read of the flag,
// issued at the start of the batch so its latency hides behind the batch's
// probes.  Returns true when the warp should stop.
__device__ __forceinline__ int overflow_peek(const int* overflow) {
    return (threadIdx.x & 31) == 0 ? *reinterpret_cast<const volatile int*>(overflow) : 0;
}

__device__ __forceinline__ bool warp_count_groups(unsigned added_now, unsigned long long* groups, uint64_t limit,
                                                  int* overflow, int seen) {
    const unsigned total = __reduce_add_sync(0xffffffffu, added_now);
    int stop = seen;
    if ((threadIdx.x & 31) == 0 && total) {
        const unsigned long long g = atomicAdd(groups, static_cast<unsigned long long>(total)) + total;
        if (g > limit) {
            atomicOr(overflow, 1);
            stop = 1;
        }
    }
    return __shfl_sync(0xffffffffu, stop, 0) != 0;
}

// Claims the key's slot in the global table (the slot word is published with
// one CAS); returns 1 when this call inserted it, 0 when the key was there,
// -1 when the probe ran past `probe_limit` slots (the overflow flag is then
// raised).  Far more threads than slots run at once, so a table sized too
// small is overfilled within the first row of every thread; the probe limit
// makes each later probe of that full table give up after a few slots
// instead of walking all of them.  The host tells a full table (grow) from a
// long cluster in a lightly loaded one (retry with no limit) by the group
// count the attempt left.
__device__ __forceinline__ int claim_slot(const Table& t, uint32_t k, uint64_t probe_limit, int* overflow) {
    const unsigned long long want = (static_cast<unsigned long long>(k) << 32) | 1ull;
    uint64_t h = home_slot(k, t.shift);
    for (uint64_t p = 0;; ++p) {
        const unsigned long long cur = __ldcg(t.slot + h);
        if (cur == want) return 0;
        if (cur == 0) {
            const unsigned long long old = atomicCAS(&t.slot[h], 0ull, want);
            if (old == 0) return 1;
            if (old == want) return 0;
        }
        h = (h + 1) & t.mask;
        if (p >= probe_limit || p > t.mask) {
            atomicOr(overflow, 1);
            return -1;
        }
    }
}

// phase 1: make sure every key has a slot; counts new groups; flags overflow.
// The row loop is warp-uniform (whole warps step together) so the group count
// can be kept per warp; a block stops claiming as soon as one of its threads
// met a full table.
__global__ void insert_keys_kernel(Table t, const uint32_t* __restrict__ keys, uint64_t n,
                                   unsigned long long* groups, uint64_t limit, uint64_t probe_limit, int* overflow) {
    __shared__ int s_stop;
    if (threadIdx.x == 0) s_stop = 0;
    __syncthreads();
    const uint64_t lane = threadIdx.x & 31;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t base = static_cast<uint64_t>(blockIdx.x) * blockDim.x + (threadIdx.x - lane); base < n;
         base += stride) {
        const int seen = overflow_peek(overflow);
        const uint64_t i = base + lane;
        unsigned added = 0;
        if (i < n && !*reinterpret_cast<volatile int*>(&s_stop)) {
            const int r = claim_slot(t, keys[i], probe_limit, overflow);
            if (r > 0) added = 1;
            if (r < 0) s_stop = 1;
        }
        if (warp_count_groups(added, groups, limit, overflow, seen)) break;
    }
}

// Phase 1 for small tables: each block first looks a key up in a shared copy
// of the slot words taken at its start; only keys missing there (new keys, or
// keys another block inserted after the copy) take the global CAS path above.
__global__ void __launch_bounds__(512) insert_keys_smem_kernel(Table t, const uint32_t* __restrict__ keys,
                                                               uint64_t n, unsigned long long* groups, uint64_t limit,
                                                               uint64_t probe_limit, int* overflow) {
    extern __shared__ __align__(16) unsigned long long i_slot[];
    __shared__ int s_stop;
    const uint32_t cap = static_cast<uint32_t>(t.mask + 1), mask = cap - 1;
    for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x) i_slot[i] = __ldcg(t.slot + i);
    if (threadIdx.x == 0) s_stop = 0;
    __syncthreads();
    const uint64_t lane = threadIdx.x & 31;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t base = static_cast<uint64_t>(blockIdx.x) * blockDim.x + (threadIdx.x - lane); base < n;
         base += 4 * stride) {
        const int seen = overflow_peek(overflow);
        const uint64_t i0 = base + lane;
        uint32_t kk[4];  // four keys in flight per thread
#pragma unroll
        for (int u = 0; u < 4; ++u) kk[u] = i0 + u * stride < n ? __ldcs(keys + i0 + u * stride) : 0u;
        unsigned added = 0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (i0 + u * stride >= n) break;
            const uint32_t k = kk[u];
            const unsigned long long want = (static_cast<unsigned long long>(k) << 32) | 1ull;
            uint32_t h = home_slot(k, t.shift);
            uint32_t probes = 0;
            unsigned long long cur;
            while ((cur = i_slot[h]) != want && cur != 0 && probes++ < mask) h = (h + 1) & mask;
            if (cur == want) continue;
            if (*reinterpret_cast<volatile int*>(&s_stop)) break;
            const int r = claim_slot(t, k, probe_limit, overflow);
            if (r > 0) ++added;
            if (r < 0) {
                s_stop = 1;
                break;
            }
        }
        if (warp_count_groups(added, groups, limit, overflow, seen)) break;
    }
}

__device__ __forceinline__ uint64_t find_slot(const Table& t, uint32_t k) {
    unsigned long long want = (static_cast<unsigned long long>(k) << 32) | 1ull;
    uint64_t h = home_slot(k, t.shift);
    for (uint64_t p = 0; p <= t.mask; ++p) {
        unsigned long long cur = __ldg(t.slot + h);
        if (cur == want) return h;
        if (cur == 0) return ~0ull;
        h = (h + 1) & t.mask;
    }
    return ~0ull;
}

// phase 2: fold values into their groups (keys all present)
__global__ void accumulate_kernel(Table t, const uint32_t* __restrict__ keys, const double* __restrict__ vals,
                                  uint64_t n, int* err) {
    bool bad = false;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t s = find_slot(t, keys[i]);
        if (s == ~0ull) { bad = true; continue; }
        double v = vals[i];
        fix_atomic_add(&t.sum[3 * s], fix_from_double(v, &bad));
        atomicAdd(&t.cnt[s], 1ull);
        uint64_t ok = f64_order_key(v);
        if (ok < t.mn[s]) atomicMin(&t.mn[s], static_cast<unsigned long long>(ok));
        if (ok > t.mx[s]) atomicMax(&t.mx[s], static_cast<unsigned long long>(ok));
    }
    if (bad) atomicOr(err, 1);
}

// Phase 2 for tables of up to kSmemSlots slots: each block folds its rows into
// a shared-memory copy of the per-slot state (native 32-bit atomics), then adds
// it to the table once.  The sum is the same 192-bit integer (LSB 2^-96) the
// global path accumulates, kept as six 32-bit words: a row adds
// trunc(|x| * 2^96) (three words at word k0, or subtracts it for x < 0) and a
// word's wrap, read from the atomic's returned old value, ripples upward, so
// concurrent rows compose to the exact sum in any order.
constexpr uint32_t kSmemSlots = 2048;
constexpr uint64_t kProbeLimit = 128;  // slots a phase-1 probe walks before it reports a full table
constexpr int kAccWords = 6;

struct Words96 {
    uint32_t c0, c1, c2;
    int k0;
};

// trunc(|x| * 2^96) as three words at word k0; false for NaN / inf / |x| >= 2^63
__device__ __forceinline__ bool words96(double x, Words96* w) {
    const uint64_t b = static_cast<uint64_t>(__double_as_longlong(x));
    const int ex = static_cast<int>((b >> 52) & 0x7FF);
    w->c0 = w->c1 = w->c2 = 0;
    w->k0 = 0;
    if (ex == 0x7FF) return false;
    if (ex == 0) return true;  // zero or subnormal: below the window
    uint64_t m = (b & ((1ull << 52) - 1)) | (1ull << 52);
    int sh = ex - 1075 + 96;  // |x| * 2^96 = m * 2^sh
    if (sh >= 107) return false;  // |x| >= 2^63
    if (sh < 0) {
        m = sh > -64 ? (m >> -sh) : 0;
        sh = 0;
    }
    const uint32_t ml = static_cast<uint32_t>(m), mh = static_cast<uint32_t>(m >> 32);
    const uint32_t r = static_cast<uint32_t>(sh) & 31;
    w->k0 = sh >> 5;  // <= 3: words k0..k0+2 lie inside the 6 words
    w->c0 = ml << r;
    w->c1 = __funnelshift_l(ml, mh, r);
    w->c2 = __funnelshift_l(mh, 0u, r);
    return true;
}

// Carry (+1) or borrow (-1) into word j and upwards while words wrap: rare
// (the first level is handled inline below).
__device__ __noinline__ void ripple96(uint32_t* acc, int j, uint32_t step, uint32_t wrap) {
    while (j < kAccWords && atomicAdd(&acc[j], step) == wrap) ++j;
}

// Adds (neg: subtracts) the row's words; each word's wrap goes into the next
// word inline and ripples further only when that word wraps too (exact under
// any interleaving of concurrent rows).
__device__ __forceinline__ void add96(uint32_t* acc, const Words96& w, bool neg) {
    const uint32_t d0 = neg ? 0u - w.c0 : w.c0, d1 = neg ? 0u - w.c1 : w.c1, d2 = neg ? 0u - w.c2 : w.c2;
    uint32_t o0 = 0, o1 = 0, o2 = 0;
    if (w.c0) o0 = atomicAdd(&acc[w.k0], d0);
    if (w.c1) o1 = atomicAdd(&acc[w.k0 + 1], d1);
    if (w.c2) o2 = atomicAdd(&acc[w.k0 + 2], d2);
    const bool r0 = w.c0 && (neg ? o0 < w.c0 : o0 + w.c0 < o0);
    const bool r1 = w.c1 && (neg ? o1 < w.c1 : o1 + w.c1 < o1);
    const bool r2 = w.c2 && (neg ? o2 < w.c2 : o2 + w.c2 < o2) && w.k0 + 3 < kAccWords;
    const uint32_t step = neg ? 0xFFFFFFFFu : 1u, wrap = neg ? 0u : 0xFFFFFFFFu;
    bool x0 = false, x1 = false, x2 = false;
    if (r0) x0 = atomicAdd(&acc[w.k0 + 1], step) == wrap;
    if (r1) x1 = atomicAdd(&acc[w.k0 + 2], step) == wrap;
    if (r2) x2 = atomicAdd(&acc[w.k0 + 3], step) == wrap;
    if (x0) ripple96(acc, w.k0 + 2, step, wrap);
    if (x1) ripple96(acc, w.k0 + 3, step, wrap);
    if (x2) ripple96(acc, w.k0 + 4, step, wrap);
}

__global__ void __launch_bounds__(512) accumulate_smem_kernel(Table t, const uint32_t* __restrict__ keys,
                                                              const double* __restrict__ vals, uint64_t n, int* err) {
    extern __shared__ __align__(16) unsigned long long a_sm[];
    const uint32_t cap = static_cast<uint32_t>(t.mask + 1);
    unsigned long long* s_slot = a_sm;  // the table's slot words (read at L2: written by the insert kernel)
    unsigned long long* s_mn = s_slot + cap;
    unsigned long long* s_mx = s_mn + cap;
    uint32_t* s_w = reinterpret_cast<uint32_t*>(s_mx + cap);
    uint32_t* s_cnt = s_w + kAccWords * cap;
    for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x) {
        s_slot[i] = __ldcg(t.slot + i);
#pragma unroll
        for (int k = 0; k < kAccWords; ++k) s_w[kAccWords * i + k] = 0;
        s_cnt[i] = 0;
        s_mn[i] = ~0ull;
        s_mx[i] = 0;
    }
    __syncthreads();
    const uint32_t mask = cap - 1;
    bool bad = false;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i0 < n; i0 += 4 * stride) {
        // four rows in flight per thread: loads first
        uint32_t kk[4];
        double vv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint64_t i = i0 + u * stride;
            kk[u] = i < n ? __ldcs(keys + i) : 0u;
            vv[u] = i < n ? __ldcs(vals + i) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (i0 + u * stride >= n) break;
            // the key's slot: linear probing in the shared copy
            const unsigned long long want = (static_cast<unsigned long long>(kk[u]) << 32) | 1ull;
            uint32_t sl = home_slot(kk[u], t.shift);
            uint32_t probes = 0;
            unsigned long long cur;
            while ((cur = s_slot[sl]) != want && cur != 0 && probes++ < mask) sl = (sl + 1) & mask;
            if (cur != want) {
                bad = true;
                continue;
            }
            const double v = vv[u];
            Words96 w;
            if (words96(v, &w)) add96(s_w + kAccWords * sl, w, v < 0.0);
            else bad = true;
            atomicAdd(&s_cnt[sl], 1u);
            const uint64_t ok = f64_order_key(v);
            if (ok < s_mn[sl]) atomicMin(&s_mn[sl], static_cast<unsigned long long>(ok));
            if (ok > s_mx[sl]) atomicMax(&s_mx[sl], static_cast<unsigned long long>(ok));
        }
    }
    if (bad) atomicOr(err, 1);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x) {
        const uint32_t c = s_cnt[i];
        if (!c) continue;
        const uint32_t* w = s_w + kAccWords * i;
        const Fix3 f{w[0] | (static_cast<uint64_t>(w[1]) << 32), w[2] | (static_cast<uint64_t>(w[3]) << 32),
                     w[4] | (static_cast<uint64_t>(w[5]) << 32)};
        fix_atomic_add(&t.sum[3 * i], f);
        atomicAdd(&t.cnt[i], static_cast<unsigned long long>(c));
        atomicMin(&t.mn[i], s_mn[i]);
        atomicMax(&t.mx[i], s_mx[i]);
    }
}

size_t smem_table_bytes(uint64_t cap) { return cap * (3 * 8 + kAccWords * 4 + 4); }

// move every occupied slot of `from` into `to` (a grow)
__global__ void rehash_kernel(Table from, Table to) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= from.mask;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        unsigned long long w = from.slot[i];
        if (!w) continue;
        uint32_t k = static_cast<uint32_t>(w >> 32);
        uint64_t h = home_slot(k, to.shift);
        for (;;) {
            if (atomicCAS(&to.slot[h], 0ull, w) == 0ull) break;
            h = (h + 1) & to.mask;
        }
        to.sum[3 * h] = from.sum[3 * i];
        to.sum[3 * h + 1] = from.sum[3 * i + 1];
        to.sum[3 * h + 2] = from.sum[3 * i + 2];
        to.cnt[h] = from.cnt[i];
        to.mn[h] = from.mn[i];
        to.mx[h] = from.mx[i];
    }
}

// occupied slots -> (key image for sorting, slot id)
__global__ void collect_kernel(Table t, int key_signed, uint32_t* out_key, uint32_t* out_slot,
                               unsigned long long* n) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= t.mask;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        unsigned long long w = t.slot[i];
        if (!w) continue;
        unsigned long long p = atomicAdd(n, 1ull);
        out_key[p] = static_cast<uint32_t>(w >> 32);
        out_slot[p] = static_cast<uint32_t>(i);
    }
    (void)key_signed;
}

__global__ void emit_groups_kernel(Table t, const uint32_t* __restrict__ skey, const uint32_t* __restrict__ sslot,
                                   uint64_t g, uint32_t* okeys, double* osum, double* omin, double* omax,
                                   uint64_t* ocount) {
    for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < g;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint32_t s = sslot[j];
        okeys[j] = skey[j];
        Fix3 f{t.sum[3 * s], t.sum[3 * s + 1], t.sum[3 * s + 2]};
        osum[j] = fix_to_double(f);
        omin[j] = f64_from_order_key(t.mn[s]);
        omax[j] = f64_from_order_key(t.mx[s]);
        ocount[j] = t.cnt[s];
    }
}

// ---- sorted (run-based) group-by ----------------------------------------------------

__global__ void grouped_sorted_kernel(const int32_t* __restrict__ keys, const double* __restrict__ vals, uint64_t n,
                                      const uint32_t* __restrict__ run_of, unsigned long long* sum,
                                      unsigned long long* cnt, unsigned long long* mn, unsigned long long* mx,
                                      int* err) {
    const int lane = threadIdx.x & 31;
    bool bad = false;
    // warps take 32 consecutive rows; runs inside a warp are contiguous lane ranges
    for (uint64_t base = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) & ~31ull; base < n;
         base += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t i = base + lane;
        bool in = i < n;
        uint32_t r = in ? run_of[i] : 0xFFFFFFFFu;
        double v = in ? vals[i] : 0.0;
        Fix3 f = in ? fix_from_double(v, &bad) : Fix3{0, 0, 0};
        uint64_t c = in ? 1 : 0;
        uint64_t okey = f64_order_key(v);
        uint64_t lo = in ? okey : ~0ull, hi = in ? okey : 0;
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t rr = __shfl_up_sync(0xffffffffu, r, d);
            Fix3 g;
            g.w0 = __shfl_up_sync(0xffffffffu, f.w0, d);
            g.w1 = __shfl_up_sync(0xffffffffu, f.w1, d);
            g.w2 = __shfl_up_sync(0xffffffffu, f.w2, d);
            uint64_t cc = __shfl_up_sync(0xffffffffu, c, d);
            uint64_t l2 = __shfl_up_sync(0xffffffffu, lo, d);
            uint64_t h2 = __shfl_up_sync(0xffffffffu, hi, d);
            if (lane >= d && rr == r) {
                fix_add(f, g);
                c += cc;
                lo = l2 < lo ? l2 : lo;
                hi = h2 > hi ? h2 : hi;
            }
        }
        uint32_t rn = __shfl_down_sync(0xffffffffu, r, 1);
        bool tail = in && (lane == 31 || rn != r);
        if (tail) {
            fix_atomic_add(&sum[3 * static_cast<uint64_t>(r)], f);
            atomicAdd(&cnt[r], static_cast<unsigned long long>(c));
            atomicMin(&mn[r], static_cast<unsigned long long>(lo));
            atomicMax(&mx[r], static_cast<unsigned long long>(hi));
        }
    }
    if (bad) atomicOr(err, 1);
    (void)keys;
}

__global__ void run_flags_kernel(const int32_t* __restrict__ keys, uint64_t n, uint32_t* __restrict__ flag) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        flag[i] = (i > 0 && keys[i] != keys[i - 1]) ? 1u : 0u;
}

// inclusive scan of 0/1 flags -> run id per row (single pass, look-back)
constexpr int kScanItems = 8;
constexpr int kScanTile = kOThreads * kScanItems;
__global__ void __launch_bounds__(kOThreads) run_ids_kernel(const uint32_t* __restrict__ flag, uint64_t n,
                                                            uint32_t* __restrict__ run, unsigned long long* status,
                                                            unsigned int* ctr, int* err) {
    __shared__ uint64_t s_tile, s_base;
    __shared__ uint32_t s_warp[kOThreads / 32];
    const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        uint64_t r0 = tile * kScanTile + threadIdx.x * kScanItems;
        uint32_t v[kScanItems], c = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            v[k] = r0 + k < n ? flag[r0 + k] : 0;
            c += v[k];
        }
        int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        uint32_t inc = c;
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += y;
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            uint32_t x = lane < kOThreads / 32 ? s_warp[lane] : 0, t = x;
            for (int d = 1; d < 32; d <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, t, d);
                if (lane >= d) t += y;
            }
            if (lane < kOThreads / 32) s_warp[lane] = t - x;
            if (lane == kOThreads / 32 - 1) s_base = lookback_exclusive(status, tile, t, err);
        }
        __syncthreads();
        uint64_t pos = s_base + s_warp[warp] + (inc - c);
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            pos += v[k];
            if (r0 + k < n) run[r0 + k] = static_cast<uint32_t>(pos);
        }
        __syncthreads();
    }
}

__global__ void emit_runs_kernel(const int32_t* __restrict__ keys, const uint32_t* __restrict__ run, uint64_t n,
                                 const unsigned long long* sum, const unsigned long long* cnt,
                                 const unsigned long long* mn, const unsigned long long* mx, int32_t* okeys,
                                 double* osum, double* omin, double* omax, uint64_t* ocount) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (i > 0 && run[i] == run[i - 1]) continue;
        uint32_t r = run[i];
        okeys[r] = keys[i];
        Fix3 f{sum[3 * r], sum[3 * r + 1], sum[3 * r + 2]};
        osum[r] = fix_to_double(f);
        omin[r] = f64_from_order_key(mn[r]);
        omax[r] = f64_from_order_key(mx[r]);
        ocount[r] = cnt[r];
    }
}

__global__ void init_runs_kernel(unsigned long long* sum, unsigned long long* cnt, unsigned long long* mn,
                                 unsigned long long* mx, uint64_t g) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < g;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        sum[3 * i] = 0;
        sum[3 * i + 1] = 0;
        sum[3 * i + 2] = 0;
        cnt[i] = 0;
        mn[i] = ~0ull;
        mx[i] = 0;
    }
}

// ---- f64 sort keys -----------------------------------------------------------------

__global__ void f64_sort_keys_kernel(const double* __restrict__ x, uint64_t n, int descending,
                                     uint64_t* __restrict__ key, uint32_t* __restrict__ idx) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        // -0.0 and +0.0 compare equal in the reference's merge: both become +0.0
        // (bit test: exact for every input, NaN included)
        uint64_t b = static_cast<uint64_t>(__double_as_longlong(x[i]));
        if ((b << 1) == 0) b = 0;
        uint64_t k = f64_order_key(__longlong_as_double(static_cast<long long>(b)));
        key[i] = descending ? ~k : k;
        idx[i] = static_cast<uint32_t>(i);
    }
}

__global__ void gather_f64_kernel(const double* __restrict__ x, const uint32_t* __restrict__ idx, uint64_t k,
                                  double* __restrict__ out) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < k;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        out[i] = x[idx[i]];
}

// dictionary build: sorted (key, row) -> dictionary values + per-row indices
__global__ void dict_heads_kernel(const uint64_t* __restrict__ skey, uint64_t n, uint32_t* __restrict__ flag) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        // NaN images never compare equal, like std::unordered_map<double> keys.
        // Order key: non-negative x -> bits | sign (magnitude in k), negative
        // x -> ~bits (magnitude in ~k).
        uint64_t k = skey[i];
        bool nan = (k >> 63) ? ((k & 0x7FFFFFFFFFFFFFFFull) > 0x7FF0000000000000ull)
                             : ((~k & 0x7FFFFFFFFFFFFFFFull) > 0x7FF0000000000000ull);
        flag[i] = (i > 0 && (skey[i] != skey[i - 1] || nan)) ? 1u : 0u;
    }
}

__global__ void dict_emit_kernel(const double* __restrict__ x, const uint32_t* __restrict__ srow,
                                 const uint32_t* __restrict__ run, uint64_t n, double* __restrict__ dict,
                                 uint32_t* __restrict__ indices) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint32_t r = run[i];
        if (i == 0 || run[i - 1] != r) dict[r] = x[srow[i]];  // first occurrence's representation
        indices[srow[i]] = r;
    }
}

__global__ void f64_dict_gather_kernel(const double* __restrict__ dict, const uint32_t* __restrict__ idx,
                                       uint64_t count, double* __restrict__ out) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        out[i] = dict[idx[i]];
}

thread_local DevBuf t_oerr;
int* oerr(cudaStream_t s) {
    if (!t_oerr.p) {
        t_oerr = DevBuf(16);
        if (t_oerr.p) cudaMemsetAsync(t_oerr.p, 0, 16, s);
    }
    return t_oerr.as<int>();
}
int ocheck(cudaStream_t s, const char* what) {
    int h = 0;
    if (int st = d2h(&h, oerr(s), 4, s)) return st;
    if (int st = sync(s)) return st;
    if (h) {
        cudaMemsetAsync(oerr(s), 0, 4, s);
        if (h & 4) { set_error(kErrDeviceTimeout, "%s: a device-side wait ran out of budget", what); return kErrDeviceTimeout; }
        set_error(kErrOverflow, "%s: a value is not finite or exceeds 2^63 in magnitude", what);
        return kErrOverflow;
    }
    return kOk;
}

// sorted run ids for n rows of keys (flags + scan); returns #runs
int run_ids(const int32_t* keys, uint64_t n, DevBuf& run, cudaStream_t s, uint64_t* nruns) {
    DevBuf flag(n * 4 + 4);
    run = DevBuf(n * 4 + 4);
    uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    DevBuf scratch((ntiles + 1) * 8 + 64);
    if (!flag.p || !run.p || !scratch.p) return kErrOutOfMemory;
    run_flags_kernel<<<ogrid(n), kOThreads, 0, s>>>(keys, n, flag.as<uint32_t>());
    VX_CUDA(cudaMemsetAsync(scratch.p, 0, scratch.n, s));
    unsigned long long* status = scratch.as<unsigned long long>();
    unsigned int* ctr = reinterpret_cast<unsigned int*>(status + ntiles);
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t b = ntiles < static_cast<uint64_t>(sms) * 4 ? ntiles : static_cast<uint64_t>(sms) * 4;
    run_ids_kernel<<<static_cast<unsigned>(b), kOThreads, 0, s>>>(flag.as<uint32_t>(), n, run.as<uint32_t>(), status,
                                                                 ctr, oerr(s));
    VX_CUDA(cudaGetLastError());
    uint32_t last = 0;
    if (int st = d2h(&last, run.as<uint32_t>() + (n - 1), 4, s)) return st;
    if (int st = ocheck(s, "run scan")) return st;
    *nruns = static_cast<uint64_t>(last) + 1;
    return kOk;
}

}  // namespace

__global__ void iota_u32_kernel(uint32_t* out, uint64_t n) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<uint32_t>(i);
}

__global__ void gather_rows_f64_kernel(const double* __restrict__ v, const uint32_t* __restrict__ idx,
                                       uint64_t n, double* __restrict__ out) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        out[i] = __ldg(v + __ldg(idx + i));
}

// ---- device hash aggregator object ------------------------------------------------

class HashAgg {
public:
    DevBuf mem;
    Table t{};
    uint64_t cap = 0, groups = 0;
    DevBuf groups_d, flag_d;

    int alloc_table(uint64_t c, Table& out, DevBuf& m, cudaStream_t s) {
        if (c > (1ull << 32)) {  // more slots than 32-bit keys could need
            set_error(kErrInvalidArg, "hash table of %llu slots exceeds 2^32", static_cast<unsigned long long>(c));
            return kErrInvalidArg;
        }
        size_t bytes = c * (8 + 24 + 8 + 8 + 8);
        m = DevBuf(bytes);
        if (!m.p) return kErrOutOfMemory;
        char* b = static_cast<char*>(m.p);
        out.slot = reinterpret_cast<unsigned long long*>(b);
        out.sum = out.slot + c;
        out.cnt = out.sum + 3 * c;
        out.mn = out.cnt + c;
        out.mx = out.mn + c;
        out.mask = c - 1;
        int lg = 0;
        while ((2ull << lg) <= c) ++lg;
        out.shift = static_cast<uint32_t>(32 - lg);
        table_init_kernel<<<ogrid(c), kOThreads, 0, s>>>(out);
        VX_CUDA(cudaGetLastError());
        return kOk;
    }

    int init(uint64_t expected, cudaStream_t s) {
        uint64_t c = 16;
        while (c < expected * 2) c <<= 1;  // nextpow2(max(2*expected, 16)) (aggregate.hpp:160)
        cap = c;
        groups = 0;
        if (!groups_d.p) groups_d = DevBuf(16);
        if (!flag_d.p) flag_d = DevBuf(16);
        if (!groups_d.p || !flag_d.p) return kErrOutOfMemory;
        VX_CUDA(cudaMemsetAsync(groups_d.p, 0, 16, s));
        return alloc_table(c, t, mem, s);
    }

    int grow(cudaStream_t s, uint64_t factor) {
        Table nt{};
        DevBuf nm;
        if (int st = alloc_table(cap * factor, nt, nm, s)) return st;
        rehash_kernel<<<ogrid(cap), kOThreads, 0, s>>>(t, nt);
        VX_CUDA(cudaGetLastError());
        mem = std::move(nm);
        t = nt;
        cap *= factor;
        return kOk;
    }

    int accumulate(const uint32_t* dk, const double* dv, uint64_t n, cudaStream_t s) {
        if (!mem.p) if (int st = init(16, s)) return st;
        if (!n) return kOk;
        // phase 1: insert keys, growing until every key fits under load 0.75.
        // An attempt that overflowed leaves the exact count of the groups it
        // inserted: a table (nearly) full grows 8x (a far-too-small size
        // hint), one past its load limit 2x, and one that gave up on a long
        // probe at a low load is retried with unbounded probes.
        uint64_t probe_limit = kProbeLimit;
        for (int attempt = 0; attempt < 64; ++attempt) {
            VX_CUDA(cudaMemsetAsync(flag_d.p, 0, 4, s));
            uint64_t limit = cap * 3 / 4;
            if (cap <= kSmemSlots) {
                const int sms = sm_count() > 0 ? sm_count() : 148;
                uint64_t blocks = (n + 511) / 512;
                if (blocks > static_cast<uint64_t>(sms) * 4) blocks = static_cast<uint64_t>(sms) * 4;
                insert_keys_smem_kernel<<<static_cast<unsigned>(blocks), 512, cap * 8, s>>>(
                    t, dk, n, groups_d.as<unsigned long long>(), limit, probe_limit, flag_d.as<int>());
            } else {
                insert_keys_kernel<<<ogrid(n), kOThreads, 0, s>>>(t, dk, n, groups_d.as<unsigned long long>(), limit,
                                                                  probe_limit, flag_d.as<int>());
            }
            VX_CUDA(cudaGetLastError());
            int ovf = 0;
            uint64_t g = 0;
            if (int st = d2h(&ovf, flag_d.p, 4, s)) return st;
            if (int st = d2h(&g, groups_d.p, 8, s)) return st;
            if (int st = sync(s)) return st;
            groups = g;
            if (!ovf) break;
            if (g >= cap - cap / 16) {
                if (int st = grow(s, 8)) return st;
            } else if (g > limit || g >= cap / 2) {
                if (int st = grow(s, 2)) return st;
            } else {
                probe_limit = ~0ull;
            }
        }
        if (cap <= kSmemSlots) {  // per-block shared-memory state, one flush per block
            const size_t smem = smem_table_bytes(cap);
            static bool attr_set = false;
            if (!attr_set) {
                VX_CUDA(cudaFuncSetAttribute(accumulate_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem_table_bytes(kSmemSlots))));
                attr_set = true;
            }
            int per_sm = 0;
            VX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, accumulate_smem_kernel, 512, smem));
            if (per_sm < 1) per_sm = 1;
            const int sms = sm_count() > 0 ? sm_count() : 148;
            uint64_t blocks = (n + 511) / 512;
            if (blocks > static_cast<uint64_t>(sms) * per_sm) blocks = static_cast<uint64_t>(sms) * per_sm;
            accumulate_smem_kernel<<<static_cast<unsigned>(blocks), 512, smem, s>>>(t, dk, dv, n, oerr(s));
        } else {
            accumulate_kernel<<<ogrid(n), kOThreads, 0, s>>>(t, dk, dv, n, oerr(s));
        }
        VX_CUDA(cudaGetLastError());
        return ocheck(s, "group-by");
    }

    // groups sorted by key (key_signed: order as i32); dev_out: the outputs are
    // device pointers (copied on the stream instead of read back)
    int results(int key_signed, void* okeys, double* osum, double* omin, double* omax, uint64_t* ocount,
                cudaStream_t s, bool dev_out = false) {
        if (!groups) return kOk;
        DevBuf k(groups * 4 + 4), sl(groups * 4 + 4), n(8);
        DevBuf ok(groups * 4), os(groups * 8), omn(groups * 8), omx(groups * 8), oc(groups * 8);
        if (!k.p || !sl.p || !n.p || !ok.p || !os.p || !omn.p || !omx.p || !oc.p) return kErrOutOfMemory;
        VX_CUDA(cudaMemsetAsync(n.p, 0, 8, s));
        collect_kernel<<<ogrid(cap), kOThreads, 0, s>>>(t, key_signed, k.as<uint32_t>(), sl.as<uint32_t>(),
                                                        n.as<unsigned long long>());
        VX_CUDA(cudaGetLastError());
        size_t tb = radix_tmp_bytes(key_signed ? I32 : U32, groups);
        DevBuf tmp(tb);
        if (!tmp.p) return kErrOutOfMemory;
        if (int st = launch_radix_sort(key_signed ? I32 : U32, k.p, sl.as<uint32_t>(), groups, tmp.p, tb, radix_err(s),
                                       s, nullptr))
            return st;
        emit_groups_kernel<<<ogrid(groups), kOThreads, 0, s>>>(t, k.as<uint32_t>(), sl.as<uint32_t>(), groups,
                                                              ok.as<uint32_t>(), os.as<double>(), omn.as<double>(),
                                                              omx.as<double>(), oc.as<uint64_t>());
        VX_CUDA(cudaGetLastError());
        auto out = [&](void* dst, const void* src, size_t bytes) -> int {
            if (!dst) return kOk;
            if (dev_out) {
                VX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
                return kOk;
            }
            return d2h(dst, src, bytes, s);
        };
        if (int st = out(okeys, ok.p, groups * 4)) return st;
        if (int st = out(osum, os.p, groups * 8)) return st;
        if (int st = out(omin, omn.p, groups * 8)) return st;
        if (int st = out(omax, omx.p, groups * 8)) return st;
        if (int st = out(ocount, oc.p, groups * 8)) return st;
        if (dev_out) if (int st = sync(s)) return st;  // the staging buffers are released on return
        return radix_check(s);
    }
};

struct DictF64 {
    DevBuf dict, indices;
    uint64_t card = 0, n = 0;
};

}  // namespace vx

using namespace vx;

extern "C" {

// ---- HashAggregator<u32,f64> (reference bindings/voxel_c.cpp:168-182) ----------------
void* voxel_agg_create(void) { return new HashAgg(); }
void voxel_agg_destroy(void* a) { delete static_cast<HashAgg*>(a); }
void voxel_agg_init(void* a, size_t expected) {
    clear_error();
    if (ensure_device()) return;
    cudaStream_t s = thread_stream();
    static_cast<HashAgg*>(a)->init(expected, s);
    sync(s);
}
void voxel_agg_accumulate(void* a, const uint32_t* keys, const double* values, size_t n) {
    clear_error();
    if (ensure_device()) return;
    cudaStream_t s = thread_stream();
    DevBuf dk(n * 4 + 4), dv(n * 8 + 8);
    if (!dk.p || !dv.p) return;
    if (h2d(dk.p, keys, n * 4, s) || h2d(dv.p, values, n * 8, s)) return;
    static_cast<HashAgg*>(a)->accumulate(dk.as<uint32_t>(), dv.as<double>(), n, s);
}
size_t voxel_agg_group_count(const void* a) { return static_cast<const HashAgg*>(a)->groups; }
int voxel_agg_accumulate_dev(void* a, const uint32_t* d_keys, const double* d_values, size_t n, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    return static_cast<HashAgg*>(a)->accumulate(d_keys, d_values, n, static_cast<cudaStream_t>(stream));
}
size_t voxel_agg_results(void* a, uint32_t* keys, double* sum, double* mn, double* mx, uint64_t* count) {
    clear_error();
    if (ensure_device()) return static_cast<size_t>(-1);
    HashAgg* h = static_cast<HashAgg*>(a);
    if (h->results(0, keys, sum, mn, mx, count, thread_stream())) return static_cast<size_t>(-1);
    return h->groups;
}

size_t voxel_groupby_u32_f64(const uint32_t* keys, const double* values, size_t n, size_t expected,
                             uint32_t* okeys, double* osum, double* omin, double* omax, uint64_t* ocount) {
    clear_error();
    if (ensure_device()) return static_cast<size_t>(-1);
    cudaStream_t s = thread_stream();
    HashAgg h;
    if (h.init(expected, s)) return static_cast<size_t>(-1);
    DevBuf dk(n * 4 + 4), dv(n * 8 + 8);
    if (!dk.p || !dv.p) return static_cast<size_t>(-1);
    if (h2d(dk.p, keys, n * 4, s) || h2d(dv.p, values, n * 8, s)) return static_cast<size_t>(-1);
    if (h.accumulate(dk.as<uint32_t>(), dv.as<double>(), n, s)) return static_cast<size_t>(-1);
    if (h.results(0, okeys, osum, omin, omax, ocount, s)) return static_cast<size_t>(-1);
    return h.groups;
}

size_t voxel_groupby_i32_f64(const int32_t* keys, const double* values, size_t n, size_t expected, int32_t* okeys,
                             double* osum, double* omin, double* omax, uint64_t* ocount) {
    clear_error();
    if (ensure_device()) return static_cast<size_t>(-1);
    cudaStream_t s = thread_stream();
    HashAgg h;
    if (h.init(expected, s)) return static_cast<size_t>(-1);
    DevBuf dk(n * 4 + 4), dv(n * 8 + 8);
    if (!dk.p || !dv.p) return static_cast<size_t>(-1);
    if (h2d(dk.p, keys, n * 4, s) || h2d(dv.p, values, n * 8, s)) return static_cast<size_t>(-1);
    if (h.accumulate(dk.as<uint32_t>(), dv.as<double>(), n, s)) return static_cast<size_t>(-1);
    if (h.results(1, okeys, osum, omin, omax, ocount, s)) return static_cast<size_t>(-1);
    return h.groups;
}

size_t voxel_grouped_sorted_i32_f64(const int32_t* sorted_keys, const double* values, size_t n, int32_t* okeys,
                                    double* osum, double* omin, double* omax, uint64_t* ocount) {
    clear_error();
    if (n == 0) return 0;
    if (ensure_device()) return static_cast<size_t>(-1);
    cudaStream_t s = thread_stream();
    DevBuf dk(n * 4), dv(n * 8);
    if (!dk.p || !dv.p) return static_cast<size_t>(-1);
    if (h2d(dk.p, sorted_keys, n * 4, s) || h2d(dv.p, values, n * 8, s)) return static_cast<size_t>(-1);
    DevBuf run;
    uint64_t g = 0;
    if (run_ids(dk.as<int32_t>(), n, run, s, &g)) return static_cast<size_t>(-1);
    DevBuf st(g * 48), ok(g * 4), os(g * 8), omn(g * 8), omx(g * 8), oc(g * 8);
    if (!st.p || !ok.p || !os.p || !omn.p || !omx.p || !oc.p) return static_cast<size_t>(-1);
    unsigned long long* sum = st.as<unsigned long long>();
    unsigned long long *cnt = sum + 3 * g, *mn = cnt + g, *mx = mn + g;
    init_runs_kernel<<<ogrid(g), kOThreads, 0, s>>>(sum, cnt, mn, mx, g);
    grouped_sorted_kernel<<<ogrid(n), kOThreads, 0, s>>>(dk.as<int32_t>(), dv.as<double>(), n, run.as<uint32_t>(),
                                                         sum, cnt, mn, mx, oerr(s));
    emit_runs_kernel<<<ogrid(n), kOThreads, 0, s>>>(dk.as<int32_t>(), run.as<uint32_t>(), n, sum, cnt, mn, mx,
                                                    ok.as<int32_t>(), os.as<double>(), omn.as<double>(),
                                                    omx.as<double>(), oc.as<uint64_t>());
    if (cudaGetLastError() != cudaSuccess) return static_cast<size_t>(-1);
    if (d2h(okeys, ok.p, g * 4, s) || d2h(osum, os.p, g * 8, s) || d2h(omin, omn.p, g * 8, s) ||
        d2h(omax, omx.p, g * 8, s) || d2h(ocount, oc.p, g * 8, s))
        return static_cast<size_t>(-1);
    if (ocheck(s, "sorted group-by")) return static_cast<size_t>(-1);
    return g;
}

// ---- group-by over device columns with a chosen plan -----------------------------------
// method 0: HashAggregator (table sized for expected_groups, grown by doubling
// if that was too small); 1: sort-based (stable radix sort of the keys with row
// ids, values gathered, GroupedAggregator over the runs).  Both sum the same
// fixed-point integers, so the outputs (groups in key order) are bit-identical;
// the plan only changes the time.  *ngroups (host) gets the group count.
int voxel_groupby_u32_f64_dev(const uint32_t* d_keys, const double* d_values, size_t n, size_t expected_groups,
                              int method, uint32_t* d_okeys, double* d_osum, double* d_omin, double* d_omax,
                              uint64_t* d_ocount, uint64_t* ngroups, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (ngroups) *ngroups = 0;
    if (method != 0 && method != 1) {
        set_error(kErrInvalidArg, "group-by method %d is neither 0 (hash) nor 1 (sort)", method);
        return kErrInvalidArg;
    }
    if (n == 0) return kOk;
    if (method == 0) {
        HashAgg h;
        if (int st = h.init(expected_groups, s)) return st;
        if (int st = h.accumulate(d_keys, d_values, n, s)) return st;
        if (int st = h.results(0, d_okeys, d_osum, d_omin, d_omax, d_ocount, s, true)) return st;
        if (ngroups) *ngroups = h.groups;
        return kOk;
    }
    if (n >= (1ull << 32)) {
        set_error(kErrInvalidArg, "sort-based group-by limited to 2^32 rows");
        return kErrInvalidArg;
    }
    DevBuf sk(n * 4), idx(n * 4), sv(n * 8);
    if (!sk.p || !idx.p || !sv.p) return kErrOutOfMemory;
    VX_CUDA(cudaMemcpyAsync(sk.p, d_keys, n * 4, cudaMemcpyDeviceToDevice, s));
    iota_u32_kernel<<<ogrid(n), kOThreads, 0, s>>>(idx.as<uint32_t>(), n);
    VX_CUDA(cudaGetLastError());
    {
        const size_t tb = radix_tmp_bytes(U32, n);
        DevBuf tmp(tb);
        if (!tmp.p) return kErrOutOfMemory;
        if (int st = launch_radix_sort(U32, sk.p, idx.as<uint32_t>(), n, tmp.p, tb, radix_err(s), s, nullptr))
            return st;
        gather_rows_f64_kernel<<<ogrid(n), kOThreads, 0, s>>>(d_values, idx.as<uint32_t>(), n, sv.as<double>());
        VX_CUDA(cudaGetLastError());
        if (int st = sync(s)) return st;  // tmp is released here
    }
    DevBuf run;
    uint64_t g = 0;
    // runs only compare keys for equality, so the u32 keys are read as i32 bits
    if (int st = run_ids(sk.as<int32_t>(), n, run, s, &g)) return st;
    DevBuf stt(g * 48);
    if (!stt.p) return kErrOutOfMemory;
    unsigned long long* sum = stt.as<unsigned long long>();
    unsigned long long *cnt = sum + 3 * g, *mn = cnt + g, *mx = mn + g;
    init_runs_kernel<<<ogrid(g), kOThreads, 0, s>>>(sum, cnt, mn, mx, g);
    grouped_sorted_kernel<<<ogrid(n), kOThreads, 0, s>>>(sk.as<int32_t>(), sv.as<double>(), n, run.as<uint32_t>(),
                                                         sum, cnt, mn, mx, oerr(s));
    emit_runs_kernel<<<ogrid(n), kOThreads, 0, s>>>(sk.as<int32_t>(), run.as<uint32_t>(), n, sum, cnt, mn, mx,
                                                    reinterpret_cast<int32_t*>(d_okeys), d_osum, d_omin, d_omax,
                                                    d_ocount);
    VX_CUDA(cudaGetLastError());
    if (int st = ocheck(s, "sorted group-by")) return st;
    if (int st = radix_check(s)) return st;
    if (ngroups) *ngroups = g;
    return kOk;
}

// ---- SortOperator / TopK (reference bindings/voxel_c.cpp:187-203) ---------------------
static int sort_f64_index(const double* data, size_t n, int desc, DevBuf& dx, DevBuf& keys, DevBuf& idx,
                          cudaStream_t s) {
    dx = DevBuf(n * 8);
    keys = DevBuf(n * 8);
    idx = DevBuf(n * 4);
    if (!dx.p || !keys.p || !idx.p) return kErrOutOfMemory;
    if (int st = h2d(dx.p, data, n * 8, s)) return st;
    f64_sort_keys_kernel<<<ogrid(n), kOThreads, 0, s>>>(dx.as<double>(), n, desc, keys.as<uint64_t>(),
                                                        idx.as<uint32_t>());
    VX_CUDA(cudaGetLastError());
    size_t tb = radix_tmp_bytes(U64, n);
    DevBuf tmp(tb);
    if (!tmp.p) return kErrOutOfMemory;
    return launch_radix_sort(U64, keys.p, idx.as<uint32_t>(), n, tmp.p, tb, radix_err(s), s, nullptr);
}

static void sort_impl(const double* data, size_t n, uint32_t* out, int desc) {
    clear_error();
    if (n == 0) return;
    if (n == 1) { out[0] = 0; return; }
    if (ensure_device()) return;
    cudaStream_t s = thread_stream();
    DevBuf dx, keys, idx;
    if (sort_f64_index(data, n, desc, dx, keys, idx, s)) return;
    if (d2h(out, idx.p, n * 4, s)) return;
    radix_check(s);
}

void voxel_sort_ascending(const double* data, size_t n, uint32_t* out) { sort_impl(data, n, out, 0); }
void voxel_sort_descending(const double* data, size_t n, uint32_t* out) { sort_impl(data, n, out, 1); }

void voxel_topk(const double* data, size_t n, size_t k, double* out, int largest) {
    clear_error();
    if (k >= n) {  // sort.hpp:491: k >= count copies the input unchanged
        if (n) std::memcpy(out, data, n * 8);
        return;
    }
    if (ensure_device()) return;
    cudaStream_t s = thread_stream();
    DevBuf dx, keys, idx;
    if (sort_f64_index(data, n, largest ? 1 : 0, dx, keys, idx, s)) return;
    DevBuf o(k * 8 + 8);
    if (!o.p) return;
    gather_f64_kernel<<<ogrid(k), kOThreads, 0, s>>>(dx.as<double>(), idx.as<uint32_t>(), k, o.as<double>());
    if (d2h(out, o.p, k * 8, s)) return;
    radix_check(s);
}

// ---- DictionaryEncoding<f64> (reference bindings/voxel_c.cpp:208-214) -----------------
void* voxel_dict_create(void) { return new DictF64(); }
void voxel_dict_destroy(void* d) { delete static_cast<DictF64*>(d); }
void voxel_dict_build(void* h, const double* data, size_t n) {
    clear_error();
    DictF64* d = static_cast<DictF64*>(h);
    d->card = 0;
    d->n = n;
    d->dict.reset();
    d->indices.reset();
    if (n == 0) return;
    if (ensure_device()) return;
    cudaStream_t s = thread_stream();
    DevBuf dx, keys, idx;
    if (sort_f64_index(data, n, 0, dx, keys, idx, s)) return;
    DevBuf flag(n * 4), run(n * 4);
    uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    DevBuf scratch((ntiles + 1) * 8 + 64);
    if (!flag.p || !run.p || !scratch.p) return;
    dict_heads_kernel<<<ogrid(n), kOThreads, 0, s>>>(keys.as<uint64_t>(), n, flag.as<uint32_t>());
    cudaMemsetAsync(scratch.p, 0, scratch.n, s);
    unsigned long long* status = scratch.as<unsigned long long>();
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t b = ntiles < static_cast<uint64_t>(sms) * 4 ? ntiles : static_cast<uint64_t>(sms) * 4;
    run_ids_kernel<<<static_cast<unsigned>(b), kOThreads, 0, s>>>(flag.as<uint32_t>(), n, run.as<uint32_t>(), status,
                                                                 reinterpret_cast<unsigned int*>(status + ntiles),
                                                                 oerr(s));
    uint32_t last = 0;
    if (d2h(&last, run.as<uint32_t>() + (n - 1), 4, s) || ocheck(s, "dictionary build")) return;
    d->card = static_cast<uint64_t>(last) + 1;
    d->dict = DevBuf(d->card * 8);
    d->indices = DevBuf(n * 4);
    if (!d->dict.p || !d->indices.p) return;
    dict_emit_kernel<<<ogrid(n), kOThreads, 0, s>>>(dx.as<double>(), idx.as<uint32_t>(), run.as<uint32_t>(), n,
                                                    d->dict.as<double>(), d->indices.as<uint32_t>());
    sync(s);
}
size_t voxel_dict_cardinality(const void* h) { return static_cast<const DictF64*>(h)->card; }
void voxel_dict_decode_batch(void* h, double* out, size_t offset, size_t count) {
    clear_error();
    DictF64* d = static_cast<DictF64*>(h);
    if (offset >= d->n) return;
    if (count > d->n - offset) count = d->n - offset;  // encoding.hpp:163
    if (!count || ensure_device()) return;
    cudaStream_t s = thread_stream();
    DevBuf o(count * 8);
    if (!o.p) return;
    f64_dict_gather_kernel<<<ogrid(count), kOThreads, 0, s>>>(d->dict.as<double>(), d->indices.as<uint32_t>() + offset,
                                                              count, o.as<double>());
    if (d2h(out, o.p, count * 8, s)) return;
    sync(s);
}
size_t voxel_dict_values(const void* h, double* out) {
    const DictF64* d = static_cast<const DictF64*>(h);
    if (d->card && out) {
        cudaStream_t s = thread_stream();
        if (d2h(out, d->dict.p, d->card * 8, s) || sync(s)) return static_cast<size_t>(-1);
    }
    return d->card;
}

}  // extern "C"
