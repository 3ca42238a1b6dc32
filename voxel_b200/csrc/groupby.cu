// Fused scan + group-by over a dictionary-encoded, bit-packed key column.
//
// Reference composition this replaces (all single-threaded CPU operators):
//   BitPackedEncoding::DecodeBatch -> DictionaryEncoding lookup
//     (include/voxel/data/encoding.hpp:397-422, 156-167)
//   VectorFilter<f64>::ApplyGT, VectorFilter<i32>::ApplyBetween, ColumnFilter::AndWith
//     (include/voxel/ops/filter.hpp:42-78, 255-288, 526-547)
//   SelectionVector::BuildFromBitmap + gather (filter.hpp:378-399)
//   HashAggregator<i32,f64>::Accumulate / Finalize (include/voxel/ops/aggregate.hpp:159-261)
//
// B200 design: one pass over the three columns, nothing materialised.  The
// reference's dictionary is sorted and unique, so a row's dictionary index is
// already a dense group id in key order: no hash table is needed.  Each block
// keeps a shared-memory table of per-group state and runs barrier-free over
// its tiles (each thread reads its rows' key bits straight through L1).  A
// passing row costs two shared atomics in the common case: its exact
// fixed-point value (LSB 2^-76) shifted left 20 bits with the row count in the
// low 20 bits goes into a 192-bit accumulator, so SUM and COUNT share words;
// MIN/MAX (as order keys) are only touched when they improve.  Blocks flush to
// a global table (exact 192-bit sums, u64 counts) before 2^20 rows could wrap
// the embedded count, and the last block to finish converts the global table
// to sorted output rows and resets it for the next launch.
#include <cstdio>
#include <mutex>
#include <type_traits>

#include "fixedpoint.cuh"
#include "groupby.h"
#include "tune.h"
#include "tma.cuh"
#include "voxel_c.h"
#include "vx_common.cuh"
#include "vx_runtime.h"
#include "vx_scan.cuh"

namespace vx {

namespace {

constexpr int kGbThreads = 512;
constexpr int kCountBits = 20;
constexpr int kFixScale = 76;  // LSB weight 2^-76 of the group sums
constexpr int kWordScale = 76; // LSB weight of the 32-bit word accumulators (the same)
constexpr int kWords = 5;      // 160-bit word accumulator per group
constexpr int kMaxWidth = 32;

struct GlobalGroups {
    unsigned long long* sum;  // 3 words per group, LSB 2^-76
    unsigned long long* cnt;
    unsigned long long* mn;   // order keys
    unsigned long long* mx;
};

// x -> 192-bit fixed point with LSB 2^-S (|x| < 2^63); *bad on NaN / inf / overflow
template <int S>
__device__ __forceinline__ Fix3 fix_from_double_s(double x, bool* bad) {
    uint64_t b = static_cast<uint64_t>(__double_as_longlong(x));
    int ex = static_cast<int>((b >> 52) & 0x7FF);
    Fix3 r{0, 0, 0};
    if (ex == 0x7FF) { *bad = true; return r; }
    if (ex == 0) return r;
    uint64_t m = (b & ((1ull << 52) - 1)) | (1ull << 52);
    int s = ex - 1075 + S;
    if (ex >= 1023 + 63) { *bad = true; return r; }
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
    if (b >> 63) {
        r.w0 = ~r.w0; r.w1 = ~r.w1; r.w2 = ~r.w2;
        r.w0 += 1;
        if (r.w0 == 0) { r.w1 += 1; if (r.w1 == 0) r.w2 += 1; }
    }
    return r;
}

// (F << 20) | 1 : the value and one row, packed for a single 192-bit add
__device__ __forceinline__ Fix3 pack_row(const Fix3& f) {
    Fix3 v;
    v.w0 = (f.w0 << kCountBits) | 1ull;
    v.w1 = (f.w1 << kCountBits) | (f.w0 >> (64 - kCountBits));
    v.w2 = (f.w2 << kCountBits) | (f.w1 >> (64 - kCountBits));
    return v;
}

// accumulator -> (value with LSB 2^-76, count)
__device__ __forceinline__ Fix3 unpack_sum(Fix3 x, unsigned int* count) {
    *count = static_cast<unsigned int>(x.w0 & ((1ull << kCountBits) - 1));
    x.w0 -= *count;
    Fix3 f;
    f.w0 = (x.w0 >> kCountBits) | (x.w1 << (64 - kCountBits));
    f.w1 = (x.w1 >> kCountBits) | (x.w2 << (64 - kCountBits));
    f.w2 = static_cast<uint64_t>(static_cast<int64_t>(x.w2) >> kCountBits);
    return f;
}

__device__ __forceinline__ uint32_t key_bits(const uint64_t* __restrict__ packed, uint64_t row, uint32_t w,
                                             uint64_t mask) {
    uint64_t bit = row * w;
    uint64_t wi = bit >> 6;
    uint32_t sh = static_cast<uint32_t>(bit & 63);
    uint64_t v = __ldg(packed + wi) >> sh;
    if (sh + w > 64) v |= __ldg(packed + wi + 1) << (64 - sh);
    return static_cast<uint32_t>(v & mask);
}

// key_bits for scans whose bit offsets fit 32 bits (rows x width < 2^32): the
// queue holds the row's bit offset, and the decode is two 32-bit loads and a
// funnel shift (nw32: 32-bit words of the packed column that hold values)
__device__ __forceinline__ uint32_t key_bits32(const uint32_t* __restrict__ p32, uint32_t bit, uint32_t nw32,
                                               uint32_t mask32) {
    const uint32_t q = bit >> 5;
    const uint32_t lo = __ldg(p32 + q);
    const uint32_t hi = q + 1 < nw32 ? __ldg(p32 + q + 1) : 0u;
    return __funnelshift_r(lo, hi, bit & 31) & mask32;
}

// Word form of a row value for the 32-bit table (MODE 1, 2): the magnitude
// trunc(|x| * 2^76) -- the integer fix_from_double_s<76> produces -- as three
// 32-bit words c0..c2 placed at word k0 of a 160-bit group accumulator.
// Returns false for NaN, inf or |x| >= 2^63; zero and subnormals give c = 0.
struct RowWords {
    uint32_t c0, c1, c2;
    int k0;
};

__device__ __forceinline__ bool row_words(double x, RowWords* w) {
    const uint64_t b = static_cast<uint64_t>(__double_as_longlong(x));
    const int ex = static_cast<int>((b >> 52) & 0x7FF);
    w->c0 = w->c1 = w->c2 = 0;
    w->k0 = 0;
    if (ex >= 1023 + 63) return false;  // inf, NaN, |x| >= 2^63
    if (ex == 0) return true;
    uint64_t m = (b & ((1ull << 52) - 1)) | (1ull << 52);
    int s = ex - 1075 + kWordScale;  // |x| * 2^76 = m * 2^s, s <= 86
    if (s < 0) {
        m = s > -64 ? (m >> -s) : 0;
        s = 0;
    }
    const uint32_t ml = static_cast<uint32_t>(m), mh = static_cast<uint32_t>(m >> 32);
    const uint32_t r = static_cast<uint32_t>(s) & 31;
    w->k0 = s >> 5;  // <= 2, so words k0..k0+2 lie inside the 5-word accumulator
    w->c0 = ml << r;
    w->c1 = __funnelshift_l(ml, mh, r);
    w->c2 = __funnelshift_l(mh, 0u, r);
    return true;
}

// Carry (+1) or borrow (-1) into word j and upwards while words wrap: rare
// (the first level is handled inline below).
__device__ __noinline__ void words_ripple(uint32_t* acc, int j, uint32_t step, uint32_t wrap) {
    while (j < kWords && atomicAdd(&acc[j], step) == wrap) ++j;
}

// Adds (neg: subtracts) a row's words to a group accumulator: the three
// atomics are issued back to back, each one's own wrap (read from its
// returned old value) goes into the next word, and a wrap of that word
// ripples further up.  Every wrap is accounted exactly once, so concurrent
// updates compose to the exact sum (modulo 2^160; no true sum needs more).
// MAYNEG = false: the caller knows every value of the warp is >= 0.
template <bool MAYNEG = true>
__device__ __forceinline__ void words_add(uint32_t* acc, const RowWords& w, bool neg) {
    if (!MAYNEG) neg = false;
    const uint32_t d0 = neg ? 0u - w.c0 : w.c0, d1 = neg ? 0u - w.c1 : w.c1, d2 = neg ? 0u - w.c2 : w.c2;
    uint32_t o0 = 0, o1 = 0, o2 = 0;
    if (w.c0) o0 = atomicAdd(&acc[w.k0], d0);
    if (w.c1) o1 = atomicAdd(&acc[w.k0 + 1], d1);
    if (w.c2) o2 = atomicAdd(&acc[w.k0 + 2], d2);
    // add: carry when old + c wraps; subtract: borrow when old < c
    const bool r0 = w.c0 && (neg ? o0 < w.c0 : o0 + w.c0 < o0);
    const bool r1 = w.c1 && (neg ? o1 < w.c1 : o1 + w.c1 < o1);
    const bool r2 = w.c2 && (neg ? o2 < w.c2 : o2 + w.c2 < o2) && w.k0 + 3 < kWords;
    const uint32_t step = neg ? 0xFFFFFFFFu : 1u, wrap = neg ? 0u : 0xFFFFFFFFu;
    bool x0 = false, x1 = false, x2 = false;
    if (r0) x0 = atomicAdd(&acc[w.k0 + 1], step) == wrap;
    if (r1) x1 = atomicAdd(&acc[w.k0 + 2], step) == wrap;
    if (r2) x2 = atomicAdd(&acc[w.k0 + 3], step) == wrap;
    if (x0) words_ripple(acc, w.k0 + 2, step, wrap);
    if (x1) words_ripple(acc, w.k0 + 3, step, wrap);
    if (x2) words_ripple(acc, w.k0 + 4, step, wrap);
}

// five signed limbs (weights 2^0, 2^32, .., 2^128) -> 192-bit two's complement
__device__ __forceinline__ Fix3 fix_from_limbs(const unsigned long long* l) {
    Fix3 r{0, 0, 0};
#pragma unroll
    for (int k = 0; k < kWords; ++k) {
        const uint64_t u = l[k];
        const uint64_t e = static_cast<int64_t>(u) < 0 ? ~0ull : 0ull;  // sign extension
        Fix3 t;
        switch (k) {
        case 0: t = Fix3{u, e, e}; break;
        case 1: t = Fix3{u << 32, (u >> 32) | (e << 32), e}; break;
        case 2: t = Fix3{0, u, e}; break;
        case 3: t = Fix3{0, u << 32, (u >> 32) | (e << 32)}; break;
        default: t = Fix3{0, 0, u}; break;
        }
        fix_add(r, t);
    }
    return r;
}

// 160-bit two's complement (5 words) -> 192-bit.
__device__ __forceinline__ Fix3 fix_from_words(const uint32_t* w) {
    const uint64_t lo = w[0] | (static_cast<uint64_t>(w[1]) << 32);
    const uint64_t mid = w[2] | (static_cast<uint64_t>(w[3]) << 32);
    const int64_t top = static_cast<int32_t>(w[4]);
    return Fix3{lo, mid, static_cast<uint64_t>(top)};
}

// Per-warp queue of passing rows (ballot compaction): the atomic path then runs
// with all 32 lanes converged instead of once per 32-row slice with ~6 lanes.
constexpr int kQueue = 64;
// Entries carry the row, its price and qty; the key decode and the price*qty
// product happen when the queue is consumed, with all 32 lanes busy.
// B32: the entry's position is the row's 32-bit bit offset in the packed
// column, else the 64-bit row index.
template <bool B32>
struct WarpQueue {
    typename std::conditional<B32, uint32_t, uint64_t>::type pos[kQueue];
    double price[kQueue];
    int32_t qty[kQueue];
};

// MODE 0: rows merged per group within the warp (match + shuffles), packed
//         192-bit sum+count words updated with carrying 64-bit atomics;
// MODE 1: every row added by its own lane to a 160-bit accumulator of five
//         32-bit words (native 32-bit shared atomics, carries propagated),
//         a 32-bit count, and min/max keys; rows reach the lanes through the
//         warp queue (all 32 lanes busy);
// MODE 2: as MODE 1, rows added where they are read (no queue).
// MODE 3: MODE 1 with the block's next tile of price and qty loaded into
//         registers before the current tile is filtered and its queue
//         consumed, so each warp keeps a tile of loads in flight while it
//         aggregates (two blocks per SM: the second register set).
template <int RPT, int MODE, bool B32 = false>
__device__ __forceinline__ void scan_groupby_body(
    const uint64_t* __restrict__ packed, uint32_t width, const int32_t* __restrict__ dict, uint32_t card,
    const double* __restrict__ price, const int32_t* __restrict__ qty, uint64_t n, double pthr, int32_t qlo,
    int32_t qhi, GlobalGroups g, unsigned int* done, int32_t* out_keys, double* out_sum, double* out_min,
    double* out_max, uint64_t* out_count, uint64_t* out_ngroups, int* status) {
    constexpr int kTile = kGbThreads * RPT;
    constexpr bool WORDS = MODE != 0;
    extern __shared__ __align__(128) unsigned char smem[];
    // MODE 0: 3 words per group (packed 192-bit sum + count), min, max.
    // MODE 1-3: min, max, then 5 32-bit words and a 32-bit count per group.
    unsigned long long* s_acc = reinterpret_cast<unsigned long long*>(smem);
    unsigned long long* s_mn = WORDS ? s_acc : s_acc + 3 * card;
    unsigned long long* s_mx = s_mn + card;
    uint32_t* s_w = reinterpret_cast<uint32_t*>(s_mx + card);  // MODE 1-3
    uint32_t* s_cnt = s_w + kWords * card;                      // MODE 1-3

    auto reset_table = [&]() {
        for (uint32_t i = threadIdx.x; i < card; i += blockDim.x) {
            if (WORDS) {
#pragma unroll
                for (int k = 0; k < kWords; ++k) s_w[kWords * i + k] = 0;
                s_cnt[i] = 0;
            } else {
                s_acc[3 * i] = 0;
                s_acc[3 * i + 1] = 0;
                s_acc[3 * i + 2] = 0;
            }
            s_mn[i] = ~0ull;
            s_mx[i] = 0;
        }
    };
    auto flush_table = [&]() {
        for (uint32_t i = threadIdx.x; i < card; i += blockDim.x) {
            unsigned int c;
            Fix3 f;
            if (WORDS) {
                c = s_cnt[i];
                if (!c) continue;
                f = fix_from_words(s_w + kWords * i);
            } else {
                Fix3 x{s_acc[3 * i], s_acc[3 * i + 1], s_acc[3 * i + 2]};
                f = unpack_sum(x, &c);
                if (!c) continue;
            }
            fix_atomic_add(&g.sum[3 * i], f);
            atomicAdd(&g.cnt[i], static_cast<unsigned long long>(c));
            atomicMin(&g.mn[i], s_mn[i]);
            atomicMax(&g.mx[i], s_mx[i]);
        }
    };

    reset_table();
    __syncthreads();
    const uint64_t mask = (width >= 64) ? ~0ull : ((1ull << width) - 1);
    const uint64_t ntiles = (n + kTile - 1) / kTile;
    // rows between flushes: MODE 0 embeds counts in 20 bits; MODES 1-3 sum
    // rows below 2^139 in 160 bits (and count in 32)
    const uint64_t tiles_per_flush = WORDS ? (1ull << 19) / kTile : ((1ull << kCountBits) - 1) / kTile;
    bool bad_value = false, bad_key = false;
    uint64_t since_flush = 0;

    __shared__ WarpQueue<B32> s_queue[kGbThreads / 32];
    const int lane = threadIdx.x & 31;
    const unsigned lanemask_lt = (1u << lane) - 1;
    WarpQueue<B32>& Q = s_queue[threadIdx.x >> 5];
    const uint32_t* const p32 = reinterpret_cast<const uint32_t*>(packed);
    const uint32_t nw32 = B32 ? static_cast<uint32_t>((n * width + 63) / 64 * 2) : 0u;
    const uint32_t mask32 = static_cast<uint32_t>(mask);
    int qn = 0;  // warp-uniform fill of Q (a ring of kQueue entries from qh)
    int qh = 0;
    // qty in [qlo, qhi] as one unsigned compare; an empty range passes nothing
    // (p > +inf never holds), and rows past n read NaN prices (never pass)
    const uint32_t qspan = qlo <= qhi ? static_cast<uint32_t>(qhi) - static_cast<uint32_t>(qlo) : 0u;
    const double pcut = qlo <= qhi ? pthr : __longlong_as_double(0x7FF0000000000000ll);
    // lanes < cnt fold queue entry `lane` into the block table, converged.
    // Entries of the same group are first combined by the lowest such lane
    // (match + shuffles), so a hot group costs one set of atomics per round
    // instead of one per row, and no two lanes of an atomic hit one address.
    // MODE 1, 2: a row is added by its own lane; same-address lanes are handled
    // by the shared-memory atomic unit (32-bit atomics stay fast under conflicts)
    auto add_row = [&](uint32_t gi, double v, double p, bool mayneg) {
        if (gi >= card) {
            bad_key = true;
            return;
        }
        RowWords w;
        if (!row_words(v, &w)) bad_value = true;
        else if (mayneg) words_add<true>(s_w + kWords * gi, w, v < 0.0);
        else words_add<false>(s_w + kWords * gi, w, false);
        atomicAdd(&s_cnt[gi], 1u);
        const uint64_t k = f64_order_key(p);
        if (k < s_mn[gi]) atomicMin(&s_mn[gi], static_cast<unsigned long long>(k));
        if (k > s_mx[gi]) atomicMax(&s_mx[gi], static_cast<unsigned long long>(k));
    };
    auto consume = [&](int cnt) {
        bool valid = lane < cnt;
        uint32_t gi = 0;
        double p = 0.0, v = 0.0;
        if (valid) {
            const int e = (qh + lane) & (kQueue - 1);
            p = Q.price[e];
            if constexpr (B32) gi = key_bits32(p32, Q.pos[e], nw32, mask32);
            else gi = key_bits(packed, Q.pos[e], width, mask);
            // one rounded multiply, as the reference materialises price*qty
            v = __dmul_rn(p, static_cast<double>(Q.qty[e]));
        }
        if (WORDS) {
            // one warp-uniform test picks the add-only path for the whole warp
            const bool mayneg = __any_sync(0xffffffffu, valid && v < 0.0);
            if (valid) add_row(gi, v, p, mayneg);
            return;
        }
        if (valid && gi >= card) {
            bad_key = true;
            valid = false;
        }
        Fix3 f{0, 0, 0};
        if (valid) f = pack_row(fix_from_double_s<kFixScale>(v, &bad_value));
        uint32_t key = valid ? gi : (0x80000000u | static_cast<uint32_t>(lane));
        unsigned peers = __match_any_sync(0xffffffffu, key);
        bool leader = valid && (__ffs(peers) - 1 == lane);
        double pmin = p, pmax = p;
        Fix3 acc = f;
        if (__any_sync(0xffffffffu, valid && __popc(peers) > 1)) {
            unsigned rest = leader ? (peers & ~(1u << lane)) : 0u;
            while (__any_sync(0xffffffffu, rest != 0)) {
                int src = rest ? __ffs(rest) - 1 : lane;
                Fix3 o;
                o.w0 = __shfl_sync(0xffffffffu, f.w0, src);
                o.w1 = __shfl_sync(0xffffffffu, f.w1, src);
                o.w2 = __shfl_sync(0xffffffffu, f.w2, src);
                double op = __shfl_sync(0xffffffffu, p, src);
                if (rest) {
                    fix_add(acc, o);
                    pmin = op < pmin ? op : pmin;
                    pmax = op > pmax ? op : pmax;
                    rest &= rest - 1;
                }
            }
        }
        if (leader) {
            fix_atomic_add(&s_acc[3 * gi], acc);
            uint64_t kmin = f64_order_key(pmin), kmax = f64_order_key(pmax);
            if (kmin < s_mn[gi]) atomicMin(&s_mn[gi], static_cast<unsigned long long>(kmin));
            if (kmax > s_mx[gi]) atomicMax(&s_mx[gi], static_cast<unsigned long long>(kmax));
        }
    };

    constexpr bool PF = MODE == 3;
    auto load_tile = [&](uint64_t tt, double (&lp)[RPT], int32_t (&lq)[RPT]) {
        const uint64_t l0 = tt * kTile + static_cast<uint64_t>(threadIdx.x) * RPT;
        if (l0 + RPT <= n) {
#pragma unroll
            for (int k = 0; k < RPT; k += 4) {
                const double2* pp = reinterpret_cast<const double2*>(price + l0 + k);
                double2 a = __ldcs(pp), b = __ldcs(pp + 1);
                int4 q = __ldcs(reinterpret_cast<const int4*>(qty + l0 + k));
                lp[k] = a.x; lp[k + 1] = a.y; lp[k + 2] = b.x; lp[k + 3] = b.y;
                lq[k] = q.x; lq[k + 1] = q.y; lq[k + 2] = q.z; lq[k + 3] = q.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                bool in = l0 + k < n;
                lp[k] = in ? price[l0 + k] : __longlong_as_double(0x7FF8000000000000ll);
                lq[k] = in ? qty[l0 + k] : 0;
            }
        }
    };
    double nextp[RPT];  // PF: the block's next tile, in flight while this one is processed
    int32_t nextq[RPT];
    if (PF && blockIdx.x < ntiles) load_tile(blockIdx.x, nextp, nextq);
    for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        if (since_flush == tiles_per_flush) {
            __syncwarp();
            consume(qn);
            qn = 0;
            __syncthreads();
            flush_table();
            __syncthreads();
            reset_table();
            __syncthreads();
            since_flush = 0;
        }
        ++since_flush;
        const uint64_t r0 = t * kTile + static_cast<uint64_t>(threadIdx.x) * RPT;
        double pv[RPT];
        int32_t qv[RPT];
        if (PF) {
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                pv[k] = nextp[k];
                qv[k] = nextq[k];
            }
            if (t + gridDim.x < ntiles) load_tile(t + gridDim.x, nextp, nextq);
        } else {
            load_tile(t, pv, qv);
        }
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            const uint64_t r = r0 + k;
            const double p = pv[k];
            const int32_t q = qv[k];
            const bool pass = p > pcut && static_cast<uint32_t>(q) - static_cast<uint32_t>(qlo) <= qspan;
            if (MODE == 2) {  // no queue: passing lanes add their rows directly
                if (pass) add_row(key_bits(packed, r, width, mask), __dmul_rn(p, static_cast<double>(q)), p, true);
                continue;
            }
            unsigned m = __ballot_sync(0xffffffffu, pass);
            if (pass) {
                const int pos = (qh + qn + __popc(m & lanemask_lt)) & (kQueue - 1);
                if constexpr (B32) Q.pos[pos] = static_cast<uint32_t>(r) * width;  // < 2^32 by the launch check
                else Q.pos[pos] = r;
                Q.price[pos] = p;
                Q.qty[pos] = q;
            }
            qn += __popc(m);
            if (qn >= 32) {
                __syncwarp();
                consume(32);
                __syncwarp();  // the consumed entries are free for the next pushes
                qh = (qh + 32) & (kQueue - 1);
                qn -= 32;
            }
        }
    }
    __syncwarp();
    consume(qn);
    if (bad_value) atomicOr(status, 1);
    if (bad_key) atomicOr(status, 2);
    __syncthreads();
    flush_table();
    __threadfence();
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();

    // last block: compact non-empty groups in key (= dictionary index) order;
    // the scan scratch reuses the warp queues, idle since the last consume
    static_assert(sizeof(s_queue) >= kGbThreads * sizeof(unsigned int), "scan scratch");
    unsigned int* const s_scan = reinterpret_cast<unsigned int*>(s_queue);
    uint32_t per = (card + blockDim.x - 1) / blockDim.x;
    uint32_t lo = threadIdx.x * per < card ? threadIdx.x * per : card;
    uint32_t hi = lo + per < card ? lo + per : card;
    unsigned int mine = 0;
    for (uint32_t i = lo; i < hi; ++i) mine += __ldcg(&g.cnt[i]) ? 1 : 0;
    s_scan[threadIdx.x] = mine;
    __syncthreads();
    for (int d = 1; d < kGbThreads; d <<= 1) {
        unsigned int v = threadIdx.x >= static_cast<unsigned>(d) ? s_scan[threadIdx.x - d] : 0;
        __syncthreads();
        s_scan[threadIdx.x] += v;
        __syncthreads();
    }
    unsigned int pos = s_scan[threadIdx.x] - mine;
    for (uint32_t i = lo; i < hi; ++i) {
        unsigned long long c = __ldcg(&g.cnt[i]);
        if (c) {
            Fix3 f{__ldcg(&g.sum[3 * i]), __ldcg(&g.sum[3 * i + 1]), __ldcg(&g.sum[3 * i + 2])};
            out_keys[pos] = dict[i];
            out_sum[pos] = fix_to_double_s<kFixScale>(f);
            out_min[pos] = f64_from_order_key(__ldcg(&g.mn[i]));
            out_max[pos] = f64_from_order_key(__ldcg(&g.mx[i]));
            out_count[pos] = c;
            ++pos;
        }
        g.sum[3 * i] = 0;
        g.sum[3 * i + 1] = 0;
        g.sum[3 * i + 2] = 0;
        g.cnt[i] = 0;
        g.mn[i] = ~0ull;
        g.mx[i] = 0;
    }
    if (threadIdx.x == blockDim.x - 1) {
        *out_ngroups = s_scan[threadIdx.x];
        *done = 0;
    }
}

#define VX_GB_PARAMS                                                                                             \
    const uint64_t *__restrict__ packed, uint32_t width, const int32_t *__restrict__ dict, uint32_t card,         \
        const double *__restrict__ price, const int32_t *__restrict__ qty, uint64_t n, double pthr, int32_t qlo,  \
        int32_t qhi, GlobalGroups g, unsigned int *done, int32_t *out_keys, double *out_sum, double *out_min,     \
        double *out_max, uint64_t *out_count, uint64_t *out_ngroups, int *status
#define VX_GB_ARGS \
    packed, width, dict, card, price, qty, n, pthr, qlo, qhi, g, done, out_keys, out_sum, out_min, out_max, \
        out_count, out_ngroups, status

template <int RPT, int MODE, bool B32 = false>
__global__ void __launch_bounds__(kGbThreads) scan_groupby_kernel(VX_GB_PARAMS) {
    scan_groupby_body<RPT, MODE, B32>(VX_GB_ARGS);
}

// MODE 3 holds a second tile in registers: sized for two blocks per SM
template <int RPT, bool B32 = false>
__global__ void __launch_bounds__(kGbThreads, 2) scan_groupby_pf_kernel(VX_GB_PARAMS) {
    scan_groupby_body<RPT, 3, B32>(VX_GB_ARGS);
}
#undef VX_GB_PARAMS
#undef VX_GB_ARGS

// ---------------------------------------------------------------------------
// TMA-fed variant for dictionaries up to kTmaMaxCard entries.
//
// A producer warp streams 2048-row tiles of price / qty / packed keys into a
// 3-stage shared-memory ring with bulk async copies (cp.async.bulk, counted on
// mbarriers).  Each of 8 consumer warps owns a private per-group table
// (compensated FP64 sum with an f32 error term, u32 count) and updates it
// without atomics: passing rows are compacted into a per-warp queue with a
// ballot, rows of the same group inside a 32-row round are folded by the
// leader lane (__match_any_sync + shuffles), and leaders have distinct groups,
// so plain read-modify-writes suffice.  MIN/MAX live in one block table and
// change rarely (conditional atomics).  At the end the warp tables are merged
// in warp order and added exactly (192-bit fixed point) to the global table.
// ---------------------------------------------------------------------------
constexpr int kTmaConsumers = 8;
constexpr int kTmaThreads = (kTmaConsumers + 1) * 32;
constexpr int kTmaRows = 2048;
constexpr int kTmaStages = 3;
constexpr uint32_t kTmaMaxCard = 1024;
constexpr long long kTmaWaitBudget = 1ll << 32;  // clock cycles

__device__ __forceinline__ size_t tma_stage_bytes(uint32_t width) { return 24576u + 256u * width; }

// Folds one row per lane (valid lanes) into the warp's private table.
__device__ __forceinline__ void warp_table_update(uint32_t gid, double v, double p, bool valid, uint32_t card,
                                                  double* ts, float* tc, uint32_t* tn, unsigned long long* s_mn,
                                                  unsigned long long* s_mx, bool* bad_key) {
    const int lane = threadIdx.x & 31;
    if (valid && gid >= card) {
        *bad_key = true;
        valid = false;
    }
    uint32_t key = valid ? gid : (0x80000000u | static_cast<uint32_t>(lane));
    unsigned peers = __match_any_sync(0xffffffffu, key);
    bool leader = valid && (__ffs(peers) - 1 == lane);
    double vs = v, pmin = p, pmax = p;
    uint32_t cn = 1;
    if (__any_sync(0xffffffffu, valid && __popc(peers) > 1)) {
        unsigned rest = leader ? (peers & ~(1u << lane)) : 0u;
        while (__any_sync(0xffffffffu, rest != 0)) {
            int src = rest ? __ffs(rest) - 1 : lane;
            double ov = __shfl_sync(0xffffffffu, v, src);
            double op = __shfl_sync(0xffffffffu, p, src);
            if (rest) {
                vs = __dadd_rn(vs, ov);
                ++cn;
                pmin = op < pmin ? op : pmin;
                pmax = op > pmax ? op : pmax;
                rest &= rest - 1;
            }
        }
    }
    if (leader) {
        double s0 = ts[gid];
        double t = __dadd_rn(s0, vs);
        double e = fabs(s0) >= fabs(vs) ? __dadd_rn(__dsub_rn(s0, t), vs) : __dadd_rn(__dsub_rn(vs, t), s0);
        ts[gid] = t;
        tc[gid] = __fadd_rn(tc[gid], static_cast<float>(e));
        tn[gid] += cn;
        uint64_t kmin = f64_order_key(pmin), kmax = f64_order_key(pmax);
        if (kmin < s_mn[gid]) atomicMin(&s_mn[gid], static_cast<unsigned long long>(kmin));
        if (kmax > s_mx[gid]) atomicMax(&s_mx[gid], static_cast<unsigned long long>(kmax));
    }
}

// Last block: compact the global table's non-empty groups in key order and
// reset it.  All threads of the block call.
template <int THREADS>
__device__ void finalize_groups(const GlobalGroups& g, const int32_t* dict, uint32_t card, unsigned int* done,
                                int32_t* out_keys, double* out_sum, double* out_min, double* out_max,
                                uint64_t* out_count, uint64_t* out_ngroups) {
    __shared__ unsigned int s_scan[THREADS];
    uint32_t per = (card + THREADS - 1) / THREADS;
    uint32_t lo = threadIdx.x * per < card ? threadIdx.x * per : card;
    uint32_t hi = lo + per < card ? lo + per : card;
    unsigned int mine = 0;
    for (uint32_t i = lo; i < hi; ++i) mine += __ldcg(&g.cnt[i]) ? 1 : 0;
    s_scan[threadIdx.x] = mine;
    __syncthreads();
    for (int d = 1; d < THREADS; d <<= 1) {
        unsigned int v = threadIdx.x >= static_cast<unsigned>(d) ? s_scan[threadIdx.x - d] : 0;
        __syncthreads();
        s_scan[threadIdx.x] += v;
        __syncthreads();
    }
    unsigned int pos = s_scan[threadIdx.x] - mine;
    for (uint32_t i = lo; i < hi; ++i) {
        unsigned long long c = __ldcg(&g.cnt[i]);
        if (c) {
            Fix3 f{__ldcg(&g.sum[3 * i]), __ldcg(&g.sum[3 * i + 1]), __ldcg(&g.sum[3 * i + 2])};
            out_keys[pos] = dict[i];
            out_sum[pos] = fix_to_double_s<kFixScale>(f);
            out_min[pos] = f64_from_order_key(__ldcg(&g.mn[i]));
            out_max[pos] = f64_from_order_key(__ldcg(&g.mx[i]));
            out_count[pos] = c;
            ++pos;
        }
        g.sum[3 * i] = 0;
        g.sum[3 * i + 1] = 0;
        g.sum[3 * i + 2] = 0;
        g.cnt[i] = 0;
        g.mn[i] = ~0ull;
        g.mx[i] = 0;
    }
    if (threadIdx.x == THREADS - 1) {
        *out_ngroups = s_scan[threadIdx.x];
        *done = 0;
    }
}

__global__ void __launch_bounds__(kTmaThreads, 1) scan_groupby_tma_kernel(
    const uint64_t* __restrict__ packed, uint32_t width, const int32_t* __restrict__ dict, uint32_t card,
    const double* __restrict__ price, const int32_t* __restrict__ qty, uint64_t n, double pthr, int32_t qlo,
    int32_t qhi, GlobalGroups g, unsigned int* done, int32_t* out_keys, double* out_sum, double* out_min,
    double* out_max, uint64_t* out_count, uint64_t* out_ngroups, int* status) {
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t stage_bytes = static_cast<uint32_t>(tma_stage_bytes(width));
    unsigned char* stages = smem;
    double* t_s = reinterpret_cast<double*>(smem + kTmaStages * stage_bytes);
    float* t_c = reinterpret_cast<float*>(t_s + kTmaConsumers * card);
    uint32_t* t_n = reinterpret_cast<uint32_t*>(t_c + kTmaConsumers * card);
    unsigned long long* s_mn = reinterpret_cast<unsigned long long*>(
        (reinterpret_cast<uintptr_t>(t_n + kTmaConsumers * card) + 7) & ~static_cast<uintptr_t>(7));
    unsigned long long* s_mx = s_mn + card;
    uint16_t* queues = reinterpret_cast<uint16_t*>(s_mx + card);
    uint64_t* full = reinterpret_cast<uint64_t*>(
        (reinterpret_cast<uintptr_t>(queues + kTmaConsumers * 64) + 7) & ~static_cast<uintptr_t>(7));
    uint64_t* empty = full + kTmaStages;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (uint32_t i = threadIdx.x; i < kTmaConsumers * card; i += blockDim.x) {
        t_s[i] = 0.0;
        t_c[i] = 0.0f;
        t_n[i] = 0;
    }
    for (uint32_t i = threadIdx.x; i < card; i += blockDim.x) {
        s_mn[i] = ~0ull;
        s_mx[i] = 0;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kTmaStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kTmaConsumers);
        }
        mbar_fence_init();
    }
    __syncthreads();

    const uint64_t nfull = n / kTmaRows;
    const uint64_t mytiles = nfull > blockIdx.x ? (nfull - blockIdx.x - 1) / gridDim.x + 1 : 0;
    const uint64_t mask = (1ull << width) - 1;
    bool bad_value = false, bad_key = false, timeout = false;

    if (warp == kTmaConsumers) {
        // producer: one lane issues the bulk copies, a stage ahead of the consumers
        if (lane == 0) {
            uint64_t issued = 0;
            for (uint64_t k = 0; k < mytiles; ++k) {
                const int s = static_cast<int>(k % kTmaStages);
                const uint64_t r = k / kTmaStages;
                if (r > 0 && !mbar_wait(&empty[s], static_cast<uint32_t>((r - 1) & 1), kTmaWaitBudget)) {
                    timeout = true;
                    break;
                }
                const uint64_t base = (blockIdx.x + k * gridDim.x) * kTmaRows;
                unsigned char* st = stages + static_cast<size_t>(s) * stage_bytes;
                mbar_arrive_expect_tx(&full[s], stage_bytes);
                bulk_g2s(st, price + base, kTmaRows * 8, &full[s]);
                bulk_g2s(st + kTmaRows * 8, qty + base, kTmaRows * 4, &full[s]);
                bulk_g2s(st + kTmaRows * 12, packed + base * width / 64, 256u * width, &full[s]);
                ++issued;
            }
            // never leave the block with copies still landing in its shared memory
            uint64_t from = issued > kTmaStages ? issued - kTmaStages : 0;
            for (uint64_t k = from; k < issued; ++k)
                if (!mbar_wait(&full[k % kTmaStages], static_cast<uint32_t>((k / kTmaStages) & 1), kTmaWaitBudget))
                    timeout = true;
        }
    } else {
        double* ts = t_s + warp * card;
        float* tc = t_c + warp * card;
        uint32_t* tn = t_n + warp * card;
        uint16_t* q = queues + warp * 64;
        const unsigned lanemask_lt = (1u << lane) - 1;
        for (uint64_t k = 0; k < mytiles; ++k) {
            const int s = static_cast<int>(k % kTmaStages);
            // every lane observes the phase (visibility of the copied bytes); the
            // warp then agrees, so the warp-wide intrinsics below stay converged
            bool ok = mbar_wait(&full[s], static_cast<uint32_t>((k / kTmaStages) & 1), kTmaWaitBudget);
            if (!__all_sync(0xffffffffu, ok)) {
                timeout = true;
                break;
            }
            const unsigned char* st = stages + static_cast<size_t>(s) * stage_bytes;
            const double* sp = reinterpret_cast<const double*>(st);
            const int32_t* sq = reinterpret_cast<const int32_t*>(st + kTmaRows * 8);
            const uint64_t* sk = reinterpret_cast<const uint64_t*>(st + kTmaRows * 12);
            int qn = 0;
            auto round = [&](int cnt) {
                bool valid = lane < cnt;
                uint32_t gid = 0;
                double v = 0.0, p = 0.0;
                if (valid) {
                    uint32_t j = q[lane];
                    p = sp[j];
                    v = __dmul_rn(p, static_cast<double>(sq[j]));  // one rounded multiply
                    uint32_t bit = j * width, wi = bit >> 6, sh = bit & 63;
                    uint64_t x = sk[wi] >> sh;
                    if (sh + width > 64) x |= sk[wi + 1] << (64 - sh);
                    gid = static_cast<uint32_t>(x & mask);
                }
                warp_table_update(gid, v, p, valid, card, ts, tc, tn, s_mn, s_mx, &bad_key);
            };
            const uint32_t r0 = static_cast<uint32_t>(warp) * (kTmaRows / kTmaConsumers);
#pragma unroll 2
            for (uint32_t sl = 0; sl < kTmaRows / kTmaConsumers; sl += 32) {
                uint32_t j = r0 + sl + lane;
                double p = sp[j];
                int32_t qq = sq[j];
                bool pass = p > pthr && qq >= qlo && qq <= qhi;
                unsigned m = __ballot_sync(0xffffffffu, pass);
                if (pass) q[qn + __popc(m & lanemask_lt)] = static_cast<uint16_t>(j);
                qn += __popc(m);
                if (qn >= 32) {
                    __syncwarp();
                    round(32);
                    __syncwarp();
                    if (lane < qn - 32) q[lane] = q[32 + lane];
                    __syncwarp();
                    qn -= 32;
                }
            }
            __syncwarp();
            round(qn);  // the queue refers to this stage: drain before releasing it
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
        }
        // the partial tail tile: block 0's consumer warps, plain loads
        if (blockIdx.x == 0 && !timeout) {
            const uint64_t tb = nfull * kTmaRows;
            for (uint64_t r = tb + static_cast<uint64_t>(warp) * 32 + lane; r - lane < n;
                 r += kTmaConsumers * 32) {
                bool in = r < n;
                double p = in ? price[r] : 0.0;
                int32_t qq = in ? qty[r] : 0;
                bool pass = in && p > pthr && qq >= qlo && qq <= qhi;
                uint32_t gid = pass ? key_bits(packed, r, width, mask) : 0;
                warp_table_update(gid, __dmul_rn(p, static_cast<double>(qq)), p, pass, card, ts, tc, tn, s_mn, s_mx,
                                  &bad_key);
            }
        }
    }
    if (timeout) atomicOr(status, 4);
    if (bad_key) atomicOr(status, 2);
    __syncthreads();
    // merge the warp tables (warp order) and add them exactly to the global table
    for (uint32_t i = threadIdx.x; i < card; i += blockDim.x) {
        KSum k{0.0, 0.0};
        unsigned long long c = 0;
        double ec = 0.0;
        for (int w = 0; w < kTmaConsumers; ++w) {
            ksum_add(k, t_s[w * card + i]);
            ec += static_cast<double>(t_c[w * card + i]);
            c += t_n[w * card + i];
        }
        if (!c) continue;
        Fix3 f = fix_from_double_s<kFixScale>(k.s, &bad_value);
        fix_add(f, fix_from_double_s<kFixScale>(__dadd_rn(k.c, ec), &bad_value));
        fix_atomic_add(&g.sum[3 * i], f);
        atomicAdd(&g.cnt[i], c);
        atomicMin(&g.mn[i], s_mn[i]);
        atomicMax(&g.mx[i], s_mx[i]);
    }
    if (bad_value) atomicOr(status, 1);
    __threadfence();
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    finalize_groups<kTmaThreads>(g, dict, card, done, out_keys, out_sum, out_min, out_max, out_count, out_ngroups);
}

// ---------------------------------------------------------------------------
// Bulk-copy-fed word table (variant 6).  The queue-fed word table above
// streams its columns with the same warps that do the shared atomics, so the
// stream stalls while they aggregate: time = filter pass + aggregation.  Here a
// producer warp keeps up to kTwStages 2048-row stages of price / qty / packed
// keys in flight with cp.async.bulk (mbarrier-counted), and 16 consumer warps
// filter each stage out of shared memory, decode the passing rows' keys there,
// and push (price, qty, group) into their ring queues; a stage is released as
// soon as it is filtered (the queue holds copies), so copies keep landing
// while the consumers aggregate.  Aggregation is the word table's (same
// integers, identical bits).  One block per SM; each block sums at most 2^19
// rows (the word table's bound), which the host checks.  On the 2^25-row,
// 1000-group workload it measured slower than the queue-fed variant (0.197
// vs 0.125 ms; 0.099 vs 0.076 ms with no row passing): 16 aggregating warps
// hide less atomic latency than 48, and the stage hand-off costs stream
// bandwidth, so the autotuner does not time it; it stays selectable.
// ---------------------------------------------------------------------------
constexpr int kTwConsumers = 16;
constexpr int kTwThreads = (kTwConsumers + 1) * 32;
constexpr int kTwRows = 2048;
constexpr int kTwMaxStages = 4;
constexpr int kTwRowsPerWarp = kTwRows / kTwConsumers;  // 128: four 32-row slices

__host__ __device__ constexpr size_t tw_stage_bytes(uint32_t width) { return 12u * kTwRows + 256u * width; }

struct TwQueue {
    double price[kQueue];
    int32_t qty[kQueue];
    uint32_t gid[kQueue];
};

__host__ __device__ constexpr size_t tw_smem_bytes(uint32_t card, uint32_t width, int stages) {
    return static_cast<size_t>(stages) * tw_stage_bytes(width) + static_cast<size_t>(card) * 16 +
           static_cast<size_t>(card) * (kWords + 1) * 4 + 16 + kTwConsumers * sizeof(TwQueue) +
           2 * kTwMaxStages * 8;
}

__global__ void __launch_bounds__(kTwThreads, 1) scan_groupby_tw_kernel(
    const uint64_t* __restrict__ packed, uint32_t width, const int32_t* __restrict__ dict, uint32_t card,
    const double* __restrict__ price, const int32_t* __restrict__ qty, uint64_t n, double pthr, int32_t qlo,
    int32_t qhi, int nstages, GlobalGroups g, unsigned int* done, int32_t* out_keys, double* out_sum,
    double* out_min, double* out_max, uint64_t* out_count, uint64_t* out_ngroups, int* status) {
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t stage_bytes = static_cast<uint32_t>(tw_stage_bytes(width));
    unsigned char* stages = smem;
    unsigned long long* s_mn = reinterpret_cast<unsigned long long*>(smem + static_cast<size_t>(nstages) * stage_bytes);
    unsigned long long* s_mx = s_mn + card;
    uint32_t* s_w = reinterpret_cast<uint32_t*>(s_mx + card);
    uint32_t* s_cnt = s_w + kWords * card;
    TwQueue* queues = reinterpret_cast<TwQueue*>(
        (reinterpret_cast<uintptr_t>(s_cnt + card) + 15) & ~static_cast<uintptr_t>(15));
    uint64_t* full = reinterpret_cast<uint64_t*>(queues + kTwConsumers);
    uint64_t* empty = full + kTwMaxStages;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (uint32_t i = threadIdx.x; i < card; i += blockDim.x) {
#pragma unroll
        for (int k = 0; k < kWords; ++k) s_w[kWords * i + k] = 0;
        s_cnt[i] = 0;
        s_mn[i] = ~0ull;
        s_mx[i] = 0;
    }
    if (threadIdx.x == 0) {
        for (int st = 0; st < nstages; ++st) {
            mbar_init(&full[st], 1);
            mbar_init(&empty[st], kTwConsumers);
        }
        mbar_fence_init();
    }
    __syncthreads();

    const uint64_t nfull = n / kTwRows;
    const uint64_t mytiles = nfull > blockIdx.x ? (nfull - blockIdx.x - 1) / gridDim.x + 1 : 0;
    const uint64_t mask = (1ull << width) - 1;
    bool bad_value = false, bad_key = false, timeout = false;

    if (warp == kTwConsumers) {
        // producer: one lane issues the bulk copies, up to nstages ahead
        if (lane == 0) {
            uint64_t issued = 0;
            for (uint64_t k = 0; k < mytiles; ++k) {
                const int st = static_cast<int>(k % static_cast<uint64_t>(nstages));
                const uint64_t r = k / static_cast<uint64_t>(nstages);
                if (r > 0 && !mbar_wait(&empty[st], static_cast<uint32_t>((r - 1) & 1), kTmaWaitBudget)) {
                    timeout = true;
                    break;
                }
                const uint64_t base = (blockIdx.x + k * gridDim.x) * kTwRows;
                unsigned char* sb = stages + static_cast<size_t>(st) * stage_bytes;
                mbar_arrive_expect_tx(&full[st], stage_bytes);
                bulk_g2s(sb, price + base, kTwRows * 8, &full[st]);
                bulk_g2s(sb + kTwRows * 8, qty + base, kTwRows * 4, &full[st]);
                bulk_g2s(sb + kTwRows * 12, packed + base * width / 64, 256u * width, &full[st]);
                ++issued;
            }
            // never leave the block with copies still landing in its shared memory
            const uint64_t ns = static_cast<uint64_t>(nstages);
            for (uint64_t k = issued > ns ? issued - ns : 0; k < issued; ++k)
                if (!mbar_wait(&full[k % ns], static_cast<uint32_t>((k / ns) & 1), kTmaWaitBudget)) timeout = true;
        }
    } else {
        TwQueue& Q = queues[warp];
        const unsigned lanemask_lt = (1u << lane) - 1;
        const uint32_t qspan = qlo <= qhi ? static_cast<uint32_t>(qhi) - static_cast<uint32_t>(qlo) : 0u;
        const double pcut = qlo <= qhi ? pthr : __longlong_as_double(0x7FF0000000000000ll);
        int qn = 0, qh = 0;
        auto consume = [&](int cnt) {
            if (lane >= cnt) return;
            const int e = (qh + lane) & (kQueue - 1);
            const double p = Q.price[e];
            const uint32_t gi = Q.gid[e];
            const double v = __dmul_rn(p, static_cast<double>(Q.qty[e]));  // one rounded multiply
            if (gi >= card) {
                bad_key = true;
                return;
            }
            RowWords w;
            if (row_words(v, &w)) words_add(s_w + kWords * gi, w, v < 0.0);
            else bad_value = true;
            atomicAdd(&s_cnt[gi], 1u);
            const uint64_t k = f64_order_key(p);
            if (k < s_mn[gi]) atomicMin(&s_mn[gi], static_cast<unsigned long long>(k));
            if (k > s_mx[gi]) atomicMax(&s_mx[gi], static_cast<unsigned long long>(k));
        };
        auto push = [&](bool pass, double p, int32_t q, uint32_t gi) {
            const unsigned m = __ballot_sync(0xffffffffu, pass);
            if (pass) {
                const int pos = (qh + qn + __popc(m & lanemask_lt)) & (kQueue - 1);
                Q.price[pos] = p;
                Q.qty[pos] = q;
                Q.gid[pos] = gi;
            }
            qn += __popc(m);
            if (qn >= 32) {
                __syncwarp();
                consume(32);
                __syncwarp();  // the consumed entries are free for the next pushes
                qh = (qh + 32) & (kQueue - 1);
                qn -= 32;
            }
        };
        for (uint64_t k = 0; k < mytiles; ++k) {
            const int st = static_cast<int>(k % static_cast<uint64_t>(nstages));
            // every lane observes the phase (visibility of the copied bytes); the
            // warp then agrees, so the warp-wide intrinsics below stay converged
            const bool ok = mbar_wait(&full[st], static_cast<uint32_t>((k / static_cast<uint64_t>(nstages)) & 1),
                                      kTmaWaitBudget);
            if (!__all_sync(0xffffffffu, ok)) {
                timeout = true;
                break;
            }
            const unsigned char* sb = stages + static_cast<size_t>(st) * stage_bytes;
            const double* sp = reinterpret_cast<const double*>(sb);
            const int32_t* sq = reinterpret_cast<const int32_t*>(sb + kTwRows * 8);
            const uint64_t* sk = reinterpret_cast<const uint64_t*>(sb + kTwRows * 12);
            double pv[kTwRowsPerWarp / 32];
            int32_t qv[kTwRowsPerWarp / 32];
            uint32_t gv[kTwRowsPerWarp / 32];
            bool pa[kTwRowsPerWarp / 32];
#pragma unroll
            for (int sl = 0; sl < kTwRowsPerWarp / 32; ++sl) {
                const uint32_t j = static_cast<uint32_t>(warp) * kTwRowsPerWarp + sl * 32 + lane;
                pv[sl] = sp[j];
                qv[sl] = sq[j];
                pa[sl] = pv[sl] > pcut && static_cast<uint32_t>(qv[sl]) - static_cast<uint32_t>(qlo) <= qspan;
                gv[sl] = 0;
                if (pa[sl]) {
                    const uint32_t bit = j * width, wi = bit >> 6, sh = bit & 63;
                    uint64_t x = sk[wi] >> sh;
                    if (sh + width > 64) x |= sk[wi + 1] << (64 - sh);
                    gv[sl] = static_cast<uint32_t>(x & mask);
                }
            }
            // the warp's rows of this stage are in registers: release it
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[st]);
#pragma unroll
            for (int sl = 0; sl < kTwRowsPerWarp / 32; ++sl) push(pa[sl], pv[sl], qv[sl], gv[sl]);
        }
        // the partial tail stage: block 0's consumer warps, plain loads
        if (blockIdx.x == 0 && !__any_sync(0xffffffffu, timeout)) {
            for (uint64_t r0 = nfull * kTwRows + static_cast<uint64_t>(warp) * 32; r0 < n; r0 += kTwConsumers * 32) {
                const uint64_t r = r0 + lane;
                const bool in = r < n;
                const double p = in ? price[r] : 0.0;
                const int32_t q = in ? qty[r] : 0;
                const bool pass = in && p > pcut && static_cast<uint32_t>(q) - static_cast<uint32_t>(qlo) <= qspan;
                push(pass, p, q, pass ? key_bits(packed, r, width, mask) : 0u);
            }
        }
        __syncwarp();
        consume(qn);
    }
    if (timeout) atomicOr(status, 4);
    if (bad_key) atomicOr(status, 2);
    if (bad_value) atomicOr(status, 1);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < card; i += blockDim.x) {
        const unsigned int c = s_cnt[i];
        if (!c) continue;
        fix_atomic_add(&g.sum[3 * i], fix_from_words(s_w + kWords * i));
        atomicAdd(&g.cnt[i], static_cast<unsigned long long>(c));
        atomicMin(&g.mn[i], s_mn[i]);
        atomicMax(&g.mx[i], s_mx[i]);
    }
    __threadfence();
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    finalize_groups<kTwThreads>(g, dict, card, done, out_keys, out_sum, out_min, out_max, out_count, out_ngroups);
}

// ---------------------------------------------------------------------------
// Lean word table (variant 7): the queue-fed word table with less work per
// passing row.
//  - A queue entry is one 16-byte slot {u32 row, i32 qty, f64 price}: one
//    shared store to push it, one load to consume it.
//  - The ring holds 160 entries (31 left over + 4 x 32 pushed per tile), so a
//    tile's pushes come first and its consumes after them, from one place.
//  - MIN / MAX are screened with the high 32 bits of the group's order keys
//    (one 8-byte shared load and two compares); only a row that can move
//    them (a new extreme, or a tie in the high bits: rare) updates the 64-bit
//    keys, straight in the global table, and then the screen.
//  - SUM and COUNT are the word table's: the same integers, so every variant
//    gives identical bits.
// Rows are indexed with 32 bits: the host runs it for n < 2^32.
// ---------------------------------------------------------------------------
constexpr int kLeanQueue = 160;

struct __align__(16) LeanEntry {
    uint32_t row;
    int32_t qty;
    double price;
};

__host__ __device__ constexpr size_t lean_smem_bytes(uint32_t card) {
    return static_cast<size_t>(card) * (kWords * 4 + 4 + 8) + 16;
}

template <int RPT>
__global__ void __launch_bounds__(kGbThreads, 3) scan_groupby_lean_kernel(
    const uint64_t* __restrict__ packed, uint32_t width, const int32_t* __restrict__ dict, uint32_t card,
    const double* __restrict__ price, const int32_t* __restrict__ qty, uint32_t n, double pthr, int32_t qlo,
    int32_t qhi, GlobalGroups g, unsigned int* done, int32_t* out_keys, double* out_sum, double* out_min,
    double* out_max, uint64_t* out_count, uint64_t* out_ngroups, int* status) {
    constexpr uint32_t kTile = kGbThreads * RPT;
    extern __shared__ __align__(16) unsigned char smem[];
    uint2* s_mm = reinterpret_cast<uint2*>(smem);                      // {hi32(min key), hi32(max key)}
    uint32_t* s_w = reinterpret_cast<uint32_t*>(s_mm + card);          // 5 words per group
    uint32_t* s_cnt = s_w + kWords * card;
    __shared__ LeanEntry s_queue[kGbThreads / 32][kLeanQueue];

    for (uint32_t i = threadIdx.x; i < card; i += blockDim.x) {
#pragma unroll
        for (int k = 0; k < kWords; ++k) s_w[kWords * i + k] = 0;
        s_cnt[i] = 0;
        s_mm[i] = make_uint2(0xFFFFFFFFu, 0u);
    }
    __syncthreads();
    auto flush_table = [&]() {
        for (uint32_t i = threadIdx.x; i < card; i += blockDim.x) {
            const unsigned int c = s_cnt[i];
            if (!c) continue;
            fix_atomic_add(&g.sum[3 * i], fix_from_words(s_w + kWords * i));
            atomicAdd(&g.cnt[i], static_cast<unsigned long long>(c));
#pragma unroll
            for (int k = 0; k < kWords; ++k) s_w[kWords * i + k] = 0;
            s_cnt[i] = 0;
        }
    };

    const uint64_t mask = (width >= 64) ? ~0ull : ((1ull << width) - 1);
    const uint32_t ntiles = (n + kTile - 1) / kTile;
    const uint32_t tiles_per_flush = (1u << 19) / kTile;  // the word table sums below 2^139 per 2^19 rows
    bool bad_value = false, bad_key = false;
    uint32_t since_flush = 0;
    const int lane = threadIdx.x & 31;
    const unsigned lanemask_lt = (1u << lane) - 1;
    LeanEntry* Q = s_queue[threadIdx.x >> 5];
    int qn = 0, qh = 0;  // warp-uniform: entries [qh, qh + qn) of the ring
    const uint32_t qspan = qlo <= qhi ? static_cast<uint32_t>(qhi) - static_cast<uint32_t>(qlo) : 0u;
    const double pcut = qlo <= qhi ? pthr : __longlong_as_double(0x7FF0000000000000ll);

    auto consume = [&](int cnt) {
        const bool valid = lane < cnt;
        uint32_t gi = 0;
        double p = 0.0, v = 0.0;
        if (valid) {
            int e = qh + lane;
            if (e >= kLeanQueue) e -= kLeanQueue;
            const LeanEntry en = Q[e];
            p = en.price;
            gi = key_bits(packed, en.row, width, mask);
            v = __dmul_rn(p, static_cast<double>(en.qty));  // one rounded multiply, as the reference materialises it
        }
        const bool mayneg = __any_sync(0xffffffffu, valid && v < 0.0);
        if (!valid) return;
        if (gi >= card) {
            bad_key = true;
            return;
        }
        RowWords w;
        if (!row_words(v, &w)) bad_value = true;
        else if (mayneg) words_add<true>(s_w + kWords * gi, w, v < 0.0);
        else words_add<false>(s_w + kWords * gi, w, false);
        atomicAdd(&s_cnt[gi], 1u);
        const uint64_t key = f64_order_key(p);
        const uint32_t khi = static_cast<uint32_t>(key >> 32);
        const uint2 mm = s_mm[gi];
        if (khi <= mm.x) {
            atomicMin(&g.mn[gi], static_cast<unsigned long long>(key));
            atomicMin(&s_mm[gi].x, khi);
        }
        if (khi >= mm.y) {
            atomicMax(&g.mx[gi], static_cast<unsigned long long>(key));
            atomicMax(&s_mm[gi].y, khi);
        }
    };
    auto drain = [&]() {
        __syncwarp();
        while (qn >= 32) {
            consume(32);
            __syncwarp();  // the consumed entries are free for the next pushes
            qh += 32;
            if (qh >= kLeanQueue) qh -= kLeanQueue;
            qn -= 32;
        }
    };

    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        if (since_flush == tiles_per_flush) {
            __syncwarp();
            consume(qn);
            qn = 0;
            __syncthreads();
            flush_table();
            __syncthreads();
            since_flush = 0;
        }
        ++since_flush;
        const uint32_t r0 = t * kTile + threadIdx.x * RPT;
        double pv[RPT];
        int32_t qv[RPT];
        if (r0 + RPT <= n) {
#pragma unroll
            for (int k = 0; k < RPT; k += 4) {
                const double2* pp = reinterpret_cast<const double2*>(price + r0 + k);
                const double2 a = __ldcs(pp), b = __ldcs(pp + 1);
                const int4 q = __ldcs(reinterpret_cast<const int4*>(qty + r0 + k));
                pv[k] = a.x; pv[k + 1] = a.y; pv[k + 2] = b.x; pv[k + 3] = b.y;
                qv[k] = q.x; qv[k + 1] = q.y; qv[k + 2] = q.z; qv[k + 3] = q.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                const bool in = r0 + k < n;
                pv[k] = in ? price[r0 + k] : __longlong_as_double(0x7FF8000000000000ll);  // NaN never passes
                qv[k] = in ? qty[r0 + k] : 0;
            }
        }
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            const bool pass =
                pv[k] > pcut && static_cast<uint32_t>(qv[k]) - static_cast<uint32_t>(qlo) <= qspan;
            const unsigned m = __ballot_sync(0xffffffffu, pass);
            if (pass) {
                int pos = qh + qn + __popc(m & lanemask_lt);
                if (pos >= kLeanQueue) pos -= kLeanQueue;
                LeanEntry en;
                en.row = r0 + k;
                en.qty = qv[k];
                en.price = pv[k];
                Q[pos] = en;
            }
            qn += __popc(m);
        }
        drain();
    }
    __syncwarp();
    consume(qn);
    if (bad_value) atomicOr(status, 1);
    if (bad_key) atomicOr(status, 2);
    __syncthreads();
    flush_table();
    __threadfence();
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    finalize_groups<kGbThreads>(g, dict, card, done, out_keys, out_sum, out_min, out_max, out_count, out_ngroups);
}

// ---------------------------------------------------------------------------
// Large dictionaries (more than kMaxGroups entries: a full shared-memory table
// does not fit).  Each block keeps a shared-memory cache of 2^slots_log2 slots,
// each a 32-bit word accumulator as in MODE 1 tagged with the group it holds.
// A group takes the first free slot of its probe sequence the first time one
// of its rows reaches the block and keeps it until the block flushes, so the
// frequent groups of a skewed column settle in every block's cache.  Rows whose
// group finds no slot go to the HBM table: per group five signed 64-bit limbs
// (limb k weighs 2^(32k) units of 2^-76), the count and the MIN / MAX order
// keys.  Every update of the HBM table (sums, count, min, max) is a reduction
// whose result is never read (no carry crosses a limb; each added piece is
// below 2^32), so no thread waits on an HBM atomic.  A scan kernel covers at most kSpillChunk rows; the
// limbs are normalised between chunks, which keeps each below 2^61.  A
// separate kernel then compacts the non-empty groups in key order (tiles of
// groups claimed in launch order, output offsets by decoupled look-back) and
// resets the table.  The sums are the same integers as the shared-table
// kernels', so the rows are bit-identical to theirs.
// ---------------------------------------------------------------------------
constexpr int kLimbWords = 8;  // per group in HBM: limbs 0-4, count, min key, max key
constexpr uint32_t kSlotEmpty = 0xFFFFFFFFu;
constexpr int kSlotProbes = 4;
constexpr uint64_t kSpillChunk = 1ull << 28;
constexpr int kSpillMaxLog2 = 11;

// shared memory of the slot cache: min, max keys, five words, count, tag per slot
size_t spill_smem_bytes(int slots_log2) { return (static_cast<size_t>(1) << slots_log2) * 44; }

// B32: queue entries hold the row's 32-bit bit offset in the packed column
// (rows x width < 2^32), else its 64-bit index
template <int RPT, int MINB, bool B32>
__global__ void __launch_bounds__(kGbThreads, MINB) scan_groupby_spill_kernel(
    const uint64_t* __restrict__ packed, uint32_t width, uint32_t card, const double* __restrict__ price,
    const int32_t* __restrict__ qty, uint64_t row0, uint64_t n, double pthr, int32_t qlo, int32_t qhi,
    unsigned long long* __restrict__ hbm, int slots_log2, int* status) {
    constexpr int kTile = kGbThreads * RPT;
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t nslots = 1u << slots_log2;
    unsigned long long* s_mn = reinterpret_cast<unsigned long long*>(smem);
    unsigned long long* s_mx = s_mn + nslots;
    uint32_t* s_w = reinterpret_cast<uint32_t*>(s_mx + nslots);
    uint32_t* s_cnt = s_w + kWords * nslots;
    uint32_t* s_tag = s_cnt + nslots;
    auto reset_slots = [&]() {
        for (uint32_t i = threadIdx.x; i < nslots; i += blockDim.x) {
#pragma unroll
            for (int k = 0; k < kWords; ++k) s_w[kWords * i + k] = 0;
            s_cnt[i] = 0;
            s_mn[i] = ~0ull;
            s_mx[i] = 0;
            s_tag[i] = kSlotEmpty;
        }
    };
    // slot -> HBM: words 0-3 as unsigned pieces, word 4 sign-extended (the
    // 160-bit two's complement value), all as reductions
    auto flush_slots = [&]() {
        for (uint32_t i = threadIdx.x; i < nslots; i += blockDim.x) {
            const uint32_t tag = s_tag[i], c = s_cnt[i];
            if (tag == kSlotEmpty || !c) continue;
            unsigned long long* e = hbm + static_cast<uint64_t>(kLimbWords) * tag;
#pragma unroll
            for (int k = 0; k < kWords - 1; ++k)
                if (const uint32_t w = s_w[kWords * i + k]) atomicAdd(&e[k], static_cast<unsigned long long>(w));
            if (const uint32_t w = s_w[kWords * i + kWords - 1]) {
                const long long top = static_cast<int32_t>(w);  // the sign word
                atomicAdd(&e[kWords - 1], static_cast<unsigned long long>(top));
            }
            atomicAdd(&e[5], static_cast<unsigned long long>(c));
            atomicMin(&e[6], s_mn[i]);
            atomicMax(&e[7], s_mx[i]);
        }
    };
    reset_slots();
    __syncthreads();

    const uint64_t mask = (width >= 64) ? ~0ull : ((1ull << width) - 1);
    const uint32_t qspan = qlo <= qhi ? static_cast<uint32_t>(qhi) - static_cast<uint32_t>(qlo) : 0u;
    const double pcut = qlo <= qhi ? pthr : __longlong_as_double(0x7FF0000000000000ll);
    const uint64_t ntiles = (n + kTile - 1) / kTile;
    const uint64_t tiles_per_flush = (1ull << 19) / kTile;  // 32-bit slot counts, 160-bit slot sums
    bool bad_value = false, bad_key = false;
    uint64_t since_flush = 0;

    __shared__ WarpQueue<B32> s_queue[kGbThreads / 32];
    const int lane = threadIdx.x & 31;
    const unsigned lanemask_lt = (1u << lane) - 1;
    WarpQueue<B32>& Q = s_queue[threadIdx.x >> 5];
    int qn = 0, qh = 0;
    volatile uint32_t* const v_tag = s_tag;
    const uint32_t* const p32 = reinterpret_cast<const uint32_t*>(packed);
    const uint32_t nw32 = B32 ? static_cast<uint32_t>(((row0 + n) * width + 63) / 64 * 2) : 0u;
    const uint32_t mask32 = static_cast<uint32_t>(mask);

    auto consume = [&](int cnt) {
        const bool valid = lane < cnt;
        const int e = (qh + lane) & (kQueue - 1);
        const double p = valid ? Q.price[e] : 0.0;
        const double v = valid ? __dmul_rn(p, static_cast<double>(Q.qty[e])) : 0.0;  // one rounded multiply
        // one warp-uniform test picks the add-only path of the slot words
        const bool mayneg = __any_sync(0xffffffffu, v < 0.0);
        if (!valid) return;
        uint32_t gi;
        if constexpr (B32) gi = key_bits32(p32, Q.pos[e], nw32, mask32);
        else gi = key_bits(packed, Q.pos[e], width, mask);
        if (gi >= card) {
            bad_key = true;
            return;
        }
        RowWords w;
        const bool ok = row_words(v, &w);
        if (!ok) bad_value = true;
        const bool neg = v < 0.0;
        const unsigned long long key = f64_order_key(p);
        // a slot is written once (empty -> tag) between flushes, so the first
        // slot of the probe sequence that holds gi or is won for it is gi's own
        uint32_t h = (gi * 0x9E3779B1u) >> (32 - slots_log2);
        int slot = -1;
#pragma unroll
        for (int pr = 0; pr < kSlotProbes; ++pr) {
            uint32_t t = v_tag[h];
            if (t == kSlotEmpty) {
                t = atomicCAS(&s_tag[h], kSlotEmpty, gi);
                if (t == kSlotEmpty) t = gi;
            }
            if (t == gi) {
                slot = static_cast<int>(h);
                break;
            }
            h = (h + 1) & (nslots - 1);
        }
        if (slot >= 0) {
            if (ok && mayneg) words_add<true>(s_w + kWords * slot, w, neg);
            else if (ok) words_add<false>(s_w + kWords * slot, w, false);
            atomicAdd(&s_cnt[slot], 1u);
            if (key < s_mn[slot]) atomicMin(&s_mn[slot], key);
            if (key > s_mx[slot]) atomicMax(&s_mx[slot], key);
            return;
        }
        unsigned long long* eb = hbm + static_cast<uint64_t>(kLimbWords) * gi;
        if (ok) {
            const unsigned long long a0 = w.c0, a1 = w.c1, a2 = w.c2;
            if (a0) atomicAdd(&eb[w.k0], neg ? 0ull - a0 : a0);
            if (a1) atomicAdd(&eb[w.k0 + 1], neg ? 0ull - a1 : a1);
            if (a2) atomicAdd(&eb[w.k0 + 2], neg ? 0ull - a2 : a2);
        }
        atomicAdd(&eb[5], 1ull);
        // MIN / MAX as reductions too: no read of the current keys to wait on
        atomicMin(&eb[6], key);
        atomicMax(&eb[7], key);
    };

    for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        if (since_flush == tiles_per_flush) {
            __syncwarp();
            consume(qn);
            qn = 0;
            __syncthreads();
            flush_slots();
            __syncthreads();
            reset_slots();
            __syncthreads();
            since_flush = 0;
        }
        ++since_flush;
        const uint64_t r0 = row0 + t * kTile + static_cast<uint64_t>(threadIdx.x) * RPT;
        const uint64_t rend = row0 + n;
        double pv[RPT];
        int32_t qv[RPT];
        if (r0 + RPT <= rend) {
#pragma unroll
            for (int k = 0; k < RPT; k += 4) {
                const double2* pp = reinterpret_cast<const double2*>(price + r0 + k);
                const double2 a = __ldcs(pp), b = __ldcs(pp + 1);
                const int4 q = __ldcs(reinterpret_cast<const int4*>(qty + r0 + k));
                pv[k] = a.x; pv[k + 1] = a.y; pv[k + 2] = b.x; pv[k + 3] = b.y;
                qv[k] = q.x; qv[k + 1] = q.y; qv[k + 2] = q.z; qv[k + 3] = q.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                const bool in = r0 + k < rend;
                pv[k] = in ? price[r0 + k] : __longlong_as_double(0x7FF8000000000000ll);  // NaN never passes
                qv[k] = in ? qty[r0 + k] : 0;
            }
        }
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            const double p = pv[k];
            const int32_t q = qv[k];
            const bool pass = p > pcut && static_cast<uint32_t>(q) - static_cast<uint32_t>(qlo) <= qspan;
            const unsigned m = __ballot_sync(0xffffffffu, pass);
            if (pass) {
                const int pos = (qh + qn + __popc(m & lanemask_lt)) & (kQueue - 1);
                if constexpr (B32) Q.pos[pos] = static_cast<uint32_t>((r0 + k) * width);  // < 2^32 by the launch check
                else Q.pos[pos] = r0 + k;
                Q.price[pos] = p;
                Q.qty[pos] = q;
            }
            qn += __popc(m);
            if (qn >= 32) {
                __syncwarp();
                consume(32);
                __syncwarp();  // the consumed entries are free for the next pushes
                qh = (qh + 32) & (kQueue - 1);
                qn -= 32;
            }
        }
    }
    __syncwarp();
    consume(qn);
    if (bad_value) atomicOr(status, 1);
    if (bad_key) atomicOr(status, 2);
    __syncthreads();
    flush_slots();
}

// carries of limbs 0-3 into the next limb: afterwards limbs 0-3 lie in
// [0, 2^32) and limb 4 holds the signed rest (between scan chunks)
__global__ void normalize_limbs_kernel(unsigned long long* hbm, uint32_t card) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < card;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        unsigned long long* e = hbm + kLimbWords * i;
        long long c = 0;
#pragma unroll
        for (int k = 0; k < kWords - 1; ++k) {
            const long long v = static_cast<long long>(e[k]) + c;
            e[k] = static_cast<unsigned long long>(v) & 0xFFFFFFFFull;
            c = v >> 32;  // arithmetic: v = c * 2^32 + low word
        }
        e[kWords - 1] = static_cast<unsigned long long>(static_cast<long long>(e[kWords - 1]) + c);
    }
}

constexpr int kFinPer = 2;                        // groups per thread
constexpr int kFinTile = kGbThreads * kFinPer;     // groups per tile

__global__ void __launch_bounds__(kGbThreads) groupby_finalize_kernel(
    unsigned long long* hbm, const int32_t* __restrict__ dict, uint32_t card, int32_t* out_keys, double* out_sum,
    double* out_min, double* out_max, uint64_t* out_count, uint64_t* out_ngroups, unsigned long long* lb,
    unsigned int* ctr, int* err) {
    __shared__ uint64_t s_tile, s_base;
    __shared__ uint64_t s_warp[kGbThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t ntiles = (card + kFinTile - 1) / kFinTile;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t i0 = tile * kFinTile + static_cast<uint64_t>(threadIdx.x) * kFinPer;
        uint32_t live = 0;
#pragma unroll
        for (int k = 0; k < kFinPer; ++k) {
            const uint64_t i = i0 + k;
            if (i < card && __ldcg(&hbm[kLimbWords * i + 5])) live |= 1u << k;
        }
        const uint64_t c = __popc(live);
        uint64_t inc = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += y;
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            const uint64_t x = lane < kGbThreads / 32 ? s_warp[lane] : 0;
            uint64_t t = x;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint64_t y = __shfl_up_sync(0xffffffffu, t, d);
                if (lane >= d) t += y;
            }
            if (lane < kGbThreads / 32) s_warp[lane] = t - x;
            const uint64_t total = __shfl_sync(0xffffffffu, t, kGbThreads / 32 - 1);
            const uint64_t e = lookback_exclusive_warp(lb, tile, total, err);
            if (lane == 0) {
                s_base = e;
                if (tile == ntiles - 1) *out_ngroups = e + total;
            }
        }
        __syncthreads();
        uint64_t pos = s_base + s_warp[warp] + (inc - c);
#pragma unroll
        for (int k = 0; k < kFinPer; ++k) {
            const uint64_t i = i0 + k;
            if (i >= card) break;
            unsigned long long* e = hbm + kLimbWords * i;
            if (live >> k & 1u) {
                unsigned long long l[kWords];
#pragma unroll
                for (int j = 0; j < kWords; ++j) l[j] = __ldcg(&e[j]);
                out_keys[pos] = dict[i];
                out_sum[pos] = fix_to_double_s<kFixScale>(fix_from_limbs(l));
                out_min[pos] = f64_from_order_key(__ldcg(&e[6]));
                out_max[pos] = f64_from_order_key(__ldcg(&e[7]));
                out_count[pos] = __ldcg(&e[5]);
                ++pos;
            }
#pragma unroll
            for (int j = 0; j < 6; ++j) e[j] = 0;
            e[6] = ~0ull;
            e[7] = 0;
        }
        __syncthreads();
    }
}

__global__ void init_groups_kernel(GlobalGroups g, uint32_t card, unsigned int* done) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < card; i += gridDim.x * blockDim.x) {
        g.sum[3 * i] = 0;
        g.sum[3 * i + 1] = 0;
        g.sum[3 * i + 2] = 0;
        g.cnt[i] = 0;
        g.mn[i] = ~0ull;
        g.mx[i] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *done = 0;
}

__global__ void init_limbs_kernel(unsigned long long* hbm, uint32_t card, unsigned int* done) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < card;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        unsigned long long* e = hbm + kLimbWords * i;
#pragma unroll
        for (int j = 0; j < 6; ++j) e[j] = 0;
        e[6] = ~0ull;
        e[7] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *done = 0;
}

// shared-table dictionaries: sums (3 words), count, min, max per group; larger
// ones: the eight-word limb layout
size_t table_bytes(uint32_t card) {
    return static_cast<size_t>(card) * (card > kMaxGroups ? kLimbWords : 6) * 8 + 256;
}

size_t tma_smem_bytes(uint32_t card, uint32_t width) {
    return kTmaStages * (24576u + 256u * width) + static_cast<size_t>(kTmaConsumers) * card * 16 +
           static_cast<size_t>(card) * 16 + kTmaConsumers * 64 * 2 + 2 * kTmaStages * 8 + 64;
}

// 227 KB per block on sm_100, less the TMA kernel's static shared memory
constexpr size_t kSmemOptIn = 232448 - 2048;

int launch_tma(ScanGroupBy& S, const uint64_t* packed, uint32_t width, const int32_t* dict, uint32_t card,
               const double* price, const int32_t* qty, uint64_t n, double pthr, int32_t qlo, int32_t qhi,
               int32_t* ok, double* os, double* omn, double* omx, uint64_t* oc, uint64_t* ong, cudaStream_t s) {
    size_t smem = tma_smem_bytes(card, width);
    static thread_local int max_dyn = 0;
    if (!max_dyn) {
        int dev = 0, optin = 0;
        VX_CUDA(cudaGetDevice(&dev));
        VX_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        cudaFuncAttributes fa;
        VX_CUDA(cudaFuncGetAttributes(&fa, scan_groupby_tma_kernel));
        max_dyn = optin - static_cast<int>(fa.sharedSizeBytes);
        VX_CUDA(cudaFuncSetAttribute(scan_groupby_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn));
    }
    if (smem > static_cast<size_t>(max_dyn)) {
        set_error(kErrInvalidArg, "TMA group-by needs %zu bytes of shared memory, %d available", smem, max_dyn);
        return kErrInvalidArg;
    }
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t nfull = n / kTmaRows;
    uint64_t grid = static_cast<uint64_t>(sms);
    if (grid > nfull) grid = nfull;
    if (grid < 1) grid = 1;
    GlobalGroups g{S.g_sum, S.g_cnt, S.g_mn, S.g_mx};
    scan_groupby_tma_kernel<<<static_cast<unsigned>(grid), kTmaThreads, smem, s>>>(
        packed, width, dict, card, price, qty, n, pthr, qlo, qhi, g, S.g_done, ok, os, omn, omx, oc, ong,
        static_cast<int*>(S.status.p));
    VX_CUDA(cudaGetLastError());
    S.last_grid = static_cast<int>(grid);
    S.last_kernel = 1;
    return kOk;
}

// Stages of the bulk-copy-fed word table that fit this shape (0: the variant
// does not apply: misaligned packed keys, fewer than one full stage, a block
// would sum more than 2^19 rows, or the table and two stages do not fit).
int tw_stages(const uint64_t* packed, uint32_t width, uint32_t card, uint64_t n, size_t max_dyn) {
    if ((reinterpret_cast<uintptr_t>(packed) & 15) || width == 0 || width > kMaxWidth) return 0;
    const uint64_t nfull = n / kTwRows;
    if (nfull == 0) return 0;
    const uint64_t sms = static_cast<uint64_t>(sm_count() > 0 ? sm_count() : 148);
    const uint64_t grid = nfull < sms ? nfull : sms;
    if (((nfull + grid - 1) / grid + 1) * kTwRows > (1ull << 19)) return 0;
    for (int st = kTwMaxStages; st >= 2; --st)
        if (tw_smem_bytes(card, width, st) <= max_dyn) return st;
    return 0;
}

size_t tw_max_dyn() {
    static thread_local size_t max_dyn = 0;
    if (!max_dyn) {
        int dev = 0, optin = 0;
        cudaFuncAttributes fa{};
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
            cudaFuncGetAttributes(&fa, scan_groupby_tw_kernel) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        const int dyn = optin - static_cast<int>(fa.sharedSizeBytes);
        if (dyn <= 0 ||
            cudaFuncSetAttribute(scan_groupby_tw_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) !=
                cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        max_dyn = static_cast<size_t>(dyn);
    }
    return max_dyn;
}

int launch_tw(ScanGroupBy& S, int nstages, const uint64_t* packed, uint32_t width, const int32_t* dict,
              uint32_t card, const double* price, const int32_t* qty, uint64_t n, double pthr, int32_t qlo,
              int32_t qhi, int32_t* ok, double* os, double* omn, double* omx, uint64_t* oc, uint64_t* ong,
              cudaStream_t s) {
    const int sms = sm_count() > 0 ? sm_count() : 148;
    const uint64_t nfull = n / kTwRows;
    const uint64_t grid = nfull < static_cast<uint64_t>(sms) ? nfull : static_cast<uint64_t>(sms);
    GlobalGroups g{S.g_sum, S.g_cnt, S.g_mn, S.g_mx};
    scan_groupby_tw_kernel<<<static_cast<unsigned>(grid), kTwThreads, tw_smem_bytes(card, width, nstages), s>>>(
        packed, width, dict, card, price, qty, n, pthr, qlo, qhi, nstages, g, S.g_done, ok, os, omn, omx, oc, ong,
        static_cast<int*>(S.status.p));
    VX_CUDA(cudaGetLastError());
    S.last_grid = static_cast<int>(grid);
    S.last_kernel = 4;
    return kOk;
}

template <int RPT, int MODE, bool B32>
auto fused_kernel_of() {
    if constexpr (MODE == 3) return scan_groupby_pf_kernel<RPT, B32>;
    else return scan_groupby_kernel<RPT, MODE, B32>;
}

// dynamic shared memory of the MODE 1, 2 table: min, max (8 bytes each), five
// accumulator words and a count (4 bytes each) per group -- the MODE 0 size
template <int RPT, int MODE>
int launch_rpt(ScanGroupBy& S, const uint64_t* packed, uint32_t width, const int32_t* dict, uint32_t card,
               const double* price, const int32_t* qty, uint64_t n, double pthr, int32_t qlo, int32_t qhi,
               int32_t* ok, double* os, double* omn, double* omx, uint64_t* oc, uint64_t* ong, cudaStream_t s) {
    constexpr int kTile = kGbThreads * RPT;
    // the queue modes keep 32-bit bit offsets when rows x width < 2^32
    constexpr bool kQueued = MODE == 1 || MODE == 3;
    const bool b32 = kQueued && n * static_cast<uint64_t>(width) < (1ull << 32);
    auto* const kern = b32 ? fused_kernel_of<RPT, MODE, kQueued>() : fused_kernel_of<RPT, MODE, false>();
    size_t smem = scan_groupby_smem_bytes(card);
    static thread_local uint32_t attr_set_for[2] = {0, 0};  // per B32 instance
    if (attr_set_for[b32] < card) {
        VX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(scan_groupby_smem_bytes(kMaxGroups))));
        attr_set_for[b32] = kMaxGroups;
    }
    int per_sm = 0;
    VX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kGbThreads, smem));
    if (per_sm < 1) per_sm = 1;
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t ntiles = (n + kTile - 1) / kTile;
    uint64_t grid = static_cast<uint64_t>(sms) * per_sm;
    if (grid > ntiles) grid = ntiles;
    if (grid < 1) grid = 1;
    GlobalGroups g{S.g_sum, S.g_cnt, S.g_mn, S.g_mx};
    kern<<<static_cast<unsigned>(grid), kGbThreads, smem, s>>>(packed, width, dict, card, price, qty, n, pthr, qlo,
                                                               qhi, g, S.g_done, ok, os, omn, omx, oc, ong,
                                                               static_cast<int*>(S.status.p));
    VX_CUDA(cudaGetLastError());
    S.last_grid = static_cast<int>(grid);
    S.last_kernel = MODE == 0 ? 0 : MODE == 3 ? 7 : MODE + 1;
    return kOk;
}

template <int RPT>
int launch_lean(ScanGroupBy& S, const uint64_t* packed, uint32_t width, const int32_t* dict, uint32_t card,
                const double* price, const int32_t* qty, uint64_t n, double pthr, int32_t qlo, int32_t qhi,
                int32_t* ok, double* os, double* omn, double* omx, uint64_t* oc, uint64_t* ong, cudaStream_t s) {
    constexpr uint64_t kTile = static_cast<uint64_t>(kGbThreads) * RPT;
    const size_t smem = lean_smem_bytes(card);
    static thread_local bool attr_set = false;
    if (!attr_set) {
        VX_CUDA(cudaFuncSetAttribute(scan_groupby_lean_kernel<RPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(lean_smem_bytes(kMaxGroups))));
        attr_set = true;
    }
    int per_sm = 0;
    VX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, scan_groupby_lean_kernel<RPT>, kGbThreads, smem));
    if (per_sm < 1) per_sm = 1;
    const int sms = sm_count() > 0 ? sm_count() : 148;
    const uint64_t ntiles = (n + kTile - 1) / kTile;
    uint64_t grid = static_cast<uint64_t>(sms) * per_sm;
    if (grid > ntiles) grid = ntiles;
    if (grid < 1) grid = 1;
    GlobalGroups g{S.g_sum, S.g_cnt, S.g_mn, S.g_mx};
    scan_groupby_lean_kernel<RPT><<<static_cast<unsigned>(grid), kGbThreads, smem, s>>>(
        packed, width, dict, card, price, qty, static_cast<uint32_t>(n), pthr, qlo, qhi, g, S.g_done, ok, os, omn,
        omx, oc, ong, static_cast<int*>(S.status.p));
    VX_CUDA(cudaGetLastError());
    S.last_grid = static_cast<int>(grid);
    S.last_kernel = 5;
    return kOk;
}

int launch_spill(ScanGroupBy& S, int slots_log2, const uint64_t* packed, uint32_t width, const int32_t* dict,
                 uint32_t card, const double* price, const int32_t* qty, uint64_t n, double pthr, int32_t qlo,
                 int32_t qhi, int32_t* ok, double* os, double* omn, double* omx, uint64_t* oc, uint64_t* ong,
                 cudaStream_t s) {
    constexpr int kRpt = 4;
    constexpr uint64_t kTile = static_cast<uint64_t>(kGbThreads) * kRpt;
    const int sms = sm_count() > 0 ? sm_count() : 148;
    unsigned long long* const hbm = S.g_limb;
    int* const status = static_cast<int*>(S.status.p);
    const size_t smem = spill_smem_bytes(slots_log2);
    // the smaller cache leaves room for a third block per SM: registers capped
    // to match; 32-bit bit offsets in the queue when rows x width < 2^32
    const bool b32 = n * static_cast<uint64_t>(width) < (1ull << 32);
    const bool small = slots_log2 < kSpillMaxLog2;
    auto* const kern = small ? (b32 ? scan_groupby_spill_kernel<kRpt, 3, true>
                                    : scan_groupby_spill_kernel<kRpt, 3, false>)
                             : (b32 ? scan_groupby_spill_kernel<kRpt, 2, true>
                                    : scan_groupby_spill_kernel<kRpt, 2, false>);
    static thread_local bool attr_set = false;
    if (!attr_set) {
        const int bytes = static_cast<int>(spill_smem_bytes(kSpillMaxLog2));
        VX_CUDA(cudaFuncSetAttribute(scan_groupby_spill_kernel<kRpt, 2, false>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        VX_CUDA(cudaFuncSetAttribute(scan_groupby_spill_kernel<kRpt, 3, false>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        VX_CUDA(cudaFuncSetAttribute(scan_groupby_spill_kernel<kRpt, 2, true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        VX_CUDA(cudaFuncSetAttribute(scan_groupby_spill_kernel<kRpt, 3, true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        attr_set = true;
    }
    int per_sm = 0;
    VX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kGbThreads, smem));
    if (per_sm < 1) per_sm = 1;
    uint64_t grid = 1;
    for (uint64_t off = 0; off < n; off += kSpillChunk) {
        const uint64_t m = n - off < kSpillChunk ? n - off : kSpillChunk;
        if (off) {  // carries out of the limbs before the next chunk adds to them
            normalize_limbs_kernel<<<static_cast<unsigned>(sms) * 4, 256, 0, s>>>(hbm, card);
            VX_CUDA(cudaGetLastError());
        }
        const uint64_t ntiles = (m + kTile - 1) / kTile;
        grid = static_cast<uint64_t>(sms) * per_sm;
        if (grid > ntiles) grid = ntiles;
        kern<<<static_cast<unsigned>(grid), kGbThreads, smem, s>>>(
            packed, width, card, price, qty, off, m, pthr, qlo, qhi, hbm, slots_log2, status);
        VX_CUDA(cudaGetLastError());
    }
    const uint64_t ftiles = (card + kFinTile - 1) / kFinTile;
    const size_t lb_bytes = (ftiles + 1) * 8 + 64;
    if (S.lookback.n < lb_bytes) {
        S.lookback = DevBuf(lb_bytes);
        if (!S.lookback.p) return kErrOutOfMemory;
    }
    VX_CUDA(cudaMemsetAsync(S.lookback.p, 0, lb_bytes, s));
    unsigned long long* lb = S.lookback.as<unsigned long long>();
    unsigned int* ctr = reinterpret_cast<unsigned int*>(lb + ftiles);
    uint64_t fgrid = static_cast<uint64_t>(sms) * 4;
    if (fgrid > ftiles) fgrid = ftiles;
    // the status word's bit 4 is the look-back timeout, reported like the bulk-copy waits
    groupby_finalize_kernel<<<static_cast<unsigned>(fgrid), kGbThreads, 0, s>>>(hbm, dict, card, ok, os, omn, omx,
                                                                                oc, ong, lb, ctr, status);
    VX_CUDA(cudaGetLastError());
    S.last_grid = static_cast<int>(grid);
    S.last_kernel = 6;
    return kOk;
}

// the slot-cache size: 2048 slots (two blocks per SM) or 1024 (three), timed
// per (dictionary size, rows) when tuning is on
int launch_global(ScanGroupBy& S, const uint64_t* packed, uint32_t width, const int32_t* dict, uint32_t card,
                  const double* price, const int32_t* qty, uint64_t n, double pthr, int32_t qlo, int32_t qhi,
                  int32_t* ok, double* os, double* omn, double* omx, uint64_t* oc, uint64_t* ong, cudaStream_t s) {
    auto variant = [&](int c) -> int {
        return launch_spill(S, c == 1 ? kSpillMaxLog2 - 1 : kSpillMaxLog2, packed, width, dict, card, price, qty, n,
                            pthr, qlo, qhi, ok, os, omn, omx, oc, ong, s);
    };
    if (!S.autotune || n < (1u << 16)) return variant(0);
    int cl = 0;
    while (cl < 31 && (2u << cl) <= card) ++cl;
    const std::string family = "scan_groupby_spill_card" + std::to_string(cl);
    const std::string key = tune_key(family.c_str(), F64, n);
    int c = 0;
    if (!tune_lookup(key, &c)) c = tune_pick(key, 2, 0, s, variant);
    return variant(c);
}

}  // namespace

size_t scan_groupby_smem_bytes(uint32_t card) { return static_cast<size_t>(card) * 5 * 8 + 16; }

int ScanGroupBy::prepare(uint32_t card, cudaStream_t s) {
    if (card == 0 || card > kMaxGlobalGroups) {
        set_error(kErrInvalidArg, "dictionary cardinality %u outside 1..%u", card, kMaxGlobalGroups);
        return kErrInvalidArg;
    }
    if (card_ != card) {
        table = DevBuf(table_bytes(card));
        status = DevBuf(16);
        if (!table.p || !status.p) return kErrOutOfMemory;
        card_ = card;
        char* b = static_cast<char*>(table.p);
        if (card > kMaxGroups) {  // the HBM table of the slot-cache kernels: eight words per group
            g_limb = reinterpret_cast<unsigned long long*>(b);
            g_sum = g_cnt = g_mn = g_mx = nullptr;
            g_done = reinterpret_cast<unsigned int*>(g_limb + static_cast<size_t>(kLimbWords) * card);
            init_limbs_kernel<<<(card + 255) / 256, 256, 0, s>>>(g_limb, card, g_done);
        } else {
            g_limb = nullptr;
            g_sum = reinterpret_cast<unsigned long long*>(b);
            g_cnt = g_sum + 3 * card;
            g_mn = g_cnt + card;
            g_mx = g_mn + card;
            g_done = reinterpret_cast<unsigned int*>(g_mx + card);
            GlobalGroups g{g_sum, g_cnt, g_mn, g_mx};
            init_groups_kernel<<<(card + 255) / 256, 256, 0, s>>>(g, card, g_done);
        }
        VX_CUDA(cudaGetLastError());
        VX_CUDA(cudaMemsetAsync(status.p, 0, 16, s));
    }
    return kOk;
}

int ScanGroupBy::launch(const uint64_t* packed, uint32_t width, const int32_t* dict, uint32_t card,
                        const double* price, const int32_t* qty, uint64_t n, double pthr, int32_t qlo,
                        int32_t qhi, int32_t* out_keys, double* out_sum, double* out_min, double* out_max,
                        uint64_t* out_count, uint64_t* out_ngroups, cudaStream_t s) {
    if (width == 0 || width > kMaxWidth) {
        set_error(kErrInvalidArg, "bit width %u outside 1..%d", width, kMaxWidth);
        return kErrInvalidArg;
    }
    if ((reinterpret_cast<uintptr_t>(price) | reinterpret_cast<uintptr_t>(qty)) & 15) {
        set_error(kErrInvalidArg, "price / qty columns must be 16-byte aligned");
        return kErrInvalidArg;
    }
    int st = prepare(card, s);
    if (st) return st;
    if (card > kMaxGroups)  // the shared-memory tables do not fit: HBM atomics, multi-block finalize
        return launch_global(*this, packed, width, dict, card, price, qty, n, pthr, qlo, qhi, out_keys, out_sum,
                             out_min, out_max, out_count, out_ngroups, s);
    if (use_tma && card <= kTmaMaxCard && tma_smem_bytes(card, width) <= kSmemOptIn && n >= kTmaRows &&
        ((reinterpret_cast<uintptr_t>(packed) & 15) == 0))
        return launch_tma(*this, packed, width, dict, card, price, qty, n, pthr, qlo, qhi, out_keys, out_sum,
                          out_min, out_max, out_count, out_ngroups, s);
#define VX_LAUNCH_RPT(R, M)                                                                                    \
    launch_rpt<R, M>(*this, packed, width, dict, card, price, qty, n, pthr, qlo, qhi, out_keys, out_sum, out_min, \
                     out_max, out_count, out_ngroups, s)
    if (use_tw && !use_tma)
        if (const int tw = tw_stages(packed, width, card, n, tw_max_dyn()))
            return launch_tw(*this, tw, packed, width, dict, card, price, qty, n, pthr, qlo, qhi, out_keys,
                             out_sum, out_min, out_max, out_count, out_ngroups, s);
    const bool lean_ok = n < (1ull << 32);
#define VX_LAUNCH_LEAN()                                                                                       \
    launch_lean<4>(*this, packed, width, dict, card, price, qty, n, pthr, qlo, qhi, out_keys, out_sum, out_min, \
                   out_max, out_count, out_ngroups, s)
    if (use_lean && lean_ok) return VX_LAUNCH_LEAN();
    if (autotune && !use_tma && n >= (1u << 16)) {  // smaller scans take the default
        // the word-table variants give identical bits: time them on this call's
        // data once per (dictionary size, rows) and keep the fastest
        auto variant = [&](int c) -> int {
            switch (c) {
            case 1: return VX_LAUNCH_RPT(8, 1);
            case 2: return VX_LAUNCH_RPT(4, 2);
            case 3: return VX_LAUNCH_RPT(8, 2);
            case 4: return lean_ok ? VX_LAUNCH_LEAN() : VX_LAUNCH_RPT(4, 1);
            case 5: return VX_LAUNCH_RPT(4, 3);
            default: return VX_LAUNCH_RPT(4, 1);
            }
        };
        int cl = 0;
        while (cl < 31 && (2u << cl) <= card) ++cl;
        const std::string family = "scan_groupby_v3_card" + std::to_string(cl);
        const std::string key = tune_key(family.c_str(), F64, n);
        int c = 0;
        if (!tune_lookup(key, &c)) c = tune_pick(key, 6, 0, s, variant);
        return variant(c);
    }
    if (mode == 3) return VX_LAUNCH_RPT(4, 3);
    if (mode == 1) return rows_per_thread == 8 ? VX_LAUNCH_RPT(8, 1) : VX_LAUNCH_RPT(4, 1);
    if (mode == 2) return rows_per_thread == 8 ? VX_LAUNCH_RPT(8, 2) : VX_LAUNCH_RPT(4, 2);
    switch (rows_per_thread) {
    case 8: return VX_LAUNCH_RPT(8, 0);
    case 16: return VX_LAUNCH_RPT(16, 0);
    default: return VX_LAUNCH_RPT(4, 0);
    }
#undef VX_LAUNCH_RPT
#undef VX_LAUNCH_LEAN
}

// Status word bits the fused scan kernels OR in: 4 a bounded bulk-copy wait ran
// out (the group rows are partial), 2 a key index outside the dictionary, 1 a
// product that is not finite or beyond 2^63.  The most serious bit wins.
int groupby_status_error(int h) {
    if (!h) return kOk;
    if (h & 4) {
        set_error(kErrDeviceTimeout,
                  "a bounded wait in the fused scan (bulk copy or tile look-back) ran out of its budget; the group rows "
                  "are partial");
        return kErrDeviceTimeout;
    }
    if (h & 2) {
        set_error(kErrInvalidArg, "a packed key index is outside the dictionary");
        return kErrInvalidArg;
    }
    if (h & 1) {
        set_error(kErrOverflow, "a price*qty product is not finite or exceeds 2^63 in magnitude");
        return kErrOverflow;
    }
    set_error(kErrInvalidArg, "unknown fused-scan status bits 0x%x", static_cast<unsigned>(h));
    return kErrInvalidArg;
}

int ScanGroupBy::check_status(cudaStream_t s) {
    if (!status.p) return kOk;  // nothing launched on this thread yet
    int h = 0;
    int st = d2h(&h, status.p, sizeof(int), s);
    if (st) return st;
    st = sync(s);
    if (st) return st;
    if (h) {
        VX_CUDA(cudaMemsetAsync(status.p, 0, 16, s));
        return groupby_status_error(h);
    }
    return kOk;
}

ScanGroupBy& scan_groupby_state() {
    static thread_local ScanGroupBy s;
    return s;
}

// ---------------------------------------------------------------------------
// Allocation-free variant (voxel_scan_groupby_noalloc_dev).
//
// The group table lives in a fixed file-scope device array laid out for the
// largest dictionary (kMaxGroups groups at a fixed stride, so a call with any
// smaller dictionary uses a prefix of each field).  Its resting state is: sum
// words 0, counts 0, min keys all ones, max keys 0, completion counter 0.  The
// loader zeroes the array; the first call on a device sets the min keys and
// waits for that; every launch's last block puts the groups it used and the
// counter back to the resting state.
namespace {

constexpr size_t kNoAllocWords = static_cast<size_t>(kMaxGroups) * 6 + 32;  // 196,864 bytes
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocWords];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_addr[kNoAllocMaxDevices] = {};
int g_noalloc_per_sm[kNoAllocMaxDevices] = {};

// One-time per-device setup: symbol address, resting state of the min keys,
// kernel attribute, occupancy.  Synchronises `s`.
int noalloc_setup(cudaStream_t s, unsigned long long** base, int* per_sm) {
    int dev = 0;
    VX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        set_error(kErrInvalidArg, "device ordinal %d outside 0..%d", dev, kNoAllocMaxDevices - 1);
        return kErrInvalidArg;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        VX_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        unsigned long long* b = static_cast<unsigned long long*>(p);
        VX_CUDA(cudaMemsetAsync(b + 4 * static_cast<size_t>(kMaxGroups), 0xFF, kMaxGroups * sizeof(unsigned long long),
                                s));
        VX_CUDA(cudaStreamSynchronize(s));
        VX_CUDA(cudaFuncSetAttribute(scan_groupby_kernel<4, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(scan_groupby_smem_bytes(kMaxGroups))));
        int occ = 0;
        VX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, scan_groupby_kernel<4, 0>, kGbThreads,
                                                              scan_groupby_smem_bytes(kMaxGroups)));
        g_noalloc_per_sm[dev] = occ < 1 ? 1 : occ;
        g_noalloc_addr[dev] = b;
    }
    *base = g_noalloc_addr[dev];
    *per_sm = g_noalloc_per_sm[dev];
    return kOk;
}

}  // namespace

}  // namespace vx

using namespace vx;

extern "C" {

int voxel_scan_groupby_dev(const uint64_t* d_packed, size_t nwords, uint32_t width, const int32_t* d_dict,
                           size_t card, const double* d_price, const int32_t* d_qty, size_t n, double pthr,
                           int32_t qlo, int32_t qhi, int32_t* d_keys, double* d_sum, double* d_min, double* d_max,
                           uint64_t* d_count, uint64_t* d_ngroups, void* stream) {
    clear_error();
    int st = ensure_device();
    if (st) return st;
    if (nwords * 64 < n * static_cast<uint64_t>(width)) {
        set_error(kErrInvalidArg, "packed key column has %zu words, %zu rows of %u bits need more", nwords, n, width);
        return kErrInvalidArg;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    return scan_groupby_state().launch(d_packed, width, d_dict, static_cast<uint32_t>(card), d_price, d_qty, n, pthr,
                                       qlo, qhi, d_keys, d_sum, d_min, d_max, d_count, d_ngroups, s);
}

int voxel_scan_groupby_tune(int variant) {
    clear_error();
    // validate before touching the state: a rejected id leaves the previous choice in place
    const bool known = variant == -1 || (variant >= 0 && variant <= 9) || variant == 16;
    if (!known) {
        set_error(kErrInvalidArg, "unknown fused-scan variant %d", variant);
        return kErrInvalidArg;
    }
    ScanGroupBy& S = scan_groupby_state();
    S.autotune = variant == -1;  // -1: the autotuner's choice per shape (word table + queue, 4 rows, untuned)
    if (variant == -1) variant = 1;
    S.use_tw = false;
    S.use_lean = false;
    if (variant == 7) {  // lean word table (16-byte queue entries, screened MIN / MAX)
        S.use_tma = false;
        S.use_lean = true;
        S.mode = 1;
        S.rows_per_thread = 4;
        return kOk;
    }
    if (variant == 0) {
        S.use_tma = true;
        return kOk;
    }
    if (variant == 9) {  // word table + queue with the next tile prefetched into registers
        S.use_tma = false;
        S.mode = 3;
        S.rows_per_thread = 4;
        return kOk;
    }
    if (variant == 6) {  // bulk-copy-fed word table where the shape allows, else variant 1
        S.use_tma = false;
        S.use_tw = true;
        S.mode = 1;
        S.rows_per_thread = 4;
        return kOk;
    }
    if (variant == 1 || variant == 2) {  // 32-bit word table, warp queue; 4 / 8 rows per thread
        S.use_tma = false;
        S.mode = 1;
        S.rows_per_thread = 4 << (variant - 1);
        return kOk;
    }
    if (variant == 3 || variant == 5) {  // 32-bit word table, direct; 4 / 8 rows per thread
        S.use_tma = false;
        S.mode = 2;
        S.rows_per_thread = variant == 3 ? 4 : 8;
        return kOk;
    }
    S.use_tma = false;  // 4, 8, 16: warp-merged rows
    S.mode = 0;
    S.rows_per_thread = variant;
    return kOk;
}

int voxel_scan_groupby_tune_state(void) {
    const ScanGroupBy& S = scan_groupby_state();
    if (S.autotune) return -1;
    if (S.use_lean) return 7;
    if (S.use_tma) return 0;
    if (S.use_tw) return 6;
    if (S.mode == 1) return S.rows_per_thread == 8 ? 2 : 1;
    if (S.mode == 2) return S.rows_per_thread == 8 ? 5 : 3;
    if (S.mode == 3) return 9;
    return S.rows_per_thread;
}

int voxel_scan_groupby_status_code(int status_word) {
    clear_error();
    return groupby_status_error(status_word);
}

int voxel_scan_groupby_check(void* stream) {
    clear_error();
    return scan_groupby_state().check_status(static_cast<cudaStream_t>(stream));
}

int voxel_scan_groupby_last_variant(void) { return scan_groupby_state().last_kernel; }

int voxel_scan_groupby_noalloc_dev(const uint64_t* d_packed, size_t nwords, uint32_t width, const int32_t* d_dict,
                                   size_t card, const double* d_price, const int32_t* d_qty, size_t n, double pthr,
                                   int32_t qlo, int32_t qhi, int32_t* d_keys, double* d_sum, double* d_min,
                                   double* d_max, uint64_t* d_count, uint64_t* d_ngroups, int* d_status,
                                   void* stream) {
    clear_error();
    int st = ensure_device();
    if (st) return st;
    if (card == 0 || card > kMaxGroups) {
        set_error(kErrInvalidArg,
                  "voxel_scan_groupby_noalloc_dev: dictionary of %zu entries; its fixed scratch holds 1..%u groups",
                  card, kMaxGroups);
        return kErrInvalidArg;
    }
    if (width == 0 || width > kMaxWidth) {
        set_error(kErrInvalidArg, "bit width %u outside 1..%d", width, kMaxWidth);
        return kErrInvalidArg;
    }
    if (nwords * 64 < n * static_cast<uint64_t>(width)) {
        set_error(kErrInvalidArg, "packed key column has %zu words, %zu rows of %u bits need more", nwords, n, width);
        return kErrInvalidArg;
    }
    if ((reinterpret_cast<uintptr_t>(d_price) | reinterpret_cast<uintptr_t>(d_qty)) & 15) {
        set_error(kErrInvalidArg, "price / qty columns must be 16-byte aligned");
        return kErrInvalidArg;
    }
    if (!d_status) {
        set_error(kErrInvalidArg, "voxel_scan_groupby_noalloc_dev needs a device status word");
        return kErrInvalidArg;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    unsigned long long* base = nullptr;
    int per_sm = 1;
    st = noalloc_setup(s, &base, &per_sm);
    if (st) return st;
    const size_t G = kMaxGroups;
    GlobalGroups g{base, base + 3 * G, base + 4 * G, base + 5 * G};
    unsigned int* done = reinterpret_cast<unsigned int*>(base + 6 * G);
    constexpr uint64_t kTile = static_cast<uint64_t>(kGbThreads) * 4;
    const uint32_t c32 = static_cast<uint32_t>(card);
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t ntiles = (n + kTile - 1) / kTile;
    uint64_t grid = static_cast<uint64_t>(sms) * per_sm;
    if (grid > ntiles) grid = ntiles;
    if (grid < 1) grid = 1;
    scan_groupby_kernel<4, 0><<<static_cast<unsigned>(grid), kGbThreads, scan_groupby_smem_bytes(c32), s>>>(
        d_packed, width, d_dict, c32, d_price, d_qty, n, pthr, qlo, qhi, g, done, d_keys, d_sum, d_min, d_max,
        d_count, d_ngroups, d_status);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

size_t voxel_scan_groupby(const uint64_t* packed, size_t nwords, uint32_t width, const int32_t* dict, size_t card,
                          const double* price, const int32_t* qty, size_t n, double pthr, int32_t qlo, int32_t qhi,
                          int32_t* out_keys, double* out_sum, double* out_min, double* out_max,
                          uint64_t* out_count) {
    clear_error();
    if (ensure_device()) return static_cast<size_t>(-1);
    cudaStream_t s = thread_stream();
    size_t bytes_words = nwords * 8, bytes_price = n * 8, bytes_qty = n * 4, bytes_dict = card * 4;
    DevBuf dw(bytes_words), dd(bytes_dict), dp(bytes_price), dq(bytes_qty);
    DevBuf ok(card * 4), os(card * 8), omn(card * 8), omx(card * 8), oc(card * 8), ong(8);
    if (!dw.ok(bytes_words) || !dd.ok(bytes_dict) || !dp.ok(bytes_price) || !dq.ok(bytes_qty) || !ok.p || !os.p ||
        !omn.p || !omx.p || !oc.p || !ong.p)
        return static_cast<size_t>(-1);
    if (h2d(dw.p, packed, bytes_words, s) || h2d(dd.p, dict, bytes_dict, s) || h2d(dp.p, price, bytes_price, s) ||
        h2d(dq.p, qty, bytes_qty, s))
        return static_cast<size_t>(-1);
    int st = voxel_scan_groupby_dev(dw.as<uint64_t>(), nwords, width, dd.as<int32_t>(), card, dp.as<double>(),
                                    dq.as<int32_t>(), n, pthr, qlo, qhi, ok.as<int32_t>(), os.as<double>(),
                                    omn.as<double>(), omx.as<double>(), oc.as<uint64_t>(), ong.as<uint64_t>(), s);
    if (st) return static_cast<size_t>(-1);
    if (scan_groupby_state().check_status(s)) return static_cast<size_t>(-1);
    uint64_t ng = 0;
    if (d2h(&ng, ong.p, 8, s) || sync(s)) return static_cast<size_t>(-1);
    if (ng) {
        if (d2h(out_keys, ok.p, ng * 4, s) || d2h(out_sum, os.p, ng * 8, s) || d2h(out_min, omn.p, ng * 8, s) ||
            d2h(out_max, omx.p, ng * 8, s) || d2h(out_count, oc.p, ng * 8, s) || sync(s))
            return static_cast<size_t>(-1);
    }
    return static_cast<size_t>(ng);
}

}  // extern "C"
