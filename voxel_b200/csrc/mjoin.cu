// Merge, semi and anti joins (reference include/voxel/ops/join.hpp:216-310).
//
//   MergeJoin<TKey>::Join (218-244), over keys sorted ascending: for each left
//     row li in order, every right row ri of the equal-key run, ascending
//     (the right cursor rewinds to the run start for the next left row), so a
//     key with p left and q right rows gives p*q pairs, left-major.
//   MergeJoin<TKey>::JoinUnique (246-268): both cursors advance on a match, so
//     the t-th left row of a key's run pairs with the t-th right row of the
//     same key while t < q.
//   SemiJoin / AntiJoin<TKey>::Join (294-310 / 273-290): the left rows (in
//     order) whose key is / is not in a hash set of the right keys
//     (HashJoin::Build + Contains); no order is assumed.
//
// B200 design: one pass over the left rows in tiles claimed in launch order.
// Merge joins: a tile finds the window of right rows that can match its keys
// with two binary searches, each row then binary-searches its key's run
// inside that window (and, for JoinUnique, its own position in the left
// run), counts its pairs, takes its output offset from a decoupled look-back
// and writes its pairs, so the pair list is exactly the reference's order.
// Semi / anti joins: the right keys go through the hash-join build (sorted
// runs + open-addressing table of distinct keys); each left row is one table
// lookup, and the passing row ids are compacted in order the same way.
#include <cstdint>

#include "join.h"
#include "join_table.cuh"
#include "radix.h"
#include "voxel_c.h"
#include "vx_common.cuh"
#include "vx_runtime.h"
#include "vx_scan.cuh"

namespace vx {

namespace {

constexpr int kMThreads = 256;
constexpr int kMItems = 4;  // left rows per thread (consecutive)
constexpr int kMTile = kMThreads * kMItems;

// first index in [lo, hi) with a[idx] >= k (UPPER: > k)
template <typename T, bool UPPER>
__device__ __forceinline__ uint64_t bsearch(const T* __restrict__ a, uint64_t lo, uint64_t hi, T k) {
    while (lo < hi) {
        const uint64_t mid = lo + ((hi - lo) >> 1);
        const T v = __ldg(a + mid);
        if (UPPER ? !(k < v) : (v < k)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Exclusive tile offset from per-thread counts c (all threads call); writes
// the thread's first output position to *pos.
__device__ __forceinline__ uint64_t tile_offsets(uint64_t c, uint64_t tile, unsigned long long* status, int* err,
                                                 uint64_t* s_warp, uint64_t* s_base) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t inc = c;
    for (int d = 1; d < 32; d <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint64_t x = lane < kMThreads / 32 ? s_warp[lane] : 0;
        uint64_t t = x;
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, t, d);
            if (lane >= d) t += y;
        }
        if (lane < kMThreads / 32) s_warp[lane] = t - x;
        const uint64_t total = __shfl_sync(0xffffffffu, t, kMThreads / 32 - 1);
        const uint64_t e = lookback_exclusive_warp(status, tile, total, err);
        if (lane == 0) *s_base = e;
    }
    __syncthreads();
    return *s_base + s_warp[warp] + (inc - c);
}

template <typename T, bool UNIQUE>
__global__ void __launch_bounds__(kMThreads) merge_join_kernel(const T* __restrict__ left, uint64_t nl,
                                                               const T* __restrict__ right, uint64_t nr,
                                                               uint64_t cap, uint32_t* __restrict__ lout,
                                                               uint32_t* __restrict__ rout,
                                                               unsigned long long* status, unsigned int* ctr,
                                                               int* err) {
    __shared__ uint64_t s_tile, s_base, s_rlo, s_rhi, s_llo;
    __shared__ uint64_t s_warp[kMThreads / 32];
    const uint64_t ntiles = (nl + kMTile - 1) / kMTile;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t t0 = tile * kMTile;
        const uint64_t t1 = t0 + kMTile < nl ? t0 + kMTile : nl;
        if (threadIdx.x == 0) {
            // the right rows any key of this tile can match, and where the
            // left run of the tile's first key starts
            s_rlo = bsearch<T, false>(right, 0, nr, __ldg(left + t0));
            s_rhi = bsearch<T, true>(right, s_rlo, nr, __ldg(left + t1 - 1));
            s_llo = UNIQUE ? bsearch<T, false>(left, 0, t0 + 1, __ldg(left + t0)) : 0;
        }
        __syncthreads();
        const uint64_t rlo = s_rlo, rhi = s_rhi, llo = s_llo;
        const uint64_t r0 = t0 + static_cast<uint64_t>(threadIdx.x) * kMItems;
        uint64_t rb[kMItems];
        uint32_t cnt[kMItems];
        uint64_t c = 0;
#pragma unroll
        for (int k = 0; k < kMItems; ++k) {
            const uint64_t i = r0 + k;
            cnt[k] = 0;
            rb[k] = 0;
            if (i >= t1) continue;
            const T key = __ldg(left + i);
            const uint64_t b = bsearch<T, false>(right, rlo, rhi, key);
            const uint64_t e = bsearch<T, true>(right, b, rhi, key);
            if (UNIQUE) {
                const uint64_t ls = bsearch<T, false>(left, llo, i + 1, key);  // the left run's first row
                const uint64_t t = i - ls;
                if (t < e - b) {
                    cnt[k] = 1;
                    rb[k] = b + t;
                }
            } else {
                cnt[k] = static_cast<uint32_t>(e - b);
                rb[k] = b;
            }
            c += cnt[k];
        }
        uint64_t pos = tile_offsets(c, tile, status, err, s_warp, &s_base);
#pragma unroll
        for (int k = 0; k < kMItems; ++k) {
            for (uint32_t j = 0; j < cnt[k] && pos < cap; ++j, ++pos) {
                lout[pos] = static_cast<uint32_t>(r0 + k);
                rout[pos] = static_cast<uint32_t>(rb[k] + j);
            }
        }
        __syncthreads();
    }
}

template <typename T, bool ANTI>
__global__ void __launch_bounds__(kMThreads) semi_join_kernel(const Slot* __restrict__ table, uint64_t mask,
                                                              const T* __restrict__ left, uint64_t nl,
                                                              uint32_t* __restrict__ out,
                                                              unsigned long long* status, unsigned int* ctr,
                                                              int* err) {
    __shared__ uint64_t s_tile, s_base;
    __shared__ uint64_t s_warp[kMThreads / 32];
    const uint64_t ntiles = (nl + kMTile - 1) / kMTile;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t r0 = tile * kMTile + static_cast<uint64_t>(threadIdx.x) * kMItems;
        uint32_t pass = 0;
#pragma unroll
        for (int k = 0; k < kMItems; ++k) {
            const uint64_t i = r0 + k;
            if (i >= nl) continue;
            const bool found = lookup(table, mask, static_cast<int64_t>(__ldcs(left + i))).len != 0;
            if (found != ANTI) pass |= 1u << k;
        }
        uint64_t pos = tile_offsets(__popc(pass), tile, status, err, s_warp, &s_base);
#pragma unroll
        for (int k = 0; k < kMItems; ++k)
            if (pass >> k & 1u) out[pos++] = static_cast<uint32_t>(r0 + k);
        __syncthreads();
    }
}

// keys of T widened to i64 (sign- or zero-extended): equality is unchanged
template <typename T>
__global__ void widen_kernel(const T* __restrict__ in, uint64_t n, int64_t* __restrict__ out) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<int64_t>(in[i]);
}

// (l << 32) | (2^32 - 1 - r): ascending order = left row ascending, then right
// row descending (the order HashJoin::ProbeAllMatches emits with the right
// side built: probe rows in order, each key's build rows newest first)
__global__ void pair_key_kernel(const uint32_t* __restrict__ l, const uint32_t* __restrict__ r, uint64_t m,
                                uint64_t* __restrict__ key, uint32_t* __restrict__ idx) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        key[i] = (static_cast<uint64_t>(l[i]) << 32) | (0xFFFFFFFFull - r[i]);
        idx[i] = static_cast<uint32_t>(i);
    }
}

__global__ void pair_split_kernel(const uint64_t* __restrict__ key, uint64_t m, uint32_t* __restrict__ l,
                                  uint32_t* __restrict__ r) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        l[i] = static_cast<uint32_t>(key[i] >> 32);
        r[i] = static_cast<uint32_t>(0xFFFFFFFFull - (key[i] & 0xFFFFFFFFull));
    }
}

__global__ void total_kernel(const unsigned long long* status, uint64_t ntiles, uint64_t cap,
                             unsigned long long* out2) {
    const uint64_t total = ntiles ? (status[ntiles - 1] & kLbValMask) : 0;
    out2[0] = total < cap ? total : cap;
    out2[1] = total;
}

int grid_for_tiles(uint64_t ntiles) {
    const int sms = sm_count() > 0 ? sm_count() : 148;
    const uint64_t cap = static_cast<uint64_t>(sms) * 8;
    return static_cast<int>(ntiles < cap ? (ntiles ? ntiles : 1) : cap);
}

bool key_type(int dtype) { return dtype == I64 || dtype == I32 || dtype == U64 || dtype == U32; }

template <typename T>
int merge_t(const void* l, uint64_t nl, const void* r, uint64_t nr, uint64_t cap, uint32_t* lo, uint32_t* ro,
            int unique, unsigned long long* status, unsigned int* ctr, int* err, cudaStream_t s) {
    const uint64_t ntiles = (nl + kMTile - 1) / kMTile;
    if (unique)
        merge_join_kernel<T, true><<<grid_for_tiles(ntiles), kMThreads, 0, s>>>(
            static_cast<const T*>(l), nl, static_cast<const T*>(r), nr, cap, lo, ro, status, ctr, err);
    else
        merge_join_kernel<T, false><<<grid_for_tiles(ntiles), kMThreads, 0, s>>>(
            static_cast<const T*>(l), nl, static_cast<const T*>(r), nr, cap, lo, ro, status, ctr, err);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

template <typename T>
int semi_t(const Slot* table, uint64_t mask, const void* l, uint64_t nl, uint32_t* out, int anti,
           unsigned long long* status, unsigned int* ctr, int* err, cudaStream_t s) {
    const uint64_t ntiles = (nl + kMTile - 1) / kMTile;
    if (anti)
        semi_join_kernel<T, true><<<grid_for_tiles(ntiles), kMThreads, 0, s>>>(table, mask, static_cast<const T*>(l),
                                                                              nl, out, status, ctr, err);
    else
        semi_join_kernel<T, false><<<grid_for_tiles(ntiles), kMThreads, 0, s>>>(
            table, mask, static_cast<const T*>(l), nl, out, status, ctr, err);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

// status words for ntiles tiles, the tile counter, then the (pairs, total) pair
struct Scratch {
    DevBuf buf;
    unsigned long long* status = nullptr;
    unsigned int* ctr = nullptr;
    unsigned long long* out2 = nullptr;
    int init(uint64_t ntiles, cudaStream_t s) {
        const size_t need = (ntiles + 1) * 8 + 16 + 64;
        buf = DevBuf(need);
        if (!buf.p) return kErrOutOfMemory;
        status = buf.as<unsigned long long>();
        ctr = reinterpret_cast<unsigned int*>(status + ntiles);
        out2 = reinterpret_cast<unsigned long long*>(static_cast<char*>(buf.p) + ((ntiles + 1) * 8 + 15) / 16 * 16);
        VX_CUDA(cudaMemsetAsync(buf.p, 0, need, s));
        return kOk;
    }
};

int finish(const Scratch& sc, uint64_t ntiles, uint64_t cap, uint64_t* d_count2, cudaStream_t s) {
    total_kernel<<<1, 1, 0, s>>>(sc.status, ntiles, cap, sc.out2);
    VX_CUDA(cudaGetLastError());
    if (d_count2) VX_CUDA(cudaMemcpyAsync(d_count2, sc.out2, 16, cudaMemcpyDeviceToDevice, s));
    return kOk;
}

}  // namespace

}  // namespace vx

using namespace vx;

extern "C" {

int voxel_merge_join_dev(int dtype, const void* d_left, size_t nl, const void* d_right, size_t nr, uint32_t* d_lout,
                         uint32_t* d_rout, size_t max_matches, int unique, uint64_t* d_count2, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    if (!key_type(dtype)) {
        set_error(kErrInvalidArg, "merge join: element type %d is not an integer key type", dtype);
        return kErrInvalidArg;
    }
    if (nl >= (1ull << 32) || nr >= (1ull << 32)) {
        set_error(kErrInvalidArg, "merge join sides limited to 2^32 rows (u32 row ids)");
        return kErrInvalidArg;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint64_t ntiles = (nl + kMTile - 1) / kMTile;
    Scratch sc;
    if (int st = sc.init(ntiles, s)) return st;
    int* err = radix_err(s);
    if (nl && nr) {
        int st = kOk;
        switch (dtype) {
        case I64: st = merge_t<int64_t>(d_left, nl, d_right, nr, max_matches, d_lout, d_rout, unique, sc.status, sc.ctr, err, s); break;
        case I32: st = merge_t<int32_t>(d_left, nl, d_right, nr, max_matches, d_lout, d_rout, unique, sc.status, sc.ctr, err, s); break;
        case U64: st = merge_t<uint64_t>(d_left, nl, d_right, nr, max_matches, d_lout, d_rout, unique, sc.status, sc.ctr, err, s); break;
        default: st = merge_t<uint32_t>(d_left, nl, d_right, nr, max_matches, d_lout, d_rout, unique, sc.status, sc.ctr, err, s); break;
        }
        if (st) return st;
    }
    if (int st = finish(sc, nl && nr ? ntiles : 0, max_matches, d_count2, s)) return st;
    if (int st = sync(s)) return st;  // the scratch is released on return
    return radix_check(s);
}

int voxel_semi_join_dev(int dtype, const void* d_left, size_t nl, const void* d_right, size_t nr, uint32_t* d_out,
                        int anti, uint64_t* d_count, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    if (!key_type(dtype)) {
        set_error(kErrInvalidArg, "semi / anti join: element type %d is not an integer key type", dtype);
        return kErrInvalidArg;
    }
    if (nl >= (1ull << 32) || nr >= (1ull << 30)) {
        set_error(kErrInvalidArg, "semi / anti join limited to 2^32 left and 2^30 right rows");
        return kErrInvalidArg;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the right keys as i64 for the hash-join build
    DevBuf wide;
    const int64_t* rk = static_cast<const int64_t*>(d_right);
    if (dtype != I64 && dtype != U64) {
        wide = DevBuf(nr * 8 + 8);
        if (!wide.p) return kErrOutOfMemory;
        const int sms = sm_count() > 0 ? sm_count() : 148;
        const unsigned g = static_cast<unsigned>(nr / 256 + 1 < static_cast<uint64_t>(sms) * 8 ? nr / 256 + 1 : sms * 8);
        if (dtype == I32)
            widen_kernel<int32_t><<<g, 256, 0, s>>>(static_cast<const int32_t*>(d_right), nr, wide.as<int64_t>());
        else
            widen_kernel<uint32_t><<<g, 256, 0, s>>>(static_cast<const uint32_t*>(d_right), nr, wide.as<int64_t>());
        VX_CUDA(cudaGetLastError());
        rk = wide.as<int64_t>();
    }
    HashJoinBuild hb;
    if (int st = hb.build(rk, nr, s)) return st;
    const uint64_t ntiles = (nl + kMTile - 1) / kMTile;
    Scratch sc;
    if (int st = sc.init(ntiles, s)) return st;
    int* err = radix_err(s);
    if (nl) {
        int st = kOk;
        switch (dtype) {
        case I64: st = semi_t<int64_t>(hb.table.as<Slot>(), hb.mask, d_left, nl, d_out, anti, sc.status, sc.ctr, err, s); break;
        case I32: st = semi_t<int32_t>(hb.table.as<Slot>(), hb.mask, d_left, nl, d_out, anti, sc.status, sc.ctr, err, s); break;
        case U64: st = semi_t<uint64_t>(hb.table.as<Slot>(), hb.mask, d_left, nl, d_out, anti, sc.status, sc.ctr, err, s); break;
        default: st = semi_t<uint32_t>(hb.table.as<Slot>(), hb.mask, d_left, nl, d_out, anti, sc.status, sc.ctr, err, s); break;
        }
        if (st) return st;
    }
    if (int st = finish(sc, nl ? ntiles : 0, ~0ull, nullptr, s)) return st;
    if (d_count) VX_CUDA(cudaMemcpyAsync(d_count, sc.out2, 8, cudaMemcpyDeviceToDevice, s));
    if (int st = sync(s)) return st;
    return radix_check(s);
}

// Pairs of a join built on the LEFT side and probed with the right (d_probe =
// right row ids, d_build = left row ids) put into the order of the same join
// built on the right and probed with the left: left rows ascending, each
// left row's right rows descending.  Lets a planner build on the smaller side
// and still return the reference's pair list.
int voxel_join_pairs_swap_order_dev(const uint32_t* d_probe, const uint32_t* d_build, size_t m, uint32_t* d_left,
                                    uint32_t* d_right, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    if (m == 0) return kOk;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DevBuf key(m * 8), idx(m * 4);
    if (!key.p || !idx.p) return kErrOutOfMemory;
    const int sms = sm_count() > 0 ? sm_count() : 148;
    const unsigned g = static_cast<unsigned>(m / 256 + 1 < static_cast<uint64_t>(sms) * 8 ? m / 256 + 1 : sms * 8);
    pair_key_kernel<<<g, 256, 0, s>>>(d_build, d_probe, m, key.as<uint64_t>(), idx.as<uint32_t>());
    VX_CUDA(cudaGetLastError());
    const size_t tb = radix_tmp_bytes(U64, m);
    DevBuf tmp(tb);
    if (!tmp.p) return kErrOutOfMemory;
    if (int st = launch_radix_sort(U64, key.p, idx.as<uint32_t>(), m, tmp.p, tb, radix_err(s), s, nullptr)) return st;
    pair_split_kernel<<<g, 256, 0, s>>>(key.as<uint64_t>(), m, d_left, d_right);
    VX_CUDA(cudaGetLastError());
    if (int st = sync(s)) return st;
    return radix_check(s);
}

size_t voxel_merge_join(int dtype, const void* left, size_t nl, const void* right, size_t nr, uint32_t* lout,
                        uint32_t* rout, size_t max_matches, int unique) {
    clear_error();
    if (ensure_device()) return static_cast<size_t>(-1);
    if (!key_type(dtype)) {
        set_error(kErrInvalidArg, "merge join: element type %d is not an integer key type", dtype);
        return static_cast<size_t>(-1);
    }
    cudaStream_t s = thread_stream();
    const size_t es = dtype_size(dtype);
    DevBuf dl(nl * es + 8), dr(nr * es + 8), ol(max_matches * 4 + 4), orr(max_matches * 4 + 4), c2(16);
    if (!dl.p || !dr.p || !ol.p || !orr.p || !c2.p) return static_cast<size_t>(-1);
    if (h2d(dl.p, left, nl * es, s) || h2d(dr.p, right, nr * es, s)) return static_cast<size_t>(-1);
    if (voxel_merge_join_dev(dtype, dl.p, nl, dr.p, nr, ol.as<uint32_t>(), orr.as<uint32_t>(), max_matches, unique,
                             c2.as<uint64_t>(), s))
        return static_cast<size_t>(-1);
    uint64_t h[2] = {0, 0};
    if (d2h(h, c2.p, 16, s) || sync(s)) return static_cast<size_t>(-1);
    if (h[0] && (d2h(lout, ol.p, h[0] * 4, s) || d2h(rout, orr.p, h[0] * 4, s) || sync(s)))
        return static_cast<size_t>(-1);
    return h[0];
}

size_t voxel_semi_join(int dtype, const void* left, size_t nl, const void* right, size_t nr, uint32_t* out,
                       int anti) {
    clear_error();
    if (ensure_device()) return static_cast<size_t>(-1);
    if (!key_type(dtype)) {
        set_error(kErrInvalidArg, "semi / anti join: element type %d is not an integer key type", dtype);
        return static_cast<size_t>(-1);
    }
    cudaStream_t s = thread_stream();
    const size_t es = dtype_size(dtype);
    DevBuf dl(nl * es + 8), dr(nr * es + 8), o(nl * 4 + 4), c(16);
    if (!dl.p || !dr.p || !o.p || !c.p) return static_cast<size_t>(-1);
    if (h2d(dl.p, left, nl * es, s) || h2d(dr.p, right, nr * es, s)) return static_cast<size_t>(-1);
    if (voxel_semi_join_dev(dtype, dl.p, nl, dr.p, nr, o.as<uint32_t>(), anti, c.as<uint64_t>(), s))
        return static_cast<size_t>(-1);
    uint64_t h = 0;
    if (d2h(&h, c.p, 8, s) || sync(s)) return static_cast<size_t>(-1);
    if (h && (d2h(out, o.p, h * 4, s) || sync(s))) return static_cast<size_t>(-1);
    return h;
}

}  // extern "C"
