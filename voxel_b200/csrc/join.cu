// Hash join build / probe (reference HashJoin<TKey>, include/voxel/ops/join.hpp:36-165).
//
// Reference semantics: Build inserts build row i at the head of its bucket's
// chain (LIFO, 50-56 / 150-165); Probe emits (probe_idx, build_row) for the
// first equal key met on the chain, i.e. the newest build row with that key
// (58-80); ProbeAllMatches emits every equal key, newest first (82-102); both
// walk probe rows in order and stop at maxMatches.
//
// B200 design: the build side is radix-sorted by key (stable, rows ascending
// within a key), so every distinct key owns a run [start, start+len) of build
// rows; an open-addressing table (16-byte slots {key, start, len}, load <= 0.5)
// maps key -> run.  The probe is one pass: each block takes the next tile of
// probe rows, looks each up (one 16-byte load per probe in the common case),
// counts its matches, gets its output offset from a decoupled look-back, and
// writes the pairs newest-first per key, so the pair list comes out in exactly
// the reference's order.  Match count and the u64 sum of build payloads over
// the emitted pairs are reduced per block and added atomically.
#include <vector>

#include "join.h"
#include "join_table.cuh"
#include "radix.h"
#include "voxel_c.h"
#include "vx_common.cuh"
#include "vx_runtime.h"
#include "vx_scan.cuh"

namespace vx {

namespace {

// sorted keys -> runs: flag the first row of every distinct key
__global__ void run_heads_kernel(const int64_t* __restrict__ skeys, uint64_t n, uint32_t* __restrict__ head) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        head[i] = (i == 0 || skeys[i] != skeys[i - 1]) ? 1u : 0u;
}

__global__ void insert_runs_kernel(const int64_t* __restrict__ skeys, const uint32_t* __restrict__ head, uint64_t n,
                                   Slot* __restrict__ table, uint64_t mask, int* err) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (!head[i]) continue;
        int64_t k = skeys[i];
        const uint64_t e = sorted_run_end(skeys, i, n);
        uint32_t len = static_cast<uint32_t>(e - i);
        uint64_t h = mix64(static_cast<uint64_t>(k)) & mask;
        uint64_t probes = 0;
        for (;;) {
            unsigned int* lp = &table[h].len;
            if (atomicCAS(lp, 0u, len) == 0u) {
                table[h].key = k;
                table[h].start = static_cast<uint32_t>(i);
                break;
            }
            h = (h + 1) & mask;
            if (++probes > mask) { atomicOr(err, 8); break; }
        }
    }
}

constexpr int kJThreads = 256;
constexpr int kJItems = 4;  // probes per thread (8 blocks per SM; measured best)
constexpr int kJTile = kJThreads * kJItems;

__global__ void __launch_bounds__(kJThreads, 8) probe_kernel(
    const Slot* __restrict__ table, uint64_t mask, const uint32_t* __restrict__ srows,
    const uint64_t* __restrict__ payload, const int64_t* __restrict__ probe, uint64_t np, int all, uint64_t cap,
    uint32_t* __restrict__ left, uint32_t* __restrict__ right, unsigned long long* count_sum,
    unsigned long long* status, unsigned int* ctr, int* err) {
    __shared__ uint64_t s_tile, s_base;
    __shared__ uint64_t s_warp[kJThreads / 32];
    __shared__ unsigned long long s_sum[kJThreads / 32];
    const uint64_t ntiles = (np + kJTile - 1) / kJTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long my_sum = 0;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        // this thread's probe rows: consecutive, so pairs stay in probe order
        const uint64_t r0 = tile * kJTile + static_cast<uint64_t>(threadIdx.x) * kJItems;
        Slot hit[kJItems];
        uint64_t c = 0;
#pragma unroll
        for (int k = 0; k < kJItems; ++k) {
            uint64_t r = r0 + k;
            if (r < np) {
                hit[k] = lookup(table, mask, __ldcs(probe + r));
                if (!all && hit[k].len > 1) {  // first match only: the newest build row
                    hit[k].start += hit[k].len - 1;
                    hit[k].len = 1;
                }
            } else {
                hit[k].len = 0;
            }
            c += hit[k].len;
        }
        uint64_t inc = c;
        for (int d = 1; d < 32; d <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += y;
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            uint64_t x = lane < kJThreads / 32 ? s_warp[lane] : 0, t = x;
            for (int d = 1; d < 32; d <<= 1) {
                uint64_t y = __shfl_up_sync(0xffffffffu, t, d);
                if (lane >= d) t += y;
            }
            if (lane < kJThreads / 32) s_warp[lane] = t - x;
            const uint64_t tile_total = __shfl_sync(0xffffffffu, t, kJThreads / 32 - 1);
            const uint64_t e = lookback_exclusive_warp(status, tile, tile_total, err);
            if (lane == 0) s_base = e;
        }
        __syncthreads();
        uint64_t pos = s_base + s_warp[warp] + (inc - c);
#pragma unroll
        for (int k = 0; k < kJItems; ++k) {
            for (uint32_t j = 0; j < hit[k].len; ++j) {
                if (pos >= cap) break;
                uint32_t b = __ldg(srows + hit[k].start + hit[k].len - 1 - j);  // newest first
                left[pos] = static_cast<uint32_t>(r0 + k);
                right[pos] = b;
                if (payload) my_sum += __ldg(payload + b);
                ++pos;
            }
        }
        __syncthreads();
    }
    for (int d = 16; d > 0; d >>= 1) my_sum += __shfl_down_sync(0xffffffffu, my_sum, d);
    if (lane == 0) s_sum[warp] = my_sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < kJThreads / 32; ++i) t += s_sum[i];
        atomicAdd(&count_sum[1], t);
    }
}

__global__ void finish_count_kernel(const unsigned long long* status, uint64_t ntiles, uint64_t cap,
                                    unsigned long long* count_sum) {
    uint64_t total = ntiles ? (status[ntiles - 1] & kLbValMask) : 0;
    count_sum[0] = total < cap ? total : cap;
    count_sum[2] = total;
}

__global__ void iota_kernel(uint32_t* out, uint64_t n) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<uint32_t>(i);
}

}  // namespace

void iota_kernel_launch(uint32_t* out, uint64_t n, cudaStream_t s) {
    if (!n) return;
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t b = (n + 255) / 256;
    if (b > static_cast<uint64_t>(sms) * 8) b = static_cast<uint64_t>(sms) * 8;
    iota_kernel<<<static_cast<unsigned>(b), 256, 0, s>>>(out, n);
}

int HashJoinBuild::build(const int64_t* d_keys, uint64_t nb, cudaStream_t s) {
    nbuild = nb;
    uint64_t cap = 64;
    while (cap < 2 * nb) cap <<= 1;  // reference sizing: nextpow2(max(2n, 64)) (join.hpp:37)
    mask = cap - 1;
    table = DevBuf(cap * sizeof(Slot));
    skeys = DevBuf(nb * 8 + 8);
    srows = DevBuf(nb * 4 + 4);
    DevBuf head(nb * 4 + 4);
    if (!table.p || !skeys.p || !srows.p || !head.p) return kErrOutOfMemory;
    VX_CUDA(cudaMemsetAsync(table.p, 0, cap * sizeof(Slot), s));
    if (nb == 0) return kOk;
    VX_CUDA(cudaMemcpyAsync(skeys.p, d_keys, nb * 8, cudaMemcpyDeviceToDevice, s));
    int sms = sm_count() > 0 ? sm_count() : 148;
    int grid = static_cast<int>(nb / 256 + 1 < static_cast<uint64_t>(sms) * 8 ? nb / 256 + 1 : sms * 8);
    iota_kernel_launch(srows.as<uint32_t>(), nb, s);
    size_t tb = radix_tmp_bytes(I64, nb);
    DevBuf tmp(tb);
    if (!tmp.p) return kErrOutOfMemory;
    int st = launch_radix_sort(I64, skeys.p, srows.as<uint32_t>(), nb, tmp.p, tb, radix_err(s), s, nullptr);
    if (st) return st;
    run_heads_kernel<<<grid, 256, 0, s>>>(skeys.as<int64_t>(), nb, head.as<uint32_t>());
    VX_CUDA(cudaGetLastError());
    insert_runs_kernel<<<grid, 256, 0, s>>>(skeys.as<int64_t>(), head.as<uint32_t>(), nb, table.as<Slot>(), mask,
                                            radix_err(s));
    VX_CUDA(cudaGetLastError());
    return sync(s);  // `head` and `tmp` are released when this returns
}

size_t probe_scratch_bytes(uint64_t np) {
    uint64_t ntiles = (np + kJTile - 1) / kJTile;
    return (ntiles + 1) * 8 + 64;
}

int HashJoinBuild::probe(const uint64_t* d_payload, const int64_t* d_probe, uint64_t np, int all, uint64_t cap,
                         uint32_t* d_left, uint32_t* d_right, uint64_t* d_count_sum, void* scratch, int* err,
                         cudaStream_t s) {
    uint64_t ntiles = (np + kJTile - 1) / kJTile;
    unsigned long long* status = static_cast<unsigned long long*>(scratch);
    unsigned int* ctr = reinterpret_cast<unsigned int*>(status + ntiles);
    VX_CUDA(cudaMemsetAsync(scratch, 0, probe_scratch_bytes(np), s));
    VX_CUDA(cudaMemsetAsync(d_count_sum, 0, 24, s));
    if (ntiles) {
        int sms = sm_count() > 0 ? sm_count() : 148;
        uint64_t grid = ntiles < static_cast<uint64_t>(sms) * 8 ? ntiles : static_cast<uint64_t>(sms) * 8;
        probe_kernel<<<static_cast<unsigned>(grid), kJThreads, 0, s>>>(
            table.as<Slot>(), mask, srows.as<uint32_t>(), d_payload, d_probe, np, all, cap, d_left, d_right,
            reinterpret_cast<unsigned long long*>(d_count_sum), status, ctr, err);
        VX_CUDA(cudaGetLastError());
    }
    finish_count_kernel<<<1, 1, 0, s>>>(status, ntiles, cap, reinterpret_cast<unsigned long long*>(d_count_sum));
    VX_CUDA(cudaGetLastError());
    return kOk;
}

}  // namespace vx

using namespace vx;

extern "C" {

int voxel_hashjoin_i64_dev(const int64_t* d_build, const uint64_t* d_payload, size_t nb, const int64_t* d_probe,
                           size_t np, uint32_t* d_left, uint32_t* d_right, size_t max_matches, int all,
                           uint64_t* d_count_sum, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    if (nb >= (1ull << 30) || np >= (1ull << 32)) {
        set_error(kErrInvalidArg, "join sides limited to 2^30 build and 2^32 probe rows (u32 row ids)");
        return kErrInvalidArg;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    HashJoinBuild hb;
    if (int st = hb.build(d_build, nb, s)) return st;
    DevBuf scratch(probe_scratch_bytes(np));
    if (!scratch.p) return kErrOutOfMemory;
    if (int st = hb.probe(d_payload, d_probe, np, all, max_matches, d_left, d_right, d_count_sum, scratch.p,
                          radix_err(s), s))
        return st;
    if (int st = sync(s)) return st;
    return radix_check(s);
}

size_t voxel_hashjoin_i64(const int64_t* build, size_t nb, const int64_t* probe, size_t np, uint32_t* left,
                          uint32_t* right, size_t max_matches, int all) {
    clear_error();
    if (ensure_device()) return static_cast<size_t>(-1);
    cudaStream_t s = thread_stream();
    size_t cap = all ? max_matches : (max_matches < np ? max_matches : np);
    DevBuf db(nb * 8 + 8), dp(np * 8 + 8), dl(cap * 4 + 4), dr(cap * 4 + 4), cs(32);
    if (!db.p || !dp.p || !dl.p || !dr.p || !cs.p) return static_cast<size_t>(-1);
    if (h2d(db.p, build, nb * 8, s) || h2d(dp.p, probe, np * 8, s)) return static_cast<size_t>(-1);
    if (voxel_hashjoin_i64_dev(db.as<int64_t>(), nullptr, nb, dp.as<int64_t>(), np, dl.as<uint32_t>(),
                               dr.as<uint32_t>(), cap, all, cs.as<uint64_t>(), s))
        return static_cast<size_t>(-1);
    uint64_t h[3] = {0, 0, 0};
    if (d2h(h, cs.p, 24, s) || sync(s)) return static_cast<size_t>(-1);
    if (h[0] && (d2h(left, dl.p, h[0] * 4, s) || d2h(right, dr.p, h[0] * 4, s) || sync(s)))
        return static_cast<size_t>(-1);
    return h[0];
}

}  // extern "C"
