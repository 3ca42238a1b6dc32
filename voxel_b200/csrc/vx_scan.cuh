// Single-pass tile prefix (decoupled look-back), shared by the compaction,
// RLE and radix-sort kernels.
//
// Tiles take their index from a global counter in launch order, so a tile
// only ever waits on tiles already owned by a running block.  Each tile
// publishes its aggregate, walks back over its predecessors' published
// aggregates / inclusive prefixes, then publishes its own inclusive prefix.
// Every wait is bounded: when the budget runs out the kernel records an error
// in *err and the tile proceeds with what it has (the host reports
// VOXEL_ETIMEOUT; no spin is unbounded).
//
// A status is one 64-bit word (flag and value together), written with one
// atomic exchange and read with one load, so no fence orders a value against
// its flag; the look-back communicates nothing else, and a publication never
// waits for the tile's earlier output stores to drain.
#pragma once

#include <stdint.h>

namespace vx {

// status word: bits 63..62 flag (0 empty, 1 aggregate, 2 inclusive), 61..0 value
constexpr uint64_t kLbAgg = 1ull << 62;
constexpr uint64_t kLbInc = 2ull << 62;
constexpr uint64_t kLbValMask = (1ull << 62) - 1;
constexpr long long kLbSpinBudget = 1ll << 31;  // clock cycles (~1 s at 2 GHz)

// Returns the exclusive prefix of `tile` (call from one thread of the tile).
__device__ __forceinline__ uint64_t lookback_exclusive(unsigned long long* status, uint64_t tile, uint64_t agg,
                                                       int* err) {
    if (tile == 0) {
        atomicExch(&status[0], kLbInc | (agg & kLbValMask));
        return 0;
    }
    atomicExch(&status[tile], kLbAgg | (agg & kLbValMask));
    uint64_t excl = 0;
    int64_t p = static_cast<int64_t>(tile) - 1;
    long long t0 = clock64();
    while (p >= 0) {
        uint64_t s = *reinterpret_cast<volatile unsigned long long*>(&status[p]);
        uint64_t flag = s & ~kLbValMask;
        if (flag == 0) {
            if (clock64() - t0 > kLbSpinBudget) {
                atomicOr(err, 4);
                break;
            }
            continue;
        }
        excl += s & kLbValMask;
        if (flag == kLbInc) break;
        --p;
    }
    atomicExch(&status[tile], kLbInc | ((excl + agg) & kLbValMask));
    return excl;
}

// Warp-wide variant (call from all 32 lanes of one warp; every lane returns
// the tile's exclusive prefix).  Each step reads the statuses of 32
// predecessors at once (lane i reads p - i), finds the nearest inclusive
// prefix among them with a ballot, and adds the aggregates back to it; it
// spins (bounded) only while an entry inside that window is still empty.
__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ uint64_t lookback_exclusive_warp(unsigned long long* status, uint64_t tile, uint64_t agg,
                                                            int* err) {
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) atomicExch(&status[0], kLbInc | (agg & kLbValMask));
        return 0;
    }
    if (lane == 0) atomicExch(&status[tile], kLbAgg | (agg & kLbValMask));
    uint64_t excl = 0;
    int64_t p = static_cast<int64_t>(tile) - 1;
    const long long t0 = clock64();
    while (p >= 0) {
        const int64_t idx = p - lane;
        // before tile 0: an inclusive prefix of 0
        const uint64_t s = idx >= 0 ? *reinterpret_cast<volatile unsigned long long*>(&status[idx]) : kLbInc;
        const uint64_t flag = s & ~kLbValMask;
        const unsigned inc = __ballot_sync(0xffffffffu, flag == kLbInc);
        const int stop = inc ? __ffs(inc) - 1 : 31;  // lanes 0..stop matter
        const unsigned empty = __ballot_sync(0xffffffffu, flag == 0) & (stop == 31 ? 0xffffffffu : ((2u << stop) - 1));
        if (empty) {
            if (clock64() - t0 > kLbSpinBudget) {
                if (lane == 0) atomicOr(err, 4);
                break;
            }
            continue;
        }
        excl += warp_sum_u64(lane <= stop ? (s & kLbValMask) : 0);
        if (inc) break;
        p -= 32;
    }
    if (lane == 0) atomicExch(&status[tile], kLbInc | ((excl + agg) & kLbValMask));
    return excl;
}

}  // namespace vx
