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
    __threadfence();
    atomicExch(&status[tile], kLbInc | ((excl + agg) & kLbValMask));
    return excl;
}

}  // namespace vx
