// Fused scan + group-by state (global group table, status word).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "vx_runtime.h"

namespace vx {

// Largest dictionary the shared-memory group table holds.
constexpr uint32_t kMaxGroups = 4096;
// Largest dictionary of the fused scan (above kMaxGroups: the global-table path).
constexpr uint32_t kMaxGlobalGroups = 1u << 26;

size_t scan_groupby_smem_bytes(uint32_t card);

struct ScanGroupBy {
    DevBuf table, status, lookback;
    uint32_t card_ = 0;
    unsigned long long *g_sum = nullptr, *g_cnt = nullptr, *g_mn = nullptr, *g_mx = nullptr;
    unsigned long long* g_limb = nullptr;  // dictionaries above kMaxGroups: limbs 0-4, count, min, max per group
    unsigned int* g_done = nullptr;
    int rows_per_thread = 4;  // rows per thread of the shared-table variants: 4, 8 (16: merged only)
    bool use_tma = false;     // TMA-fed private-table variant when the dictionary fits
    bool use_tw = false;      // bulk-copy-fed word table (when the shape allows it)
    bool use_lean = false;    // lean word table (16-byte queue entries, screened MIN / MAX), when n < 2^32
    int mode = 1;             // 0: merged 192-bit atomics, 1: 32-bit word table + warp queue, 2: word table direct
    bool autotune = true;     // pick among the bit-identical word-table variants per shape (unless one was forced)
    int last_grid = 0;
    int last_kernel = 0;      // 0: merged 192-bit atomics, 1: TMA-fed, 2: word table + queue, 3: word table direct,
                              // 4: bulk-copy-fed word table, 5: lean word table,
                              // 6: slot caches spilling to the HBM table (dictionaries above kMaxGroups),
                              // 7: word table with next-tile prefetch

    int prepare(uint32_t card, cudaStream_t s);
    int launch(const uint64_t* packed, uint32_t width, const int32_t* dict, uint32_t card, const double* price,
               const int32_t* qty, uint64_t n, double pthr, int32_t qlo, int32_t qhi, int32_t* out_keys,
               double* out_sum, double* out_min, double* out_max, uint64_t* out_count, uint64_t* out_ngroups,
               cudaStream_t s);
    // reads (and clears) the kernel's status word; synchronises the stream
    int check_status(cudaStream_t s);
};

ScanGroupBy& scan_groupby_state();

}  // namespace vx
