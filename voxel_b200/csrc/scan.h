// Fused filter/compare/aggregate scan: launch interface.
#pragma once

#include <cuda_runtime.h>

#include "vx_types.h"

namespace vx {

// Scratch the scan kernel needs between its blocks: per-block partials plus a
// completion counter (zeroed once; each launch's last block re-zeroes it).
size_t scan_scratch_bytes();
int scan_scratch_init(void* scratch, cudaStream_t s);

// One fused launch over the lowered loop described by `p`; the final register
// values land in *d_out (device memory).  Returns a Status.
int launch_scan(const ScanParams& p, ScanResult* d_out, void* scratch, cudaStream_t s);

// Which kernel launch_scan runs for `p`: "fsum" (one atom, one masked SUM),
// "range" (one reduction over an interval), "mrange" (2-4 reductions sharing
// one interval) or "generic" (per-lane interpretation).  Host code only.
const char* scan_kernel_name(const ScanParams& p);

// Number of blocks launch_scan uses for `ngroups` groups of element type dt.
int scan_grid(int dtype, uint64_t ndata, int ncols, int nred);

// Segment aggregate (AGG_COUNT/SUM/MIN/MAX over rows [begin, end) of a column,
// engine.hpp:499-569).  kind: 0 count(nonzero) 1 sum 3 min 4 max.  Writes a
// 3-word result {u64 count | i64 sum | T-bits min/max, f64 sum, f64 compensation}.
// Min/max start from init_bits (the slot's running value).
int launch_segment_agg(int dtype, const void* col, uint64_t begin, uint64_t end, int kind,
                       uint64_t init_bits, uint64_t* d_out3, void* scratch, cudaStream_t s);

}  // namespace vx
