// Hash join: build-side table and probe launch.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "vx_runtime.h"

namespace vx {

// fills out[i] = i for i < n
void iota_kernel_launch(uint32_t* out, uint64_t n, cudaStream_t s);

struct HashJoinBuild {
    DevBuf table, skeys, srows;
    uint64_t mask = 0, nbuild = 0;
    // sorts the build keys (stable, with row ids) and inserts one slot per distinct key
    int build(const int64_t* d_keys, uint64_t nb, cudaStream_t s);
    // d_count_sum[0] = emitted pairs (<= cap), [1] = u64 sum of payload over them, [2] = all matches
    int probe(const uint64_t* d_payload, const int64_t* d_probe, uint64_t np, int all, uint64_t cap,
              uint32_t* d_left, uint32_t* d_right, uint64_t* d_count_sum, void* scratch, int* err, cudaStream_t s);
};

size_t probe_scratch_bytes(uint64_t np);

}  // namespace vx
