// Stable LSD radix sort: launch interface.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace vx {

size_t radix_tmp_bytes(int dtype, uint64_t n);
// keys (dtype 2..5) and idx sorted in place; *passes = digit passes executed
int launch_radix_sort(int dtype, void* keys, uint32_t* idx, uint64_t n, void* tmp, size_t tmp_bytes, int* err,
                      cudaStream_t s, int* passes);
int* radix_err(cudaStream_t s);
int radix_check(cudaStream_t s);

}  // namespace vx
