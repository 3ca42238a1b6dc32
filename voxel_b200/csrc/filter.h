// VectorFilter / ColumnFilter / SelectionVector kernels: launch interface.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>

namespace vx {

// bitmap of rows passing `op` (0..5 compare with a, 6 = a <= v <= b); *count = passes
int launch_vfilter(int dtype, const void* d, uint64_t n, int op, uint64_t a_bits, uint64_t b_bits, uint64_t* bitmap,
                   unsigned long long* count, cudaStream_t s);
// ascending row ids of set bits; scratch from selection_scratch_bytes(rows)
size_t selection_scratch_bytes(uint64_t rows);
int launch_selection(const uint64_t* bitmap, uint64_t rows, uint32_t* out, unsigned long long* count, void* scratch,
                     int* err, cudaStream_t s);
int launch_bitmap_and(const uint64_t* const* d_bitmaps, int nbm, uint64_t rows, uint64_t* out,
                      unsigned long long* count, cudaStream_t s);
// up to kAndInline bitmaps whose device pointers sit in a host array: passed
// to the kernel by value (no pointer table is uploaded)
constexpr int kAndInline = 16;
struct BitmapList {
    const uint64_t* p[kAndInline];
};
int launch_bitmap_and_host_list(const uint64_t* const* h_bitmaps, int nbm, uint64_t rows, uint64_t* out,
                                unsigned long long* count, cudaStream_t s);

}  // namespace vx
