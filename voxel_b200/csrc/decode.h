// Column decoders: launch interface.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace vx {

int launch_bitunpack(const uint64_t* words, uint64_t nwords, uint32_t w, uint64_t value_count, uint64_t offset,
                     uint64_t count, uint32_t* out, cudaStream_t s);
int launch_dict_bitunpack_i32(const uint64_t* words, uint64_t nwords, uint32_t w, const int32_t* dict, uint32_t card,
                              uint64_t value_count, uint64_t offset, uint64_t count, int32_t* out, int* err,
                              cudaStream_t s);
int launch_dict_gather(int dtype, const void* dict, uint32_t card, const uint32_t* idx, uint64_t count, void* out,
                       int* err, cudaStream_t s);
size_t rle_scratch_bytes(uint64_t nruns);
int launch_rle_decode_i64(const int64_t* values, const uint32_t* runs, uint64_t nruns, uint64_t offset,
                          uint64_t count, int64_t* out, void* scratch, int* err, cudaStream_t s);

// delta.cu: DeltaEncoding / FrameOfReferenceEncoding codecs
size_t delta_scratch_bytes(uint64_t limit);
int launch_delta_decode(int dtype, const void* deltas, uint64_t n, uint64_t base_bits, uint64_t offset,
                        uint64_t count, void* out, void* scratch, int* err, cudaStream_t s);
int launch_delta_encode(int dtype, const void* data, uint64_t n, void* deltas, cudaStream_t s);
int launch_for_decode_f64(const int32_t* code, uint64_t n, double base, double scale, uint64_t offset,
                          uint64_t count, double* out, cudaStream_t s);

}  // namespace vx
