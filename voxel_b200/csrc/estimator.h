// Learned estimator: column sketches, exact labels and the FP32 MLP.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "vx_runtime.h"

namespace vx {

constexpr int kHllP = 12;
constexpr int kHllRegs = 1 << kHllP;
constexpr int kHistBins = 64;

// Per-column device sketch, copied to the host (plain C layout for the ABI).
struct ColumnSketch {
    uint64_t n;
    double min, max;
    uint64_t hist[kHistBins];  // equi-width over [min, max]
    uint8_t hll[kHllRegs];     // HyperLogLog registers (p = 12)
};

// Up to 4 conjunctive "value op threshold" atoms (T bits), as in a program.
struct PredSet {
    int32_t natoms;
    int32_t op[4];
    int32_t pad;
    uint64_t thr[4];
};

struct Mlp {
    DevBuf params, mom, vel, gbuf, lbuf;
    int step = 0;
    int last_blocks = 0;
    int init(uint64_t seed, cudaStream_t s);
    int set_params(const float* host, cudaStream_t s);
    int get_params(float* host, cudaStream_t s) const;
    // gradient of the summed squared error over samples idx[0..m); optional host copies
    int grad(const float* dX, const float* dY, const uint32_t* didx, uint32_t m, float* host_grad, float* host_loss,
             cudaStream_t s);
    int adam_step(uint32_t m, float lr, cudaStream_t s);
    int infer(const float* dX, uint64_t n, float* dY, cudaStream_t s);
};

int sketch_column(int dtype, const void* d, uint64_t n, ColumnSketch* out, cudaStream_t s);
int exact_labels(int dtype, const void* d, uint64_t n, const PredSet* sets, uint32_t nsets, uint64_t* rows,
                 uint64_t* distinct, cudaStream_t s);

}  // namespace vx
