// Learned cardinality / selectivity estimator (no reference counterpart; the
// closest reference structure is the per-segment zone map,
// include/voxel/data/segment.hpp:187-211).
//
//   Column sketches (one pass after min/max): min / max, a 64-bucket
//   equi-width histogram over [min, max], and HyperLogLog registers (p = 12,
//   splitmix64 of the value's bits) for the distinct count.
//
//   Exact labels: a column's sorted unique values with their multiplicities
//   (radix sort + run counts) let one small kernel measure, for many
//   predicate sets at once, the exact number of selected rows and of distinct
//   selected values.
//
//   MLP 48 -> 64 -> 64 -> 64 -> 2 (ReLU), 11,586 FP32 parameters, trained on the
//   GPU with hand-written kernels: each block runs forward + backward for its
//   slice of the minibatch with the weights staged in shared memory and owns
//   its gradient entries (no atomics), a second kernel reduces the per-block
//   gradients in block order and applies Adam.  Inference uses the same
//   forward.  Estimates only size buffers and choose plans: results never
//   depend on them (an underestimate falls back to the exact two-pass path).
#include <cmath>
#include <cstring>
#include <vector>

#include "estimator.h"
#include "radix.h"
#include "voxel_c.h"
#include "vx_common.cuh"
#include "vx_runtime.h"

namespace vx {

namespace {

constexpr int kIn = 48, kH = 64, kOut = 2;
constexpr int kL1 = kH * kIn + kH;      // 3136
constexpr int kL2 = kH * kH + kH;       // 4160
constexpr int kL3 = kH * kH + kH;       // 4160
constexpr int kL4 = kOut * kH + kOut;   // 130
constexpr int kParams = kL1 + kL2 + kL3 + kL4;  // 11586
static_assert(kParams == 11586, "MLP parameter count");
constexpr int kMThreads = 256;
constexpr int kChunk = 8;  // samples per block step

// ---- sketches ---------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ double as_double(T v) { return static_cast<double>(v); }

__device__ __forceinline__ uint64_t splitmix(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

template <typename T>
__global__ void minmax_hll_kernel(const T* __restrict__ col, uint64_t n, unsigned long long* mnk,
                                  unsigned long long* mxk, unsigned int* hll) {
    __shared__ unsigned int sh[kHllRegs];
    for (int i = threadIdx.x; i < kHllRegs; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    double lo = INFINITY, hi = -INFINITY;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    // four elements in flight per thread: loads first, then the updates
    for (uint64_t i0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i0 < n; i0 += 4 * stride) {
        T vv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint64_t i = i0 + u * stride;
            vv[u] = i < n ? __ldcs(col + i) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (i0 + u * stride >= n) break;
            const T v = vv[u];
            double d = as_double(v);
            lo = d < lo ? d : lo;
            hi = d > hi ? d : hi;
            uint64_t h = splitmix(to_bits<T>(v));
            uint32_t reg = static_cast<uint32_t>(h >> (64 - kHllP));
            uint64_t rest = h << kHllP;
            uint32_t rank = rest ? static_cast<uint32_t>(__clzll(static_cast<long long>(rest))) + 1 : 64 - kHllP + 1;
            if (rank > sh[reg]) atomicMax(&sh[reg], rank);
        }
    }
    auto okey = [](double x) {
        uint64_t b = static_cast<uint64_t>(__double_as_longlong(x));
        return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
    };
    for (int d = 16; d > 0; d >>= 1) {
        lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, d));
        hi = fmax(hi, __shfl_down_sync(0xffffffffu, hi, d));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(mnk, okey(lo));
        atomicMax(mxk, okey(hi));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kHllRegs; i += blockDim.x)
        if (sh[i]) atomicMax(&hll[i], sh[i]);
}

// order key (minmax_hll_kernel's okey) -> the double
__host__ __device__ __forceinline__ double from_order_key(unsigned long long k) {
    const uint64_t b = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
    double x;
    memcpy(&x, &b, 8);
    return x;
}

// bins [lo, hi] (read from the min / max order keys the first pass left in
// device memory, so no host round trip sits between the passes) in 64 equal widths
template <typename T>
__global__ void histogram64_kernel(const T* __restrict__ col, uint64_t n, const unsigned long long* mnk,
                                   const unsigned long long* mxk, unsigned long long* hist) {
    __shared__ unsigned int sh[kHistBins];
    if (threadIdx.x < kHistBins) sh[threadIdx.x] = 0;
    __syncthreads();
    const double lo = from_order_key(*mnk), hi = from_order_key(*mxk);
    double w = hi > lo ? (hi - lo) / kHistBins : 1.0;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i0 < n; i0 += 4 * stride) {
        T vv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint64_t i = i0 + u * stride;
            vv[u] = i < n ? __ldcs(col + i) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (i0 + u * stride >= n) break;
            double d = as_double(vv[u]);
            int b = static_cast<int>((d - lo) / w);
            b = b < 0 ? 0 : (b >= kHistBins ? kHistBins - 1 : b);
            atomicAdd(&sh[b], 1u);
        }
    }
    __syncthreads();
    if (threadIdx.x < kHistBins && sh[threadIdx.x]) atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
}

// ---- exact labels over unique values -------------------------------------------------

template <typename T>
__global__ void to_sort_key_kernel(const T* __restrict__ col, uint64_t n, uint64_t* key, uint32_t* idx) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        T v = col[i];
        uint64_t b = to_bits<T>(v);
        uint64_t k;
        if constexpr (std::is_same<T, double>::value) {
            if (v == 0.0) b = 0;
            k = (b >> 63) ? ~b : (b | 0x8000000000000000ull);
        } else if constexpr (std::is_same<T, float>::value) {
            if (v == 0.0f) b = 0;
            uint32_t u = static_cast<uint32_t>(b);
            k = (u >> 31) ? (~u & 0xFFFFFFFFu) : (u | 0x80000000u);
        } else if constexpr (std::is_signed<T>::value) {
            k = static_cast<uint64_t>(static_cast<int64_t>(v)) ^ 0x8000000000000000ull;
        } else {
            k = static_cast<uint64_t>(v);
        }
        key[i] = k;
        idx[i] = static_cast<uint32_t>(i);
    }
}

template <typename T>
__global__ void unique_runs_kernel(const T* __restrict__ col, const uint64_t* __restrict__ skey,
                                   const uint32_t* __restrict__ sidx, uint64_t n, T* uval, unsigned int* ucnt,
                                   unsigned long long* nu) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (i > 0 && skey[i] == skey[i - 1]) continue;
        const uint64_t e = sorted_run_end(skey, i, n);
        unsigned long long slot = atomicAdd(nu, 1ull);
        uval[slot] = col[sidx[i]];
        ucnt[slot] = static_cast<unsigned int>(e - i);
    }
}

// One block per predicate set: count selected rows and distinct selected values.
template <typename T>
__global__ void label_kernel(const T* __restrict__ uval, const unsigned int* __restrict__ ucnt, uint64_t nu,
                             const PredSet* __restrict__ sets, uint64_t* out_rows, uint64_t* out_distinct) {
    const PredSet ps = sets[blockIdx.x];
    unsigned long long rows = 0, dist = 0;
    for (uint64_t i = threadIdx.x; i < nu; i += blockDim.x) {
        T v = uval[i];
        bool ok = true;
        for (int a = 0; a < ps.natoms; ++a) ok = ok && t_cmp<T>(v, from_bits<T>(ps.thr[a]), ps.op[a]);
        if (ok) {
            rows += ucnt[i];
            dist += 1;
        }
    }
    for (int d = 16; d > 0; d >>= 1) {
        rows += __shfl_down_sync(0xffffffffu, rows, d);
        dist += __shfl_down_sync(0xffffffffu, dist, d);
    }
    __shared__ unsigned long long sr[32], sd[32];
    if ((threadIdx.x & 31) == 0) {
        sr[threadIdx.x >> 5] = rows;
        sd[threadIdx.x >> 5] = dist;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long r = 0, d = 0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) {
            r += sr[w];
            d += sd[w];
        }
        out_rows[blockIdx.x] = r;
        out_distinct[blockIdx.x] = d;
    }
}

// ---- MLP ------------------------------------------------------------------------------

struct MlpView {
    const float* w1; const float* b1;
    const float* w2; const float* b2;
    const float* w3; const float* b3;
    const float* w4; const float* b4;
};

__device__ __forceinline__ MlpView mlp_view(const float* p) {
    MlpView v;
    v.w1 = p; v.b1 = p + kH * kIn;
    v.w2 = v.b1 + kH; v.b2 = v.w2 + kH * kH;
    v.w3 = v.b2 + kH; v.b3 = v.w3 + kH * kH;
    v.w4 = v.b3 + kH; v.b4 = v.w4 + kOut * kH;
    return v;
}

// out[s][j] = act(sum_k in[s][k] * W[j][k] + b[j]) for kChunk samples
__device__ __forceinline__ void dense(const float* __restrict__ in, int nin, const float* __restrict__ W,
                                      const float* __restrict__ b, int nout, float* __restrict__ pre,
                                      float* __restrict__ out, bool relu) {
    for (int t = threadIdx.x; t < kChunk * nout; t += blockDim.x) {
        int s = t / nout, j = t % nout;
        float acc = b[j];
        const float* x = in + s * nin;
        const float* w = W + j * nin;
        for (int k = 0; k < nin; ++k) acc = __fmaf_rn(x[k], w[k], acc);
        pre[s * nout + j] = acc;
        out[s * nout + j] = relu ? fmaxf(acc, 0.0f) : acc;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kMThreads) mlp_infer_kernel(const float* __restrict__ params,
                                                              const float* __restrict__ X, uint64_t n,
                                                              float* __restrict__ Y) {
    extern __shared__ __align__(16) float sm[];
    float* P = sm;
    float* a0 = P + kParams;
    float* z1 = a0 + kChunk * kIn;
    float* a1 = z1 + kChunk * kH;
    float* z2 = a1 + kChunk * kH;
    float* a2 = z2 + kChunk * kH;
    float* z3 = a2 + kChunk * kH;
    float* a3 = z3 + kChunk * kH;
    float* z4 = a3 + kChunk * kH;
    float* a4 = z4 + kChunk * kOut;
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    MlpView v = mlp_view(P);
    for (uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * kChunk; c0 < n; c0 += static_cast<uint64_t>(gridDim.x) * kChunk) {
        for (int t = threadIdx.x; t < kChunk * kIn; t += blockDim.x) {
            uint64_t s = c0 + t / kIn;
            a0[t] = s < n ? X[s * kIn + t % kIn] : 0.0f;
        }
        __syncthreads();
        dense(a0, kIn, v.w1, v.b1, kH, z1, a1, true);
        dense(a1, kH, v.w2, v.b2, kH, z2, a2, true);
        dense(a2, kH, v.w3, v.b3, kH, z3, a3, true);
        dense(a3, kH, v.w4, v.b4, kOut, z4, a4, false);
        for (int t = threadIdx.x; t < kChunk * kOut; t += blockDim.x) {
            uint64_t s = c0 + t / kOut;
            if (s < n) Y[s * kOut + t % kOut] = a4[t];
        }
        __syncthreads();
    }
}

// grad of one dense layer for a chunk: dW[j][k] += sum_s d[s][j] in[s][k]; db[j] += sum_s d[s][j];
// din[s][k] = sum_j d[s][j] W[j][k] (times relu' of the input's pre-activation when given)
__device__ __forceinline__ void dense_back(const float* __restrict__ in, int nin, const float* __restrict__ W,
                                           const float* __restrict__ d, int nout, float* __restrict__ gW,
                                           float* __restrict__ gb, float* __restrict__ din,
                                           const float* __restrict__ in_pre) {
    for (int t = threadIdx.x; t < nout * nin; t += blockDim.x) {
        int j = t / nin, k = t % nin;
        float acc = 0.0f;
        for (int s = 0; s < kChunk; ++s) acc = __fmaf_rn(d[s * nout + j], in[s * nin + k], acc);
        gW[t] += acc;
    }
    for (int j = threadIdx.x; j < nout; j += blockDim.x) {
        float acc = 0.0f;
        for (int s = 0; s < kChunk; ++s) acc += d[s * nout + j];
        gb[j] += acc;
    }
    if (din) {
        for (int t = threadIdx.x; t < kChunk * nin; t += blockDim.x) {
            int s = t / nin, k = t % nin;
            float acc = 0.0f;
            for (int j = 0; j < nout; ++j) acc = __fmaf_rn(d[s * nout + j], W[j * nin + k], acc);
            din[t] = (in_pre && in_pre[t] <= 0.0f) ? 0.0f : acc;
        }
    }
    __syncthreads();
}

// Forward + backward of mean-squared error for samples idx[0..m) of (X, Y);
// this block's gradient sum goes to grads[blockIdx.x], its loss sum to loss[blockIdx.x].
__global__ void __launch_bounds__(kMThreads) mlp_grad_kernel(const float* __restrict__ params,
                                                             const float* __restrict__ X,
                                                             const float* __restrict__ Yt,
                                                             const uint32_t* __restrict__ idx, uint32_t m,
                                                             float* __restrict__ grads, float* __restrict__ loss) {
    extern __shared__ __align__(16) float sm[];
    float* P = sm;
    float* G = P + kParams;
    float* a0 = G + kParams;
    float* z1 = a0 + kChunk * kIn;
    float* a1 = z1 + kChunk * kH;
    float* z2 = a1 + kChunk * kH;
    float* a2 = z2 + kChunk * kH;
    float* z3 = a2 + kChunk * kH;
    float* a3 = z3 + kChunk * kH;
    float* z4 = a3 + kChunk * kH;
    float* a4 = z4 + kChunk * kOut;
    float* d4 = a4 + kChunk * kOut;
    float* d3 = d4 + kChunk * kOut;
    float* d2 = d3 + kChunk * kH;
    float* d1 = d2 + kChunk * kH;
    __shared__ float s_loss;
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
        P[i] = params[i];
        G[i] = 0.0f;
    }
    if (threadIdx.x == 0) s_loss = 0.0f;
    __syncthreads();
    MlpView v = mlp_view(P);
    float* gw1 = G;
    float* gb1 = gw1 + kH * kIn;
    float* gw2 = gb1 + kH;
    float* gb2 = gw2 + kH * kH;
    float* gw3 = gb2 + kH;
    float* gb3 = gw3 + kH * kH;
    float* gw4 = gb3 + kH;
    float* gb4 = gw4 + kOut * kH;
    for (uint32_t c0 = blockIdx.x * kChunk; c0 < m; c0 += gridDim.x * kChunk) {
        for (int t = threadIdx.x; t < kChunk * kIn; t += blockDim.x) {
            uint32_t s = c0 + t / kIn;
            a0[t] = s < m ? X[static_cast<uint64_t>(idx[s]) * kIn + t % kIn] : 0.0f;
        }
        __syncthreads();
        dense(a0, kIn, v.w1, v.b1, kH, z1, a1, true);
        dense(a1, kH, v.w2, v.b2, kH, z2, a2, true);
        dense(a2, kH, v.w3, v.b3, kH, z3, a3, true);
        dense(a3, kH, v.w4, v.b4, kOut, z4, a4, false);
        // d(mean squared error)/d out, summed over the minibatch (the Adam step divides by m)
        for (int t = threadIdx.x; t < kChunk * kOut; t += blockDim.x) {
            uint32_t s = c0 + t / kOut;
            float diff = s < m ? a4[t] - Yt[static_cast<uint64_t>(idx[s]) * kOut + t % kOut] : 0.0f;
            d4[t] = 2.0f * diff;
            if (s < m) atomicAdd(&s_loss, diff * diff);
        }
        __syncthreads();
        dense_back(a3, kH, v.w4, d4, kOut, gw4, gb4, d3, z3);
        dense_back(a2, kH, v.w3, d3, kH, gw3, gb3, d2, z2);
        dense_back(a1, kH, v.w2, d2, kH, gw2, gb2, d1, z1);
        dense_back(a0, kIn, v.w1, d1, kH, gw1, gb1, nullptr, nullptr);
    }
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) grads[static_cast<uint64_t>(blockIdx.x) * kParams + i] = G[i];
    if (threadIdx.x == 0) loss[blockIdx.x] = s_loss;
}

__global__ void adam_kernel(float* __restrict__ params, float* __restrict__ mom, float* __restrict__ vel,
                            const float* __restrict__ grads, int nblocks, float inv_m, float lr, float b1,
                            float b2, float eps, float bc1, float bc2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x) {
        float g = 0.0f;
        for (int b = 0; b < nblocks; ++b) g += grads[static_cast<uint64_t>(b) * kParams + i];
        g *= inv_m;
        float mm = b1 * mom[i] + (1.0f - b1) * g;
        float vv = b2 * vel[i] + (1.0f - b2) * g * g;
        mom[i] = mm;
        vel[i] = vv;
        params[i] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
    }
}

size_t infer_smem() { return (kParams + kChunk * (kIn + 6 * kH + 2 * kOut)) * sizeof(float); }
size_t grad_smem() { return (2 * kParams + kChunk * (kIn + 6 * kH + 3 * kOut + 3 * kH)) * sizeof(float); }

int sgrid(uint64_t n, int per_sm = 4) {
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t b = (n + 255) / 256;
    uint64_t cap = static_cast<uint64_t>(sms) * per_sm;
    if (b > cap) b = cap;
    return b < 1 ? 1 : static_cast<int>(b);
}

template <typename T>
int sketch_t(const T* d, uint64_t n, ColumnSketch* out, cudaStream_t s) {
    // [min key, max key][HLL registers][histogram], kept between calls; one
    // read-back at the end
    constexpr size_t kBytes = 16 + kHllRegs * 4 + kHistBins * 8;
    static thread_local DevBuf buf;
    if (!buf.p) buf = DevBuf(kBytes);
    if (!buf.p) return kErrOutOfMemory;
    unsigned long long* mm = buf.as<unsigned long long>();
    unsigned int* hll = reinterpret_cast<unsigned int*>(mm + 2);
    unsigned long long* hist = reinterpret_cast<unsigned long long*>(hll + kHllRegs);
    VX_CUDA(cudaMemsetAsync(mm, 0xFF, 8, s));
    VX_CUDA(cudaMemsetAsync(mm + 1, 0, kBytes - 8, s));
    out->n = n;
    if (n) {
        minmax_hll_kernel<T><<<sgrid(n, 8), 256, 0, s>>>(d, n, mm, mm + 1, hll);
        VX_CUDA(cudaGetLastError());
        histogram64_kernel<T><<<sgrid(n, 8), 256, 0, s>>>(d, n, mm, mm + 1, hist);
        VX_CUDA(cudaGetLastError());
    }
    std::vector<unsigned char> h(kBytes);
    if (int st = d2h(h.data(), buf.p, kBytes, s)) return st;
    if (int st = sync(s)) return st;
    if (n) {
        unsigned long long k[2];
        std::memcpy(k, h.data(), 16);
        out->min = from_order_key(k[0]);
        out->max = from_order_key(k[1]);
    } else {
        out->min = out->max = 0.0;
    }
    std::memcpy(out->hist, h.data() + 16 + kHllRegs * 4, kHistBins * 8);
    for (int i = 0; i < kHllRegs; ++i) {
        unsigned int r;
        std::memcpy(&r, h.data() + 16 + i * 4, 4);
        out->hll[i] = static_cast<uint8_t>(r);
    }
    return kOk;
}

template <typename T>
int labels_t(const T* d, uint64_t n, const PredSet* sets, uint32_t nsets, uint64_t* rows, uint64_t* distinct,
             cudaStream_t s) {
    if (n == 0) {
        for (uint32_t i = 0; i < nsets; ++i) rows[i] = distinct[i] = 0;
        return kOk;
    }
    DevBuf key(n * 8), idx(n * 4), uval(n * sizeof(T) + 8), ucnt(n * 4), nu(8);
    size_t tb = radix_tmp_bytes(U64, n);
    DevBuf tmp(tb), dsets(nsets * sizeof(PredSet) + 8), drows(nsets * 8 + 8), ddist(nsets * 8 + 8);
    if (!key.p || !idx.p || !uval.p || !ucnt.p || !nu.p || !tmp.p || !dsets.p || !drows.p || !ddist.p)
        return kErrOutOfMemory;
    to_sort_key_kernel<T><<<sgrid(n, 8), 256, 0, s>>>(d, n, key.as<uint64_t>(), idx.as<uint32_t>());
    if (int st = launch_radix_sort(U64, key.p, idx.as<uint32_t>(), n, tmp.p, tb, radix_err(s), s, nullptr)) return st;
    VX_CUDA(cudaMemsetAsync(nu.p, 0, 8, s));
    unique_runs_kernel<T><<<sgrid(n, 8), 256, 0, s>>>(d, key.as<uint64_t>(), idx.as<uint32_t>(), n, uval.as<T>(),
                                                      ucnt.as<unsigned int>(), nu.as<unsigned long long>());
    uint64_t h_nu = 0;
    if (int st = d2h(&h_nu, nu.p, 8, s)) return st;
    if (int st = sync(s)) return st;
    if (int st = h2d(dsets.p, sets, nsets * sizeof(PredSet), s)) return st;
    label_kernel<T><<<nsets, 256, 0, s>>>(uval.as<T>(), ucnt.as<unsigned int>(), h_nu, dsets.as<PredSet>(),
                                          drows.as<uint64_t>(), ddist.as<uint64_t>());
    VX_CUDA(cudaGetLastError());
    if (int st = d2h(rows, drows.p, nsets * 8, s)) return st;
    if (int st = d2h(distinct, ddist.p, nsets * 8, s)) return st;
    return radix_check(s);
}

}  // namespace

int Mlp::init(uint64_t seed, cudaStream_t s) {
    params = DevBuf(kParams * 4);
    mom = DevBuf(kParams * 4);
    vel = DevBuf(kParams * 4);
    if (!params.p || !mom.p || !vel.p) return kErrOutOfMemory;
    // He-uniform initialisation from a splitmix64 stream (host, once)
    std::vector<float> h(kParams, 0.0f);
    uint64_t st = seed;
    auto uni = [&st]() {
        st += 0x9e3779b97f4a7c15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        z ^= z >> 31;
        return static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);
    };
    const int fan[4] = {kIn, kH, kH, kH}, outs[4] = {kH, kH, kH, kOut};
    size_t off = 0;
    for (int l = 0; l < 4; ++l) {
        double lim = std::sqrt(6.0 / fan[l]);
        for (int i = 0; i < outs[l] * fan[l]; ++i) h[off + i] = static_cast<float>((2.0 * uni() - 1.0) * lim);
        off += outs[l] * fan[l] + outs[l];  // biases stay zero
    }
    step = 0;
    if (int e = h2d(params.p, h.data(), kParams * 4, s)) return e;
    VX_CUDA(cudaMemsetAsync(mom.p, 0, kParams * 4, s));
    VX_CUDA(cudaMemsetAsync(vel.p, 0, kParams * 4, s));
    return sync(s);
}

int Mlp::set_params(const float* host, cudaStream_t s) {
    if (!params.p) {
        if (int st = init(1, s)) return st;
    }
    if (int st = h2d(params.p, host, kParams * 4, s)) return st;
    return sync(s);
}

int Mlp::get_params(float* host, cudaStream_t s) const {
    if (int st = d2h(host, params.p, kParams * 4, s)) return st;
    return sync(s);
}

int Mlp::grad(const float* dX, const float* dY, const uint32_t* didx, uint32_t m, float* host_grad, float* host_loss,
              cudaStream_t s) {
    int blocks = sm_count() > 0 ? sm_count() : 148;
    uint32_t need = (m + kChunk - 1) / kChunk;
    if (static_cast<uint32_t>(blocks) > need) blocks = static_cast<int>(need ? need : 1);
    if (gbuf.n < static_cast<size_t>(blocks) * kParams * 4) gbuf = DevBuf(static_cast<size_t>(blocks) * kParams * 4);
    if (lbuf.n < static_cast<size_t>(blocks) * 4) lbuf = DevBuf(static_cast<size_t>(blocks) * 4 + 16);
    if (!gbuf.p || !lbuf.p) return kErrOutOfMemory;
    static thread_local bool attr = false;
    if (!attr) {
        VX_CUDA(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(grad_smem())));
        VX_CUDA(cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(infer_smem())));
        attr = true;
    }
    mlp_grad_kernel<<<blocks, kMThreads, grad_smem(), s>>>(params.as<float>(), dX, dY, didx, m, gbuf.as<float>(),
                                                           lbuf.as<float>());
    VX_CUDA(cudaGetLastError());
    last_blocks = blocks;
    if (host_grad || host_loss) {
        std::vector<float> g(static_cast<size_t>(blocks) * kParams), l(blocks);
        if (int st = d2h(g.data(), gbuf.p, g.size() * 4, s)) return st;
        if (int st = d2h(l.data(), lbuf.p, l.size() * 4, s)) return st;
        if (int st = sync(s)) return st;
        if (host_grad) {
            for (int i = 0; i < kParams; ++i) {
                double acc = 0.0;
                for (int b = 0; b < blocks; ++b) acc += g[static_cast<size_t>(b) * kParams + i];
                host_grad[i] = static_cast<float>(acc);
            }
        }
        if (host_loss) {
            double acc = 0.0;
            for (float x : l) acc += x;
            *host_loss = static_cast<float>(acc);
        }
    }
    return kOk;
}

int Mlp::adam_step(uint32_t m, float lr, cudaStream_t s) {
    ++step;
    const float b1 = 0.9f, b2 = 0.999f;
    float bc1 = 1.0f - std::pow(b1, static_cast<float>(step));
    float bc2 = 1.0f - std::pow(b2, static_cast<float>(step));
    adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(params.as<float>(), mom.as<float>(), vel.as<float>(),
                                                      gbuf.as<float>(), last_blocks, 1.0f / m, lr, b1, b2, 1e-8f, bc1,
                                                      bc2);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

int Mlp::infer(const float* dX, uint64_t n, float* dY, cudaStream_t s) {
    static thread_local bool attr = false;
    if (!attr) {
        VX_CUDA(cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(infer_smem())));
        attr = true;
    }
    int blocks = sm_count() > 0 ? sm_count() : 148;
    uint64_t need = (n + kChunk - 1) / kChunk;
    if (static_cast<uint64_t>(blocks) > need) blocks = static_cast<int>(need ? need : 1);
    mlp_infer_kernel<<<blocks, kMThreads, infer_smem(), s>>>(params.as<float>(), dX, n, dY);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

int sketch_column(int dtype, const void* d, uint64_t n, ColumnSketch* out, cudaStream_t s) {
    switch (dtype) {
    case F64: return sketch_t<double>(static_cast<const double*>(d), n, out, s);
    case F32: return sketch_t<float>(static_cast<const float*>(d), n, out, s);
    case I64: return sketch_t<int64_t>(static_cast<const int64_t*>(d), n, out, s);
    case I32: return sketch_t<int32_t>(static_cast<const int32_t*>(d), n, out, s);
    case U64: return sketch_t<uint64_t>(static_cast<const uint64_t*>(d), n, out, s);
    case U32: return sketch_t<uint32_t>(static_cast<const uint32_t*>(d), n, out, s);
    default: set_error(kErrInvalidArg, "unknown element type %d", dtype); return kErrInvalidArg;
    }
}

int exact_labels(int dtype, const void* d, uint64_t n, const PredSet* sets, uint32_t nsets, uint64_t* rows,
                 uint64_t* distinct, cudaStream_t s) {
    switch (dtype) {
    case F64: return labels_t<double>(static_cast<const double*>(d), n, sets, nsets, rows, distinct, s);
    case F32: return labels_t<float>(static_cast<const float*>(d), n, sets, nsets, rows, distinct, s);
    case I64: return labels_t<int64_t>(static_cast<const int64_t*>(d), n, sets, nsets, rows, distinct, s);
    case I32: return labels_t<int32_t>(static_cast<const int32_t*>(d), n, sets, nsets, rows, distinct, s);
    case U64: return labels_t<uint64_t>(static_cast<const uint64_t*>(d), n, sets, nsets, rows, distinct, s);
    case U32: return labels_t<uint32_t>(static_cast<const uint32_t*>(d), n, sets, nsets, rows, distinct, s);
    default: set_error(kErrInvalidArg, "unknown element type %d", dtype); return kErrInvalidArg;
    }
}

}  // namespace vx

using namespace vx;

extern "C" {

size_t voxel_mlp_param_count(void) { return kParams; }
void* voxel_mlp_create(uint64_t seed) {
    clear_error();
    if (ensure_device()) return nullptr;
    Mlp* m = new Mlp();
    if (m->init(seed, thread_stream())) {
        delete m;
        return nullptr;
    }
    return m;
}
void voxel_mlp_destroy(void* m) { delete static_cast<Mlp*>(m); }
int voxel_mlp_set_params(void* m, const float* host) { return static_cast<Mlp*>(m)->set_params(host, thread_stream()); }
int voxel_mlp_get_params(const void* m, float* host) {
    return static_cast<const Mlp*>(m)->get_params(host, thread_stream());
}
int voxel_mlp_grad(void* m, const float* d_x, const float* d_y, const uint32_t* d_idx, uint32_t count, float* grad,
                   float* loss) {
    clear_error();
    return static_cast<Mlp*>(m)->grad(d_x, d_y, d_idx, count, grad, loss, thread_stream());
}
int voxel_mlp_train_step(void* m, const float* d_x, const float* d_y, const uint32_t* d_idx, uint32_t count,
                         float lr) {
    clear_error();
    Mlp* M = static_cast<Mlp*>(m);
    cudaStream_t s = thread_stream();
    if (int st = M->grad(d_x, d_y, d_idx, count, nullptr, nullptr, s)) return st;
    return M->adam_step(count, lr, s);
}
int voxel_mlp_infer(void* m, const float* d_x, size_t n, float* d_y, void* stream) {
    clear_error();
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : thread_stream();
    int st = static_cast<Mlp*>(m)->infer(d_x, n, d_y, s);
    if (st || stream) return st;
    return sync(s);
}
static_assert(sizeof(voxel_column_sketch) == sizeof(ColumnSketch), "sketch layout");
static_assert(sizeof(voxel_pred_set) == sizeof(PredSet), "predicate-set layout");

int voxel_sketch_column_dev(int dtype, const void* d_col, size_t n, voxel_column_sketch* out) {
    clear_error();
    if (int st = ensure_device()) return st;
    return sketch_column(dtype, d_col, n, reinterpret_cast<ColumnSketch*>(out), thread_stream());
}
int voxel_exact_labels_dev(int dtype, const void* d_col, size_t n, const voxel_pred_set* sets, uint32_t nsets,
                           uint64_t* rows, uint64_t* distinct) {
    clear_error();
    if (int st = ensure_device()) return st;
    return exact_labels(dtype, d_col, n, reinterpret_cast<const PredSet*>(sets), nsets, rows, distinct,
                        thread_stream());
}

}  // extern "C"
