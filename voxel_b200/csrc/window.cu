// Window functions of Engine<T> (reference include/voxel/exec/engine.hpp:176-300).
//
//   WindowDelta (182-192):    out[i] = data[i+1] - data[i], i < min(count-1, outLen).
//   WindowSum (195-214):      out[j] = data[j] + ... + data[j+w-1], summed left to
//                             right in T, j < min(count-w+1, outLen); w >= 1.
//   WindowMean (217-222):     WindowSum, then out[j] /= (T)w.
//   TimeWindowSum (228-241):  out[(ts[i] - start) / dur] += values[i] for buckets in
//                             [0, outLen) (C++ division: truncation toward zero);
//                             returns the largest bucket touched + 1 (1 if none).
//   WindowStdDev / Variance (244-275): per window, sum -> mean = sum / w ->
//                             ssq = sum of (x - mean)^2, all in T; out = sqrt(ssq / w)
//                             (integers: the double square root truncated back to T)
//                             or ssq / w; w >= 2.
//   WindowQuantile (278-300): the first min(w, 128) values of each window; pos =
//                             q * (w'-1), lo = floor(pos), hi = lo + 1 (clamped);
//                             vLo, vHi = the lo-th and hi-th smallest; out = vLo +
//                             (T)((f64)(vHi - vLo) * (pos - lo)); w >= 2, 0 <= q <= 1.
//
// Each window is evaluated in exactly the reference's operation order (the same
// left-to-right sums, one rounding per operation, no fused multiply-add), so the
// outputs are bit-identical for every element type.  B200 design: blocks stage a
// tile of outputs plus its halo of w-1 inputs in shared memory with coalesced
// loads, and each thread evaluates windows from there (O(w) shared reads per
// output, as the definition is; sums and means of windows up to 16 inputs
// evaluate 9 consecutive outputs per thread from registers); the quantile
// keeps each thread's window sorted -- in registers up to 16 inputs, in local
// memory above -- and slides it (one removal and one insertion per output);
// the time-bucketed sum steps warps through 32 consecutive rows, sums runs of
// one bucket with a segmented warp scan and adds each finished run to the
// output once with a global atomic.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>

#include "voxel_c.h"
#include "vx_common.cuh"
#include "vx_runtime.h"

namespace vx {

namespace {

constexpr int kWThreads = 256;
constexpr int kWTile = 2048;    // outputs per block step
constexpr int kWMaxWin = 256;   // u8 windows: at most 255 inputs per window
constexpr int kQMax = 128;      // WindowQuantile's buffer (engine.hpp:284)
constexpr int kQRun = 32;       // consecutive quantile outputs per thread

enum WinKind : int { kDelta = 0, kSum = 1, kMean = 2, kStdDev = 3, kVariance = 4, kQuantile = 5 };

template <typename T>
__device__ __forceinline__ T w_add(T a, T b) {
    if constexpr (std::is_same<T, double>::value) return __dadd_rn(a, b);
    else return static_cast<T>(a + b);
}
template <typename T>
__device__ __forceinline__ T w_sub(T a, T b) {
    if constexpr (std::is_same<T, double>::value) return __dsub_rn(a, b);
    else return static_cast<T>(a - b);
}
template <typename T>
__device__ __forceinline__ T w_mul(T a, T b) {
    if constexpr (std::is_same<T, double>::value) return __dmul_rn(a, b);
    else return static_cast<T>(a * b);
}
template <typename T>
__device__ __forceinline__ T w_div(T a, T b) {
    if constexpr (std::is_same<T, double>::value) return __ddiv_rn(a, b);
    else return static_cast<T>(a / b);
}
template <typename T>
__device__ __forceinline__ T w_sqrt(T a) {
    if constexpr (std::is_same<T, double>::value) return __dsqrt_rn(a);
    else return static_cast<T>(__dsqrt_rn(static_cast<double>(a)));  // std::sqrt of an integer, back to T
}

// Copies src[0, m) into shared memory with every load of the thread issued
// before its first store (a rolled copy loop waits for each load in turn),
// between two block barriers.  LOADS * kWThreads >= m.
template <typename T, int LOADS>
__device__ __forceinline__ void stage_tile(const T* __restrict__ src, uint32_t m, T* s) {
    T v[LOADS];
#pragma unroll
    for (int q = 0; q < LOADS; ++q) {
        const uint32_t i = threadIdx.x + q * kWThreads;
        v[q] = i < m ? __ldg(src + i) : T(0);
    }
    __syncthreads();  // the previous tile's readers are done
#pragma unroll
    for (int q = 0; q < LOADS; ++q) {
        const uint32_t i = threadIdx.x + q * kWThreads;
        if (i < m) s[i] = v[q];
    }
    __syncthreads();
}

template <typename T, int KIND>
__global__ void __launch_bounds__(kWThreads) window_kernel(const T* __restrict__ data, uint64_t nout, uint32_t w,
                                                           T* __restrict__ out) {
    __shared__ T s[kWTile + kWMaxWin];
    const uint32_t halo = KIND == kDelta ? 1u : w - 1u;
    const T tw = static_cast<T>(w);
    for (uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * kWTile; t0 < nout;
         t0 += static_cast<uint64_t>(gridDim.x) * kWTile) {
        const uint32_t nt = static_cast<uint32_t>(nout - t0 < kWTile ? nout - t0 : kWTile);
        stage_tile<T, (kWTile + kWMaxWin + kWThreads - 1) / kWThreads>(data + t0, nt + halo, s);
        for (uint32_t j = threadIdx.x; j < nt; j += blockDim.x) {
            T r;
            if constexpr (KIND == kDelta) {
                r = w_sub<T>(s[j + 1], s[j]);
            } else {
                T sum = T(0);
                for (uint32_t k = 0; k < w; ++k) sum = w_add<T>(sum, s[j + k]);
                if constexpr (KIND == kSum) {
                    r = sum;
                } else if constexpr (KIND == kMean) {
                    r = w_div<T>(sum, tw);
                } else {
                    const T mean = w_div<T>(sum, tw);
                    T ssq = T(0);
                    for (uint32_t k = 0; k < w; ++k) {
                        const T d = w_sub<T>(s[j + k], mean);
                        ssq = w_add<T>(ssq, w_mul<T>(d, d));
                    }
                    r = KIND == kVariance ? w_div<T>(ssq, tw) : w_sqrt<T>(w_div<T>(ssq, tw));
                }
            }
            out[t0 + j] = r;
        }
    }
}

// Register-tiled form of window_kernel (WindowSum, WindowMean) for windows of
// at most kRW inputs: each thread evaluates kRR consecutive outputs from
// kRR + w - 1 inputs held in registers (read once from shared memory instead of w times per output),
// each output still summed left to right from T(0) as the definition is.
// kRR is odd, so the threads' strided shared-memory reads fall in distinct
// banks; outputs are staged in shared memory and stored coalesced.
constexpr int kRW = 16;                 // largest window of the register form
constexpr int kRR = 9;                  // consecutive outputs per thread
constexpr int kRTile = kWThreads * kRR; // 2304 outputs per block step

template <typename T, int KIND>
__global__ void __launch_bounds__(kWThreads) window_reg_kernel(const T* __restrict__ data, uint64_t nout, uint32_t w,
                                                               T* __restrict__ out) {
    __shared__ T s[kRTile + kRW];
    __shared__ T so[kRTile];
    const T tw = static_cast<T>(w);
    const uint32_t halo = w - 1u;
    for (uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * kRTile; t0 < nout;
         t0 += static_cast<uint64_t>(gridDim.x) * kRTile) {
        const uint32_t nt = static_cast<uint32_t>(nout - t0 < kRTile ? nout - t0 : kRTile);
        stage_tile<T, (kRTile + kRW + kWThreads - 1) / kWThreads>(data + t0, nt + halo, s);
        const uint32_t j0 = threadIdx.x * kRR;
        T x[kRR + kRW - 1];
#pragma unroll
        for (int k = 0; k < kRR + kRW - 1; ++k) x[k] = j0 + k < nt + halo ? s[j0 + k] : T(0);
#pragma unroll
        for (int r = 0; r < kRR; ++r) {
            T sum = T(0);
#pragma unroll
            for (int k = 0; k < kRW; ++k)
                if (k < static_cast<int>(w)) sum = w_add<T>(sum, x[r + k]);
            const T res = KIND == kSum ? sum : w_div<T>(sum, tw);
            if (j0 + r < nt) so[j0 + r] = res;
        }
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < nt; j += blockDim.x) out[t0 + j] = so[j];
    }
}

// WindowQuantile for windows of at most kRW inputs: the sorted window lives in
// registers (every index below is a compile-time constant).  The first window
// is sorted by odd-even transposition; each slide drops data[j] and takes
// data[j + wq] in one pass that builds every entry from its old neighbours.
template <typename T>
__device__ __forceinline__ T pick_entry(const T (&a)[kRW], int idx) {
    // a[idx] as an OR of masked entries, so the array stays in registers (a
    // plain select on idx is turned into an indexed local-memory load)
    using B = typename std::conditional<sizeof(T) == 8, unsigned long long, unsigned int>::type;
    B acc = 0;
#pragma unroll
    for (int i = 0; i < kRW; ++i) {
        B bits;
        memcpy(&bits, &a[i], sizeof(T));
        acc |= bits & (B(0) - B(i == idx));
    }
    T r;
    memcpy(&r, &acc, sizeof(T));
    return r;
}

template <typename T>
__global__ void __launch_bounds__(kWThreads) quantile_reg_kernel(const T* __restrict__ data, uint64_t nout, int wq,
                                                                 int lo, int hi, double frac, T* __restrict__ out) {
    const uint64_t nruns = (nout + kQRun - 1) / kQRun;
    for (uint64_t run = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; run < nruns;
         run += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t j0 = run * kQRun;
        const uint64_t j1 = j0 + kQRun < nout ? j0 + kQRun : nout;
        T a[kRW];
#pragma unroll
        for (int i = 0; i < kRW; ++i) a[i] = i < wq ? __ldg(data + j0 + i) : T(0);
#pragma unroll
        for (int round = 0; round < kRW; ++round) {
#pragma unroll
            for (int i = round & 1; i + 1 < kRW; i += 2) {
                if (i + 1 < wq && a[i + 1] < a[i]) {
                    const T t = a[i];
                    a[i] = a[i + 1];
                    a[i + 1] = t;
                }
            }
        }
        for (uint64_t j = j0; j < j1; ++j) {
            const T vlo = pick_entry<T>(a, lo), vhi = pick_entry<T>(a, hi);
            T r = vlo;
            if (lo != hi) {
                if constexpr (std::is_same<T, double>::value) {
                    r = __dadd_rn(vlo, __dmul_rn(__dsub_rn(vhi, vlo), frac));
                } else {
                    const double d = static_cast<double>(static_cast<T>(vhi - vlo));
                    r = static_cast<T>(vlo + static_cast<T>(__dmul_rn(d, frac)));
                }
            }
            out[j] = r;
            if (j + 1 < j1) {  // slide: drop data[j], take data[j + wq]
                const T gone = __ldg(data + j), come = __ldg(data + j + wq);
                int p = 0, ins = 0;  // p: the dropped entry; ins: where `come` goes once it is gone
#pragma unroll
                for (int i = 0; i < kRW; ++i)
                    if (i < wq && a[i] < gone) ++p;
                if (p >= wq) p = wq - 1;  // NaN-free input always finds it
#pragma unroll
                for (int i = 0; i < kRW; ++i)
                    if (i < wq && i != p && a[i] < come) ++ins;
                T b[kRW];
#pragma unroll
                for (int i = 0; i < kRW; ++i) {
                    const T dn = i + 1 < kRW ? a[i + 1] : a[i];  // entries left of the drop shift down
                    const T up = i > 0 ? a[i - 1] : a[i];        // entries right of the insert shift up
                    const T left = i < p ? a[i] : dn;            // the array without the dropped entry, at i
                    const T right = i - 1 < p ? up : a[i];       // ... at i - 1
                    b[i] = i < ins ? left : (i == ins ? come : right);
                }
#pragma unroll
                for (int i = 0; i < kRW; ++i) a[i] = b[i];
            }
        }
    }
}

// first index in buf[0, n) with buf[i] >= v (strict weak order of T)
template <typename T>
__device__ __forceinline__ int lower_idx(const T* buf, int n, T v) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (buf[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

template <typename T>
__global__ void __launch_bounds__(kWThreads) quantile_kernel(const T* __restrict__ data, uint64_t nout, int wq,
                                                             int lo, int hi, double frac, T* __restrict__ out) {
    T buf[kQMax];
    const uint64_t nruns = (nout + kQRun - 1) / kQRun;
    for (uint64_t run = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; run < nruns;
         run += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t j0 = run * kQRun;
        const uint64_t j1 = j0 + kQRun < nout ? j0 + kQRun : nout;
        // the first window, insertion-sorted
        for (int k = 0; k < wq; ++k) {
            const T v = __ldg(data + j0 + k);
            int p = k;
            while (p > 0 && v < buf[p - 1]) {
                buf[p] = buf[p - 1];
                --p;
            }
            buf[p] = v;
        }
        for (uint64_t j = j0; j < j1; ++j) {
            const T vlo = buf[lo];
            T r = vlo;
            if (lo != hi) {
                const T vhi = buf[hi];
                if constexpr (std::is_same<T, double>::value) {
                    r = __dadd_rn(vlo, __dmul_rn(__dsub_rn(vhi, vlo), frac));
                } else {
                    const double d = static_cast<double>(static_cast<T>(vhi - vlo));
                    r = static_cast<T>(vlo + static_cast<T>(__dmul_rn(d, frac)));
                }
            }
            out[j] = r;
            if (j + 1 < j1) {  // slide: drop data[j], take data[j + wq]
                const T gone = __ldg(data + j), come = __ldg(data + j + wq);
                int p = lower_idx<T>(buf, wq, gone);
                if (p >= wq) p = wq - 1;  // NaN-free input always finds it
                for (int q = p; q + 1 < wq; ++q) buf[q] = buf[q + 1];
                int ins = lower_idx<T>(buf, wq - 1, come);
                for (int q = wq - 1; q > ins; --q) buf[q] = buf[q - 1];
                buf[ins] = come;
            }
        }
    }
}

// out[bucket] += v (integer buckets wrap like the reference's T additions)
template <typename T>
__device__ __forceinline__ void add_out(T* out, uint64_t b, T v) {
    if constexpr (std::is_same<T, double>::value) atomicAdd(out + b, v);
    else if constexpr (sizeof(T) == 8) atomicAdd(reinterpret_cast<unsigned long long*>(out + b), static_cast<unsigned long long>(v));
    else atomicAdd(reinterpret_cast<unsigned int*>(out + b), static_cast<unsigned int>(v));
}

// trunc(x / d) for d > 0 (C++ division): for |x| < 2^50 from the double
// product x * (1/d), whose error is below 1/4, corrected by one step on the
// integer remainder; other x take the integer division.
__device__ __forceinline__ int64_t div_trunc(int64_t x, int64_t d, double inv) {
    if (x > -(1ll << 50) && x < (1ll << 50)) {
        int64_t q = static_cast<int64_t>(__dmul_rn(static_cast<double>(x), inv));
        int64_t r = x - q * d;
        if (x >= 0) {
            if (r < 0) --q;
            else if (r >= d) ++q;
        } else {
            if (r > 0) ++q;
            else if (r <= -d) --q;
        }
        return q;
    }
    return x / d;
}

// Warp form of the time-bucketed sum: a warp takes chunks of 1024 rows and
// steps through them 32 consecutive rows at a time (coalesced loads), sums
// each run of equal buckets with a segmented warp scan, adds every finished
// run to the output once and carries the run that reaches lane 31 into the
// next step.  Integer sums are exact; f64 sums group the additions by run
// instead of the reference's row order.
constexpr uint64_t kTChunk = 1024;
constexpr int kTUnroll = 4;

template <typename T>
__global__ void __launch_bounds__(kWThreads) time_window_warp_kernel(const int64_t* __restrict__ ts,
                                                                     const T* __restrict__ vals, uint64_t n,
                                                                     int64_t start, int64_t dur, double inv,
                                                                     uint64_t nout, T* __restrict__ out,
                                                                     unsigned long long* maxb) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const uint64_t nwarps = static_cast<uint64_t>(gridDim.x) * (blockDim.x / 32);
    const uint64_t wid = static_cast<uint64_t>(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5);
    unsigned long long mymax = 0;
    for (uint64_t c0 = wid * kTChunk; c0 < n; c0 += nwarps * kTChunk) {
        const uint64_t c1 = c0 + kTChunk < n ? c0 + kTChunk : n;
        long long cb = -1;  // the carried run's bucket (warp-uniform), -1 none
        T cacc = T(0);
        for (uint64_t r0 = c0; r0 < c1; r0 += 32 * kTUnroll) {
            int64_t tv[kTUnroll];
            T vv[kTUnroll];
#pragma unroll
            for (int u = 0; u < kTUnroll; ++u) {
                const uint64_t i = r0 + u * 32 + lane;
                tv[u] = i < c1 ? __ldcs(ts + i) : 0;
                vv[u] = i < c1 ? __ldcs(vals + i) : T(0);
            }
#pragma unroll
            for (int u = 0; u < kTUnroll; ++u) {
                const uint64_t i = r0 + u * 32 + lane;
                long long b = -1;
                T v = T(0);
                if (i < c1) {
                    const int64_t q = div_trunc(tv[u] - start, dur, inv);
                    if (q >= 0 && static_cast<uint64_t>(q) < nout) {
                        b = q;
                        v = vv[u];
                        if (static_cast<unsigned long long>(q) > mymax) mymax = static_cast<unsigned long long>(q);
                    }
                }
                const long long bprev = __shfl_up_sync(full, b, 1);
                const unsigned heads = __ballot_sync(full, lane == 0 || bprev != b);
                const int sstart = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
                T sv = v;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const T y = __shfl_up_sync(full, sv, d);
                    if (lane - d >= sstart) sv = w_add<T>(sv, y);
                }
                const long long b0 = __shfl_sync(full, b, 0);
                if (cb >= 0) {
                    if (b0 == cb) {
                        if (sstart == 0) sv = w_add<T>(sv, cacc);  // the first run continues the carried one
                    } else if (lane == 0) {
                        add_out<T>(out, static_cast<uint64_t>(cb), cacc);
                    }
                }
                const long long bnext = __shfl_down_sync(full, b, 1);
                if (lane != 31 && bnext != b && b >= 0) add_out<T>(out, static_cast<uint64_t>(b), sv);
                cb = __shfl_sync(full, b, 31);
                cacc = __shfl_sync(full, sv, 31);
            }
        }
        if (cb >= 0 && lane == 0) add_out<T>(out, static_cast<uint64_t>(cb), cacc);
    }
    unsigned long long m = mymax;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync(full, m, o);
        m = y > m ? y : m;
    }
    if (lane == 0 && m) atomicMax(maxb, m);
}

int w_grid(uint64_t work, int per_sm = 8) {
    const int sms = sm_count() > 0 ? sm_count() : 148;
    const uint64_t cap = static_cast<uint64_t>(sms) * per_sm;
    return static_cast<int>(work < 1 ? 1 : (work < cap ? work : cap));
}

bool win_type(int dtype) { return dtype == F64 || dtype == I64 || dtype == I32 || dtype == U64 || dtype == U32; }

// number of outputs the reference writes (0: nothing)
uint64_t win_count(int kind, uint64_t count, uint64_t out_len, uint32_t w, double q) {
    if (kind == kDelta) return count < 2 ? 0 : (count - 1 < out_len ? count - 1 : out_len);
    if (w == 0 || count < w) return 0;
    if ((kind == kStdDev || kind == kVariance || kind == kQuantile) && w < 2) return 0;
    if (kind == kQuantile && !(q >= 0.0 && q <= 1.0)) return 0;
    const uint64_t nw = count - w + 1;
    return nw < out_len ? nw : out_len;
}

template <typename T>
int launch_t(int kind, const void* d_data, uint64_t nout, uint32_t w, double q, void* d_out, cudaStream_t s) {
    const T* in = static_cast<const T*>(d_data);
    T* o = static_cast<T*>(d_out);
    const uint64_t tiles = (nout + kWTile - 1) / kWTile;
    const uint64_t rtiles = (nout + kRTile - 1) / kRTile;
    // sums and means of short windows from registers; the statistics stay on
    // the shared-memory kernel, where more resident warps hide the latency of
    // their FP64 chains (measured faster)
    if (w <= static_cast<uint32_t>(kRW) && (kind == kSum || kind == kMean)) {
        if (kind == kSum) window_reg_kernel<T, kSum><<<w_grid(rtiles), kWThreads, 0, s>>>(in, nout, w, o);
        else window_reg_kernel<T, kMean><<<w_grid(rtiles), kWThreads, 0, s>>>(in, nout, w, o);
        VX_CUDA(cudaGetLastError());
        return kOk;
    }
    switch (kind) {
    case kDelta: window_kernel<T, kDelta><<<w_grid(tiles), kWThreads, 0, s>>>(in, nout, w, o); break;
    case kSum: window_kernel<T, kSum><<<w_grid(tiles), kWThreads, 0, s>>>(in, nout, w, o); break;
    case kMean: window_kernel<T, kMean><<<w_grid(tiles), kWThreads, 0, s>>>(in, nout, w, o); break;
    case kStdDev: window_kernel<T, kStdDev><<<w_grid(tiles), kWThreads, 0, s>>>(in, nout, w, o); break;
    case kVariance: window_kernel<T, kVariance><<<w_grid(tiles), kWThreads, 0, s>>>(in, nout, w, o); break;
    default: {
        const int wq = static_cast<int>(w < static_cast<uint32_t>(kQMax) ? w : kQMax);
        const double pos = q * static_cast<double>(wq - 1);
        int lo = static_cast<int>(pos);
        if (lo >= wq) lo = wq - 1;
        int hi = lo + 1;
        if (hi >= wq) hi = lo;
        const double frac = pos - static_cast<double>(lo);
        const uint64_t runs = (nout + kQRun - 1) / kQRun;
        if (wq <= kRW)
            quantile_reg_kernel<T><<<w_grid((runs + kWThreads - 1) / kWThreads), kWThreads, 0, s>>>(in, nout, wq, lo,
                                                                                                    hi, frac, o);
        else
            quantile_kernel<T><<<w_grid((runs + kWThreads - 1) / kWThreads), kWThreads, 0, s>>>(in, nout, wq, lo, hi,
                                                                                                frac, o);
        break;
    }
    }
    VX_CUDA(cudaGetLastError());
    return kOk;
}

int launch_window(int dtype, int kind, const void* d_data, uint64_t nout, uint32_t w, double q, void* d_out,
                  cudaStream_t s) {
    if (!nout) return kOk;
    switch (dtype) {
    case F64: return launch_t<double>(kind, d_data, nout, w, q, d_out, s);
    case I64: return launch_t<int64_t>(kind, d_data, nout, w, q, d_out, s);
    case I32: return launch_t<int32_t>(kind, d_data, nout, w, q, d_out, s);
    case U64: return launch_t<uint64_t>(kind, d_data, nout, w, q, d_out, s);
    default: return launch_t<uint32_t>(kind, d_data, nout, w, q, d_out, s);
    }
}

int check_args(int dtype, int kind) {
    if (!win_type(dtype)) {
        set_error(kErrInvalidArg, "window functions: element type %d has no engine (f64, i64, i32, u64, u32)", dtype);
        return kErrInvalidArg;
    }
    if (kind < kDelta || kind > kQuantile) {
        set_error(kErrInvalidArg, "window function kind %d outside 0..5", kind);
        return kErrInvalidArg;
    }
    return kOk;
}

template <typename T>
int launch_time_t(const int64_t* ts, const void* vals, uint64_t n, int64_t start, int64_t dur, void* out,
                  uint64_t nout, unsigned long long* maxb, cudaStream_t s) {
    const uint64_t chunks = (n + kTChunk - 1) / kTChunk;  // one warp per chunk
    const double inv = 1.0 / static_cast<double>(dur);
    time_window_warp_kernel<T><<<w_grid((chunks + kWThreads / 32 - 1) / (kWThreads / 32)), kWThreads, 0, s>>>(
        ts, static_cast<const T*>(vals), n, start, dur, inv, nout, static_cast<T*>(out), maxb);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

int launch_time_window(int dtype, const int64_t* ts, const void* vals, uint64_t n, int64_t start, int64_t dur,
                       void* out, uint64_t nout, unsigned long long* maxb, cudaStream_t s) {
    switch (dtype) {
    case F64: return launch_time_t<double>(ts, vals, n, start, dur, out, nout, maxb, s);
    case I64: return launch_time_t<int64_t>(ts, vals, n, start, dur, out, nout, maxb, s);
    case I32: return launch_time_t<int32_t>(ts, vals, n, start, dur, out, nout, maxb, s);
    case U64: return launch_time_t<uint64_t>(ts, vals, n, start, dur, out, nout, maxb, s);
    default: return launch_time_t<uint32_t>(ts, vals, n, start, dur, out, nout, maxb, s);
    }
}

}  // namespace

}  // namespace vx

using namespace vx;

extern "C" {

int voxel_window_dev(int dtype, int kind, const void* d_data, size_t count, void* d_out, size_t out_len,
                     uint8_t window, double quantile, size_t* n_out, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    if (int st = check_args(dtype, kind)) return st;
    const uint64_t nout = win_count(kind, count, out_len, window, quantile);
    if (n_out) *n_out = nout;
    return launch_window(dtype, kind, d_data, nout, window, quantile, d_out, static_cast<cudaStream_t>(stream));
}

size_t voxel_window(int dtype, int kind, const void* data, size_t count, void* out, size_t out_len, uint8_t window,
                    double quantile) {
    clear_error();
    if (ensure_device() || check_args(dtype, kind)) return 0;
    const uint64_t nout = win_count(kind, count, out_len, window, quantile);
    if (!nout) return 0;
    const uint64_t nin = kind == kDelta ? nout + 1 : nout + window - 1;  // inputs the outputs read
    const size_t es = dtype_size(dtype);
    cudaStream_t s = thread_stream();
    DevBuf din(nin * es), dout(nout * es);
    if (!din.ok(nin * es) || !dout.ok(nout * es)) return 0;
    if (h2d(din.p, data, nin * es, s)) return 0;
    if (launch_window(dtype, kind, din.p, nout, window, quantile, dout.p, s)) return 0;
    if (d2h(out, dout.p, nout * es, s) || sync(s)) return 0;
    return nout;
}

int voxel_time_window_sum_dev(int dtype, const int64_t* d_ts, const void* d_values, size_t count, int64_t start,
                              int64_t duration, void* d_out, size_t out_len, size_t* n_out, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    if (int st = check_args(dtype, kSum)) return st;
    if (duration <= 0 || count == 0 || out_len == 0) {
        if (n_out) *n_out = 0;
        return kOk;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    static thread_local DevBuf mb;
    if (!mb.p) {
        mb = DevBuf(16);
        if (!mb.p) return kErrOutOfMemory;
    }
    VX_CUDA(cudaMemsetAsync(mb.p, 0, 8, s));
    if (int st = launch_time_window(dtype, d_ts, d_values, count, start, duration, d_out, out_len,
                                    mb.as<unsigned long long>(), s))
        return st;
    uint64_t m = 0;
    if (int st = d2h(&m, mb.p, 8, s)) return st;
    if (int st = sync(s)) return st;
    if (n_out) *n_out = m + 1;  // engine.hpp:240: the largest bucket touched + 1
    return kOk;
}

size_t voxel_time_window_sum(int dtype, const int64_t* ts, const void* values, size_t count, int64_t start,
                             int64_t duration, void* out, size_t out_len) {
    clear_error();
    if (ensure_device() || check_args(dtype, kSum)) return 0;
    if (duration <= 0 || count == 0 || out_len == 0) return 0;
    const size_t es = dtype_size(dtype);
    cudaStream_t s = thread_stream();
    DevBuf dts(count * 8), dv(count * es), dout(out_len * es);
    if (!dts.ok(count * 8) || !dv.ok(count * es) || !dout.ok(out_len * es)) return 0;
    if (h2d(dts.p, ts, count * 8, s) || h2d(dv.p, values, count * es, s) || h2d(dout.p, out, out_len * es, s))
        return 0;
    size_t n = 0;
    if (voxel_time_window_sum_dev(dtype, dts.as<int64_t>(), dv.p, count, start, duration, dout.p, out_len, &n, s))
        return 0;
    if (d2h(out, dout.p, out_len * es, s) || sync(s)) return 0;
    return n;
}

}  // extern "C"
