// Delta and frame-of-reference column codecs (reference
// include/voxel/data/encoding.hpp).
//
//   DeltaEncoding<T>::Build (281-306): deltas[i] = data[i] - data[i-1], with
//     data[-1] = T{} and BaseValue = T{}.
//   DeltaEncoding<T>::DecodeBatch (317-330): out[i] = BaseValue + deltas[0] +
//     ... + deltas[offset + i], wrapping in T, for i < count and
//     offset + i < size (later outputs are not written).
//   FrameOfReferenceEncoding::Build (456-482): BaseValue = min, Scale =
//     (max - min) / INT32_MAX (1 when max == min), code = (i32) llround((x -
//     BaseValue) / Scale).
//   FrameOfReferenceEncoding::DecodeBatch (489-500): out[i] = BaseValue +
//     (f64) code[offset + i] * Scale, one rounding per operation (no fused
//     multiply-add), for offset + i < size.
//
// B200 design: the delta decode is one single-pass prefix sum (tiles of 4096
// values per 256-thread block, tile prefixes by decoupled look-back over
// fence-free two-word statuses, since the wrapping sums use all 64 bits),
// outputs staged in shared memory and written coalesced.  The FOR codecs are
// elementwise streams (the encode adds one min/max reduction).  Everything is
// HBM-bound integer / FP64 work; nothing uses tensor cores.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "decode.h"
#include "fixedpoint.cuh"
#include "voxel_c.h"
#include "vx_common.cuh"
#include "vx_runtime.h"

namespace vx {

namespace {

constexpr int kThreads = 256;
constexpr int kPer = 16;                       // values per thread
constexpr int kTile = kThreads * kPer;         // 4096 values per tile
// shared-memory index of tile value j: one pad slot per 16 values, so a
// thread's own 16 consecutive values and the warp's coalesced store order
// both fall in distinct banks
__device__ __forceinline__ uint32_t pad16(uint32_t j) { return j + (j >> 4); }
constexpr long long kSpinBudget = 1ll << 31;   // clock cycles (about 1 s)

// Tile status: the tile's aggregate and its inclusive prefix, each a 64-bit
// value published as two words (low half, high half), each word the half
// shifted up 32 bits with bit 0 set -- zero means not yet written.  A word is
// written with one single-copy-atomic 64-bit store and a reader takes a
// value only once both of its words are set, so no fence is needed to order
// a value against its flag (a release store would wait for the tile's
// earlier output stores to drain, on the critical path of every tile).
struct Status64 {
    unsigned long long* agg;  // 2 words per tile
    unsigned long long* inc;  // 2 words per tile
};

__device__ __forceinline__ void st_relaxed64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void publish64(unsigned long long* w, uint64_t tile, uint64_t v) {
    st_relaxed64(w + 2 * tile, (v << 32) | 1ull);
    st_relaxed64(w + 2 * tile + 1, (v & 0xffffffff00000000ull) | 1ull);
}

// 0 empty, 1 aggregate, 2 inclusive prefix; *v the value
__device__ __forceinline__ uint32_t read_status64(Status64 st, int64_t idx, uint64_t* v) {
    // all four words in one round trip
    const unsigned long long i0 = ld_relaxed64(st.inc + 2 * idx), i1 = ld_relaxed64(st.inc + 2 * idx + 1);
    const unsigned long long a0 = ld_relaxed64(st.agg + 2 * idx), a1 = ld_relaxed64(st.agg + 2 * idx + 1);
    if ((i0 & i1 & 1ull) != 0) {
        *v = (i0 >> 32) | (i1 & 0xffffffff00000000ull);
        return 2;
    }
    if ((a0 & a1 & 1ull) != 0) {
        *v = (a0 >> 32) | (a1 & 0xffffffff00000000ull);
        return 1;
    }
    return 0;
}

// Exclusive prefix (mod 2^64) of `tile` from its predecessors; all 32 lanes of
// one warp call it and get the same value.  Each step reads 32 predecessors
// (lane l reads p - l), finds the nearest inclusive prefix with a ballot and
// adds the aggregates back to it; it spins only while an entry inside that
// window is still empty.  Bounded: when the budget runs out it sets bit 4 of
// *err and returns what it has.
__device__ uint64_t lookback64_warp(Status64 st, uint64_t tile, uint64_t agg, int* err) {
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) publish64(st.inc, 0, agg);
        return 0;
    }
    if (lane == 0) publish64(st.agg, tile, agg);
    uint64_t excl = 0;
    int64_t p = static_cast<int64_t>(tile) - 1;
    const long long t0 = clock64();
    while (p >= 0) {
        const int64_t idx = p - lane;
        uint64_t v = 0;
        const uint32_t f = idx >= 0 ? read_status64(st, idx, &v) : 2u;  // before tile 0: an inclusive 0
        const unsigned incl = __ballot_sync(0xffffffffu, f == 2);
        const int stop = incl ? __ffs(incl) - 1 : 31;
        const unsigned empty = __ballot_sync(0xffffffffu, f == 0) & (stop == 31 ? 0xffffffffu : ((2u << stop) - 1));
        if (empty) {
            if (clock64() - t0 > kSpinBudget) {
                if (lane == 0) atomicOr(err, 4);
                break;
            }
            continue;
        }
        uint64_t s = lane <= stop ? v : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        excl += s;
        if (incl) break;
        p -= 32;
    }
    if (lane == 0) publish64(st.inc, tile, excl + agg);
    return excl;
}

// Inclusive wrapping prefix sums of the first `limit` deltas (U = the
// unsigned type of T's width), base added; outputs for rows [offset, limit)
// go to out[row - offset].  Tiles are claimed in launch order from *ctr.
template <typename U>
__global__ void __launch_bounds__(kThreads, 4) delta_decode_kernel(const U* __restrict__ deltas, uint64_t limit,
                                                                U base, uint64_t offset, U* __restrict__ out,
                                                                Status64 st, unsigned int* ctr, int vec, int* err) {
    __shared__ uint64_t s_tile;
    __shared__ uint64_t s_warp[kThreads / 32];
    __shared__ uint64_t s_base;
    __shared__ U s_out[kTile + kTile / 16];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t ntiles = (limit + kTile - 1) / kTile;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t r0 = tile * kTile + static_cast<uint64_t>(threadIdx.x) * kPer;
        U v[kPer];
        if (vec && r0 + kPer <= limit) {
#pragma unroll
            for (int k = 0; k < kPer; k += 16 / sizeof(U)) {
                const uint4 q = __ldcs(reinterpret_cast<const uint4*>(deltas + r0 + k));
                const U* pq = reinterpret_cast<const U*>(&q);
#pragma unroll
                for (int j = 0; j < static_cast<int>(16 / sizeof(U)); ++j) v[k + j] = pq[j];
            }
        } else {
#pragma unroll
            for (int k = 0; k < kPer; ++k) v[k] = r0 + k < limit ? deltas[r0 + k] : U(0);
        }
        // thread-local inclusive sums (wrapping in U)
#pragma unroll
        for (int k = 1; k < kPer; ++k) v[k] = static_cast<U>(v[k] + v[k - 1]);
        uint64_t incl = static_cast<uint64_t>(v[kPer - 1]);
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += y;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const uint64_t x = lane < kThreads / 32 ? s_warp[lane] : 0;
            uint64_t t = x;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint64_t y = __shfl_up_sync(0xffffffffu, t, d);
                if (lane >= d) t += y;
            }
            if (lane < kThreads / 32) s_warp[lane] = t - x;
            const uint64_t total = __shfl_sync(0xffffffffu, t, kThreads / 32 - 1);
            const uint64_t e = lookback64_warp(st, tile, total, err);
            if (lane == 0) s_base = e;
        }
        __syncthreads();
        const U pre = static_cast<U>(base + static_cast<U>(s_base + s_warp[warp] + incl -
                                                          static_cast<uint64_t>(v[kPer - 1])));
#pragma unroll
        for (int k = 0; k < kPer; ++k) s_out[pad16(threadIdx.x * kPer + k)] = static_cast<U>(pre + v[k]);
        __syncthreads();
        // coalesced stores of the tile's rows that lie in [offset, limit)
        const uint64_t t0 = tile * kTile;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const uint32_t j = threadIdx.x + k * kThreads;
            const uint64_t r = t0 + j;
            if (r >= offset && r < limit) out[r - offset] = s_out[pad16(j)];
        }
        __syncthreads();
    }
}

// out[i] = base + (f64) code[offset + i] * scale, rounded per operation
__global__ void __launch_bounds__(kThreads) for_decode_kernel(const int32_t* __restrict__ code, uint64_t offset,
                                                              uint64_t count, double base, double scale,
                                                              double* __restrict__ out) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i0 < count; i0 += 4 * stride) {
        int32_t c[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint64_t i = i0 + k * stride;
            c[k] = i < count ? __ldcs(code + offset + i) : 0;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint64_t i = i0 + k * stride;
            if (i < count) __stcs(out + i, __dadd_rn(base, __dmul_rn(static_cast<double>(c[k]), scale)));
        }
    }
}

// deltas[i] = data[i] - data[i-1] (data[-1] = 0), wrapping
template <typename U>
__global__ void __launch_bounds__(kThreads) delta_encode_kernel(const U* __restrict__ data, uint64_t n,
                                                                U* __restrict__ deltas) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const U prev = i ? __ldg(data + i - 1) : U(0);
        deltas[i] = static_cast<U>(__ldg(data + i) - prev);
    }
}

// min / max of the column as order keys (one atomic pair per block)
__global__ void __launch_bounds__(kThreads) minmax_f64_kernel(const double* __restrict__ x, uint64_t n,
                                                              unsigned long long* mm) {
    uint64_t lo = ~0ull, hi = 0;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t k = f64_order_key(__ldcs(x + i));
        lo = k < lo ? k : lo;
        hi = k > hi ? k : hi;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const uint64_t a = __shfl_xor_sync(0xffffffffu, lo, o), b = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&mm[0], static_cast<unsigned long long>(lo));
        atomicMax(&mm[1], static_cast<unsigned long long>(hi));
    }
}

// code[i] = (i32) llround((x[i] - base) / scale): round half away from zero,
// then the low 32 bits, as the reference's static_cast<i32> of a long long
__global__ void __launch_bounds__(kThreads) for_encode_kernel(const double* __restrict__ x, uint64_t n, double base,
                                                              double scale, int32_t* __restrict__ code) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double t = __ddiv_rn(__dsub_rn(__ldcs(x + i), base), scale);
        code[i] = static_cast<int32_t>(static_cast<uint32_t>(static_cast<unsigned long long>(llround(t))));
    }
}

int stream_grid(uint64_t n, int per_sm = 8) {
    const int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t g = (n + kThreads * 4 - 1) / (kThreads * 4);
    const uint64_t cap = static_cast<uint64_t>(sms) * per_sm;
    if (g > cap) g = cap;
    return g < 1 ? 1 : static_cast<int>(g);
}

bool delta_type(int dtype) { return dtype == I64 || dtype == I32 || dtype == U64 || dtype == U32; }

}  // namespace

size_t delta_scratch_bytes(uint64_t limit) {
    const uint64_t ntiles = (limit + kTile - 1) / kTile;
    return ntiles * 32 + 64;  // two 2-word statuses per tile + the tile counter
}

int launch_delta_decode(int dtype, const void* deltas, uint64_t n, uint64_t base_bits, uint64_t offset,
                        uint64_t count, void* out, void* scratch, int* err, cudaStream_t s) {
    if (offset >= n || count == 0) return kOk;
    const uint64_t limit = offset + (count < n - offset ? count : n - offset);
    const uint64_t ntiles = (limit + kTile - 1) / kTile;
    Status64 st;
    st.agg = static_cast<unsigned long long*>(scratch);
    st.inc = st.agg + 2 * ntiles;
    unsigned int* ctr = reinterpret_cast<unsigned int*>(st.inc + 2 * ntiles);
    VX_CUDA(cudaMemsetAsync(scratch, 0, ntiles * 32 + 4, s));
    const int sms = sm_count() > 0 ? sm_count() : 148;
    const int vec = (reinterpret_cast<uintptr_t>(deltas) & 15) == 0 ? 1 : 0;
    const uint64_t grid = ntiles < static_cast<uint64_t>(sms) * 4 ? ntiles : static_cast<uint64_t>(sms) * 4;
    if (dtype_size(dtype) == 8)
        delta_decode_kernel<uint64_t><<<static_cast<unsigned>(grid), kThreads, 0, s>>>(
            static_cast<const uint64_t*>(deltas), limit, base_bits, offset, static_cast<uint64_t*>(out), st, ctr,
            vec, err);
    else
        delta_decode_kernel<uint32_t><<<static_cast<unsigned>(grid), kThreads, 0, s>>>(
            static_cast<const uint32_t*>(deltas), limit, static_cast<uint32_t>(base_bits), offset,
            static_cast<uint32_t*>(out), st, ctr, vec, err);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

int launch_delta_encode(int dtype, const void* data, uint64_t n, void* deltas, cudaStream_t s) {
    if (!n) return kOk;
    if (dtype_size(dtype) == 8)
        delta_encode_kernel<uint64_t><<<stream_grid(n), kThreads, 0, s>>>(static_cast<const uint64_t*>(data), n,
                                                                          static_cast<uint64_t*>(deltas));
    else
        delta_encode_kernel<uint32_t><<<stream_grid(n), kThreads, 0, s>>>(static_cast<const uint32_t*>(data), n,
                                                                          static_cast<uint32_t*>(deltas));
    VX_CUDA(cudaGetLastError());
    return kOk;
}

int launch_for_decode_f64(const int32_t* code, uint64_t n, double base, double scale, uint64_t offset,
                          uint64_t count, double* out, cudaStream_t s) {
    if (offset >= n || count == 0) return kOk;
    const uint64_t m = count < n - offset ? count : n - offset;
    for_decode_kernel<<<stream_grid(m), kThreads, 0, s>>>(code, offset, m, base, scale, out);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

}  // namespace vx

using namespace vx;

namespace {

thread_local DevBuf t_err;
int* dev_err(cudaStream_t s) {
    if (!t_err.p) {
        t_err = DevBuf(16);
        if (t_err.p) cudaMemsetAsync(t_err.p, 0, 16, s);
    }
    return t_err.as<int>();
}

int check_err(int* e, cudaStream_t s) {
    int h = 0;
    if (int st = d2h(&h, e, 4, s)) return st;
    if (int st = sync(s)) return st;
    if (h) {
        cudaMemsetAsync(e, 0, 4, s);
        set_error(kErrDeviceTimeout, "a tile-prefix wait of the delta decode ran out of budget");
        return kErrDeviceTimeout;
    }
    return kOk;
}

int delta_decode_dev_impl(int dtype, const void* d_deltas, size_t n, uint64_t base_bits, size_t offset, size_t count,
                          void* d_out, cudaStream_t s, bool check) {
    if (!delta_type(dtype)) {
        set_error(kErrInvalidArg, "delta decode: element type %d is not an integer type", dtype);
        return kErrInvalidArg;
    }
    static thread_local DevBuf scratch;
    const uint64_t limit = offset < n ? offset + (count < n - offset ? count : n - offset) : 0;
    const size_t need = delta_scratch_bytes(limit);
    if (scratch.n < need) {
        scratch = DevBuf(need);
        if (!scratch.p) return kErrOutOfMemory;
    }
    int* e = dev_err(s);
    if (!e) return kErrOutOfMemory;
    if (int st = launch_delta_decode(dtype, d_deltas, n, base_bits, offset, count, d_out, scratch.p, e, s)) return st;
    return check ? check_err(e, s) : kOk;
}

}  // namespace

extern "C" {

int voxel_delta_decode_dev(int dtype, const void* d_deltas, size_t n, uint64_t base_bits, size_t offset,
                           size_t count, void* d_out, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    return delta_decode_dev_impl(dtype, d_deltas, n, base_bits, offset, count, d_out,
                                 static_cast<cudaStream_t>(stream), true);
}

int voxel_delta_decode(int dtype, const void* deltas, size_t n, uint64_t base_bits, size_t offset, size_t count,
                       void* out) {
    clear_error();
    if (int st = ensure_device()) return st;
    if (!delta_type(dtype)) {
        set_error(kErrInvalidArg, "delta decode: element type %d is not an integer type", dtype);
        return kErrInvalidArg;
    }
    cudaStream_t s = thread_stream();
    const size_t es = dtype_size(dtype);
    const uint64_t limit = offset < n ? offset + (count < n - offset ? count : n - offset) : 0;
    const uint64_t m = limit > offset ? limit - offset : 0;
    DevBuf dd(limit * es), o(m * es);
    if (!dd.ok(limit * es) || !o.ok(m * es)) return kErrOutOfMemory;
    if (int st = h2d(dd.p, deltas, limit * es, s)) return st;
    if (int st = delta_decode_dev_impl(dtype, dd.p, limit, base_bits, offset, count, o.p, s, false)) return st;
    if (int st = d2h(out, o.p, m * es, s)) return st;
    return check_err(dev_err(s), s);
}

int voxel_delta_encode_dev(int dtype, const void* d_data, size_t n, void* d_deltas, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    if (!delta_type(dtype)) {
        set_error(kErrInvalidArg, "delta encode: element type %d is not an integer type", dtype);
        return kErrInvalidArg;
    }
    return launch_delta_encode(dtype, d_data, n, d_deltas, static_cast<cudaStream_t>(stream));
}

int voxel_delta_encode(int dtype, const void* data, size_t n, void* deltas) {
    clear_error();
    if (int st = ensure_device()) return st;
    if (!delta_type(dtype)) {
        set_error(kErrInvalidArg, "delta encode: element type %d is not an integer type", dtype);
        return kErrInvalidArg;
    }
    cudaStream_t s = thread_stream();
    const size_t es = dtype_size(dtype);
    DevBuf dd(n * es), o(n * es);
    if (!dd.ok(n * es) || !o.ok(n * es)) return kErrOutOfMemory;
    if (int st = h2d(dd.p, data, n * es, s)) return st;
    if (int st = launch_delta_encode(dtype, dd.p, n, o.p, s)) return st;
    if (int st = d2h(deltas, o.p, n * es, s)) return st;
    return sync(s);
}

int voxel_for_decode_f64_dev(const int32_t* d_code, size_t n, double base, double scale, size_t offset, size_t count,
                             double* d_out, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    return launch_for_decode_f64(d_code, n, base, scale, offset, count, d_out, static_cast<cudaStream_t>(stream));
}

int voxel_for_decode_f64(const int32_t* code, size_t n, double base, double scale, size_t offset, size_t count,
                         double* out) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = thread_stream();
    const uint64_t m = offset < n ? (count < n - offset ? count : n - offset) : 0;
    DevBuf dc(m * 4), o(m * 8);
    if (!dc.ok(m * 4) || !o.ok(m * 8)) return kErrOutOfMemory;
    if (int st = h2d(dc.p, code + offset, m * 4, s)) return st;
    if (int st = launch_for_decode_f64(dc.as<int32_t>(), m, base, scale, 0, m, o.as<double>(), s)) return st;
    if (int st = d2h(out, o.p, m * 8, s)) return st;
    return sync(s);
}

int voxel_for_encode_f64_dev(const double* d_data, size_t n, int32_t* d_code, double* base, double* scale,
                             void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (n == 0) {
        if (base) *base = 0.0;
        if (scale) *scale = 1.0;
        return kOk;
    }
    static thread_local DevBuf mm;
    if (!mm.p) {
        mm = DevBuf(16);
        if (!mm.p) return kErrOutOfMemory;
    }
    const unsigned long long init[2] = {~0ull, 0ull};
    if (int st = h2d(mm.p, init, 16, s)) return st;
    minmax_f64_kernel<<<stream_grid(n, 4), kThreads, 0, s>>>(d_data, n, mm.as<unsigned long long>());
    VX_CUDA(cudaGetLastError());
    unsigned long long h[2];
    if (int st = d2h(h, mm.p, 16, s)) return st;
    if (int st = sync(s)) return st;
    auto from_key = [](unsigned long long k) {
        const uint64_t b = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
        double d;
        memcpy(&d, &b, 8);
        return d;
    };
    // encoding.hpp:464-476: the first value seeds min / max and only < / >
    // replace them, which the order keys reproduce for non-NaN columns
    const double lo = from_key(h[0]), hi = from_key(h[1]);
    const double range = hi - lo;
    const double sc = range <= 0.0 ? 1.0 : range / static_cast<double>(INT32_MAX);
    for_encode_kernel<<<stream_grid(n), kThreads, 0, s>>>(d_data, n, lo, sc, d_code);
    VX_CUDA(cudaGetLastError());
    if (base) *base = lo;
    if (scale) *scale = sc;
    return kOk;
}

int voxel_for_encode_f64(const double* data, size_t n, int32_t* code, double* base, double* scale) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = thread_stream();
    DevBuf dd(n * 8), o(n * 4);
    if (!dd.ok(n * 8) || !o.ok(n * 4)) return kErrOutOfMemory;
    if (int st = h2d(dd.p, data, n * 8, s)) return st;
    if (int st = voxel_for_encode_f64_dev(dd.as<double>(), n, o.as<int32_t>(), base, scale, s)) return st;
    if (int st = d2h(code, o.p, n * 4, s)) return st;
    return sync(s);
}

}  // extern "C"
