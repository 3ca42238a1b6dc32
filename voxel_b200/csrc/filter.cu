// VectorFilter / ColumnFilter / SelectionVector on the GPU.
//
// Reference (include/voxel/ops/filter.hpp):
//   VectorFilter<T>::Apply{GT,GE,LT,LE,EQ,NE,Between} (42-288): bit i&63 of word
//     i>>6 is set iff row i passes; PassCount = popcount of the bitmap.
//   ColumnFilter::Init + AndWith (526-547): word-wise AND, tail bits cleared.
//   SelectionVector::BuildFromBitmap (378-399): ascending u32 row ids.
// Here a warp builds one 64-bit word from two ballots per 64 rows (lanes read
// consecutive rows, so every load is coalesced), counts with popc and one
// atomic per block, and compaction is a single pass whose block offsets come
// from a decoupled look-back over per-tile popcounts.
#include "filter.h"
#include "voxel_c.h"
#include "vx_common.cuh"
#include "vx_runtime.h"
#include "vx_scan.cuh"

namespace vx {

namespace {

constexpr int kFThreads = 256;
constexpr int kWordsPerWarp = 4;  // 256 rows per warp iteration

template <typename T>
__device__ __forceinline__ bool pred(T v, int op, T a, T b) {
    if (op == 6) return v >= a && v <= b;  // Between is lo <= v <= hi (filter.hpp:272)
    return t_cmp<T>(v, a, op);
}

template <typename T>
__global__ void __launch_bounds__(kFThreads) vfilter_kernel(const T* __restrict__ data, uint64_t n, int op, T a, T b,
                                                            uint64_t* __restrict__ bitmap,
                                                            unsigned long long* count) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const uint64_t nwords = (n + 63) / 64;
    unsigned int cnt = 0;
    for (uint64_t w0 = warp * kWordsPerWarp; w0 < nwords; w0 += nwarps * kWordsPerWarp) {
        T v[kWordsPerWarp][2];
#pragma unroll
        for (int k = 0; k < kWordsPerWarp; ++k) {
            uint64_t r = (w0 + k) * 64 + lane;
            v[k][0] = r < n ? __ldcs(data + r) : T(0);
            v[k][1] = r + 32 < n ? __ldcs(data + r + 32) : T(0);
        }
#pragma unroll
        for (int k = 0; k < kWordsPerWarp; ++k) {
            uint64_t r = (w0 + k) * 64 + lane;
            unsigned lo = __ballot_sync(0xffffffffu, r < n && pred<T>(v[k][0], op, a, b));
            unsigned hi = __ballot_sync(0xffffffffu, r + 32 < n && pred<T>(v[k][1], op, a, b));
            if (lane == k && w0 + k < nwords) {
                bitmap[w0 + k] = static_cast<uint64_t>(lo) | (static_cast<uint64_t>(hi) << 32);
                cnt += __popc(lo) + __popc(hi);
            }
        }
    }
    // block total -> one atomic
    for (int d = 16; d > 0; d >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, d);
    __shared__ unsigned int s[kFThreads / 32];
    if (lane == 0) s[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < kFThreads / 32; ++i) t += s[i];
        if (t) atomicAdd(count, t);
    }
}

__global__ void bitmap_and_kernel(const uint64_t* const* bms, int nbm, uint64_t rows, uint64_t* out,
                                  unsigned long long* count) {
    const uint64_t nwords = (rows + 63) / 64;
    unsigned int cnt = 0;
    for (uint64_t w = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; w < nwords;
         w += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t x = ~0ull;
        if (w == nwords - 1 && (rows & 63)) x = (1ull << (rows & 63)) - 1;
        for (int k = 0; k < nbm; ++k) x &= bms[k][w];
        out[w] = x;
        cnt += __popcll(x);
    }
    for (int d = 16; d > 0; d >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, d);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(count, static_cast<unsigned long long>(cnt));
}

// Selection vector: tile = kSelWords words per block iteration.
constexpr int kSelThreads = 256;
constexpr int kSelWords = kSelThreads * 4;  // 1024 words = 65536 rows per tile

__global__ void __launch_bounds__(kSelThreads) selection_kernel(const uint64_t* __restrict__ bitmap, uint64_t nwords,
                                                                uint64_t rows, uint32_t* __restrict__ out,
                                                                unsigned long long* count,
                                                                unsigned long long* status, unsigned int* tile_ctr,
                                                                int* err) {
    __shared__ uint64_t s_tile;
    __shared__ unsigned int s_warp[kSelThreads / 32];
    __shared__ uint64_t s_base;
    const uint64_t ntiles = (nwords + kSelWords - 1) / kSelWords;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t w0 = tile * kSelWords + threadIdx.x * 4;
        uint64_t wv[4];
        unsigned int c = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uint64_t w = w0 + k;
            uint64_t x = w < nwords ? bitmap[w] : 0;
            if (w == nwords - 1 && (rows & 63)) x &= (1ull << (rows & 63)) - 1;
            wv[k] = x;
            c += __popcll(x);
        }
        // block exclusive scan of c
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        unsigned int inc = c;
        for (int d = 1; d < 32; d <<= 1) {
            unsigned int y = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += y;
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            unsigned int v = lane < kSelThreads / 32 ? s_warp[lane] : 0;
            unsigned int t = v;
            for (int d = 1; d < 32; d <<= 1) {
                unsigned int y = __shfl_up_sync(0xffffffffu, t, d);
                if (lane >= d) t += y;
            }
            if (lane < kSelThreads / 32) s_warp[lane] = t - v;
            if (lane == kSelThreads / 32 - 1) {
                uint64_t agg = t;
                s_base = lookback_exclusive(status, tile, agg, err);
            }
        }
        __syncthreads();
        uint64_t pos = s_base + s_warp[warp] + (inc - c);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uint64_t x = wv[k];
            uint64_t baseRow = (w0 + k) * 64;
            while (x) {
                out[pos++] = static_cast<uint32_t>(baseRow + __ffsll(static_cast<long long>(x)) - 1);
                x &= x - 1;
            }
        }
        if (tile == ntiles - 1 && threadIdx.x == kSelThreads - 1) *count = pos;
        __syncthreads();
    }
}

template <typename T>
int launch_vfilter_t(const void* d, uint64_t n, int op, uint64_t a, uint64_t b, uint64_t* bm,
                     unsigned long long* count, cudaStream_t s) {
    T ta, tb;
    std::memcpy(&ta, &a, sizeof(T));
    std::memcpy(&tb, &b, sizeof(T));
    uint64_t words = (n + 63) / 64;
    uint64_t warps_needed = (words + kWordsPerWarp - 1) / kWordsPerWarp;
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t blocks = (warps_needed * 32 + kFThreads - 1) / kFThreads;
    uint64_t cap = static_cast<uint64_t>(sms) * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    vfilter_kernel<T><<<static_cast<unsigned>(blocks), kFThreads, 0, s>>>(static_cast<const T*>(d), n, op, ta, tb, bm,
                                                                          count);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

}  // namespace

int launch_vfilter(int dtype, const void* d, uint64_t n, int op, uint64_t a, uint64_t b, uint64_t* bm,
                   unsigned long long* count, cudaStream_t s) {
    if (op < 0 || op > 6) {
        set_error(kErrInvalidArg, "comparison code %d outside 0..6", op);
        return kErrInvalidArg;
    }
    VX_CUDA(cudaMemsetAsync(count, 0, 8, s));
    if (n == 0) return kOk;
    switch (dtype) {
    case F64: return launch_vfilter_t<double>(d, n, op, a, b, bm, count, s);
    case F32: return launch_vfilter_t<float>(d, n, op, a, b, bm, count, s);
    case I64: return launch_vfilter_t<int64_t>(d, n, op, a, b, bm, count, s);
    case I32: return launch_vfilter_t<int32_t>(d, n, op, a, b, bm, count, s);
    case U64: return launch_vfilter_t<uint64_t>(d, n, op, a, b, bm, count, s);
    case U32: return launch_vfilter_t<uint32_t>(d, n, op, a, b, bm, count, s);
    default: set_error(kErrInvalidArg, "unknown element type %d", dtype); return kErrInvalidArg;
    }
}

size_t selection_scratch_bytes(uint64_t rows) {
    uint64_t nwords = (rows + 63) / 64;
    uint64_t ntiles = (nwords + kSelWords - 1) / kSelWords;
    return (ntiles + 1) * 8 + 64;
}

int launch_selection(const uint64_t* bm, uint64_t rows, uint32_t* out, unsigned long long* count, void* scratch,
                     int* err, cudaStream_t s) {
    uint64_t nwords = (rows + 63) / 64;
    uint64_t ntiles = (nwords + kSelWords - 1) / kSelWords;
    VX_CUDA(cudaMemsetAsync(scratch, 0, selection_scratch_bytes(rows), s));
    VX_CUDA(cudaMemsetAsync(count, 0, 8, s));
    if (ntiles == 0) return kOk;
    unsigned long long* status = static_cast<unsigned long long*>(scratch);
    unsigned int* ctr = reinterpret_cast<unsigned int*>(status + ntiles);
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t blocks = ntiles < static_cast<uint64_t>(sms) * 8 ? ntiles : static_cast<uint64_t>(sms) * 8;
    selection_kernel<<<static_cast<unsigned>(blocks), kSelThreads, 0, s>>>(bm, nwords, rows, out, count, status, ctr,
                                                                          err);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

int launch_bitmap_and(const uint64_t* const* d_bms, int nbm, uint64_t rows, uint64_t* out, unsigned long long* count,
                      cudaStream_t s) {
    VX_CUDA(cudaMemsetAsync(count, 0, 8, s));
    uint64_t words = (rows + 63) / 64;
    if (!words) return kOk;
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t blocks = (words + 255) / 256;
    if (blocks > static_cast<uint64_t>(sms) * 8) blocks = static_cast<uint64_t>(sms) * 8;
    bitmap_and_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(d_bms, nbm, rows, out, count);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

}  // namespace vx

using namespace vx;

namespace {
struct ErrWord {
    DevBuf b;
    int* get(cudaStream_t s) {
        if (!b.p) {
            b = DevBuf(16);
            if (b.p) cudaMemsetAsync(b.p, 0, 16, s);
        }
        return b.as<int>();
    }
};
thread_local ErrWord t_err;

int check_err(int* d_err, cudaStream_t s) {
    int h = 0;
    int st = d2h(&h, d_err, 4, s);
    if (st) return st;
    st = sync(s);
    if (st) return st;
    if (h) {
        cudaMemsetAsync(d_err, 0, 4, s);
        set_error(kErrDeviceTimeout, "a device-side wait ran out of budget (code %d)", h);
        return kErrDeviceTimeout;
    }
    return kOk;
}
}  // namespace

extern "C" {

int voxel_vfilter_dev(int dtype, int op, const void* d_data, size_t n, uint64_t lo, uint64_t hi, uint64_t* d_bitmap,
                      uint64_t* d_count, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    return launch_vfilter(dtype, d_data, n, op, lo, hi, d_bitmap, reinterpret_cast<unsigned long long*>(d_count), s);
}

size_t voxel_vfilter(int dtype, int op, const void* data, size_t n, uint64_t lo, uint64_t hi, uint64_t* bitmap) {
    clear_error();
    if (ensure_device()) return static_cast<size_t>(-1);
    cudaStream_t s = thread_stream();
    size_t es = dtype_size(dtype), words = (n + 63) / 64;
    DevBuf d(n * es), bm(words * 8), c(8);
    if (!d.ok(n * es) || !bm.ok(words * 8) || !c.p) return static_cast<size_t>(-1);
    if (h2d(d.p, data, n * es, s)) return static_cast<size_t>(-1);
    if (launch_vfilter(dtype, d.p, n, op, lo, hi, bm.as<uint64_t>(), c.as<unsigned long long>(), s))
        return static_cast<size_t>(-1);
    uint64_t cnt = 0;
    if (d2h(bitmap, bm.p, words * 8, s) || d2h(&cnt, c.p, 8, s) || sync(s)) return static_cast<size_t>(-1);
    return cnt;
}

int voxel_selection_from_bitmap_dev(const uint64_t* d_bitmap, size_t rows, uint32_t* d_out, uint64_t* d_count,
                                    void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    DevBuf scratch(selection_scratch_bytes(rows));
    if (!scratch.p) return kErrOutOfMemory;
    int* err = t_err.get(s);
    int st = launch_selection(d_bitmap, rows, d_out, reinterpret_cast<unsigned long long*>(d_count), scratch.p, err, s);
    if (st) return st;
    return check_err(err, s);
}

size_t voxel_selection_from_bitmap(const uint64_t* bitmap, size_t rows, uint32_t* out) {
    clear_error();
    if (ensure_device()) return static_cast<size_t>(-1);
    cudaStream_t s = thread_stream();
    size_t words = (rows + 63) / 64;
    DevBuf bm(words * 8), o(rows * 4), c(8);
    if (!bm.ok(words * 8) || !o.ok(rows * 4) || !c.p) return static_cast<size_t>(-1);
    if (h2d(bm.p, bitmap, words * 8, s)) return static_cast<size_t>(-1);
    if (voxel_selection_from_bitmap_dev(bm.as<uint64_t>(), rows, o.as<uint32_t>(), c.as<uint64_t>(), s))
        return static_cast<size_t>(-1);
    uint64_t cnt = 0;
    if (d2h(&cnt, c.p, 8, s) || sync(s)) return static_cast<size_t>(-1);
    if (cnt && (d2h(out, o.p, cnt * 4, s) || sync(s))) return static_cast<size_t>(-1);
    return cnt;
}

size_t voxel_bitmap_and(const uint64_t* const* bitmaps, size_t nbm, size_t rows, uint64_t* out) {
    clear_error();
    if (ensure_device()) return static_cast<size_t>(-1);
    cudaStream_t s = thread_stream();
    size_t words = (rows + 63) / 64;
    std::vector<DevBuf> bufs;
    std::vector<const uint64_t*> ptrs;
    for (size_t k = 0; k < nbm; ++k) {
        bufs.emplace_back(words * 8);
        if (!bufs.back().ok(words * 8) || h2d(bufs.back().p, bitmaps[k], words * 8, s)) return static_cast<size_t>(-1);
        ptrs.push_back(bufs.back().as<uint64_t>());
    }
    DevBuf dptrs(nbm * sizeof(void*) + 8), o(words * 8), c(8);
    if (!dptrs.p || !o.ok(words * 8) || !c.p) return static_cast<size_t>(-1);
    if (nbm && h2d(dptrs.p, ptrs.data(), nbm * sizeof(void*), s)) return static_cast<size_t>(-1);
    if (launch_bitmap_and(static_cast<const uint64_t* const*>(dptrs.p), static_cast<int>(nbm), rows, o.as<uint64_t>(),
                          c.as<unsigned long long>(), s))
        return static_cast<size_t>(-1);
    uint64_t cnt = 0;
    if (d2h(out, o.p, words * 8, s) || d2h(&cnt, c.p, 8, s) || sync(s)) return static_cast<size_t>(-1);
    return cnt;
}

}  // extern "C"
