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
#include "tune.h"
#include "voxel_c.h"
#include "vx_common.cuh"
#include "vx_runtime.h"
#include "vx_scan.cuh"

namespace vx {

namespace {

constexpr int kFThreads = 256;
// bitmap words per warp iteration (256 rows; 8 loads in flight per thread;
// 8 words for 4-byte types measured slower)
template <typename T>
constexpr int words_per_warp() { return 4; }

// OP is the comparison code, fixed per kernel instance (no per-row dispatch)
template <typename T, int OP>
__device__ __forceinline__ bool pred(T v, T a, T b) {
    if constexpr (OP == 6) return v >= a && v <= b;  // Between is lo <= v <= hi (filter.hpp:272)
    else if constexpr (OP == 0) return v == a;
    else if constexpr (OP == 1) return v != a;
    else if constexpr (OP == 2) return v < a;
    else if constexpr (OP == 3) return v <= a;
    else if constexpr (OP == 4) return v > a;
    else return v >= a;
}

template <typename T, int OP>
__global__ void __launch_bounds__(kFThreads) vfilter_kernel(const T* __restrict__ data, uint64_t n, T a, T b,
                                                            uint64_t* __restrict__ bitmap,
                                                            unsigned long long* count) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const uint64_t nwords = (n + 63) / 64;
    constexpr int kWordsPerWarp = words_per_warp<T>();
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
            unsigned lo = __ballot_sync(0xffffffffu, r < n && pred<T, OP>(v[k][0], a, b));
            unsigned hi = __ballot_sync(0xffffffffu, r + 32 < n && pred<T, OP>(v[k][1], a, b));
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

constexpr int kAndMax = 64;  // bitmaps whose pointers are held in shared memory

// inl.p[k] by a chain of selects over the parameter words (an indexed read
// would copy the whole list to local memory first)
__device__ __forceinline__ const uint64_t* list_at(const BitmapList& inl, int k) {
    const uint64_t* r = nullptr;
#pragma unroll
    for (int j = 0; j < kAndInline; ++j) r = j == k ? inl.p[j] : r;
    return r;
}

// bms: a device array of nbm bitmap pointers, or null with the pointers passed
// by value in inl (nbm <= kAndInline: no pointer table to upload first)
__global__ void bitmap_and_kernel(BitmapList inl, const uint64_t* const* bms, int nbm, uint64_t rows, uint64_t* out,
                                  unsigned long long* count) {
    constexpr int kU = 4;   // words per thread per step
    constexpr int kB = 4;   // bitmaps whose loads are issued together
    __shared__ const uint64_t* s_bm[kAndMax];
    const int nsm = nbm < kAndMax ? nbm : kAndMax;
    for (int k = threadIdx.x; k < nsm; k += blockDim.x) s_bm[k] = bms ? bms[k] : list_at(inl, k);
    __syncthreads();
    const uint64_t nwords = (rows + 63) / 64;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    unsigned int cnt = 0;
    for (uint64_t w0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; w0 < nwords; w0 += kU * stride) {
        uint64_t x[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint64_t w = w0 + u * stride;
            x[u] = ~0ull;
            if (w == nwords - 1 && (rows & 63)) x[u] = (1ull << (rows & 63)) - 1;
        }
        // kB bitmaps x kU words of loads in flight before any of them is used
        for (int k = 0; k < nbm; k += kB) {
            uint64_t v[kB][kU];
#pragma unroll
            for (int j = 0; j < kB; ++j) {
                const int kk = k + j;
                const uint64_t* b = kk < nbm ? (kk < kAndMax ? s_bm[kk] : bms[kk]) : nullptr;
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const uint64_t w = w0 + u * stride;
                    v[j][u] = b && w < nwords ? __ldcs(b + w) : ~0ull;
                }
            }
#pragma unroll
            for (int j = 0; j < kB; ++j)
#pragma unroll
                for (int u = 0; u < kU; ++u) x[u] &= v[j][u];
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint64_t w = w0 + u * stride;
            if (w >= nwords) break;
            out[w] = x[u];
            cnt += __popcll(x[u]);
        }
    }
    for (int d = 16; d > 0; d >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, d);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(count, static_cast<unsigned long long>(cnt));
}

// Selection vector: tile = kSelWords words per block iteration.  Warp w of the
// block takes words [w*512, w*512+512) of the tile in 16 rounds of 32 (lane l
// reads word round*32 + l, coalesced); a round's rows are gathered in the
// warp's shared-memory stage and stored as one contiguous run.
constexpr int kSelThreads = 128;
constexpr int kSelRounds = 8;
constexpr int kSelWords = kSelThreads * kSelRounds;  // 1024 words = 65536 rows per tile

__global__ void __launch_bounds__(kSelThreads) selection_kernel(const uint64_t* __restrict__ bitmap, uint64_t nwords,
                                                                uint64_t rows, uint32_t* __restrict__ out,
                                                                unsigned long long* count,
                                                                unsigned long long* status, unsigned int* tile_ctr,
                                                                int* err) {
    __shared__ uint64_t s_tile;
    __shared__ uint64_t s_warp[kSelThreads / 32];
    __shared__ uint64_t s_base;
    __shared__ uint32_t s_stage[kSelThreads / 32][32 * 64];
    const uint64_t ntiles = (nwords + kSelWords - 1) / kSelWords;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t* const stage = s_stage[warp];
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t wbase = tile * kSelWords + static_cast<uint64_t>(warp) * 32 * kSelRounds;
        uint64_t wv[kSelRounds];
        uint32_t rt[kSelRounds], wt = 0;
#pragma unroll
        for (int k = 0; k < kSelRounds; ++k) {
            const uint64_t w = wbase + k * 32 + lane;
            uint64_t x = w < nwords ? bitmap[w] : 0;
            if (w == nwords - 1 && (rows & 63)) x &= (1ull << (rows & 63)) - 1;  // tail word: existing rows only
            wv[k] = x;
            rt[k] = __reduce_add_sync(0xffffffffu, static_cast<unsigned>(__popcll(x)));
            wt += rt[k];
        }
        if (lane == 0) s_warp[warp] = wt;
        __syncthreads();
        if (warp == 0) {  // warp offsets, then the tile's offset from a warp-wide look-back
            uint64_t run = 0, mine = 0;
#pragma unroll
            for (int w = 0; w < kSelThreads / 32; ++w) {
                if (lane == w) mine = run;
                run += s_warp[w];
            }
            __syncwarp();
            if (lane < kSelThreads / 32) s_warp[lane] = mine;
            const uint64_t e = lookback_exclusive_warp(status, tile, run, err);
            if (lane == 0) s_base = e;
        }
        __syncthreads();
        uint64_t pos = s_base + s_warp[warp];
#pragma unroll
        for (int k = 0; k < kSelRounds; ++k) {
            const uint32_t rk = rt[k];
            if (rk == 0) continue;  // uniform over the warp
            uint64_t x = wv[k];
            const uint32_t c = __popcll(x);
            uint32_t incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            uint32_t q = incl - c;
            const uint32_t row0 = static_cast<uint32_t>((wbase + k * 32 + lane) * 64);
            while (x) {
                stage[q++] = row0 + static_cast<uint32_t>(__ffsll(static_cast<long long>(x)) - 1);
                x &= x - 1;
            }
            __syncwarp();
            for (uint32_t i = lane; i < rk; i += 32) out[pos + i] = stage[i];
            __syncwarp();
            pos += rk;
        }
        if (tile == ntiles - 1 && threadIdx.x == kSelThreads - 1) *count = s_base + s_warp[warp] + wt;
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
    constexpr int kWordsPerWarp = words_per_warp<T>();
    uint64_t warps_needed = (words + kWordsPerWarp - 1) / kWordsPerWarp;
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t blocks = (warps_needed * 32 + kFThreads - 1) / kFThreads;
    uint64_t cap = static_cast<uint64_t>(sms) * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
#define VX_VF(OPC) \
    vfilter_kernel<T, OPC><<<static_cast<unsigned>(blocks), kFThreads, 0, s>>>(static_cast<const T*>(d), n, ta, tb, bm, count)
    switch (op) {
    case 0: VX_VF(0); break;
    case 1: VX_VF(1); break;
    case 2: VX_VF(2); break;
    case 3: VX_VF(3); break;
    case 4: VX_VF(4); break;
    case 5: VX_VF(5); break;
    default: VX_VF(6); break;
    }
#undef VX_VF
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

namespace {
// one selection pass with `per_sm` resident blocks per SM (tiles are claimed
// dynamically, so any grid gives the same rows)
int selection_pass(const uint64_t* bm, uint64_t rows, uint32_t* out, unsigned long long* count, void* scratch,
                   int* err, cudaStream_t s, int per_sm) {
    uint64_t nwords = (rows + 63) / 64;
    uint64_t ntiles = (nwords + kSelWords - 1) / kSelWords;
    VX_CUDA(cudaMemsetAsync(scratch, 0, selection_scratch_bytes(rows), s));
    VX_CUDA(cudaMemsetAsync(count, 0, 8, s));
    if (ntiles == 0) return kOk;
    unsigned long long* status = static_cast<unsigned long long*>(scratch);
    unsigned int* ctr = reinterpret_cast<unsigned int*>(status + ntiles);
    int sms = sm_count() > 0 ? sm_count() : 148;
    const uint64_t cap = static_cast<uint64_t>(sms) * per_sm;
    uint64_t blocks = ntiles < cap ? ntiles : cap;
    selection_kernel<<<static_cast<unsigned>(blocks), kSelThreads, 0, s>>>(bm, nwords, rows, out, count, status, ctr,
                                                                          err);
    VX_CUDA(cudaGetLastError());
    return kOk;
}
}  // namespace

// Fewer resident tiles shorten every tile's look-back walk (the walk passes
// over the tiles still in flight) but keep fewer loads in flight: the
// autotuner times 1, 2, 4 and 8 blocks per SM once per (GPU, log2 rows) on the
// call's own bitmap (every choice writes the same rows) and keeps the fastest.
int launch_selection(const uint64_t* bm, uint64_t rows, uint32_t* out, unsigned long long* count, void* scratch,
                     int* err, cudaStream_t s) {
    static const int kPerSm[4] = {1, 2, 4, 8};
    int c = 3;  // 8 blocks per SM unless tuned
    if (rows >= (1ull << 22)) {
        const std::string key = tune_key("selection_grid", U32, rows);
        if (!tune_lookup(key, &c))
            c = tune_pick(key, 4, 3, s, [&](int k) { return selection_pass(bm, rows, out, count, scratch, err, s,
                                                                           kPerSm[k]); });
        if (c < 0 || c > 3) c = 3;
    }
    return selection_pass(bm, rows, out, count, scratch, err, s, kPerSm[c]);
}

int launch_bitmap_and_from(const BitmapList& inl, const uint64_t* const* d_bms, int nbm, uint64_t rows,
                           uint64_t* out, unsigned long long* count, cudaStream_t s) {
    VX_CUDA(cudaMemsetAsync(count, 0, 8, s));
    uint64_t words = (rows + 63) / 64;
    if (!words) return kOk;
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t blocks = (words + 1023) / 1024;  // 256 threads x 4 words per step
    if (blocks > static_cast<uint64_t>(sms) * 4) blocks = static_cast<uint64_t>(sms) * 4;  // resident at 64 registers
    bitmap_and_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(inl, d_bms, nbm, rows, out, count);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

int launch_bitmap_and(const uint64_t* const* d_bms, int nbm, uint64_t rows, uint64_t* out, unsigned long long* count,
                      cudaStream_t s) {
    return launch_bitmap_and_from(BitmapList{}, d_bms, nbm, rows, out, count, s);
}

// host array of device bitmap pointers: passed by value when they fit
int launch_bitmap_and_host_list(const uint64_t* const* h_bms, int nbm, uint64_t rows, uint64_t* out,
                                unsigned long long* count, cudaStream_t s) {
    BitmapList inl{};
    for (int k = 0; k < nbm; ++k) inl.p[k] = h_bms[k];
    return launch_bitmap_and_from(inl, nullptr, nbm, rows, out, count, s);
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
    static thread_local int* h_err = nullptr;  // pinned: the read-back is one small DMA
    if (!h_err && cudaHostAlloc(reinterpret_cast<void**>(&h_err), sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        h_err = nullptr;
    }
    int local = 0;
    int& h = h_err ? *h_err : local;
    h = 0;
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
    static thread_local DevBuf scratch;  // look-back words, kept between calls
    const size_t need = selection_scratch_bytes(rows);
    if (scratch.n < need) {
        scratch = DevBuf(need);
        if (!scratch.p) return kErrOutOfMemory;
    }
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

int voxel_bitmap_and_dev(const uint64_t* const* d_bitmaps, size_t nbm, size_t rows, uint64_t* d_out,
                         uint64_t* d_count, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    if (nbm <= static_cast<size_t>(kAndInline))
        return launch_bitmap_and_host_list(d_bitmaps, static_cast<int>(nbm), rows, d_out,
                                           reinterpret_cast<unsigned long long*>(d_count), s);
    static thread_local DevBuf table;  // the device copy of the pointer table
    if (table.n < nbm * sizeof(void*) + 8) {
        table = DevBuf(nbm * sizeof(void*) + 8);
        if (!table.p) return kErrOutOfMemory;
    }
    if (nbm) {
        if (int st = h2d(table.p, d_bitmaps, nbm * sizeof(void*), s)) return st;
    }
    return launch_bitmap_and(static_cast<const uint64_t* const*>(table.p), static_cast<int>(nbm), rows, d_out,
                             reinterpret_cast<unsigned long long*>(d_count), s);
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
    if (nbm <= static_cast<size_t>(kAndInline)) {
        if (launch_bitmap_and_host_list(ptrs.data(), static_cast<int>(nbm), rows, o.as<uint64_t>(),
                                        c.as<unsigned long long>(), s))
            return static_cast<size_t>(-1);
    } else {
        if (h2d(dptrs.p, ptrs.data(), nbm * sizeof(void*), s)) return static_cast<size_t>(-1);
        if (launch_bitmap_and(static_cast<const uint64_t* const*>(dptrs.p), static_cast<int>(nbm), rows,
                              o.as<uint64_t>(), c.as<unsigned long long>(), s))
            return static_cast<size_t>(-1);
    }
    uint64_t cnt = 0;
    if (d2h(out, o.p, words * 8, s) || d2h(&cnt, c.p, 8, s) || sync(s)) return static_cast<size_t>(-1);
    return cnt;
}

}  // extern "C"
