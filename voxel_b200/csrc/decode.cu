// Column decoders (reference include/voxel/data/encoding.hpp).
//
//   BitPackedEncoding::Decode / DecodeBatch (397-422): value i lives at bit i*w
//     of little-endian u64 words, LSB first, straddling into the next word.
//   DictionaryEncoding<T>::DecodeBatch (156-167): out[i] = Dictionary[Indices[i]].
//   RLEEncoding<T>::DecodeBatch (231-257): (value, run length) pairs expanded
//     from row `offset`; rows past the last run decode to T{}.
// Outputs are written once, coalesced; the packed words are read through L1
// (neighbouring threads share words); the RLE decode scans each tile of run
// lengths into row starts in shared memory (tile offsets by decoupled
// look-back) and expands the tile's runs from there in the same pass.
#include "decode.h"
#include "voxel_c.h"
#include "vx_common.cuh"
#include "vx_runtime.h"
#include "vx_scan.cuh"

namespace vx {

namespace {

constexpr int kDThreads = 256;
constexpr size_t kGatherSmem = 32768;  // dictionaries up to 32 KB are read from shared memory

// Bit-unpack (and dictionary lookup) per tile of kUnpackRows rows: the block
// stages the tile's packed words in shared memory with independent coalesced
// loads, then each thread decodes rows j, j+256, ... (coalesced stores).
// Words past nwords read as zero.
constexpr int kUnpackRows = 4096;
constexpr int kUnpackWords = kUnpackRows * 32 / 64 + 2;  // widths up to 32

template <bool DICT>
__global__ void __launch_bounds__(kDThreads) unpack_tile_kernel(const uint64_t* __restrict__ words, uint64_t nwords,
                                                                uint32_t w, const int32_t* __restrict__ dict,
                                                                uint32_t card, uint64_t offset, uint64_t count,
                                                                uint32_t* __restrict__ out, int vec_out, int* err) {
    __shared__ uint64_t s_w[kUnpackWords + 1];  // + one word read (masked off) past the last value
    extern __shared__ __align__(16) int32_t s_dict[];
    const bool dict_smem = DICT && card <= 8192;
    if (dict_smem)
        for (uint32_t i = threadIdx.x; i < card; i += blockDim.x) s_dict[i] = dict[i];
    const uint32_t mask = w >= 32 ? ~0u : ((1u << w) - 1u);
    const uint32_t* s_w32 = reinterpret_cast<const uint32_t*>(s_w);  // little-endian halves of s_w
    bool bad = false;
    for (uint64_t tile = blockIdx.x; tile * kUnpackRows < count; tile += gridDim.x) {
        const uint64_t r0 = offset + tile * kUnpackRows;
        const uint32_t nb = static_cast<uint32_t>(min(static_cast<uint64_t>(kUnpackRows), count - tile * kUnpackRows));
        const uint64_t wi0 = (r0 * w) >> 6;
        uint64_t wi1 = ((r0 + nb) * w + 63) >> 6;  // past the last row's last bit: at most nb*w/64 + 2 words
        if (wi1 > nwords) wi1 = nwords;
        const uint32_t nwl = wi1 > wi0 ? static_cast<uint32_t>(wi1 - wi0) : 0;
#pragma unroll
        for (int e = 0; e < (kUnpackWords + kDThreads - 1) / kDThreads; ++e) {
            const uint32_t i = threadIdx.x + e * kDThreads;
            if (i < nwl) s_w[i] = __ldg(words + wi0 + i);
        }
        if (threadIdx.x == 0) s_w[nwl] = 0;  // words past nwords read as zero
        __syncthreads();
        const uint32_t b0 = static_cast<uint32_t>(r0 * w - wi0 * 64);  // the tile's first bit in s_w (< 64)
        if (vec_out && nb == kUnpackRows) {
            // a whole tile: each thread decodes groups of 4 consecutive values (one
            // 16-byte store; lanes store consecutive groups), bit positions stepped
            // by w, no per-value bounds (the staged words cover the tile, and the
            // zero word after them covers the second word of the last value)
            uint4* out4 = reinterpret_cast<uint4*>(out + tile * kUnpackRows);
#pragma unroll
            for (int e = 0; e < kUnpackRows / (4 * kDThreads); ++e) {
                const uint32_t g = threadIdx.x + e * kDThreads;
                uint32_t bit = b0 + g * 4 * w;
                uint32_t o[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const uint32_t q = bit >> 5;
                    uint32_t k = __funnelshift_r(s_w32[q], s_w32[q + 1], bit & 31) & mask;
                    bit += w;
                    if constexpr (DICT) {
                        if (k >= card) {
                            bad = true;
                            k = 0;
                        } else {
                            k = static_cast<uint32_t>(dict_smem ? s_dict[k] : __ldg(dict + k));
                        }
                    }
                    o[i] = k;
                }
                out4[g] = make_uint4(o[0], o[1], o[2], o[3]);
            }
            __syncthreads();
            continue;
        }
#pragma unroll 4
        for (int e = 0; e < kUnpackRows / kDThreads; ++e) {
            const uint32_t j = threadIdx.x + e * kDThreads;
            if (j >= nb) break;
            const uint32_t bit = b0 + j * w;  // < 64 + 4096 * 32
            // a value of <= 32 bits spans at most two 32-bit words
            const uint32_t q = bit >> 5;
            const uint32_t k = q < 2 * nwl ? __funnelshift_r(s_w32[q], s_w32[q + 1], bit & 31) & mask : 0u;
            uint32_t o = k;
            if constexpr (DICT) {
                if (k >= card) {
                    bad = true;
                    o = 0;
                } else {
                    o = static_cast<uint32_t>(dict_smem ? s_dict[k] : __ldg(dict + k));
                }
            }
            out[tile * kUnpackRows + j] = o;
        }
        __syncthreads();
    }
    if (DICT && bad) atomicOr(err, 2);
}

// out[i] = dict[idx[i]]: four rows in flight per thread, the dictionary in
// shared memory when it fits (dynamic shared memory of card entries).
template <typename T>
__global__ void __launch_bounds__(kDThreads) dict_gather_kernel(const T* __restrict__ dict, uint32_t card,
                                                                const uint32_t* __restrict__ idx, uint64_t count,
                                                                T* __restrict__ out, int* err) {
    extern __shared__ __align__(16) unsigned char g_sm[];
    T* sd = reinterpret_cast<T*>(g_sm);
    const bool in_smem = card * sizeof(T) <= kGatherSmem;
    if (in_smem)
        for (uint32_t i = threadIdx.x; i < card; i += blockDim.x) sd[i] = dict[i];
    __syncthreads();
    bool bad = false;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i0 < count; i0 += 4 * stride) {
        uint32_t k[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint64_t i = i0 + u * stride;
            k[u] = i < count ? __ldcs(idx + i) : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint64_t i = i0 + u * stride;
            if (i >= count) break;
            if (k[u] >= card) {
                bad = true;
                out[i] = T(0);
            } else {
                out[i] = in_smem ? sd[k[u]] : __ldg(dict + k[u]);
            }
        }
    }
    if (bad) atomicOr(err, 2);
}

// RLE decode in one pass.  A block takes tiles of kRleTileRuns runs in launch
// order: it loads their lengths and values, scans the lengths into the tile's
// local row starts (shared memory), gets the tile's first row from a
// decoupled look-back over the tiles before it, and writes the tile's rows
// that fall in [offset, offset + count).  Each warp expands steps of
// kRleStepRows rows: it finds the run covering the step's first row by a
// binary search over the local starts, marks the row where each later
// non-empty run of the step begins (two non-empty runs never share a first
// row), takes an inclusive max-scan over the marks (each row's run is the last
// one begun at or before it) and stores the rows' values coalesced.  The tile
// holding the last run writes 0 to the requested rows past the data.
constexpr int kRleRunsPerThread = 8;
constexpr int kRleTileRuns = kDThreads * kRleRunsPerThread;  // 2048 runs per tile
constexpr int kRleStepRows = 512;                             // rows per warp step, 16 per lane
constexpr int kRleWarps = kDThreads / 32;
// 16-bit marks, two pad entries per 16: a lane's 16 marks sit 9 words after its neighbour's
__device__ __forceinline__ uint32_t rle_pad(uint32_t j) { return j + ((j >> 4) << 1); }
// runs' starts and values: one pad entry per 8 runs, so a thread's 8 runs and
// its neighbour's sit 9 entries apart (conflict-free stores)
__device__ __forceinline__ int run_pad(int r) { return r + (r >> 3); }
constexpr int kRlePadRuns = kRleTileRuns + kRleTileRuns / 8 + 1;

template <typename T>
__global__ void __launch_bounds__(kDThreads, 4) rle_decode_kernel(const T* __restrict__ values,
                                                               const uint32_t* __restrict__ runs, uint64_t nruns,
                                                               uint64_t offset, uint64_t count, T* __restrict__ out,
                                                               unsigned long long* status, unsigned int* ctr,
                                                               int* err) {
    __shared__ uint64_t s_start[kRlePadRuns];  // local first row of each run (run_pad); run kRleTileRuns: tile rows
    __shared__ T s_val[kRlePadRuns];
    __shared__ uint16_t s_mark[kRleWarps][kRleStepRows + kRleStepRows / 8];  // run index - k0 (< 2^11)
    __shared__ uint64_t s_warp[kRleWarps];
    __shared__ uint64_t s_tile, s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t ntiles = (nruns + kRleTileRuns - 1) / kRleTileRuns;
    const uint64_t end = offset + count;
    uint16_t* const mark = s_mark[warp];
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t t0 = tile * kRleTileRuns;
        const int nin = static_cast<int>(nruns - t0 < kRleTileRuns ? nruns - t0 : kRleTileRuns);
        const uint64_t r0 = t0 + static_cast<uint64_t>(threadIdx.x) * kRleRunsPerThread;
        uint32_t len[kRleRunsPerThread];
        T val[kRleRunsPerThread];
        if (r0 + kRleRunsPerThread <= nruns && ((reinterpret_cast<uintptr_t>(runs + r0) |
                                                  reinterpret_cast<uintptr_t>(values + r0)) & 15) == 0) {
            const uint4* lp = reinterpret_cast<const uint4*>(runs + r0);
            const uint4 a = __ldcs(lp), b = __ldcs(lp + 1);
            len[0] = a.x; len[1] = a.y; len[2] = a.z; len[3] = a.w;
            len[4] = b.x; len[5] = b.y; len[6] = b.z; len[7] = b.w;
#pragma unroll
            for (int k = 0; k < kRleRunsPerThread; ++k) val[k] = __ldcs(values + r0 + k);
        } else {
#pragma unroll
            for (int k = 0; k < kRleRunsPerThread; ++k) {
                const bool in = r0 + k < nruns;
                len[k] = in ? runs[r0 + k] : 0u;
                val[k] = in ? values[r0 + k] : T(0);
            }
        }
        uint64_t c = 0;
#pragma unroll
        for (int k = 0; k < kRleRunsPerThread; ++k) c += len[k];
        uint64_t inc = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += y;
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            const uint64_t x = lane < kRleWarps ? s_warp[lane] : 0;
            uint64_t t = x;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint64_t y = __shfl_up_sync(0xffffffffu, t, d);
                if (lane >= d) t += y;
            }
            if (lane < kRleWarps) s_warp[lane] = t - x;
            const uint64_t total = __shfl_sync(0xffffffffu, t, 31);
            const uint64_t e = lookback_exclusive_warp(status, tile, total, err);
            if (lane == 0) s_base = e;
        }
        __syncthreads();
        {
            uint64_t st = s_warp[warp] + (inc - c);
#pragma unroll
            for (int k = 0; k < kRleRunsPerThread; ++k) {
                s_start[run_pad(threadIdx.x * kRleRunsPerThread + k)] = st;
                s_val[run_pad(threadIdx.x * kRleRunsPerThread + k)] = val[k];
                st += len[k];
            }
            if (threadIdx.x == kDThreads - 1) s_start[run_pad(kRleTileRuns)] = st;  // runs past nruns are empty
        }
        __syncthreads();
        const uint64_t base = s_base, trows = s_start[run_pad(kRleTileRuns)];
        const uint64_t lo = base > offset ? base : offset;
        const uint64_t hi = base + trows < end ? base + trows : end;
        for (uint64_t cs = lo + static_cast<uint64_t>(warp) * kRleStepRows; cs < hi;
             cs += static_cast<uint64_t>(kRleWarps) * kRleStepRows) {
            const uint32_t nb = static_cast<uint32_t>(hi - cs < kRleStepRows ? hi - cs : kRleStepRows);
            const uint64_t x0 = cs - base;  // the step's first row, local: below trows
            // the last run beginning at or before x0 (non-empty: an empty run
            // shares its first row with the run after it, or begins at trows)
            int ka = 0, kb = nin;
            while (kb - ka > 1) {
                const int m = (ka + kb) >> 1;
                if (s_start[run_pad(m)] <= x0) ka = m;
                else kb = m;
            }
            const int k0 = ka;
#pragma unroll
            for (int e = 0; e < kRleStepRows / 32; ++e) mark[rle_pad(lane * (kRleStepRows / 32) + e)] = 0;
            __syncwarp();
            for (int k = k0 + 1 + lane; k < nin; k += 32) {
                const uint64_t sk = s_start[run_pad(k)];
                if (sk >= x0 + nb) break;  // starts are non-decreasing
                if (s_start[run_pad(k + 1)] > sk)
                    mark[rle_pad(static_cast<uint32_t>(sk - x0))] = static_cast<uint16_t>(k - k0);
            }
            __syncwarp();
            uint32_t loc[kRleStepRows / 32], m = 0;
#pragma unroll
            for (int e = 0; e < kRleStepRows / 32; ++e) {
                m = max(m, static_cast<uint32_t>(mark[rle_pad(lane * (kRleStepRows / 32) + e)]));
                loc[e] = m;
            }
            uint32_t incl = m;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl = max(incl, y);
            }
            uint32_t pre = __shfl_up_sync(0xffffffffu, incl, 1);
            if (lane == 0) pre = 0;
            __syncwarp();
#pragma unroll
            for (int e = 0; e < kRleStepRows / 32; ++e)
                mark[rle_pad(lane * (kRleStepRows / 32) + e)] = static_cast<uint16_t>(max(pre, loc[e]));
            __syncwarp();
#pragma unroll
            for (int i = 0; i < kRleStepRows / 32; ++i) {
                const uint32_t j = lane + 32 * i;
                if (j < nb) out[cs + j - offset] = s_val[run_pad(k0 + static_cast<int>(mark[rle_pad(j)]))];
            }
            __syncwarp();  // the marks are cleared for the next step
        }
        if (tile == ntiles - 1) {  // requested rows past the last run
            const uint64_t past = base + trows > offset ? base + trows : offset;
            for (uint64_t r = past + threadIdx.x; r < end; r += kDThreads) out[r - offset] = T(0);
        }
        __syncthreads();
    }
}

int unpack_grid(uint64_t count) {
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t b = (count + kUnpackRows - 1) / kUnpackRows;
    uint64_t cap = static_cast<uint64_t>(sms) * 8;
    if (b > cap) b = cap;
    return b < 1 ? 1 : static_cast<int>(b);
}

int grid_for(uint64_t n, int per_sm = 8) {
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t b = (n + kDThreads - 1) / kDThreads;
    uint64_t cap = static_cast<uint64_t>(sms) * per_sm;
    if (b > cap) b = cap;
    return b < 1 ? 1 : static_cast<int>(b);
}

}  // namespace

int launch_bitunpack(const uint64_t* words, uint64_t nwords, uint32_t w, uint64_t value_count, uint64_t offset,
                     uint64_t count, uint32_t* out, cudaStream_t s) {
    if (w == 0 || w > 32) {
        set_error(kErrInvalidArg, "bit width %u outside 1..32", w);
        return kErrInvalidArg;
    }
    if (offset >= value_count) return kOk;
    if (count > value_count - offset) count = value_count - offset;  // reference stops at ValueCount
    if (!count) return kOk;
    const int vec_out = (reinterpret_cast<uintptr_t>(out) & 15) == 0 ? 1 : 0;
    unpack_tile_kernel<false><<<unpack_grid(count), kDThreads, 0, s>>>(words, nwords, w, nullptr, 0, offset, count,
                                                                      out, vec_out, nullptr);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

int launch_dict_bitunpack_i32(const uint64_t* words, uint64_t nwords, uint32_t w, const int32_t* dict, uint32_t card,
                              uint64_t value_count, uint64_t offset, uint64_t count, int32_t* out, int* err,
                              cudaStream_t s) {
    if (w == 0 || w > 32) {
        set_error(kErrInvalidArg, "bit width %u outside 1..32", w);
        return kErrInvalidArg;
    }
    if (offset >= value_count) return kOk;
    if (count > value_count - offset) count = value_count - offset;
    if (!count) return kOk;
    size_t smem = card <= 8192 ? card * sizeof(int32_t) : 0;
    const int vec_out = (reinterpret_cast<uintptr_t>(out) & 15) == 0 ? 1 : 0;
    unpack_tile_kernel<true><<<unpack_grid(count), kDThreads, smem, s>>>(words, nwords, w, dict, card, offset, count,
                                                                        reinterpret_cast<uint32_t*>(out), vec_out,
                                                                        err);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

int launch_dict_gather(int dtype, const void* dict, uint32_t card, const uint32_t* idx, uint64_t count, void* out,
                       int* err, cudaStream_t s) {
    if (!count) return kOk;
    const size_t es = dtype_size(dtype);
    const size_t smem = card * es <= kGatherSmem ? card * es : 0;
    if (dtype == F64)
        dict_gather_kernel<double><<<grid_for(count), kDThreads, smem, s>>>(static_cast<const double*>(dict), card, idx,
                                                                         count, static_cast<double*>(out), err);
    else if (dtype == I32)
        dict_gather_kernel<int32_t><<<grid_for(count), kDThreads, smem, s>>>(static_cast<const int32_t*>(dict), card,
                                                                          idx, count, static_cast<int32_t*>(out), err);
    else if (dtype == I64 || dtype == U64)
        dict_gather_kernel<uint64_t><<<grid_for(count), kDThreads, smem, s>>>(static_cast<const uint64_t*>(dict), card,
                                                                           idx, count, static_cast<uint64_t*>(out),
                                                                           err);
    else
        dict_gather_kernel<uint32_t><<<grid_for(count), kDThreads, smem, s>>>(static_cast<const uint32_t*>(dict), card,
                                                                           idx, count, static_cast<uint32_t*>(out),
                                                                           err);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

size_t rle_scratch_bytes(uint64_t nruns) {
    uint64_t ntiles = (nruns + kRleTileRuns - 1) / kRleTileRuns;
    return (ntiles + 1) * 8 + 64;  // look-back statuses, then the tile counter
}

int launch_rle_decode_i64(const int64_t* values, const uint32_t* runs, uint64_t nruns, uint64_t offset,
                          uint64_t count, int64_t* out, void* scratch, int* err, cudaStream_t s) {
    if (!count) return kOk;
    if (nruns == 0) {
        VX_CUDA(cudaMemsetAsync(out, 0, count * 8, s));
        return kOk;
    }
    const uint64_t ntiles = (nruns + kRleTileRuns - 1) / kRleTileRuns;
    unsigned long long* status = static_cast<unsigned long long*>(scratch);
    unsigned int* ctr = reinterpret_cast<unsigned int*>(status + ntiles);
    VX_CUDA(cudaMemsetAsync(status, 0, (ntiles + 1) * 8, s));
    const int sms = sm_count() > 0 ? sm_count() : 148;
    const uint64_t cap = static_cast<uint64_t>(sms) * 4;
    const uint64_t blocks = ntiles < cap ? ntiles : cap;
    rle_decode_kernel<int64_t><<<static_cast<unsigned>(blocks), kDThreads, 0, s>>>(values, runs, nruns, offset, count,
                                                                                  out, status, ctr, err);
    VX_CUDA(cudaGetLastError());
    return kOk;
}

}  // namespace vx

using namespace vx;

namespace {
thread_local DevBuf t_derr;
int* derr(cudaStream_t s) {
    if (!t_derr.p) {
        t_derr = DevBuf(16);
        if (t_derr.p) cudaMemsetAsync(t_derr.p, 0, 16, s);
    }
    return t_derr.as<int>();
}
int check(int* e, cudaStream_t s) {
    int h = 0;
    if (int st = d2h(&h, e, 4, s)) return st;
    if (int st = sync(s)) return st;
    if (h) {
        cudaMemsetAsync(e, 0, 4, s);
        if (h & 4) { set_error(kErrDeviceTimeout, "a device-side wait ran out of budget"); return kErrDeviceTimeout; }
        set_error(kErrInvalidArg, "an index is outside the dictionary");
        return kErrInvalidArg;
    }
    return kOk;
}
}  // namespace

extern "C" {

int voxel_bitpack_decode_dev(const uint64_t* d_words, size_t nwords, uint32_t width, size_t value_count,
                             size_t offset, size_t count, uint32_t* d_out, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    return launch_bitunpack(d_words, nwords, width, value_count, offset, count, d_out, s);
}

int voxel_bitpack_decode(const uint64_t* words, size_t nwords, uint32_t width, size_t value_count, size_t offset,
                         size_t count, uint32_t* out) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = thread_stream();
    uint64_t n = offset < value_count ? (count < value_count - offset ? count : value_count - offset) : 0;
    DevBuf dw(nwords * 8), o(n * 4);
    if (!dw.ok(nwords * 8) || !o.ok(n * 4)) return kErrOutOfMemory;
    if (int st = h2d(dw.p, words, nwords * 8, s)) return st;
    if (int st = launch_bitunpack(dw.as<uint64_t>(), nwords, width, value_count, offset, count, o.as<uint32_t>(), s))
        return st;
    if (int st = d2h(out, o.p, n * 4, s)) return st;
    return sync(s);
}

int voxel_dict_bitpack_decode_i32(const uint64_t* words, size_t nwords, uint32_t width, const int32_t* dict,
                                  size_t card, size_t value_count, size_t offset, size_t count, int32_t* out) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = thread_stream();
    uint64_t n = offset < value_count ? (count < value_count - offset ? count : value_count - offset) : 0;
    DevBuf dw(nwords * 8), dd(card * 4), o(n * 4);
    if (!dw.ok(nwords * 8) || !dd.ok(card * 4) || !o.ok(n * 4)) return kErrOutOfMemory;
    if (int st = h2d(dw.p, words, nwords * 8, s)) return st;
    if (int st = h2d(dd.p, dict, card * 4, s)) return st;
    int* e = derr(s);
    if (int st = launch_dict_bitunpack_i32(dw.as<uint64_t>(), nwords, width, dd.as<int32_t>(),
                                           static_cast<uint32_t>(card), value_count, offset, count, o.as<int32_t>(),
                                           e, s))
        return st;
    if (int st = d2h(out, o.p, n * 4, s)) return st;
    return check(e, s);
}

int voxel_dict_decode(int dtype, const void* dict, size_t card, const uint32_t* indices, size_t n, size_t offset,
                      size_t count, void* out) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = thread_stream();
    uint64_t m = offset < n ? (count < n - offset ? count : n - offset) : 0;  // encoding.hpp:163-166
    size_t es = dtype_size(dtype);
    DevBuf dd(card * es), di(m * 4), o(m * es);
    if (!dd.ok(card * es) || !di.ok(m * 4) || !o.ok(m * es)) return kErrOutOfMemory;
    if (int st = h2d(dd.p, dict, card * es, s)) return st;
    if (int st = h2d(di.p, indices + offset, m * 4, s)) return st;
    int* e = derr(s);
    if (int st = launch_dict_gather(dtype, dd.p, static_cast<uint32_t>(card), di.as<uint32_t>(), m, o.p, e, s))
        return st;
    if (int st = d2h(out, o.p, m * es, s)) return st;
    return check(e, s);
}

int voxel_dict_bitpack_decode_i32_dev(const uint64_t* d_words, size_t nwords, uint32_t width, const int32_t* d_dict,
                                      size_t card, size_t value_count, size_t offset, size_t count, int32_t* d_out,
                                      void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    int* e = derr(s);
    if (int st = launch_dict_bitunpack_i32(d_words, nwords, width, d_dict, static_cast<uint32_t>(card), value_count,
                                           offset, count, d_out, e, s))
        return st;
    return check(e, s);
}

int voxel_dict_decode_dev(int dtype, const void* d_dict, size_t card, const uint32_t* d_indices, size_t count,
                          void* d_out, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    int* e = derr(s);
    if (int st = launch_dict_gather(dtype, d_dict, static_cast<uint32_t>(card), d_indices, count, d_out, e, s))
        return st;
    return check(e, s);
}

int voxel_rle_decode_i64_dev(const int64_t* d_values, const uint32_t* d_runs, size_t nruns, size_t offset,
                             size_t count, int64_t* d_out, void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    static thread_local DevBuf scratch;
    size_t need = rle_scratch_bytes(nruns);
    if (scratch.n < need) {
        scratch = DevBuf(need);
        if (!scratch.p) return kErrOutOfMemory;
    }
    int* e = derr(s);
    if (int st = launch_rle_decode_i64(d_values, d_runs, nruns, offset, count, d_out, scratch.p, e, s)) return st;
    return kOk;
}

int voxel_rle_decode_i64(const int64_t* values, const uint32_t* runs, size_t nruns, size_t offset, size_t count,
                         int64_t* out) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = thread_stream();
    DevBuf dv(nruns * 8), dr(nruns * 4), o(count * 8);
    if (!dv.ok(nruns * 8) || !dr.ok(nruns * 4) || !o.ok(count * 8)) return kErrOutOfMemory;
    if (int st = h2d(dv.p, values, nruns * 8, s)) return st;
    if (int st = h2d(dr.p, runs, nruns * 4, s)) return st;
    if (int st = voxel_rle_decode_i64_dev(dv.as<int64_t>(), dr.as<uint32_t>(), nruns, offset, count, o.as<int64_t>(),
                                          s))
        return st;
    if (int st = d2h(out, o.p, count * 8, s)) return st;
    return check(derr(s), s);
}

}  // extern "C"
