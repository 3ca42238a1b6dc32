// Column decoders (reference include/voxel/data/encoding.hpp).
//
//   BitPackedEncoding::Decode / DecodeBatch (397-422): value i lives at bit i*w
//     of little-endian u64 words, LSB first, straddling into the next word.
//   DictionaryEncoding<T>::DecodeBatch (156-167): out[i] = Dictionary[Indices[i]].
//   RLEEncoding<T>::DecodeBatch (231-257): (value, run length) pairs expanded
//     from row `offset`; rows past the last run decode to T{}.
// Outputs are written once, coalesced; the packed words are read through L1
// (neighbouring threads share words); the RLE decode scans the run lengths
// into row starts (decoupled look-back) and each block expands the runs that
// cover its row range from shared memory.
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

// exclusive prefix of u32 run lengths -> u64 row starts (single pass)
constexpr int kRunsPer = 16;  // runs per thread
constexpr int kRunsPerTile = kDThreads * kRunsPer;

__global__ void __launch_bounds__(kDThreads) run_starts_kernel(const uint32_t* __restrict__ runs, uint64_t nruns,
                                                               uint64_t* __restrict__ starts,
                                                               unsigned long long* status, unsigned int* ctr,
                                                               int* err) {
    __shared__ uint64_t s_tile, s_base;
    __shared__ uint64_t s_warp[kDThreads / 32];
    const uint64_t ntiles = (nruns + kRunsPerTile - 1) / kRunsPerTile;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(ctr, 1u);
        __syncthreads();
        uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        uint64_t r0 = tile * kRunsPerTile + threadIdx.x * kRunsPer;
        uint32_t v[kRunsPer];
        uint64_t c = 0;
        if (r0 + kRunsPer <= nruns && (reinterpret_cast<uintptr_t>(runs + r0) & 15) == 0) {
#pragma unroll
            for (int k = 0; k < kRunsPer; k += 4) {
                const uint4 q = __ldcs(reinterpret_cast<const uint4*>(runs + r0 + k));
                v[k] = q.x; v[k + 1] = q.y; v[k + 2] = q.z; v[k + 3] = q.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < kRunsPer; ++k) v[k] = r0 + k < nruns ? runs[r0 + k] : 0;
        }
#pragma unroll
        for (int k = 0; k < kRunsPer; ++k) c += v[k];
        int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        uint64_t inc = c;
        for (int d = 1; d < 32; d <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += y;
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            uint64_t x = lane < kDThreads / 32 ? s_warp[lane] : 0, t = x;
            for (int d = 1; d < 32; d <<= 1) {
                uint64_t y = __shfl_up_sync(0xffffffffu, t, d);
                if (lane >= d) t += y;
            }
            if (lane < kDThreads / 32) s_warp[lane] = t - x;
            const uint64_t tile_total = __shfl_sync(0xffffffffu, t, 31);
            const uint64_t e = lookback_exclusive_warp(status, tile, tile_total, err);
            if (lane == 0) s_base = e;
        }
        __syncthreads();
        uint64_t pos = s_base + s_warp[warp] + (inc - c);
#pragma unroll
        for (int k = 0; k < kRunsPer; ++k) {
            if (r0 + k < nruns) starts[r0 + k] = pos;
            pos += v[k];
        }
        if (r0 < nruns && r0 + kRunsPer >= nruns) starts[nruns] = pos;  // the thread holding the last run: total rows
        __syncthreads();
    }
}

// rows [offset, offset+count): block b expands rows [b*R, (b+1)*R) of the
// output.  The block knows the run covering its first row, marks each later
// run's first row in shared memory with its run index (and stages the runs'
// values there), takes an inclusive max-scan over the R rows (each row's
// covering run is the last run starting at or before it), and writes the
// rows' values coalesced.
constexpr int kRleRows = 2048;
constexpr int kRlePer = kRleRows / kDThreads;  // rows per thread in the scan
__device__ __forceinline__ uint32_t rle_pad(uint32_t j) { return j + (j >> 5); }  // bank-conflict padding

template <typename T>
__global__ void __launch_bounds__(kDThreads) rle_expand_kernel(const T* __restrict__ values,
                                                               const uint64_t* __restrict__ starts, uint64_t nruns,
                                                               uint64_t offset, uint64_t count, T* __restrict__ out) {
    __shared__ uint32_t s_idx[kRleRows + kRleRows / 32];
    __shared__ T s_val[kRleRows];  // values of runs k0 .. k0 + kRleRows - 1
    __shared__ uint32_t s_wmax[kDThreads / 32];
    __shared__ uint64_t s_k0;
    const uint64_t total = starts[nruns];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // each block expands a contiguous range of tiles: one binary search for
    // its first tile, then the covering run of each next tile's first row is
    // found by walking forward from the previous tile's last run
    const uint64_t ntiles = (count + kRleRows - 1) / kRleRows;
    const uint64_t per = (ntiles + gridDim.x - 1) / gridDim.x;
    const uint64_t tb = blockIdx.x * per, te = min(ntiles, tb + per);
    if (threadIdx.x == 0 && tb < te) {
        const uint64_t key = offset + tb * kRleRows;
        uint64_t lo = 0, hi = nruns;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (starts[mid] <= key) lo = mid + 1;
            else hi = mid;
        }
        s_k0 = lo ? lo - 1 : 0;
    }
    for (uint64_t blk = tb; blk < te; ++blk) {
        const uint64_t row0 = offset + blk * kRleRows;
        const uint32_t nb = static_cast<uint32_t>(min(static_cast<uint64_t>(kRleRows), count - blk * kRleRows));
#pragma unroll
        for (int e = 0; e < kRlePer; ++e) s_idx[rle_pad(threadIdx.x + e * kDThreads)] = 0;
        __syncthreads();
        const uint64_t k0 = s_k0;
        if (threadIdx.x == 0) s_val[0] = __ldg(values + k0);
        // runs after k0 start after row0 (starts are non-decreasing); each
        // thread stops at its first run past the tile
        for (uint64_t k = k0 + 1 + threadIdx.x; k < nruns; k += kDThreads) {
            const uint64_t st = __ldg(starts + k);
            if (st - row0 >= nb) break;
            const uint32_t rel = static_cast<uint32_t>(k - k0);
            atomicMax(&s_idx[rle_pad(static_cast<uint32_t>(st - row0))], rel);
            if (rel < kRleRows) s_val[rel] = __ldg(values + k);
        }
        __syncthreads();
        // inclusive max-scan: each thread a segment of kRlePer rows, then warps, then the block
        uint32_t loc[kRlePer], m = 0;
#pragma unroll
        for (int e = 0; e < kRlePer; ++e) {
            m = max(m, s_idx[rle_pad(threadIdx.x * kRlePer + e)]);
            loc[e] = m;
        }
        uint32_t inc = m;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc = max(inc, y);
        }
        if (lane == 31) s_wmax[warp] = inc;
        __syncthreads();
        uint32_t pre = __shfl_up_sync(0xffffffffu, inc, 1);
        if (lane == 0) pre = 0;
        for (int w = 0; w < warp; ++w) pre = max(pre, s_wmax[w]);
#pragma unroll
        for (int e = 0; e < kRlePer; ++e) s_idx[rle_pad(threadIdx.x * kRlePer + e)] = max(pre, loc[e]);
        __syncthreads();
#pragma unroll
        for (int e = 0; e < kRlePer; ++e) {
            const uint32_t j = threadIdx.x + e * kDThreads;
            if (j < nb) {
                const uint32_t rel = s_idx[rle_pad(j)];
                // more than kRleRows runs start in the tile only with empty runs
                const T x = rel < kRleRows ? s_val[rel] : __ldg(values + k0 + rel);
                out[blk * kRleRows + j] = row0 + j < total ? x : T(0);
            }
        }
        if (threadIdx.x == 0) {  // the next tile's first row: from the run covering this tile's last row
            uint64_t k = k0 + s_idx[rle_pad(nb - 1)];
            const uint64_t next = row0 + nb;
            while (k + 1 < nruns && __ldg(starts + k + 1) <= next) ++k;
            s_k0 = k;
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
    uint64_t ntiles = (nruns + kRunsPerTile - 1) / kRunsPerTile;
    return (nruns + 1) * 8 + (ntiles + 1) * 8 + 64;
}

int launch_rle_decode_i64(const int64_t* values, const uint32_t* runs, uint64_t nruns, uint64_t offset,
                          uint64_t count, int64_t* out, void* scratch, int* err, cudaStream_t s) {
    if (!count) return kOk;
    if (nruns == 0) {
        VX_CUDA(cudaMemsetAsync(out, 0, count * 8, s));
        return kOk;
    }
    uint64_t ntiles = (nruns + kRunsPerTile - 1) / kRunsPerTile;
    uint64_t* starts = static_cast<uint64_t*>(scratch);
    unsigned long long* status = reinterpret_cast<unsigned long long*>(starts + nruns + 1);
    unsigned int* ctr = reinterpret_cast<unsigned int*>(status + ntiles);
    VX_CUDA(cudaMemsetAsync(status, 0, (ntiles + 1) * 8, s));
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t b = ntiles < static_cast<uint64_t>(sms) * 4 ? ntiles : static_cast<uint64_t>(sms) * 4;
    run_starts_kernel<<<static_cast<unsigned>(b), kDThreads, 0, s>>>(runs, nruns, starts, status, ctr, err);
    VX_CUDA(cudaGetLastError());
    uint64_t blocks = (count + kRleRows - 1) / kRleRows;
    if (blocks > static_cast<uint64_t>(sms) * 8) blocks = static_cast<uint64_t>(sms) * 8;
    rle_expand_kernel<int64_t><<<static_cast<unsigned>(blocks), kDThreads, 0, s>>>(values, starts, nruns, offset,
                                                                                  count, out);
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
