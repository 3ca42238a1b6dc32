// Stable LSD radix sort of keys with a u32 payload (reference RadixSort<T>::Sort,
// include/voxel/ops/sort.hpp:83-160: 8-bit digits, sizeof(T) counting passes of
// histogram -> exclusive prefix -> stable scatter, then for signed T a stable
// pass that moves negatives first).
//
// B200 design (onesweep): one read of the keys builds every pass's digit
// histogram (block-local shared-memory histograms, merged with global atomics);
// each pass is then ONE kernel: a block takes the next tile (dynamic tile
// order), ranks its keys stably per digit with a warp multisplit
// (__match_any_sync) plus per-warp digit counters, gets each digit's global
// offset from a decoupled look-back over the previous tiles' per-digit counts,
// reorders the tile in shared memory and writes digit runs out coalesced.
// Signed keys are sorted with the sign bit flipped, which yields exactly the
// reference's order: negatives first, each side ascending, ties stable.
#include <cstring>
#include <vector>

#include "radix.h"
#include "tune.h"
#include "voxel_c.h"
#include "vx_common.cuh"
#include "vx_runtime.h"

namespace vx {

namespace {

constexpr int kRBits = 8;
constexpr int kRadix = 1 << kRBits;
constexpr int kRThreads = 512;
constexpr int kRWarps = kRThreads / 32;
// keys per thread in the onesweep pass: 16 (8192-key tiles, one block per SM)
// or 8 (4096-key tiles, two blocks per SM), chosen per shape by the autotuner
constexpr int kRItemsMax = 16;
constexpr int kRItemsMin = 8;
constexpr int kRTileMin = kRThreads * kRItemsMin;  // the smallest tile sizes the scratch

constexpr uint32_t kStAgg = 1u << 30;
constexpr uint32_t kStInc = 2u << 30;
constexpr uint32_t kStMask = (1u << 30) - 1;
constexpr long long kSpinBudget = 1ll << 31;
constexpr int kLbBatch = 4;  // look-back statuses loaded per round trip
constexpr uint64_t kSkipMinKeys = 1ull << 16;  // smaller sorts run every pass (no histogram read-back)

template <typename K>
__device__ __forceinline__ uint32_t digit_of(K k, int shift) {
    return static_cast<uint32_t>((k >> shift) & (kRadix - 1));
}

template <typename K>
__global__ void __launch_bounds__(256) histogram_kernel(const K* __restrict__ keys, uint64_t n, int passes, K flip,
                                                        unsigned int* __restrict__ hist) {
    __shared__ unsigned int sh[8][kRadix];
    for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x) sh[i / kRadix][i % kRadix] = 0;
    __syncthreads();
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        K k = __ldcs(keys + i) ^ flip;
        for (int p = 0; p < passes; ++p) atomicAdd(&sh[p][digit_of(k, p * kRBits)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x) {
        unsigned int v = sh[i / kRadix][i % kRadix];
        if (v) atomicAdd(&hist[i], v);
    }
}

// exclusive prefix over the digits of each pass (one block per pass)
__global__ void hist_scan_kernel(const unsigned int* hist, unsigned int* offs) {
    __shared__ unsigned int s[kRadix];
    int p = blockIdx.x, d = threadIdx.x;
    s[d] = hist[p * kRadix + d];
    __syncthreads();
    for (int o = 1; o < kRadix; o <<= 1) {
        unsigned int v = d >= o ? s[d - o] : 0;
        __syncthreads();
        s[d] += v;
        __syncthreads();
    }
    offs[p * kRadix + d] = s[d] - hist[p * kRadix + d];
}

template <typename K, int ITEMS>
__global__ void __launch_bounds__(kRThreads, ITEMS >= 16 ? 1 : 2) onesweep_kernel(
    const K* __restrict__ kin, K* __restrict__ kout, const uint32_t* __restrict__ vin, uint32_t* __restrict__ vout,
    uint64_t n, int shift, K flip_in, K flip_out, const unsigned int* __restrict__ digit_offs,
    unsigned int* status, unsigned int* tile_ctr, int* err) {
    extern __shared__ __align__(16) unsigned char smem[];
    K* s_keys = reinterpret_cast<K*>(smem);
    uint32_t* s_vals = reinterpret_cast<uint32_t*>(s_keys + (kRThreads * ITEMS));
    unsigned int* s_cnt = s_vals + (kRThreads * ITEMS);                // [kRWarps][kRadix]
    unsigned int* s_tstart = s_cnt + kRWarps * kRadix;     // [kRadix]
    unsigned int* s_gstart = s_tstart + kRadix;            // [kRadix] (low 32 bits)
    unsigned int* s_gstart_hi = s_gstart + kRadix;
    __shared__ uint64_t s_tile;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t ntiles = (n + (kRThreads * ITEMS) - 1) / (kRThreads * ITEMS);
    const unsigned lanemask_lt = (1u << lane) - 1;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
        for (int i = threadIdx.x; i < kRWarps * kRadix; i += kRThreads) s_cnt[i] = 0;
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t base = tile * (kRThreads * ITEMS);
        const uint64_t wbase = base + static_cast<uint64_t>(warp) * 32 * ITEMS;
        K key[ITEMS];
        uint32_t val[ITEMS];
        uint32_t rank[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            uint64_t pos = wbase + i * 32 + lane;
            if (pos < n) {
                key[i] = __ldcs(kin + pos) ^ flip_in;
                val[i] = __ldcs(vin + pos);
            } else {
                key[i] = 0;
                val[i] = 0;
            }
        }
        unsigned int* wc = s_cnt + warp * kRadix;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            uint64_t pos = wbase + i * 32 + lane;
            bool valid = pos < n;
            uint32_t d = valid ? digit_of(key[i], shift) : 0u;
            // lanes holding the same digit: one ballot per digit bit (and one
            // for validity) -- far cheaper here than __match_any_sync
            unsigned peers = __ballot_sync(0xffffffffu, valid);
            if (!valid) peers = ~peers;
#pragma unroll
            for (int b = 0; b < kRBits; ++b) {
                const bool bit = (d >> b) & 1u;
                const unsigned v = __ballot_sync(0xffffffffu, bit);
                peers &= bit ? v : ~v;
            }
            unsigned int before = valid ? wc[d] : 0;
            __syncwarp();
            if (valid) {
                rank[i] = before + __popc(peers & lanemask_lt);
                if ((peers & lanemask_lt) == 0) wc[d] = before + __popc(peers);
            }
            __syncwarp();
        }
        __syncthreads();
        // per digit: exclusive over warps, tile total
        unsigned int tcount = 0;
        if (threadIdx.x < kRadix) {
            int d = threadIdx.x;
            unsigned int run = 0;
            for (int w = 0; w < kRWarps; ++w) {
                unsigned int t = s_cnt[w * kRadix + d];
                s_cnt[w * kRadix + d] = run;
                run += t;
            }
            tcount = run;
            s_tstart[d] = run;
        }
        __syncthreads();
        // tile-local digit starts: inclusive scan of tcount over the 256 digits
        // (warp shuffles within each of the 8 digit warps, then the warp totals)
        __shared__ unsigned int s_wsum[kRadix / 32];
        unsigned int incl = 0;
        if (threadIdx.x < kRadix) {
            incl = tcount;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane == 31) s_wsum[warp] = incl;
        }
        __syncthreads();
        if (threadIdx.x < kRadix) {
            for (int w = 0; w < warp; ++w) incl += s_wsum[w];
            int d = threadIdx.x;
            // decoupled look-back for this digit's global offset
            unsigned int* st = status + tile * kRadix + d;
            uint64_t excl = 0;
            if (tile == 0) {
                atomicExch(st, kStInc | (tcount & kStMask));
            } else {
                atomicExch(st, kStAgg | (tcount & kStMask));
                // walk back kLbBatch predecessors per round trip (all loads
                // issued, then consumed newest first)
                int64_t p = static_cast<int64_t>(tile) - 1;
                long long t0 = clock64();
                bool done = false;
                while (!done && p >= 0) {
                    unsigned int sv[kLbBatch];
#pragma unroll
                    for (int j = 0; j < kLbBatch; ++j)
                        sv[j] = p - j >= 0 ? static_cast<unsigned int>(*reinterpret_cast<volatile unsigned int*>(
                                                 status + (p - j) * kRadix + d))
                                           : static_cast<unsigned int>(kStInc);  // before tile 0: an inclusive 0
                    int used = 0;
#pragma unroll
                    for (int j = 0; j < kLbBatch; ++j) {
                        if (done || used < j) continue;  // stopped at an empty entry or the inclusive one
                        const unsigned int flag = sv[j] & ~kStMask;
                        if (flag == 0) continue;
                        if (p - j >= 0) excl += sv[j] & kStMask;
                        used = j + 1;
                        if (flag == kStInc) done = true;
                    }
                    p -= used;
                    if (!done && used == 0 && clock64() - t0 > kSpinBudget) {
                        atomicOr(err, 4);
                        break;
                    }
                }
                // one status word carries flag and value: no fence needed
                atomicExch(st, kStInc | static_cast<unsigned int>((excl + tcount) & kStMask));
            }
            uint64_t g = static_cast<uint64_t>(digit_offs[d]) + excl;
            s_gstart[d] = static_cast<unsigned int>(g);
            s_gstart_hi[d] = static_cast<unsigned int>(g >> 32);
            s_tstart[d] = incl - tcount;  // back to exclusive
        }
        __syncthreads();
        // scatter into shared memory in (digit, stable rank) order
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            uint64_t pos = wbase + i * 32 + lane;
            if (pos < n) {
                uint32_t d = digit_of(key[i], shift);
                unsigned int lp = s_tstart[d] + wc[d] + rank[i];
                s_keys[lp] = key[i];
                s_vals[lp] = val[i];
            }
        }
        __syncthreads();
        const uint32_t tn = static_cast<uint32_t>(n - base < static_cast<uint64_t>((kRThreads * ITEMS)) ? n - base : (kRThreads * ITEMS));
        for (uint32_t j = threadIdx.x; j < tn; j += kRThreads) {
            K k = s_keys[j];
            uint32_t d = digit_of(k, shift);
            uint64_t g = (static_cast<uint64_t>(s_gstart_hi[d]) << 32 | s_gstart[d]) + (j - s_tstart[d]);
            kout[g] = k ^ flip_out;
            vout[g] = s_vals[j];
        }
        __syncthreads();
    }
}

template <typename K>
size_t tmp_bytes_t(uint64_t n) {
    uint64_t ntiles = (n + kRTileMin - 1) / kRTileMin;
    size_t b = n * sizeof(K) + n * 4;                    // ping-pong buffers
    b = (b + 255) / 256 * 256;
    b += ntiles * kRadix * 4 + 256;                       // look-back status
    b += 8 * kRadix * 4 * 2 + 256;                        // histograms + offsets
    b += 256;                                             // tile counter + error word
    return b;
}

size_t smem_bytes_t(size_t ksize, int items) {
    return static_cast<size_t>(kRThreads) * items * (ksize + 4) + (kRWarps * kRadix + 3 * kRadix) * 4;
}

// the passes with ITEMS keys per thread (scratch laid out as tmp_bytes_t)
template <typename K, int ITEMS>
int sort_run(K* keys, uint32_t* idx, uint64_t n, bool is_signed, void* tmp, int* err, cudaStream_t s) {
    constexpr uint64_t kTile = static_cast<uint64_t>(kRThreads) * ITEMS;
    const int passes = static_cast<int>(sizeof(K) * 8 / kRBits);
    const uint64_t ntiles = (n + kTile - 1) / kTile;
    const uint64_t status_words = ((n + kRTileMin - 1) / kRTileMin) * kRadix;  // sized for the smallest tile
    char* b = static_cast<char*>(tmp);
    K* ktmp = reinterpret_cast<K*>(b);
    uint32_t* vtmp = reinterpret_cast<uint32_t*>(b + n * sizeof(K));
    size_t off = (n * sizeof(K) + n * 4 + 255) / 256 * 256;
    unsigned int* status = reinterpret_cast<unsigned int*>(b + off);
    off += status_words * 4 + 256;
    unsigned int* hist = reinterpret_cast<unsigned int*>(b + off);
    unsigned int* offs = hist + 8 * kRadix;
    off += 8 * kRadix * 4 * 2 + 256;
    unsigned int* ctr = reinterpret_cast<unsigned int*>(b + off);
    const K signbit = static_cast<K>(1) << (sizeof(K) * 8 - 1);
    const K flip = is_signed ? signbit : 0;

    VX_CUDA(cudaMemsetAsync(hist, 0, 8 * kRadix * 4, s));
    int sms = sm_count() > 0 ? sm_count() : 148;
    uint64_t hb = (n + 255) / 256;
    if (hb > static_cast<uint64_t>(sms) * 4) hb = static_cast<uint64_t>(sms) * 4;
    histogram_kernel<K><<<static_cast<unsigned>(hb), 256, 0, s>>>(keys, n, passes, flip, hist);
    VX_CUDA(cudaGetLastError());
    hist_scan_kernel<<<passes, kRadix, 0, s>>>(hist, offs);
    VX_CUDA(cudaGetLastError());
    const size_t smem = smem_bytes_t(sizeof(K), ITEMS);
    VX_CUDA(cudaFuncSetAttribute(onesweep_kernel<K, ITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    const uint64_t per_sm = ITEMS >= 16 ? 1 : 2;  // resident blocks per SM (shared memory)
    uint64_t grid = static_cast<uint64_t>(sms) * per_sm;
    if (grid > ntiles) grid = ntiles;
    // A pass whose digit is the same for every key is the identity (the sort is
    // stable): its histogram holds n in one bin.  Such passes are skipped --
    // keys of narrower range than their type (row ids in u64, small signed
    // values) sort in fewer passes -- unless the stream is being captured into
    // a graph, which the histogram read-back would break.
    bool run_pass[8];
    int nrun = passes;
    for (int p = 0; p < passes; ++p) run_pass[p] = true;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
        cudaGetLastError();
        cap = cudaStreamCaptureStatusActive;
    }
    if (cap == cudaStreamCaptureStatusNone && n >= kSkipMinKeys) {
        unsigned int h[8 * kRadix];
        if (int st = d2h(h, hist, static_cast<size_t>(passes) * kRadix * 4, s)) return st;
        if (int st = sync(s)) return st;
        for (int p = 0; p < passes; ++p)
            for (int d = 0; d < kRadix; ++d)
                if (h[p * kRadix + d] == n) {
                    run_pass[p] = false;
                    --nrun;
                }
    }
    const K* kin = keys;
    const uint32_t* vin = idx;
    K* kout = ktmp;
    uint32_t* vout = vtmp;
    int done = 0;
    for (int p = 0; p < passes; ++p) {
        if (!run_pass[p]) continue;
        VX_CUDA(cudaMemsetAsync(status, 0, ntiles * kRadix * 4, s));
        VX_CUDA(cudaMemsetAsync(ctr, 0, 4, s));
        // the sign flip goes on at the first pass run and off at the last
        K fin = done == 0 ? flip : 0;
        K fout = done == nrun - 1 ? flip : 0;
        onesweep_kernel<K, ITEMS><<<static_cast<unsigned>(grid), kRThreads, smem, s>>>(
            kin, kout, vin, vout, n, p * kRBits, fin, fout, offs + p * kRadix, status, ctr, err);
        VX_CUDA(cudaGetLastError());
        ++done;
        // ping-pong
        const K* nk = kout;
        const uint32_t* nv = vout;
        kout = const_cast<K*>(kin);
        vout = const_cast<uint32_t*>(vin);
        kin = nk;
        vin = nv;
    }
    if (done & 1) {  // an odd number of passes left the result in the scratch halves
        VX_CUDA(cudaMemcpyAsync(keys, ktmp, n * sizeof(K), cudaMemcpyDeviceToDevice, s));
        VX_CUDA(cudaMemcpyAsync(idx, vtmp, n * 4, cudaMemcpyDeviceToDevice, s));
    }
    return kOk;
}

template <typename K>
__global__ void tune_sample_kernel(K* keys, uint32_t* idx, uint64_t n, uint64_t seed) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t z = (i + 1) * 0x9e3779b97f4a7c15ull + seed;  // splitmix64 of the row
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        keys[i] = static_cast<K>(z ^ (z >> 31));
        idx[i] = static_cast<uint32_t>(i);
    }
}

constexpr uint64_t kTuneMinKeys = 1ull << 16;     // smaller sorts take the default
constexpr uint64_t kTuneSampleKeys = 1ull << 24;  // tuning sorts at most this many random keys

template <typename K>
int sort_t(int dtype, K* keys, uint32_t* idx, uint64_t n, bool is_signed, void* tmp, size_t tmp_bytes, int* err,
           cudaStream_t s, int* passes_out) {
    if (n <= 1) return kOk;  // sort.hpp:84
    if (n >= (1ull << 30)) {
        set_error(kErrInvalidArg, "radix sort supports fewer than 2^30 keys per call");
        return kErrInvalidArg;
    }
    if (tmp_bytes < tmp_bytes_t<K>(n)) {
        set_error(kErrInvalidArg, "radix sort scratch too small (%zu < %zu)", tmp_bytes, tmp_bytes_t<K>(n));
        return kErrInvalidArg;
    }
    // keys per thread: the autotuner's choice for this (type, size), timed on
    // random keys of the same type (the caller's keys are sorted only once)
    int choice = 0;  // 0: 16 keys per thread, 1: 8
    if (n >= kTuneMinKeys) {
        const std::string key = tune_key("radix_onesweep", dtype, n);
        if (!tune_lookup(key, &choice) && tune_may_time(s)) {
            const uint64_t m = n < kTuneSampleKeys ? n : kTuneSampleKeys;
            DevBuf sk(m * sizeof(K)), si(m * 4), st(tmp_bytes_t<K>(m));
            if (sk.p && si.p && st.p) {
                choice = tune_pick(key, 2, 0, s, [&](int c) -> int {
                    tune_sample_kernel<K><<<static_cast<unsigned>(sm_count() > 0 ? sm_count() * 4 : 592), 256, 0, s>>>(
                        sk.as<K>(), si.as<uint32_t>(), m, 0x5eedull);
                    return c == 0 ? sort_run<K, kRItemsMax>(sk.as<K>(), si.as<uint32_t>(), m, is_signed, st.p, err, s)
                                  : sort_run<K, kRItemsMin>(sk.as<K>(), si.as<uint32_t>(), m, is_signed, st.p, err, s);
                });
            }
        }
    }
    const int r = choice == 1 ? sort_run<K, kRItemsMin>(keys, idx, n, is_signed, tmp, err, s)
                              : sort_run<K, kRItemsMax>(keys, idx, n, is_signed, tmp, err, s);
    if (passes_out) *passes_out = static_cast<int>(sizeof(K) * 8 / kRBits);
    return r;
}

}  // namespace

size_t radix_tmp_bytes(int dtype, uint64_t n) {
    return dtype_size(dtype) == 8 ? tmp_bytes_t<uint64_t>(n) : tmp_bytes_t<uint32_t>(n);
}

int launch_radix_sort(int dtype, void* keys, uint32_t* idx, uint64_t n, void* tmp, size_t tmp_bytes, int* err,
                      cudaStream_t s, int* passes) {
    switch (dtype) {
    case U64: return sort_t<uint64_t>(dtype, static_cast<uint64_t*>(keys), idx, n, false, tmp, tmp_bytes, err, s, passes);
    case I64: return sort_t<uint64_t>(dtype, static_cast<uint64_t*>(keys), idx, n, true, tmp, tmp_bytes, err, s, passes);
    case U32: return sort_t<uint32_t>(dtype, static_cast<uint32_t*>(keys), idx, n, false, tmp, tmp_bytes, err, s, passes);
    case I32: return sort_t<uint32_t>(dtype, static_cast<uint32_t*>(keys), idx, n, true, tmp, tmp_bytes, err, s, passes);
    default:
        set_error(kErrInvalidArg, "radix sort key type %d must be an integer type (2..5)", dtype);
        return kErrInvalidArg;
    }
}

}  // namespace vx

using namespace vx;

namespace {
thread_local DevBuf t_rerr;
int* rerr(cudaStream_t s) {
    if (!t_rerr.p) {
        t_rerr = DevBuf(16);
        if (t_rerr.p) cudaMemsetAsync(t_rerr.p, 0, 16, s);
    }
    return t_rerr.as<int>();
}
}  // namespace

namespace vx {
int radix_check(cudaStream_t s) {
    int h = 0;
    int* e = rerr(s);
    if (int st = d2h(&h, e, 4, s)) return st;
    if (int st = sync(s)) return st;
    if (h) {
        cudaMemsetAsync(e, 0, 4, s);
        set_error(kErrDeviceTimeout, "radix sort look-back wait ran out of budget");
        return kErrDeviceTimeout;
    }
    return kOk;
}
int* radix_err(cudaStream_t s) { return rerr(s); }
}  // namespace vx

extern "C" {

size_t voxel_radix_sort_tmp_bytes(int dtype, size_t n) { return radix_tmp_bytes(dtype, n); }

int voxel_radix_sort_dev(int dtype, void* d_keys, uint32_t* d_idx, size_t n, void* d_tmp, size_t tmp_bytes,
                         void* stream) {
    clear_error();
    if (int st = ensure_device()) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    return launch_radix_sort(dtype, d_keys, d_idx, n, d_tmp, tmp_bytes, rerr(s), s, nullptr);
}

int voxel_radix_sort(int dtype, void* keys, uint32_t* idx, size_t n) {
    clear_error();
    if (int st = ensure_device()) return st;
    if (n <= 1) return kOk;
    cudaStream_t s = thread_stream();
    size_t es = dtype_size(dtype);
    size_t tb = radix_tmp_bytes(dtype, n);
    DevBuf dk(n * es), di(n * 4), tmp(tb);
    if (!dk.p || !di.p || !tmp.p) return kErrOutOfMemory;
    if (int st = h2d(dk.p, keys, n * es, s)) return st;
    if (int st = h2d(di.p, idx, n * 4, s)) return st;
    if (int st = launch_radix_sort(dtype, dk.p, di.as<uint32_t>(), n, tmp.p, tb, rerr(s), s, nullptr)) return st;
    if (int st = d2h(keys, dk.p, n * es, s)) return st;
    if (int st = d2h(idx, di.p, n * 4, s)) return st;
    return radix_check(s);
}

}  // extern "C"
