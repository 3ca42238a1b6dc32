// Host runtime: errors, device pool, pinned staging, streams.
#include "vx_runtime.h"

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <atomic>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace vx {

namespace {
thread_local char g_err[512] = "";
thread_local int g_status = kOk;

std::mutex g_pool_mu;
// size class -> free blocks
std::map<size_t, std::vector<void*>> g_free;
std::unordered_map<void*, size_t> g_live;
size_t g_cached = 0;

size_t size_class(size_t bytes) {
    if (bytes <= 4096) {
        size_t c = 256;
        while (c < bytes) c <<= 1;
        return c;
    }
    // 1/8-step geometric classes above 4 KiB bound the waste to 12.5%
    size_t p = 4096;
    while (p * 2 <= bytes) p <<= 1;
    size_t step = p / 8;
    return (bytes + step - 1) / step * step;
}

struct Staging {
    void* p = nullptr;
    size_t n = 0;
    ~Staging() {
        if (p) cudaFreeHost(p);
    }
};
thread_local Staging g_staging;
thread_local cudaStream_t g_stream = nullptr;
int g_sms = 0;
std::once_flag g_dev_once;
int g_dev_status = kOk;
}  // namespace

void set_error(int status, const char* fmt, ...) {
    g_status = status;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

void clear_error() {
    g_status = kOk;
    g_err[0] = 0;
}

const char* last_error() { return g_err; }
int last_status() { return g_status; }

int cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return kOk;
    set_error(e == cudaErrorMemoryAllocation ? kErrOutOfMemory : kErrCuda, "CUDA error %d (%s) in %s",
              static_cast<int>(e), cudaGetErrorString(e), what);
    return g_status;
}

int ensure_device() {
    std::call_once(g_dev_once, [] {
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess || n == 0) {
            g_dev_status = kErrNoDevice;
            return;
        }
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    });
    if (g_dev_status != kOk) {
        set_error(kErrNoDevice, "voxel_b200: no CUDA device is available (this backend has no CPU path)");
        return kErrNoDevice;
    }
    return kOk;
}

int sm_count() {
    if (ensure_device() != kOk) return 0;
    // per device ordinal: grid sizing follows the calling thread's current device
    constexpr int kDevs = 64;
    static std::atomic<int> per_dev[kDevs];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevs) {
        cudaGetLastError();
        return g_sms;
    }
    int v = per_dev[dev].load(std::memory_order_relaxed);
    if (v <= 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
            cudaGetLastError();
            return g_sms;
        }
        per_dev[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

void* dev_alloc(size_t bytes) {
    if (bytes == 0) bytes = 1;
    size_t c = size_class(bytes);
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        auto it = g_free.find(c);
        if (it != g_free.end() && !it->second.empty()) {
            void* p = it->second.back();
            it->second.pop_back();
            g_cached -= c;
            g_live[p] = c;
            return p;
        }
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, c);
    if (e != cudaSuccess) {
        // release the cache and retry once before reporting out-of-memory
        dev_pool_trim();
        cudaGetLastError();
        e = cudaMalloc(&p, c);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error(kErrOutOfMemory, "device allocation of %zu bytes failed", bytes);
            return nullptr;
        }
    }
    std::lock_guard<std::mutex> lk(g_pool_mu);
    g_live[p] = c;
    return p;
}

void dev_free(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_live.find(p);
    if (it == g_live.end()) return;
    g_free[it->second].push_back(p);
    g_cached += it->second;
    g_live.erase(it);
}

size_t dev_pool_cached_bytes() {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    return g_cached;
}

void dev_pool_trim() {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    for (auto& kv : g_free)
        for (void* p : kv.second) cudaFree(p);
    g_free.clear();
    g_cached = 0;
}

void* pinned_staging(size_t bytes) {
    if (g_staging.n < bytes) {
        if (g_staging.p) cudaFreeHost(g_staging.p);
        g_staging.p = nullptr;
        g_staging.n = 0;
        size_t want = bytes < (1u << 20) ? (1u << 20) : bytes;
        if (cudaHostAlloc(&g_staging.p, want, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            set_error(kErrOutOfMemory, "pinned host allocation of %zu bytes failed", want);
            return nullptr;
        }
        g_staging.n = want;
    }
    return g_staging.p;
}

cudaStream_t thread_stream() {
    if (!g_stream) cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking);
    return g_stream;
}

// Copies between the device and pageable host memory go through two pinned
// chunks of this thread's own (the host-side memcpy of one chunk overlaps the
// DMA of the other).  Left to the driver, a pageable copy passes through its
// shared staging path, and one thread's large pageable copy then holds up
// every other thread's -- the serving loop's workers copy results out
// concurrently.  Pinned host memory and small copies go straight.
namespace {
constexpr size_t kStageChunk = 8u << 20;
constexpr size_t kStageMin = 64u << 10;
struct CopyStage {
    char* p = nullptr;  // 2 x kStageChunk, pinned
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool used[2] = {false, false};
    bool failed = false;
    ~CopyStage() {
        if (p) cudaFreeHost(p);
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
    }
};
thread_local CopyStage g_copy;

bool stage_ready() {
    if (g_copy.p) return true;
    if (g_copy.failed) return false;
    void* p = nullptr;
    if (cudaHostAlloc(&p, 2 * kStageChunk, cudaHostAllocDefault) != cudaSuccess ||
        cudaEventCreateWithFlags(&g_copy.ev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&g_copy.ev[1], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (p) cudaFreeHost(p);
        g_copy.failed = true;  // the driver's own path then
        return false;
    }
    g_copy.p = static_cast<char*>(p);
    return true;
}

bool pageable(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

// waits until this thread's staging chunk k is no longer read or written by a copy
int stage_wait(int k) {
    if (g_copy.used[k]) {
        VX_CUDA(cudaEventSynchronize(g_copy.ev[k]));
        g_copy.used[k] = false;
    }
    return kOk;
}
}  // namespace

int h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return kOk;
    if (bytes < kStageMin || !pageable(src) || !stage_ready()) {
        VX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        return kOk;
    }
    const char* in = static_cast<const char*>(src);
    char* out = static_cast<char*>(dst);
    int k = 0;
    for (size_t off = 0; off < bytes; off += kStageChunk, k ^= 1) {
        const size_t c = bytes - off < kStageChunk ? bytes - off : kStageChunk;
        if (int st = stage_wait(k)) return st;
        char* chunk = g_copy.p + k * kStageChunk;
        std::memcpy(chunk, in + off, c);
        VX_CUDA(cudaMemcpyAsync(out + off, chunk, c, cudaMemcpyHostToDevice, s));
        VX_CUDA(cudaEventRecord(g_copy.ev[k], s));
        g_copy.used[k] = true;
    }
    return kOk;  // the source may be reused: every byte is in a staging chunk or on the device
}

int d2h(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return kOk;
    if (bytes < kStageMin || !pageable(dst) || !stage_ready()) {
        VX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        return kOk;
    }
    const char* in = static_cast<const char*>(src);
    char* out = static_cast<char*>(dst);
    size_t pend_off = 0, pend_len = 0;  // the chunk in flight in the other half
    int k = 0;
    for (size_t off = 0; off < bytes; off += kStageChunk, k ^= 1) {
        const size_t c = bytes - off < kStageChunk ? bytes - off : kStageChunk;
        if (int st = stage_wait(k)) return st;
        VX_CUDA(cudaMemcpyAsync(g_copy.p + k * kStageChunk, in + off, c, cudaMemcpyDeviceToHost, s));
        VX_CUDA(cudaEventRecord(g_copy.ev[k], s));
        g_copy.used[k] = true;
        if (pend_len) {  // drain the previous chunk while this one is copied
            if (int st = stage_wait(k ^ 1)) return st;
            std::memcpy(out + pend_off, g_copy.p + (k ^ 1) * kStageChunk, pend_len);
        }
        pend_off = off;
        pend_len = c;
    }
    if (int st = stage_wait(k ^ 1)) return st;
    std::memcpy(out + pend_off, g_copy.p + (k ^ 1) * kStageChunk, pend_len);
    return kOk;  // like a pageable copy, complete on return
}

int sync(cudaStream_t s) {
    VX_CUDA(cudaStreamSynchronize(s));
    return kOk;
}

}  // namespace vx
