// Host runtime of the B200 backend: error reporting, the device-memory pool,
// pinned staging buffers and the per-thread stream.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

#include "vx_types.h"

namespace vx {

// Last error of the calling thread (what voxel_last_error returns).
void set_error(int status, const char* fmt, ...);
void clear_error();
const char* last_error();
int last_status();

// Turns a CUDA error into a status + message; returns kOk or kErrCuda.
int cuda_status(cudaError_t e, const char* what);

#define VX_CUDA(call)                                      \
    do {                                                   \
        cudaError_t _e = (call);                           \
        if (_e != cudaSuccess) return ::vx::cuda_status(_e, #call); \
    } while (0)

// Device selection / properties.  ensure_device() fails loudly (kErrNoDevice)
// when no CUDA device is present: there is no CPU fallback.
int ensure_device();
int sm_count();

// Caching device allocator: blocks are rounded up to a size class and kept on
// a free list when released, so steady-state calls do not hit cudaMalloc.
void* dev_alloc(size_t bytes);
void dev_free(void* p);
size_t dev_pool_cached_bytes();
void dev_pool_trim();

// Pinned host staging buffer owned by the calling thread, grown on demand.
void* pinned_staging(size_t bytes);

// Stream the calling thread's host entry points use.
cudaStream_t thread_stream();

// RAII device buffer from the pool.
struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t bytes) : p(bytes ? dev_alloc(bytes) : nullptr), n(bytes) {}
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { reset(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { reset(); }
    void reset() { if (p) dev_free(p); p = nullptr; n = 0; }
    template <typename T> T* as() const { return static_cast<T*>(p); }
    bool ok(size_t want) const { return want == 0 || p != nullptr; }
};

// Copy helpers on the thread stream (asynchronous; caller synchronises).
int h2d(void* dst, const void* src, size_t bytes, cudaStream_t s);
int d2h(void* dst, const void* src, size_t bytes, cudaStream_t s);
int sync(cudaStream_t s);

}  // namespace vx
