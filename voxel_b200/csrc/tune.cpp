// Autotuner cache (see tune.h).
#include "tune.h"

#include <dlfcn.h>
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <vector>

#include "voxel_c.h"
#include "vx_runtime.h"

namespace vx {

namespace {

std::mutex g_mu;
std::map<std::string, int> g_cache;
bool g_loaded = false;
int g_enabled = -1;  // -1: from VOXEL_TUNE
std::string g_path;

std::string default_path() {
    if (const char* e = std::getenv("VOXEL_TUNE_CACHE")) return e;
    Dl_info info{};
    if (dladdr(reinterpret_cast<void*>(&tune_key), &info) && info.dli_fname) {
        std::string lib = info.dli_fname;
        const size_t slash = lib.rfind('/');
        if (slash != std::string::npos) return lib.substr(0, slash) + "/tune_cache.json";
    }
    return "tune_cache.json";
}

// {"key": int, ...}; keys hold no quotes or backslashes
void load_locked() {
    if (g_loaded) return;
    g_loaded = true;
    if (g_path.empty()) g_path = default_path();
    std::ifstream f(g_path);
    if (!f) return;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string t = ss.str();
    size_t i = 0;
    while ((i = t.find('"', i)) != std::string::npos) {
        const size_t j = t.find('"', i + 1);
        if (j == std::string::npos) break;
        const std::string key = t.substr(i + 1, j - i - 1);
        const size_t colon = t.find(':', j);
        if (colon == std::string::npos) break;
        char* end = nullptr;
        const long v = std::strtol(t.c_str() + colon + 1, &end, 10);
        if (end != t.c_str() + colon + 1) g_cache[key] = static_cast<int>(v);
        i = end ? static_cast<size_t>(end - t.c_str()) : j + 1;
    }
}

void save_locked() {
    if (g_path.empty()) g_path = default_path();
    // a temporary name of this process's own, so processes saving at once
    // never write into one file; the rename then replaces the cache whole
    const std::string tmp = g_path + "." + std::to_string(static_cast<long>(getpid())) + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "w");
    if (!f) return;  // an unwritable cache only costs re-tuning in the next process
    std::fputs("{\n", f);
    size_t k = 0;
    for (const auto& e : g_cache)
        std::fprintf(f, "  \"%s\": %d%s\n", e.first.c_str(), e.second, ++k < g_cache.size() ? "," : "");
    std::fputs("}\n", f);
    // a short write (full disk) must not replace a good cache with a truncated one
    const bool write_failed = std::ferror(f) != 0;
    const bool close_failed = std::fclose(f) != 0;
    if (write_failed || close_failed) {
        std::remove(tmp.c_str());
        return;
    }
    std::rename(tmp.c_str(), g_path.c_str());
}

std::string gpu_name(int dev) {
    cudaDeviceProp p{};
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) {
        cudaGetLastError();
        return "unknown";
    }
    std::string n = p.name;
    for (char& c : n)
        if (c == '"' || c == '\\' || c == '|') c = '_';
    return n + "-" + std::to_string(p.multiProcessorCount) + "sm";
}

}  // namespace

std::string tune_key(const char* family, int dtype, uint64_t n) {
    int lg = 0;
    while (lg < 63 && (1ull << (lg + 1)) <= n) ++lg;  // floor(log2 n)
    // the GPU part of the key belongs to the calling thread's current device
    constexpr int kDevs = 64;
    static std::string names[kDevs];
    static std::mutex names_mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        dev = -1;
    }
    std::string gpu = "unknown";
    if (dev >= 0 && dev < kDevs) {
        std::lock_guard<std::mutex> lk(names_mu);
        if (names[dev].empty()) names[dev] = gpu_name(dev);
        gpu = names[dev];
    }
    return gpu + "|" + family + "|" + std::to_string(dtype) + "|" + std::to_string(lg);
}

bool tune_enabled() {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_enabled < 0) {
        const char* e = std::getenv("VOXEL_TUNE");
        g_enabled = (e && std::strcmp(e, "0") == 0) ? 0 : 1;
    }
    return g_enabled != 0;
}

bool tune_may_time(cudaStream_t s) {
    if (!tune_enabled()) return false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return cs == cudaStreamCaptureStatusNone;
}

void tune_set_enabled(bool on) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_enabled = on ? 1 : 0;
}

void tune_set_path(const std::string& path) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_path = path;
    g_loaded = false;
    g_cache.clear();
}

void tune_clear() {
    std::lock_guard<std::mutex> lk(g_mu);
    g_cache.clear();
    g_loaded = true;
    save_locked();
}

bool tune_lookup(const std::string& key, int* choice) {
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    auto it = g_cache.find(key);
    if (it == g_cache.end()) return false;
    *choice = it->second;
    return true;
}

int tune_pick(const std::string& key, int ncand, int fallback, cudaStream_t s, const std::function<int(int)>& run) {
    if (ncand <= 1 || !tune_may_time(s)) return fallback;
    int c = 0;
    if (tune_lookup(key, &c) && c >= 0 && c < ncand) return c;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        return fallback;
    }
    std::vector<float> best(ncand, INFINITY);
    for (int rep = 0; rep < 3; ++rep) {  // the first round warms each candidate up
        for (int k = 0; k < ncand; ++k) {
            cudaEventRecord(e0, s);
            const int st = run(k);
            cudaEventRecord(e1, s);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            float ms = 0.f;
            if (st == 0 && rep > 0 && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms < best[k]) best[k] = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int bi = -1;
    for (int k = 0; k < ncand; ++k)
        if (std::isfinite(best[k]) && (bi < 0 || best[k] < best[bi])) bi = k;
    if (bi < 0) return fallback;
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    g_cache[key] = bi;
    save_locked();
    return bi;
}

}  // namespace vx

using namespace vx;

extern "C" {

void voxel_tune_enable(int on) { tune_set_enabled(on != 0); }

void voxel_tune_set_cache_path(const char* path) { tune_set_path(path ? path : ""); }

void voxel_tune_clear(void) { tune_clear(); }

int voxel_tune_lookup(const char* family, int dtype, size_t n) {
    int c = -1;
    if (!tune_lookup(tune_key(family, dtype, n), &c)) return -1;
    return c;
}

}  // extern "C"
