// Autotuner: per (GPU, kernel family, element type, log2 size) the fastest of a
// family's candidate configurations, measured once with CUDA events and kept
// in a JSON cache file (one object of "key": choice entries).  The file is
// `$VOXEL_TUNE_CACHE` when set, else `tune_cache.json` beside the library.
// VOXEL_TUNE=0 turns tuning off (every family uses its default).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <string>

namespace vx {

// Cache key of one decision: "<gpu>|<family>|<dtype>|<log2 n>".
std::string tune_key(const char* family, int dtype, uint64_t n);

// The cached choice for `key` (true), or false when none is cached.
bool tune_lookup(const std::string& key, int* choice);

// Times candidates 0..ncand-1 with `run(c)` (which enqueues candidate c on
// `s`; a non-zero status skips that candidate), caches and returns the
// fastest.  With tuning off, on a capturing stream, or when every candidate
// fails, returns `fallback` without caching.
int tune_pick(const std::string& key, int ncand, int fallback, cudaStream_t s,
              const std::function<int(int)>& run);

bool tune_enabled();
// Tuning is on and `s` is not being captured into a graph (timing needs a
// synchronise, which a capture forbids).
bool tune_may_time(cudaStream_t s);
void tune_set_enabled(bool on);
void tune_set_path(const std::string& path);
void tune_clear();

}  // namespace vx
