// Engine facade: the host object behind the voxel_engine_* C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "lower.h"
#include "vx_runtime.h"
#include "vx_types.h"

namespace vx {

// AGG_* slot state (reference engine.hpp AggState, used by HandleAggregate
// engine.hpp:499-569); persists across runs like the reference's.
struct AggSlot {
    bool init = false;
    uint64_t count = 0;
    double sum_f64 = 0.0;
    int64_t sum_i64 = 0;
    uint64_t min_bits = 0, max_bits = 0;
};

struct SegmentRef {
    const void* host = nullptr;    // borrowed caller buffer, read at run time
    const void* device = nullptr;  // device-resident column (not owned)
    uint64_t count = 0;
};

class Engine {
public:
    explicit Engine(int dtype);
    ~Engine();

    int dtype() const { return dtype_; }
    size_t add_segment(const void* host, size_t count);
    size_t add_segment_device(const void* dev, size_t count);
    void load_program(const uint32_t* code, size_t len);
    int run();
    // Lowers every data region without touching the device; explain() then
    // holds the schedules (register results of regions read as zero).
    int plan();
    // Lowers the loaded program to its data regions without running it; the
    // host-side scalar glue before each region is stepped with the current
    // registers.  Used by the batched executor.
    int lower_regions(std::vector<LoweredRegion>& out);
    int run_parallel(size_t seg_id, uint32_t threads, uint8_t result_reg);
    void reset();
    uint64_t& reg(size_t i) { return R_[i & 63]; }
    const std::string& explain() const { return explain_; }
    double last_device_ms() const { return last_ms_; }

private:
    int run_from_pc();
    int ensure_device_data(int seg, const void** dptr);
    int run_region(LoweredRegion& lr);
    int exec_agg(uint32_t raw, int kind);
    void drop_uploads();

    int dtype_;
    uint64_t R_[64] = {0};
    HostVec V_[16];
    uint32_t flags_ = 0;
    std::vector<uint32_t> code_;
    std::vector<size_t> loop_end_;  // loop head pc -> index of its back branch
    size_t pc_ = 0;
    bool running_ = false;
    FastPath fast_;
    std::vector<SegmentRef> segs_;
    AggSlot agg_[16];

    // device state
    cudaStream_t stream_ = nullptr;
    DevBuf scratch_;
    DevBuf result_;
    void* host_result_ = nullptr;  // pinned ScanResult
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    std::vector<DevBuf> uploads_;
    std::vector<const void*> dev_of_seg_;
    std::string explain_;
    double last_ms_ = 0.0;
    bool dry_ = false;
    std::vector<LoweredRegion>* capture_ = nullptr;
};

}  // namespace vx
