// Batched persistent executor: host object.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "lower.h"
#include "vx_runtime.h"
#include "vx_types.h"

namespace vx {

struct __align__(16) BatchProg {
    ScanParams p;
    uint32_t sel_mask;    // atoms whose conjunction selects rows (0: no selection)
    uint32_t want_sel;    // write row ids (else only count)
    uint32_t* sel_out;
    uint64_t sel_cap;     // capacity of sel_out in row ids
    uint64_t item0;       // first work item of this program
    uint32_t nitems;
    uint32_t vec;         // 16-byte aligned column: vector loads
    // range form (0: none): 1 + 2 * reduction kind + (excluded values present);
    // the predicate is lo <= x <= hi, x != ne[0], x != ne[1] (T bits)
    uint32_t fast;
    uint32_t pad0;
    uint64_t lo, hi;
    uint64_t ne[2];
};

struct BatchOut {
    ScanResult res;
    unsigned long long sel_count;  // exact count of selected rows
    int overflow;                  // the selection did not fit sel_cap (rows past it went to the spill arena)
    int spill_lost;                // ... and some of them did not fit the spill arena either
};

// Rows past a program's capacity: each item claims one contiguous range of the
// spill arena and records it as a fragment (at most one per item).
struct SpillFrag {
    uint32_t pid;       // program
    uint32_t n;         // rows
    uint64_t dst;       // output position of the fragment's first row
    uint64_t src;       // arena offset
};

struct SpillArgs {
    uint32_t* rows;                // the arena
    uint64_t cap;                  // arena capacity in rows
    unsigned long long* cursor;    // rows claimed
    SpillFrag* frags;
    unsigned int* nfrags;
};

class Batch {
public:
    static constexpr int kClasses = 60;  // element type x {8 range forms, one reduction, several}
    static constexpr int kBranches = 4;  // parallel graph branches the class kernels are spread over
    ~Batch();
    int add(int dtype, const uint32_t* code, size_t len, const uint64_t* regs, const void* d_col, uint64_t count,
            bool want_sel, uint64_t sel_cap, uint32_t* d_sel);
    void set_capacity(size_t i, uint64_t cap, uint32_t* d_sel);
    // one persistent launch for the whole batch (replayed from a CUDA graph when use_graph)
    int launch(cudaStream_t s, bool use_graph);
    int fetch(cudaStream_t s);  // copies the per-program outputs back (synchronises)
    size_t size() const { return host_.size(); }
    size_t fetched() const { return outs_.size(); }
    const BatchOut& out(size_t i) const { return outs_[i]; }
    const BatchProg& prog(size_t i) const { return host_[i]; }
    void registers(size_t i, uint64_t* regs) const;
    // After fetch: program idx[k]'s whole selection (its count rows) into d_pool
    // at caps... offsets (the counts of idx[0..k)), assembled from its buffer
    // and its spilled fragments; kErrCapacity if a listed program lost rows
    // (its spill did not fit the arena), which then needs rerun().
    int gather_overflow(size_t n, const size_t* idx, uint32_t* d_pool, cudaStream_t s);
    void set_spill_capacity(uint64_t rows) {
        spill_cap_ = rows;
        dirty_ = true;
    }
    // After fetch: re-runs programs idx[0..n) with selection capacities caps[k]
    // into d_pool (program k's rows at d_pool + caps[0] + ... + caps[k-1]),
    // from their already-lowered descriptors, one launch, and takes their
    // outputs in place of the fetched ones.
    int rerun(size_t n, const size_t* idx, const size_t* caps, uint32_t* d_pool, cudaStream_t s);
    uint64_t items() const { return nitems_; }

private:
    int upload(cudaStream_t s);
    int enqueue(cudaStream_t s, bool branches);

    std::vector<BatchProg> host_;
    std::vector<std::vector<RegWrite>> writes_;
    std::vector<std::vector<uint64_t>> regs_;
    std::vector<BatchOut> outs_;
    DevBuf d_progs_, d_start_, d_pids_, d_outs_, d_parts_, d_status_, d_pdone_, d_err_;
    DevBuf d_spill_, d_frags_, d_spill_ctr_, d_offmap_, d_glist_;
    uint64_t spill_cap_ = 1ull << 24;  // rows
    uint64_t nitems_ = 0;
    // per class: its programs
    // (d_pids_ + pid_off), item starts (d_start_ + cs_off) and item count
    struct ClassQueue {
        uint32_t pid_off = 0, cs_off = 0, np = 0;
        uint64_t items = 0;
    };
    ClassQueue cls_[kClasses];
    bool dirty_ = true;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    cudaStream_t capture_ = nullptr;  // private stream the graph is recorded on
    std::unique_ptr<Batch> sub_;      // re-run batch (its device buffers are reused)
    cudaStream_t branch_[kBranches] = {};
    cudaEvent_t fork_ = nullptr, join_[kBranches] = {};
};

}  // namespace vx
