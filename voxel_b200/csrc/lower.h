// Host-side lowering of VoxelVM bytecode regions to fused scan schedules.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "vx_types.h"

namespace vx {

// Host model of one 256-bit vector register: either 32 known bytes or
// data-dependent (unknown to the host).
struct HostVec {
    bool known = true;
    uint8_t bytes[32] = {0};
};

// Register writes a lowered region performs, applied on the host after the
// kernel's results come back.
struct RegWrite {
    enum Kind : uint8_t { kAcc, kLast, kValue } kind;
    uint8_t reg;
    uint8_t red;     // reduction index for kAcc / kLast
    uint64_t value;  // for kValue
};

struct LoweredRegion {
    ScanParams params{};          // columns are filled in by the engine (segment ids below)
    int seg_of_col[kMaxCols] = {0, 0, 0, 0};
    std::vector<RegWrite> writes;
    size_t resume_pc = 0;          // instruction after the region
    bool set_flags = false;        // flags after the region come from a CMP / ADD
    int64_t flag_value = 0;        // the i64 result those flags reflect
    bool fast_path = false;
};

// The fused filter+sum pattern Engine<T>::DetectFastPath recognises
// (include/voxel/exec/engine.hpp:84-107).
struct FastPath {
    bool ok = false;
    int seg = 0, thr = 3, acc = 0, off = 1, tot = 2;
    int mode = 0xC5;
};
FastPath detect_fast_path(const std::vector<uint32_t>& code);

// Lowers the fast path with the current registers (engine.hpp:109-141).
int lower_fast_path(const FastPath& fp, int dtype, const uint64_t* regs,
                    const std::vector<uint64_t>& seg_counts, LoweredRegion& out);

// Lowers the region that starts at `pc` (a loop head or a straight-line run
// with vector loads).  `loop_end` is the index of the loop's backward branch,
// or SIZE_MAX for a straight-line run ending at the next control transfer.
// Returns kOk or kErrUnsupportedProgram / kErrNonTerminating with a message
// in `why`.
int lower_region(const std::vector<uint32_t>& code, size_t pc, size_t loop_end, int dtype,
                 const uint64_t* regs, const HostVec* vregs,
                 const std::vector<uint64_t>& seg_counts, LoweredRegion& out, std::string& why);

// Text form of a lowered schedule (used by tests and diagnostics).
std::string describe(const LoweredRegion& r);

}  // namespace vx
