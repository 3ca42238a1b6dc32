// Plain data types shared by the host lowering and the CUDA kernels.
#pragma once

#include <stddef.h>
#include <stdint.h>
#include <type_traits>

namespace vx {

// Element types; the numbering is the one the C ABI uses.
enum DType : int { F64 = 0, F32 = 1, I64 = 2, I32 = 3, U64 = 4, U32 = 5 };

inline constexpr size_t dtype_size(int dt) { return (dt == F64 || dt == I64 || dt == U64) ? 8 : 4; }
// Engine<T>::kLanes: a 256-bit vector register holds 4 (64-bit) or 8 (32-bit) lanes
// (include/voxel/core/registers.hpp:170-178 in the reference).
inline constexpr size_t dtype_lanes(int dt) { return 32 / dtype_size(dt); }
inline constexpr bool dtype_is_float(int dt) { return dt == F64 || dt == F32; }

// Status codes returned by every status-returning entry point.
enum Status : int {
    kOk = 0,
    kErrInvalidArg = 1,
    kErrUnsupportedProgram = 2,
    kErrNonTerminating = 3,
    kErrCuda = 4,
    kErrOutOfMemory = 5,
    kErrDeviceTimeout = 6,
    kErrOverflow = 7,
    kErrNoDevice = 8,
    kErrCapacity = 9,
};

// ---- fused scan schedule (one lowered bytecode loop) -----------------------

constexpr int kMaxCols = 4;
constexpr int kMaxAtoms = 4;
constexpr int kMaxRed = 8;

// Per-group reductions: the vector reduction opcodes over one kLanes group.
enum RedKind : uint8_t { kRedSum = 0, kRedCount = 1, kRedMin = 2, kRedMax = 3 };
// How the per-group result is folded into its loop-carried scalar register.
enum AccOp : uint8_t {
    kAccNone = 0,  // temporary: only the last group's value is kept
    kAccAdd = 1,   // ADD   acc, acc, r   (i64, wraps)
    kAccSub = 2,   // SUB   acc, acc, r   (i64, wraps)
    kAccAddF = 3,  // ADDF  acc, acc, r   (f64, compensated)
    kAccMin = 4,   // MIN   acc, acc, r   (signed i64 compare)
    kAccMax = 5,   // MAX   acc, acc, r   (signed i64 compare)
    kAccTAdd = 6,  // fused fast path: acc += groupSum in T (f32: in f64)
};
enum OpndKind : uint8_t { kOpZero = 0, kOpCol = 1, kOpConst = 2 };

struct Atom {
    uint8_t col;
    uint8_t op;  // EQ NE LT LE GT GE = 0..5
    uint8_t pad[6];
    uint64_t thr;  // threshold as T bits
};

struct Opnd {
    uint8_t kind;
    uint8_t col;
    uint8_t pad[6];
    uint64_t bits;  // constant as T bits
};

// lane value = (all atoms in pmask hold) ? a : b ; pmask bit 31 = constant false
struct Red {
    uint8_t kind;
    uint8_t acc;
    uint8_t pad[2];
    uint32_t pmask;
    Opnd a, b;
};

constexpr uint32_t kMaskFalse = 0x80000000u;

struct ScanParams {
    int32_t dtype;
    int32_t ncols, natoms, nred;
    const void* col[kMaxCols];
    uint64_t count[kMaxCols];  // rows per column; VLOAD zero-pads past it
    uint64_t off0;             // first row of group 0
    uint64_t ngroups;          // groups the loop executes
    uint64_t ndata;            // leading groups that may touch data (rest are all-zero lanes)
    Atom atom[kMaxAtoms];
    Red red[kMaxRed];
    uint64_t acc0[kMaxRed];    // register values before the loop
};

struct ScanResult {
    uint64_t acc[kMaxRed];   // final register value per reduction (accumulators)
    uint64_t last[kMaxRed];  // value of the reduction in the last executed group
    int32_t status;
    int32_t pad;
};

}  // namespace vx
