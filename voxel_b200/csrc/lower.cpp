// Lowering of VoxelVM bytecode loops to fused scan schedules.
//
// The reference executes a filter/aggregate loop one instruction at a time
// (Engine<T>::Run, include/voxel/exec/engine.hpp:70-81) or, for the one
// pattern DetectFastPath accepts (engine.hpp:84-107), as a scalar C++ loop
// (RunFastPath, engine.hpp:109-141).  Here the host evaluates one iteration of
// the loop body symbolically, with loop-invariant registers as constants:
//
//   vector registers become lane expressions  lanes = F ? A : B
//     (F a conjunction of predicate atoms "column op threshold", A/B a column,
//      a constant splat or zero),
//   VSUM / VCOUNT / VRED_MIN / VRED_MAX become per-group reductions,
//   ADD / SUB / ADDF / MIN / MAX of a register with itself and a reduction
//     result become accumulators, ADD/ADDI of a constant become induction
//     variables, and the CMP + conditional branch give the trip count.
//
// The result is a ScanParams the fused kernel executes for all iterations in
// one launch.  Anything the schedule cannot reproduce exactly is rejected with
// a reason; there is no per-row interpretation on the device and no CPU path.
#include "lower.h"
#include "scan.h"

#include <cstdio>
#include <cstring>
#include <limits>
#include <set>
#include <sstream>

namespace vx {

namespace {

// ---- opcode numbers (include/voxel/bytecode/opcodes.hpp:11-262) -------------
enum : uint8_t {
    OP_NOP = 0x00, OP_HALT = 0x01,
    OP_MOV = 0x10, OP_MOVR = 0x11, OP_ADDI = 0x12, OP_SUBI = 0x13,
    OP_ADD = 0x20, OP_SUB = 0x21, OP_MUL = 0x22, OP_MIN = 0x27, OP_MAX = 0x28,
    OP_ADDF = 0x2A, OP_SUBF = 0x2B, OP_MULF = 0x2C,
    OP_CMP = 0x40,
    OP_JMP = 0x50, OP_JZ = 0x51, OP_JNZ = 0x52, OP_JS = 0x53, OP_JNS = 0x54,
    OP_JL = 0x59, OP_JLE = 0x5A, OP_JG = 0x5B, OP_JGE = 0x5C,
    OP_VLOAD = 0x70, OP_VSPLAT = 0x78,
    OP_VCMPEQ = 0xA0, OP_VCMPGE = 0xA5,
    OP_VAND = 0xB0, OP_VOR = 0xB1, OP_VXOR = 0xB2, OP_VNOT = 0xB3, OP_VANDN = 0xB4,
    OP_VFILTER = 0xC0, OP_VFILTER_EQ = 0xC1, OP_VFILTER_GE = 0xC6, OP_VBLEND = 0xC7,
    OP_VSUM = 0xD0, OP_VRED_MIN = 0xD5, OP_VRED_MAX = 0xD6, OP_VCOUNT = 0xD7,
};

inline unsigned f_rd(uint32_t r) { return (r >> 8) & 0xF; }
inline unsigned f_ra(uint32_t r) { return (r >> 12) & 0xF; }
inline unsigned f_rb(uint32_t r) { return (r >> 16) & 0xF; }
inline unsigned f_imm(uint32_t r) { return (r >> 20) & 0xFFF; }
inline int16_t f_simm(uint32_t r) {
    uint16_t v = (r >> 20) & 0xFFF;
    return (v & 0x800) ? static_cast<int16_t>(v | 0xF000) : static_cast<int16_t>(v);
}

double as_f64(uint64_t b) { double d; std::memcpy(&d, &b, 8); return d; }
uint64_t f64_bits(double d) { uint64_t b; std::memcpy(&b, &d, 8); return b; }
float as_f32(uint64_t b) { uint32_t u = static_cast<uint32_t>(b); float f; std::memcpy(&f, &u, 4); return f; }
uint64_t f32_bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

// Engine<T>::ScalarAsT (engine.hpp:395-401); f32 registers hold f64 values.
uint64_t scalar_as_t(int dt, uint64_t reg) {
    switch (dt) {
    case F32: return f32_bits(static_cast<float>(as_f64(reg)));
    case I32: case U32: return static_cast<uint32_t>(reg);
    default: return reg;
    }
}

uint64_t lane_mask(int dt) { return dtype_size(dt) == 8 ? ~0ull : 0xFFFFFFFFull; }

bool host_cmp(int dt, int op, uint64_t a, uint64_t b) {
    auto cmp = [op](auto x, auto y) {
        switch (op) {
        case 0: return x == y; case 1: return x != y; case 2: return x < y;
        case 3: return x <= y; case 4: return x > y; default: return x >= y;
        }
    };
    switch (dt) {
    case F64: return cmp(as_f64(a), as_f64(b));
    case F32: return cmp(as_f32(a), as_f32(b));
    case I64: return cmp(static_cast<int64_t>(a), static_cast<int64_t>(b));
    case I32: return cmp(static_cast<int32_t>(static_cast<uint32_t>(a)), static_cast<int32_t>(static_cast<uint32_t>(b)));
    case U64: return cmp(a, b);
    default: return cmp(static_cast<uint32_t>(a), static_cast<uint32_t>(b));
    }
}

int mirror_op(int op) {  // a op b  ==  b mirror(op) a
    switch (op) { case 2: return 4; case 3: return 5; case 4: return 2; case 5: return 3; default: return op; }
}

// ---- lane expressions ---------------------------------------------------------

struct Formula {
    uint32_t mask = 0;
    bool is_false = false;
    bool valid = true;
    bool is_true() const { return valid && !is_false && mask == 0; }
    bool operator==(const Formula& o) const {
        if (!valid || !o.valid) return false;
        if (is_false || o.is_false) return is_false == o.is_false;
        return mask == o.mask;
    }
};
Formula f_true() { return Formula{}; }
Formula f_false() { Formula f; f.is_false = true; return f; }
Formula f_invalid() { Formula f; f.valid = false; return f; }
Formula f_and(const Formula& a, const Formula& b) {
    if (!a.valid || !b.valid) return f_invalid();
    if (a.is_false || b.is_false) return f_false();
    Formula f;
    f.mask = a.mask | b.mask;
    return f;
}

struct LOp {
    uint8_t kind = kOpZero;  // kOpZero / kOpCol / kOpConst
    uint8_t col = 0;
    uint64_t bits = 0;
    bool operator==(const LOp& o) const {
        return kind == o.kind && (kind != kOpCol || col == o.col) && (kind != kOpConst || bits == o.bits);
    }
};
LOp op_zero() { return LOp{}; }
LOp op_const(uint64_t b) { LOp o; if (b) { o.kind = kOpConst; o.bits = b; } return o; }
LOp op_col(int c) { LOp o; o.kind = kOpCol; o.col = static_cast<uint8_t>(c); return o; }

struct LExpr {
    bool valid = false;
    Formula f;
    LOp a, b;  // lanes = f ? a : b
};
LExpr ex_simple(LOp a) { LExpr e; e.valid = true; e.f = f_true(); e.a = a; e.b = op_zero(); return e; }
LExpr ex_sel(Formula f, LOp a, LOp b) {
    LExpr e;
    e.valid = f.valid;
    e.f = f;
    e.a = a;
    e.b = b;
    if (f.is_false) { e.f = f_true(); e.a = b; e.b = op_zero(); }
    if (e.f.is_true()) e.b = op_zero();
    if (e.a == e.b) { e.f = f_true(); e.b = op_zero(); }
    return e;
}
bool is_simple(const LExpr& e) { return e.valid && e.f.is_true(); }

// bitwise combinations of operands; ok=false when not representable
LOp op_and(const LOp& x, const LOp& y, int dt, bool& ok) {
    uint64_t ones = lane_mask(dt);
    if (x.kind == kOpZero || y.kind == kOpZero) return op_zero();
    if (x.kind == kOpConst && y.kind == kOpConst) return op_const(x.bits & y.bits);
    if (x.kind == kOpConst && x.bits == ones) return y;
    if (y.kind == kOpConst && y.bits == ones) return x;
    if (x.kind == kOpCol && y.kind == kOpCol && x.col == y.col) return x;
    ok = false;
    return op_zero();
}
LOp op_or(const LOp& x, const LOp& y, int dt, bool& ok) {
    uint64_t ones = lane_mask(dt);
    if (x.kind == kOpZero) return y;
    if (y.kind == kOpZero) return x;
    if (x.kind == kOpConst && y.kind == kOpConst) return op_const(x.bits | y.bits);
    if ((x.kind == kOpConst && x.bits == ones) || (y.kind == kOpConst && y.bits == ones)) return op_const(ones);
    if (x.kind == kOpCol && y.kind == kOpCol && x.col == y.col) return x;
    ok = false;
    return op_zero();
}
LOp op_not(const LOp& x, int dt, bool& ok) {
    uint64_t ones = lane_mask(dt);
    if (x.kind == kOpZero) return op_const(ones);
    if (x.kind == kOpConst) return op_const(~x.bits & ones);
    ok = false;
    return op_zero();
}

using BinOp = LOp (*)(const LOp&, const LOp&, int, bool&);

LExpr ex_bin(const LExpr& x, const LExpr& y, int dt, BinOp fn) {
    LExpr bad;
    if (!x.valid || !y.valid) return bad;
    bool ok = true;
    if (x.f == y.f) {
        LExpr e = ex_sel(x.f, fn(x.a, y.a, dt, ok), fn(x.b, y.b, dt, ok));
        return ok ? e : bad;
    }
    if (x.f.is_true()) {
        LExpr e = ex_sel(y.f, fn(x.a, y.a, dt, ok), fn(x.a, y.b, dt, ok));
        return ok ? e : bad;
    }
    if (y.f.is_true()) {
        LExpr e = ex_sel(x.f, fn(x.a, y.a, dt, ok), fn(x.b, y.a, dt, ok));
        return ok ? e : bad;
    }
    // two different conjunctions: representable when every lane outside F&G is zero
    LOp aa = fn(x.a, y.a, dt, ok), ab = fn(x.a, y.b, dt, ok), ba = fn(x.b, y.a, dt, ok), bb = fn(x.b, y.b, dt, ok);
    if (!ok) return bad;
    if (ab.kind == kOpZero && ba.kind == kOpZero && bb.kind == kOpZero) return ex_sel(f_and(x.f, y.f), aa, op_zero());
    return bad;
}

// ---- scalar symbolic state ------------------------------------------------------

struct SVal {
    enum K : uint8_t { Known, Carried, Induct, Temp, Acc } k = Known;
    uint64_t v = 0;      // Known value / Induct delta
    int red = -1;        // Temp / Acc reduction
};

struct FlagSrc {
    enum K : uint8_t { None, Const, IndCmp, IndArith, Data } k = None;
    int reg = -1;
    int64_t delta = 0;   // induction delta at the CMP
    int64_t limit = 0;
    int sign = 1;
    int64_t value = 0;   // Const
};

struct Builder {
    int dt;
    size_t kl;
    const std::vector<uint64_t>& counts;
    LoweredRegion& out;
    std::string& why;
    int ncols = 0;
    int natoms = 0;
    int nred = 0;
    int load_reg = -1;        // induction register the loads use (-1: constant offset)
    int64_t load_delta = 0;
    uint64_t load_const = 0;
    bool have_load = false;

    Builder(int d, const std::vector<uint64_t>& c, LoweredRegion& o, std::string& w)
        : dt(d), kl(dtype_lanes(d)), counts(c), out(o), why(w) {}

    bool fail(const char* msg, size_t pc) {
        char buf[200];
        std::snprintf(buf, sizeof buf, "%s (instruction %zu)", msg, pc);
        why = buf;
        return false;
    }

    int column(int seg) {
        for (int c = 0; c < ncols; ++c)
            if (out.seg_of_col[c] == seg) return c;
        if (ncols == kMaxCols) return -1;
        out.seg_of_col[ncols] = seg;
        return ncols++;
    }

    int atom(int col, int op, uint64_t thr) {
        for (int a = 0; a < natoms; ++a) {
            const Atom& at = out.params.atom[a];
            if (at.col == col && at.op == op && at.thr == thr) return a;
        }
        if (natoms == kMaxAtoms) return -1;
        Atom& at = out.params.atom[natoms];
        at.col = static_cast<uint8_t>(col);
        at.op = static_cast<uint8_t>(op);
        at.thr = thr;
        return natoms++;
    }
};

int64_t floor_div(int64_t a, int64_t b) {
    int64_t q = a / b, r = a % b;
    return (r != 0 && ((r < 0) != (b < 0))) ? q - 1 : q;
}
int64_t ceil_div(int64_t a, int64_t b) { return -floor_div(-a, b); }

}  // namespace

FastPath detect_fast_path(const std::vector<uint32_t>& c) {
    // engine.hpp:84-107, including its operand-aliasing checks
    FastPath f;
    if (c.size() < 8) return f;
    uint32_t r0 = c[0], r1 = c[1], r2 = c[2], r3 = c[3], r4 = c[4], r5 = c[5], r6 = c[6];
    unsigned o0 = r0 & 0xFF, o1 = r1 & 0xFF, o2 = r2 & 0xFF, o3 = r3 & 0xFF, o4 = r4 & 0xFF,
             o5 = r5 & 0xFF, o6 = r6 & 0xFF;
    bool isf = o1 >= 0xC1 && o1 <= 0xC6;
    if (o0 == 0x70 && isf && o2 == 0xD0 && o3 == 0x2A && o4 == 0x20 && o5 == 0x40 && o6 == 0x52 &&
        f_ra(r1) == f_rd(r0) && f_ra(r2) == f_rd(r1) && f_rb(r3) == f_rd(r2) && f_ra(r4) == f_ra(r0) &&
        f_ra(r5) == f_ra(r0) && f_simm(r6) == -6) {
        f.ok = true;
        f.seg = (r0 >> 28) & 0xF;
        f.thr = static_cast<int>(f_rb(r1));
        f.acc = static_cast<int>(f_rd(r3));
        f.off = static_cast<int>(f_ra(r0));
        f.tot = static_cast<int>(f_rb(r5));
        f.mode = static_cast<int>(o1);
    }
    return f;
}

int lower_fast_path(const FastPath& fp, int dt, const uint64_t* regs,
                    const std::vector<uint64_t>& seg_counts, LoweredRegion& out) {
    out = LoweredRegion{};
    out.fast_path = true;
    if (fp.seg < 0 || static_cast<size_t>(fp.seg) >= seg_counts.size()) return kErrInvalidArg;
    ScanParams& p = out.params;
    size_t kl = dtype_lanes(dt);
    p.dtype = dt;
    p.ncols = 1;
    out.seg_of_col[0] = fp.seg;
    p.count[0] = seg_counts[fp.seg];
    uint64_t total = static_cast<uint64_t>(static_cast<int64_t>(regs[fp.tot]));
    if (seg_counts[fp.seg] < total) total = seg_counts[fp.seg];
    uint64_t off = static_cast<uint64_t>(static_cast<int64_t>(regs[fp.off]));
    // while (offset + kLanes <= total): whole groups only, the tail is dropped
    uint64_t n = (off + kl >= off && off + kl <= total) ? (total - off) / kl : 0;
    p.off0 = off;
    p.ngroups = n;
    p.ndata = n;
    p.natoms = 1;
    p.atom[0].col = 0;
    p.atom[0].op = static_cast<uint8_t>(fp.mode - 0xC1);
    p.atom[0].thr = scalar_as_t(dt, regs[fp.thr]);
    p.nred = 1;
    Red& r = p.red[0];
    r.kind = kRedSum;
    r.acc = kAccTAdd;
    r.pmask = 1;
    r.a.kind = kOpCol;
    r.a.col = 0;
    r.b.kind = kOpZero;
    p.acc0[0] = regs[fp.acc];
    out.writes.push_back({RegWrite::kAcc, static_cast<uint8_t>(fp.acc), 0, 0});
    out.writes.push_back({RegWrite::kValue, static_cast<uint8_t>(fp.off), 0, off + n * kl});
    return kOk;
}

int lower_region(const std::vector<uint32_t>& code, size_t pc0, size_t loop_end, int dt,
                 const uint64_t* regs, const HostVec* vregs, const std::vector<uint64_t>& seg_counts,
                 LoweredRegion& out, std::string& why) {
    out = LoweredRegion{};
    out.params.dtype = dt;
    Builder B(dt, seg_counts, out, why);
    const bool loop = loop_end != SIZE_MAX;
    size_t end = loop ? loop_end : pc0;
    if (!loop) {
        while (end < code.size()) {
            uint8_t op = code[end] & 0xFF;
            if (op == OP_HALT || (op >= OP_JMP && op <= 0x5F)) break;
            ++end;
        }
    }

    // registers written anywhere in the region are loop-carried at the head
    std::set<int> written;
    for (size_t i = pc0; i < end; ++i) {
        uint32_t raw = code[i];
        uint8_t op = raw & 0xFF;
        bool writes_rd = (op >= OP_MOV && op <= 0x1E) || (op >= OP_ADD && op <= 0x3F) ||
                         op == OP_VSUM || op == OP_VCOUNT || op == OP_VRED_MIN || op == OP_VRED_MAX;
        if (writes_rd) written.insert(static_cast<int>(f_rd(raw)));
    }

    SVal R[16];
    for (int r = 0; r < 16; ++r) {
        R[r].k = (loop && written.count(r)) ? SVal::Carried : SVal::Known;
        R[r].v = regs[r];
    }
    LExpr V[16];
    bool Vcarried[16] = {false};
    std::set<int> vwritten;
    for (size_t i = pc0; i < end; ++i) {
        uint8_t op = code[i] & 0xFF;
        if (op == OP_VLOAD || op == OP_VSPLAT || (op >= OP_VCMPEQ && op <= OP_VCMPGE) ||
            (op >= OP_VAND && op <= OP_VANDN) || (op >= OP_VFILTER && op <= OP_VBLEND))
            vwritten.insert(static_cast<int>(f_rd(code[i])));
    }
    for (int v = 0; v < 16; ++v) {
        if (loop && vwritten.count(v)) { Vcarried[v] = true; continue; }
        const HostVec& hv = vregs[v];
        if (!hv.known) continue;  // invalid LExpr: unusable if read
        size_t es = dtype_size(dt);
        uint64_t l0 = 0;
        std::memcpy(&l0, hv.bytes, es);
        bool uniform = true;
        for (size_t l = 1; l < 32 / es; ++l) {
            uint64_t x = 0;
            std::memcpy(&x, hv.bytes + l * es, es);
            if (x != l0) uniform = false;
        }
        if (uniform) V[v] = ex_simple(op_const(l0));
    }
    Formula M[8];
    for (int m = 0; m < 8; ++m) M[m] = f_invalid();

    FlagSrc flags;
    int red_acc_reg[kMaxRed];
    for (int k = 0; k < kMaxRed; ++k) red_acc_reg[k] = -1;

    auto vread = [&](unsigned v, size_t pc, LExpr& e) -> bool {
        if (Vcarried[v]) return B.fail("vector register carried across loop iterations", pc);
        e = V[v];
        if (!e.valid) return B.fail("vector operand not representable", pc);
        return true;
    };
    auto vwrite = [&](unsigned v, const LExpr& e) { V[v] = e; Vcarried[v] = false; };
    auto known = [&](unsigned r) { return R[r].k == SVal::Known; };

    for (size_t pc = pc0; pc < end; ++pc) {
        uint32_t raw = code[pc];
        uint8_t op = raw & 0xFF;
        unsigned rd = f_rd(raw), ra = f_ra(raw), rb = f_rb(raw), imm = f_imm(raw);
        int16_t si = f_simm(raw);
        switch (op) {
        case OP_NOP: break;
        case OP_MOV: R[rd].k = SVal::Known; R[rd].v = static_cast<uint64_t>(static_cast<int64_t>(si)); break;
        case OP_MOVR:
            if (!known(ra)) return B.fail("MOVR of a loop-carried register", pc), kErrUnsupportedProgram;
            R[rd] = R[ra];
            break;
        case OP_ADDI:
        case OP_SUBI: {
            int64_t d = op == OP_ADDI ? si : -static_cast<int64_t>(si);
            if (known(ra)) { R[rd].k = SVal::Known; R[rd].v = R[ra].v + static_cast<uint64_t>(d); }
            else if (rd == ra && (R[ra].k == SVal::Carried || R[ra].k == SVal::Induct)) {
                if (R[ra].k == SVal::Carried) { R[ra].k = SVal::Induct; R[ra].v = 0; }
                R[rd].v += static_cast<uint64_t>(d);
            } else return B.fail("unsupported ADDI/SUBI form", pc), kErrUnsupportedProgram;
            break;
        }
        case OP_ADD: case OP_SUB: case OP_MUL: case OP_MIN: case OP_MAX:
        case OP_ADDF: case OP_SUBF: case OP_MULF: {
            bool fl = op >= OP_ADDF;
            if (known(ra) && known(rb)) {
                uint64_t a = R[ra].v, b = R[rb].v, r;
                int64_t ia = static_cast<int64_t>(a), ib = static_cast<int64_t>(b);
                switch (op) {
                case OP_ADD: r = a + b; break;
                case OP_SUB: r = a - b; break;
                case OP_MUL: r = a * b; break;
                case OP_MIN: r = static_cast<uint64_t>(ia < ib ? ia : ib); break;
                case OP_MAX: r = static_cast<uint64_t>(ia > ib ? ia : ib); break;
                case OP_ADDF: r = f64_bits(as_f64(a) + as_f64(b)); break;
                case OP_SUBF: r = f64_bits(as_f64(a) - as_f64(b)); break;
                default: r = f64_bits(as_f64(a) * as_f64(b)); break;
                }
                R[rd].k = SVal::Known;
                R[rd].v = r;
                if (!fl) { flags = FlagSrc{}; flags.k = FlagSrc::Const; flags.value = static_cast<int64_t>(r); }
                else flags.k = FlagSrc::Data;  // partial float flag update: not modelled
                break;
            }
            // induction update: r = r +/- invariant
            if ((op == OP_ADD || op == OP_SUB) && rd == ra && known(rb) &&
                (R[ra].k == SVal::Carried || R[ra].k == SVal::Induct)) {
                if (R[ra].k == SVal::Carried) { R[ra].k = SVal::Induct; R[ra].v = 0; }
                R[rd].v += op == OP_ADD ? R[rb].v : (0 - R[rb].v);
                flags = FlagSrc{};
                flags.k = FlagSrc::IndArith;
                flags.reg = static_cast<int>(rd);
                flags.delta = static_cast<int64_t>(R[rd].v);
                break;
            }
            if (op == OP_ADD && rd == rb && known(ra) && (R[rb].k == SVal::Carried || R[rb].k == SVal::Induct)) {
                if (R[rb].k == SVal::Carried) { R[rb].k = SVal::Induct; R[rb].v = 0; }
                R[rd].v += R[ra].v;
                flags = FlagSrc{};
                flags.k = FlagSrc::IndArith;
                flags.reg = static_cast<int>(rd);
                flags.delta = static_cast<int64_t>(R[rd].v);
                break;
            }
            // accumulator: r = r op temp  (commutative ops also r = temp op r)
            int other = -1;
            bool self_ok = loop ? (R[rd].k == SVal::Carried) : known(rd);
            if (rd == ra && self_ok && R[rb].k == SVal::Temp) other = static_cast<int>(rb);
            else if (rd == rb && self_ok && R[ra].k == SVal::Temp && op != OP_SUB && op != OP_SUBF)
                other = static_cast<int>(ra);
            uint8_t accop = 0;
            switch (op) {
            case OP_ADD: accop = kAccAdd; break;
            case OP_SUB: accop = kAccSub; break;
            case OP_ADDF: accop = kAccAddF; break;
            case OP_MIN: accop = kAccMin; break;
            case OP_MAX: accop = kAccMax; break;
            default: other = -1; break;
            }
            if (other < 0 || (loop && ra == rb)) return B.fail("unsupported scalar operation in loop", pc), kErrUnsupportedProgram;
            int k = R[other].red;
            if (red_acc_reg[k] >= 0) return B.fail("reduction folded into two accumulators", pc), kErrUnsupportedProgram;
            red_acc_reg[k] = static_cast<int>(rd);
            out.params.red[k].acc = accop;
            out.params.acc0[k] = regs[rd];
            if (!loop) out.params.acc0[k] = R[rd].v;
            R[rd].k = SVal::Acc;
            R[rd].red = k;
            flags.k = FlagSrc::Data;
            break;
        }
        case OP_CMP: {
            flags = FlagSrc{};
            // `CMP acc, r; JLE 2; MOVR acc, r` (JGE: max) keeps the smaller (larger) of
            // the accumulator and a reduction result in signed 64-bit order -- the
            // MIN / MAX fold the Python query builder emits (bindings/voxel_query.py:
            // 116-139; JLE / JGE jump on the signed flags of ra - rb)
            if (pc + 2 < end) {
                const uint32_t jr = code[pc + 1], mr = code[pc + 2];
                const uint8_t jop = jr & 0xFF;
                const bool self_ok = loop ? (R[ra].k == SVal::Carried) : known(ra);
                if ((jop == OP_JLE || jop == OP_JGE) && f_simm(jr) == 2 && (mr & 0xFF) == OP_MOVR &&
                    f_rd(mr) == ra && f_ra(mr) == rb && ra != rb && R[rb].k == SVal::Temp && self_ok) {
                    const int k = R[rb].red;
                    if (red_acc_reg[k] >= 0)
                        return B.fail("reduction folded into two accumulators", pc), kErrUnsupportedProgram;
                    red_acc_reg[k] = static_cast<int>(ra);
                    out.params.red[k].acc = jop == OP_JLE ? kAccMin : kAccMax;
                    out.params.acc0[k] = loop ? regs[ra] : R[ra].v;
                    R[ra].k = SVal::Acc;
                    R[ra].red = k;
                    flags.k = FlagSrc::Data;
                    pc += 2;
                    break;
                }
            }
            if (known(ra) && known(rb)) {
                flags.k = FlagSrc::Const;
                flags.value = static_cast<int64_t>(R[ra].v - R[rb].v);
            } else if ((R[ra].k == SVal::Induct || R[ra].k == SVal::Carried) && known(rb)) {
                flags.k = FlagSrc::IndCmp;
                flags.reg = static_cast<int>(ra);
                flags.delta = R[ra].k == SVal::Induct ? static_cast<int64_t>(R[ra].v) : 0;
                flags.limit = static_cast<int64_t>(R[rb].v);
                flags.sign = 1;
            } else if ((R[rb].k == SVal::Induct || R[rb].k == SVal::Carried) && known(ra)) {
                flags.k = FlagSrc::IndCmp;
                flags.reg = static_cast<int>(rb);
                flags.delta = R[rb].k == SVal::Induct ? static_cast<int64_t>(R[rb].v) : 0;
                flags.limit = static_cast<int64_t>(R[ra].v);
                flags.sign = -1;
            } else {
                return B.fail("CMP on data-dependent registers", pc), kErrUnsupportedProgram;
            }
            break;
        }
        case OP_VLOAD: {
            unsigned seg = (imm >> 8) & 0xF, cnt = imm & 0xFF;
            if (cnt != 0 && cnt != B.kl) return B.fail("partial-width VLOAD", pc), kErrUnsupportedProgram;
            if (seg >= seg_counts.size()) {
                // VLOAD from a missing segment loads zeros (engine.hpp:1963-1965)
                vwrite(rd, ex_simple(op_zero()));
                break;
            }
            int lreg = -1;
            int64_t ldelta = 0;
            uint64_t lconst = 0;
            if (known(ra)) lconst = R[ra].v;
            else if (R[ra].k == SVal::Induct || R[ra].k == SVal::Carried) {
                lreg = static_cast<int>(ra);
                ldelta = R[ra].k == SVal::Induct ? static_cast<int64_t>(R[ra].v) : 0;
                if (R[ra].k == SVal::Carried) { R[ra].k = SVal::Induct; R[ra].v = 0; }
            } else return B.fail("VLOAD offset is data-dependent", pc), kErrUnsupportedProgram;
            if (loop && lreg < 0) return B.fail("loop VLOAD offset does not advance", pc), kErrUnsupportedProgram;
            if (B.have_load && (lreg != B.load_reg || ldelta != B.load_delta || (lreg < 0 && lconst != B.load_const)))
                return B.fail("VLOADs at different offsets", pc), kErrUnsupportedProgram;
            B.have_load = true;
            B.load_reg = lreg;
            B.load_delta = ldelta;
            B.load_const = lconst;
            int c = B.column(static_cast<int>(seg));
            if (c < 0) return B.fail("more than 4 columns", pc), kErrUnsupportedProgram;
            vwrite(rd, ex_simple(op_col(c)));
            break;
        }
        case OP_VSPLAT:
            if (!known(ra)) return B.fail("VSPLAT of a loop-carried register", pc), kErrUnsupportedProgram;
            vwrite(rd, ex_simple(op_const(scalar_as_t(dt, R[ra].v))));
            break;
        case 0xA0: case 0xA1: case 0xA2: case 0xA3: case 0xA4: case 0xA5: {
            LExpr x, y;
            if (!vread(ra, pc, x) || !vread(rb, pc, y)) return kErrUnsupportedProgram;
            if (!is_simple(x) || !is_simple(y)) return B.fail("VCMP of a masked vector", pc), kErrUnsupportedProgram;
            int cop = op - 0xA0;
            Formula f;
            auto tconst = [](const LOp& o) { return o.kind == kOpConst ? o.bits : 0ull; };
            if (x.a.kind == kOpCol && y.a.kind != kOpCol) {
                int a = B.atom(x.a.col, cop, tconst(y.a));
                if (a < 0) return B.fail("more than 4 predicate atoms", pc), kErrUnsupportedProgram;
                f.mask = 1u << a;
            } else if (y.a.kind == kOpCol && x.a.kind != kOpCol) {
                int a = B.atom(y.a.col, mirror_op(cop), tconst(x.a));
                if (a < 0) return B.fail("more than 4 predicate atoms", pc), kErrUnsupportedProgram;
                f.mask = 1u << a;
            } else if (x.a.kind != kOpCol && y.a.kind != kOpCol) {
                f = host_cmp(dt, cop, tconst(x.a), tconst(y.a)) ? f_true() : f_false();
            } else {
                return B.fail("VCMP between two columns", pc), kErrUnsupportedProgram;
            }
            vwrite(rd, ex_sel(f, op_const(lane_mask(dt)), op_zero()));
            M[0] = f;
            break;
        }
        case OP_VAND: case OP_VOR: case OP_VANDN: {
            LExpr x, y;
            if (!vread(ra, pc, x) || !vread(rb, pc, y)) return kErrUnsupportedProgram;
            LExpr r;
            if (op == OP_VAND) r = ex_bin(x, y, dt, op_and);
            else if (op == OP_VOR) r = ex_bin(x, y, dt, op_or);
            else {
                bool ok = true;
                LExpr nx = ex_sel(x.f, op_not(x.a, dt, ok), op_not(x.b, dt, ok));
                if (!ok) return B.fail("VANDN of a data vector", pc), kErrUnsupportedProgram;
                r = ex_bin(nx, y, dt, op_and);
            }
            if (!r.valid) return B.fail("bitwise combination not representable", pc), kErrUnsupportedProgram;
            vwrite(rd, r);
            break;
        }
        case OP_VFILTER: case 0xC1: case 0xC2: case 0xC3: case 0xC4: case 0xC5: case 0xC6: {
            if (!known(rb)) return B.fail("VFILTER threshold is loop-carried", pc), kErrUnsupportedProgram;
            LExpr x;
            if (!vread(ra, pc, x)) return kErrUnsupportedProgram;
            int cop = op == OP_VFILTER ? static_cast<int>(imm & 7) : op - 0xC1;
            uint64_t t = scalar_as_t(dt, R[rb].v);
            unsigned mreg = imm & 7;
            if (cop > 5) {  // generic VFILTER with an undefined mode passes nothing
                vwrite(rd, ex_simple(op_zero()));
                M[mreg] = f_false();
                break;
            }
            bool zero_passes = host_cmp(dt, cop, 0, t);
            if (x.b.kind != kOpZero) return B.fail("VFILTER of a blended vector", pc), kErrUnsupportedProgram;
            if (x.a.kind == kOpCol) {
                int a = B.atom(x.a.col, cop, t);
                if (a < 0) return B.fail("more than 4 predicate atoms", pc), kErrUnsupportedProgram;
                Formula at;
                at.mask = 1u << a;
                Formula f = f_and(x.f, at);
                vwrite(rd, ex_sel(f, x.a, op_zero()));
                M[mreg] = (!zero_passes || x.f.is_true()) ? f : f_invalid();
            } else if (x.a.kind == kOpConst) {
                bool p = host_cmp(dt, cop, x.a.bits, t);
                vwrite(rd, p ? x : ex_simple(op_zero()));
                Formula f = p ? x.f : f_false();
                M[mreg] = (!zero_passes || x.f.is_true()) ? f : f_invalid();
            } else {
                vwrite(rd, ex_simple(op_zero()));
                M[mreg] = zero_passes ? f_true() : f_false();
            }
            break;
        }
        case OP_VBLEND: {
            LExpr x, y;
            if (!vread(ra, pc, x) || !vread(rb, pc, y)) return kErrUnsupportedProgram;
            Formula m = M[imm & 7];
            if (!m.valid) return B.fail("VBLEND mask not representable", pc), kErrUnsupportedProgram;
            LOp on, off;
            if (y.f.is_true()) on = y.a;
            else if (y.f == m) on = y.a;
            else return B.fail("VBLEND operand not representable", pc), kErrUnsupportedProgram;
            if (x.f.is_true()) off = x.a;
            else if (x.f == m) off = x.b;
            else return B.fail("VBLEND operand not representable", pc), kErrUnsupportedProgram;
            vwrite(rd, ex_sel(m, on, off));
            break;
        }
        case OP_VSUM: case OP_VCOUNT: case OP_VRED_MIN: case OP_VRED_MAX: {
            LExpr x;
            if (!vread(ra, pc, x)) return kErrUnsupportedProgram;
            if (B.nred == kMaxRed) return B.fail("more than 8 reductions", pc), kErrUnsupportedProgram;
            int k = B.nred++;
            Red& r = out.params.red[k];
            r.kind = op == OP_VSUM ? kRedSum : op == OP_VCOUNT ? kRedCount : op == OP_VRED_MIN ? kRedMin : kRedMax;
            r.acc = kAccNone;
            r.pmask = x.f.is_false ? kMaskFalse : x.f.mask;
            r.a.kind = x.a.kind; r.a.col = x.a.col; r.a.bits = x.a.bits;
            r.b.kind = x.b.kind; r.b.col = x.b.col; r.b.bits = x.b.bits;
            R[rd].k = SVal::Temp;
            R[rd].red = k;
            break;
        }
        default:
            return B.fail("opcode outside the lowered set", pc), kErrUnsupportedProgram;
        }
    }

    ScanParams& p = out.params;
    p.ncols = B.ncols;
    p.natoms = B.natoms;
    p.nred = B.nred;
    if (B.nred == 0 && !B.have_load) return B.fail("region has no vector work", pc0), kErrUnsupportedProgram;

    // trip count
    uint64_t n = 1;
    int64_t step = 0;
    if (loop) {
        if (!B.have_load) return B.fail("loop without VLOAD", pc0), kErrUnsupportedProgram;
        if (R[B.load_reg].k != SVal::Induct) return B.fail("load offset register is not an induction variable", pc0), kErrUnsupportedProgram;
        step = static_cast<int64_t>(R[B.load_reg].v);
        uint8_t bop = code[loop_end] & 0xFF;
        if (flags.k != FlagSrc::IndCmp && flags.k != FlagSrc::IndArith)
            return B.fail("loop exit does not test the induction variable", loop_end), kErrUnsupportedProgram;
        int ireg = flags.reg;
        if (R[ireg].k != SVal::Induct) return B.fail("loop exit register is not an induction variable", loop_end), kErrUnsupportedProgram;
        int64_t istep = static_cast<int64_t>(R[ireg].v);
        __int128 head = static_cast<int64_t>(regs[ireg]);
        __int128 A, Bc;
        if (flags.k == FlagSrc::IndCmp) {
            A = flags.sign * (head + flags.delta - flags.limit);
            Bc = static_cast<__int128>(flags.sign) * istep;
        } else {
            A = head + flags.delta;
            Bc = istep;
        }
        // f_j = A + (j-1)*Bc ; continue while cond(f_j); n = first j >= 1 that stops
        const __int128 kMaxTrip = static_cast<__int128>(1) << 44;
        __int128 tn = -1;
        auto ceil128 = [](__int128 a, __int128 b) { __int128 q = a / b, r = a % b; return (r != 0 && ((r > 0) == (b > 0))) ? q + 1 : q; };
        auto floor128 = [](__int128 a, __int128 b) { __int128 q = a / b, r = a % b; return (r != 0 && ((r < 0) != (b < 0))) ? q - 1 : q; };
        switch (bop) {
        case OP_JNZ:
            if (A == 0) tn = 1;
            else if (Bc != 0 && (-A) % Bc == 0 && (-A) / Bc > 0) tn = (-A) / Bc + 1;
            break;
        case OP_JZ:
            tn = A != 0 ? 1 : (Bc != 0 ? 2 : -1);
            break;
        case OP_JL: case OP_JS:
            if (A >= 0) tn = 1; else if (Bc > 0) tn = 1 + ceil128(-A, Bc);
            break;
        case OP_JLE:
            if (A > 0) tn = 1; else if (Bc > 0) tn = 2 + floor128(-A, Bc);
            break;
        case OP_JG:
            if (A <= 0) tn = 1; else if (Bc < 0) tn = 1 + ceil128(A, -Bc);
            break;
        case OP_JGE: case OP_JNS:
            if (A < 0) tn = 1; else if (Bc < 0) tn = 2 + floor128(A, -Bc);
            break;
        default:
            return B.fail("unsupported loop branch", loop_end), kErrUnsupportedProgram;
        }
        if (tn < 1 || tn > kMaxTrip) {
            why = "loop never reaches its exit condition";
            return kErrNonTerminating;
        }
        n = static_cast<uint64_t>(tn);
        __int128 fin = A + (tn - 1) * Bc;
        out.set_flags = true;
        out.flag_value = static_cast<int64_t>(fin);
        if (B.nred > 0 && step != static_cast<int64_t>(B.kl) && n > 1)
            return B.fail("load stride differs from the vector width", pc0), kErrUnsupportedProgram;
        out.resume_pc = loop_end + 1;
    } else {
        out.resume_pc = end;
        if (flags.k == FlagSrc::Const) { out.set_flags = true; out.flag_value = flags.value; }
    }

    // rows: group j covers [off0 + j*kl, off0 + (j+1)*kl)
    uint64_t off0 = B.load_reg >= 0 ? static_cast<uint64_t>(static_cast<int64_t>(regs[B.load_reg]) + B.load_delta)
                                    : B.load_const;
    if (static_cast<int64_t>(off0) < 0 && n > 1) return B.fail("negative load offset", pc0), kErrUnsupportedProgram;
    p.off0 = off0;
    p.ngroups = n;
    uint64_t maxc = 0;
    for (int c = 0; c < B.ncols; ++c) {
        p.count[c] = seg_counts[out.seg_of_col[c]];
        if (p.count[c] > maxc) maxc = p.count[c];
    }
    uint64_t nd = 0;
    if (maxc > off0 && static_cast<int64_t>(off0) >= 0) nd = (maxc - off0 + B.kl - 1) / B.kl;
    p.ndata = nd < n ? nd : n;

    // register writes once the kernel is done
    for (int r = 0; r < 16; ++r) {
        switch (R[r].k) {
        case SVal::Known:
            if (written.count(r) || (!loop && R[r].v != regs[r]))
                out.writes.push_back({RegWrite::kValue, static_cast<uint8_t>(r), 0, R[r].v});
            break;
        case SVal::Induct:
            out.writes.push_back({RegWrite::kValue, static_cast<uint8_t>(r), 0,
                                  regs[r] + n * R[r].v});
            break;
        case SVal::Temp:
            out.writes.push_back({RegWrite::kLast, static_cast<uint8_t>(r), static_cast<uint8_t>(R[r].red), 0});
            break;
        case SVal::Acc:
            out.writes.push_back({RegWrite::kAcc, static_cast<uint8_t>(r), static_cast<uint8_t>(R[r].red), 0});
            break;
        case SVal::Carried:
            break;
        }
    }
    (void)step;
    return kOk;
}

std::string describe(const LoweredRegion& r) {
    std::ostringstream os;
    const ScanParams& p = r.params;
    static const char* kOps[] = {"==", "!=", "<", "<=", ">", ">="};
    static const char* kRed[] = {"sum", "count", "min", "max"};
    static const char* kAcc[] = {"none", "add", "sub", "addf", "min", "max", "tadd"};
    os << (r.fast_path ? "fast" : "loop") << " dtype=" << p.dtype << " cols=" << p.ncols << " off0=" << p.off0
       << " groups=" << p.ngroups << " data=" << p.ndata;
    for (int c = 0; c < p.ncols; ++c) os << " c" << c << "=seg" << r.seg_of_col[c];
    for (int a = 0; a < p.natoms; ++a)
        os << " a" << a << "=(c" << int(p.atom[a].col) << kOps[p.atom[a].op % 6] << std::hex << "0x" << p.atom[a].thr << std::dec << ")";
    for (int k = 0; k < p.nred; ++k) {
        const Red& d = p.red[k];
        os << " r" << k << "=" << kRed[d.kind % 4] << "/" << kAcc[d.acc % 7] << "[m=" << d.pmask << " a=" << int(d.a.kind)
           << ":" << int(d.a.col) << " b=" << int(d.b.kind) << ":" << int(d.b.col) << "]";
    }
    os << " kernel=" << scan_kernel_name(p);
    return os.str();
}

}  // namespace vx
