// Engine facade behind the voxel_engine_* C ABI.
//
// Mirrors the observable behaviour of the reference Engine<T>
// (include/voxel/exec/engine.hpp): segments are borrowed caller buffers read at
// run time (AddSegment, 35-38), programs are copied at load (LoadProgram,
// 43-48), and the scalar register file is the program's interface.  Running a
// program works differently: the fused filter+sum pattern (DetectFastPath,
// 84-107) and every loop whose body touches column data are lowered to one
// fused CUDA launch each (lower.cpp / scan.cu); the scalar glue around them
// (MOV / ADD / CMP / branches / VSPLAT of constants) is stepped on the host with
// the reference's register and flag semantics.  Data-dependent work never runs
// on the CPU: a region the lowering cannot express fails with
// VOXEL_EUNSUPPORTED.
#include "engine.h"

#include <cmath>
#include <cstring>
#include <thread>

#include "scan.h"

namespace vx {

namespace {

constexpr uint32_t F_ZERO = 1u, F_CARRY = 2u, F_SIGN = 4u, F_OVF = 8u, F_NAN = 32u;

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

uint64_t scalar_as_t(int dt, uint64_t reg) {
    switch (dt) {
    case F32: return f32_bits(static_cast<float>(as_f64(reg)));
    case I32: case U32: return static_cast<uint32_t>(reg);
    default: return reg;
    }
}
uint64_t set_scalar_t(int dt, uint64_t bits) {
    switch (dt) {
    case F32: return f64_bits(static_cast<double>(as_f32(bits)));
    case I32: return static_cast<uint64_t>(static_cast<int64_t>(static_cast<int32_t>(static_cast<uint32_t>(bits))));
    case U32: return static_cast<uint32_t>(bits);
    default: return bits;
    }
}
bool t_less(int dt, uint64_t a, uint64_t b) {
    switch (dt) {
    case F64: return as_f64(a) < as_f64(b);
    case F32: return as_f32(a) < as_f32(b);
    case I64: return static_cast<int64_t>(a) < static_cast<int64_t>(b);
    case I32: return static_cast<int32_t>(static_cast<uint32_t>(a)) < static_cast<int32_t>(static_cast<uint32_t>(b));
    case U64: return a < b;
    default: return static_cast<uint32_t>(a) < static_cast<uint32_t>(b);
    }
}

void arith_flags(uint32_t& fl, int64_t r) {  // registers.hpp:96-101
    fl &= ~(F_ZERO | F_SIGN | F_CARRY | F_OVF);
    if (r == 0) fl |= F_ZERO;
    if (r < 0) fl |= F_SIGN;
}
void float_flags(uint32_t& fl, double r) {  // registers.hpp:103-110
    fl &= ~(F_NAN | 64u | F_OVF | 128u | 256u | 512u);
    if (r == 0.0) { fl |= F_ZERO; fl &= ~F_SIGN; }
    if (r < 0.0) fl |= F_SIGN;
    if (std::isnan(r)) fl |= F_NAN;
}

bool is_vector_data_op(uint8_t op) {
    return op == 0x70 || (op >= 0xA0 && op <= 0xA5) || (op >= 0xB0 && op <= 0xB4) ||
           (op >= 0xC0 && op <= 0xC7) || op == 0xD0 || (op >= 0xD5 && op <= 0xD7);
}

}  // namespace

Engine::Engine(int dtype) : dtype_(dtype) {}

Engine::~Engine() {
    drop_uploads();
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (host_result_) cudaFreeHost(host_result_);
    if (stream_) cudaStreamDestroy(stream_);
}

size_t Engine::add_segment(const void* host, size_t count) {
    SegmentRef s;
    s.host = host;
    s.count = count;
    segs_.push_back(s);
    return segs_.size() - 1;
}

size_t Engine::add_segment_device(const void* dev, size_t count) {
    SegmentRef s;
    s.device = dev;
    s.count = count;
    segs_.push_back(s);
    return segs_.size() - 1;
}

void Engine::load_program(const uint32_t* code, size_t len) {
    code_.assign(code, code + len);
    pc_ = 0;
    running_ = true;
    fast_ = detect_fast_path(code_);
    // loop structure: a backward branch at b with target t makes [t, b] a loop
    loop_end_.assign(code_.size(), SIZE_MAX);
    for (size_t b = 0; b < code_.size(); ++b) {
        uint8_t op = code_[b] & 0xFF;
        if (op >= 0x51 && op <= 0x5C && op != 0x5D) {
            int64_t t = static_cast<int64_t>(b) + f_simm(code_[b]);
            if (t >= 0 && t <= static_cast<int64_t>(b) && loop_end_[t] == SIZE_MAX) loop_end_[t] = b;
        }
    }
}

void Engine::reset() {
    std::memset(R_, 0, sizeof R_);
    for (auto& v : V_) v = HostVec{};
    flags_ = 0;
    code_.clear();
    loop_end_.clear();
    segs_.clear();
    pc_ = 0;
    running_ = false;
    for (auto& a : agg_) a = AggSlot{};
}

void Engine::drop_uploads() {
    uploads_.clear();
    dev_of_seg_.clear();
}

int Engine::ensure_device_data(int seg, const void** dptr) {
    if (seg < 0 || static_cast<size_t>(seg) >= segs_.size()) {
        set_error(kErrInvalidArg, "segment %d does not exist", seg);
        return kErrInvalidArg;
    }
    if (dev_of_seg_.size() < segs_.size()) dev_of_seg_.resize(segs_.size(), nullptr);
    if (dev_of_seg_[seg]) { *dptr = dev_of_seg_[seg]; return kOk; }
    const SegmentRef& s = segs_[seg];
    if (s.device) {
        dev_of_seg_[seg] = s.device;
    } else {
        size_t bytes = s.count * dtype_size(dtype_);
        DevBuf b(bytes);
        if (!b.ok(bytes)) return kErrOutOfMemory;
        int st = h2d(b.p, s.host, bytes, stream_);
        if (st) return st;
        dev_of_seg_[seg] = b.p;
        uploads_.push_back(std::move(b));
    }
    *dptr = dev_of_seg_[seg];
    return kOk;
}

int Engine::run_region(LoweredRegion& lr) {
    ScanParams& p = lr.params;
    if (dry_) {
        if (capture_) capture_->push_back(lr);
        for (const RegWrite& w : lr.writes) R_[w.reg] = w.kind == RegWrite::kValue ? w.value : 0;
        if (lr.set_flags) arith_flags(flags_, lr.flag_value);
        explain_ += describe(lr);
        explain_ += "\n";
        return kOk;
    }
    for (int c = 0; c < p.ncols; ++c) {
        const void* d = nullptr;
        int st = ensure_device_data(lr.seg_of_col[c], &d);
        if (st) return st;
        p.col[c] = d;
    }
    if (!scratch_.p) {
        scratch_ = DevBuf(scan_scratch_bytes());
        result_ = DevBuf(sizeof(ScanResult));
        if (!scratch_.p || !result_.p) return kErrOutOfMemory;
        int st = scan_scratch_init(scratch_.p, stream_);
        if (st) return st;
    }
    VX_CUDA(cudaEventRecord(ev0_, stream_));
    int st = launch_scan(p, result_.as<ScanResult>(), scratch_.p, stream_);
    if (st) return st;
    VX_CUDA(cudaEventRecord(ev1_, stream_));
    st = d2h(host_result_, result_.p, sizeof(ScanResult), stream_);
    if (st) return st;
    st = sync(stream_);
    if (st) return st;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    last_ms_ += ms;
    const ScanResult& res = *static_cast<const ScanResult*>(host_result_);
    for (const RegWrite& w : lr.writes) {
        switch (w.kind) {
        case RegWrite::kAcc: R_[w.reg] = res.acc[w.red]; break;
        case RegWrite::kLast: if (p.ngroups > 0) R_[w.reg] = res.last[w.red]; break;
        case RegWrite::kValue: R_[w.reg] = w.value; break;
        }
    }
    if (lr.set_flags) arith_flags(flags_, lr.flag_value);
    explain_ += describe(lr);
    explain_ += "\n";
    return kOk;
}

int Engine::exec_agg(uint32_t raw, int kind) {
    // HandleAggregate (engine.hpp:499-569): rd = slot and result register,
    // ra = segment id, rb = start row register, imm = row count (0 = all)
    unsigned rd = f_rd(raw), seg = f_ra(raw), rb = f_rb(raw), imm = f_imm(raw);
    if (seg >= segs_.size()) return kOk;  // the reference skips the instruction
    uint64_t start = static_cast<uint64_t>(static_cast<int64_t>(R_[rb]));
    uint64_t count = imm == 0 ? 0xFFFFFFFFull : (imm & 0xFFF);
    uint64_t end = start + count;
    if (end > segs_[seg].count) end = segs_[seg].count;
    if (dry_) {
        R_[rd] = 0;
        return kOk;
    }
    AggSlot& s = agg_[rd & 0xF];
    int dt = dtype_;
    uint64_t init_bits = 0;
    if (kind == 3 || kind == 4) {
        if (!s.init) {
            uint64_t v;
            switch (dt) {
            case F64: v = f64_bits(kind == 3 ? 1.7976931348623157e308 : -1.7976931348623157e308); break;
            case F32: v = f32_bits(kind == 3 ? 3.40282347e38f : -3.40282347e38f); break;
            case I64: v = kind == 3 ? 0x7FFFFFFFFFFFFFFFull : 0x8000000000000000ull; break;
            case I32: v = kind == 3 ? 0x7FFFFFFFull : 0x80000000ull; break;
            case U64: v = kind == 3 ? ~0ull : 0ull; break;
            default: v = kind == 3 ? 0xFFFFFFFFull : 0ull; break;
            }
            if (kind == 3) s.min_bits = v; else s.max_bits = v;
            s.init = true;
        }
        init_bits = kind == 3 ? s.min_bits : s.max_bits;
    } else if (!s.init) {
        s.count = 0;
        s.sum_f64 = 0;
        s.sum_i64 = 0;
        s.init = true;
    }
    if (end > start) {
        const void* d = nullptr;
        int st = ensure_device_data(static_cast<int>(seg), &d);
        if (st) return st;
        if (!scratch_.p) {
            scratch_ = DevBuf(scan_scratch_bytes());
            result_ = DevBuf(sizeof(ScanResult));
            if (!scratch_.p || !result_.p) return kErrOutOfMemory;
            st = scan_scratch_init(scratch_.p, stream_);
            if (st) return st;
        }
        st = launch_segment_agg(dt, d, start, end, kind, init_bits, result_.as<uint64_t>(), scratch_.p, stream_);
        if (st) return st;
        st = d2h(host_result_, result_.p, 3 * sizeof(uint64_t), stream_);
        if (st) return st;
        st = sync(stream_);
        if (st) return st;
        const uint64_t* o = static_cast<const uint64_t*>(host_result_);
        switch (kind) {
        case 0: s.count += o[0]; break;
        case 1:
            if (dtype_is_float(dt)) s.sum_f64 += as_f64(o[1]) + as_f64(o[2]);
            else s.sum_i64 = static_cast<int64_t>(static_cast<uint64_t>(s.sum_i64) + o[0]);
            break;
        case 3: s.min_bits = o[0]; break;
        case 4: s.max_bits = o[0]; break;
        }
    }
    switch (kind) {
    case 0: R_[rd] = s.count; break;
    case 1:
        if (dt == F64) R_[rd] = f64_bits(s.sum_f64);
        else if (dt == F32) R_[rd] = f64_bits(static_cast<double>(static_cast<float>(s.sum_f64)));
        else R_[rd] = static_cast<uint64_t>(s.sum_i64);
        break;
    case 3: R_[rd] = set_scalar_t(dt, s.min_bits); break;
    case 4: R_[rd] = set_scalar_t(dt, s.max_bits); break;
    }
    return kOk;
}

int Engine::run() {
    clear_error();
    int st = ensure_device();
    if (st) return st;
    if (!stream_) {
        VX_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        VX_CUDA(cudaEventCreate(&ev0_));
        VX_CUDA(cudaEventCreate(&ev1_));
        VX_CUDA(cudaHostAlloc(&host_result_, sizeof(ScanResult), cudaHostAllocDefault));
    }
    explain_.clear();
    last_ms_ = 0.0;
    drop_uploads();
    std::vector<uint64_t> counts(segs_.size());
    for (size_t i = 0; i < segs_.size(); ++i) counts[i] = segs_[i].count;

    if (fast_.ok) {  // Run(): RunFastPath whenever the pattern was detected (engine.hpp:70-74)
        LoweredRegion lr;
        st = lower_fast_path(fast_, dtype_, R_, counts, lr);
        if (st) {
            set_error(st, "fast-path segment %d does not exist", fast_.seg);
            drop_uploads();
            return st;
        }
        st = run_region(lr);
        running_ = false;
        drop_uploads();
        return st;
    }
    st = run_from_pc();
    drop_uploads();
    return st;
}

int Engine::plan() {
    clear_error();
    explain_.clear();
    uint64_t saved[64];
    std::memcpy(saved, R_, sizeof R_);
    size_t pc = pc_;
    bool running = running_;
    uint32_t fl = flags_;
    dry_ = true;
    int st = kOk;
    if (fast_.ok) {
        std::vector<uint64_t> counts(segs_.size());
        for (size_t i = 0; i < segs_.size(); ++i) counts[i] = segs_[i].count;
        LoweredRegion lr;
        st = lower_fast_path(fast_, dtype_, R_, counts, lr);
        if (st) set_error(st, "fast-path segment %d does not exist", fast_.seg);
        else st = run_region(lr);
    } else {
        st = run_from_pc();
    }
    dry_ = false;
    std::memcpy(R_, saved, sizeof R_);
    pc_ = pc;
    running_ = running;
    flags_ = fl;
    return st;
}

int Engine::lower_regions(std::vector<LoweredRegion>& out) {
    out.clear();
    capture_ = &out;
    int st = plan();
    capture_ = nullptr;
    return st;
}

int Engine::run_from_pc() {
    std::vector<uint64_t> counts(segs_.size());
    for (size_t i = 0; i < segs_.size(); ++i) counts[i] = segs_[i].count;
    const uint64_t kMaxHostSteps = 1ull << 32;
    uint64_t steps = 0;
    while (pc_ < code_.size()) {
        if (++steps > kMaxHostSteps) {
            set_error(kErrNonTerminating, "program exceeded %llu host steps", (unsigned long long)kMaxHostSteps);
            return kErrNonTerminating;
        }
        // a loop whose body touches column data runs as one fused launch
        if (loop_end_[pc_] != SIZE_MAX) {
            size_t b = loop_end_[pc_];
            bool vec = false;
            for (size_t i = pc_; i <= b; ++i) vec |= is_vector_data_op(code_[i] & 0xFF);
            if (vec) {
                LoweredRegion lr;
                std::string why;
                int st = lower_region(code_, pc_, b, dtype_, R_, V_, counts, lr, why);
                if (st) {
                    set_error(st, "cannot lower loop at %zu: %s", pc_, why.c_str());
                    return st;
                }
                st = run_region(lr);
                if (st) return st;
                for (size_t i = pc_; i <= b; ++i) {
                    uint8_t op = code_[i] & 0xFF;
                    if (is_vector_data_op(op) || op == 0x78) V_[f_rd(code_[i])].known = false;
                }
                pc_ = lr.resume_pc;
                continue;
            }
        }
        uint32_t raw = code_[pc_];
        uint8_t op = raw & 0xFF;
        unsigned rd = f_rd(raw), ra = f_ra(raw), rb = f_rb(raw);
        int16_t si = f_simm(raw);
        if (is_vector_data_op(op)) {
            // straight-line vector work outside a loop: lower the run that starts here
            bool data = false;
            for (size_t i = pc_; i < code_.size(); ++i) {
                uint8_t o = code_[i] & 0xFF;
                if (o == 0x01 || (o >= 0x50 && o <= 0x5F)) break;
                if (o == 0x70) data = true;
            }
            if (data) {
                LoweredRegion lr;
                std::string why;
                int st = lower_region(code_, pc_, SIZE_MAX, dtype_, R_, V_, counts, lr, why);
                if (st) {
                    set_error(st, "cannot lower vector block at %zu: %s", pc_, why.c_str());
                    return st;
                }
                st = run_region(lr);
                if (st) return st;
                for (size_t i = pc_; i < lr.resume_pc; ++i) {
                    uint8_t o = code_[i] & 0xFF;
                    if (is_vector_data_op(o) || o == 0x78) V_[f_rd(code_[i])].known = false;
                }
                pc_ = lr.resume_pc;
                continue;
            }
            set_error(kErrUnsupportedProgram, "vector instruction 0x%02x at %zu outside a data region", op, pc_);
            return kErrUnsupportedProgram;
        }
        uint64_t* R = R_;
        switch (op) {
        case 0x00: case 0x04: case 0x05: case 0x06: case 0x07: case 0x08: case 0x09: pc_++; break;
        case 0x01: running_ = false; return kOk;  // HALT
        case 0x02: case 0x03: flags_ |= 512u; running_ = false; return kOk;  // TRAP / BREAK
        case 0x10: R[rd] = static_cast<uint64_t>(static_cast<int64_t>(si)); pc_++; break;
        case 0x11: R[rd] = R[ra]; pc_++; break;
        case 0x12: R[rd] = static_cast<uint64_t>(static_cast<int64_t>(R[ra]) + si); pc_++; break;
        case 0x13: R[rd] = static_cast<uint64_t>(static_cast<int64_t>(R[ra]) - si); pc_++; break;
        case 0x14: R[rd] = static_cast<uint64_t>(static_cast<int64_t>(R[ra]) * si); pc_++; break;
        case 0x20: case 0x21: case 0x22: case 0x27: case 0x28: {
            int64_t a = static_cast<int64_t>(R[ra]), b = static_cast<int64_t>(R[rb]), r;
            switch (op) {
            case 0x20: r = static_cast<int64_t>(R[ra] + R[rb]); break;
            case 0x21: r = static_cast<int64_t>(R[ra] - R[rb]); break;
            case 0x22: r = static_cast<int64_t>(R[ra] * R[rb]); break;
            case 0x27: r = a < b ? a : b; break;
            default: r = a > b ? a : b; break;
            }
            R[rd] = static_cast<uint64_t>(r);
            arith_flags(flags_, r);
            pc_++;
            break;
        }
        case 0x23: case 0x24: {  // DIV / MOD
            int64_t b = static_cast<int64_t>(R[rb]);
            if (b == 0) { flags_ |= 256u; running_ = false; return kOk; }
            int64_t a = static_cast<int64_t>(R[ra]);
            int64_t r = op == 0x23 ? a / b : a % b;
            R[rd] = static_cast<uint64_t>(r);
            arith_flags(flags_, r);
            pc_++;
            break;
        }
        case 0x2A: case 0x2B: case 0x2C: {
            double a = as_f64(R[ra]), b = as_f64(R[rb]);
            double r = op == 0x2A ? a + b : op == 0x2B ? a - b : a * b;
            R[rd] = f64_bits(r);
            float_flags(flags_, r);
            pc_++;
            break;
        }
        case 0x2D: {
            double b = as_f64(R[rb]);
            if (b == 0.0) { flags_ |= 256u; running_ = false; return kOk; }
            double r = as_f64(R[ra]) / b;
            R[rd] = f64_bits(r);
            float_flags(flags_, r);
            pc_++;
            break;
        }
        case 0x30: R[rd] = R[ra] & R[rb]; pc_++; break;
        case 0x31: R[rd] = R[ra] | R[rb]; pc_++; break;
        case 0x32: R[rd] = R[ra] ^ R[rb]; pc_++; break;
        case 0x40: arith_flags(flags_, static_cast<int64_t>(R[ra] - R[rb])); pc_++; break;
        case 0x50: pc_ += si; break;
        case 0x51: if (flags_ & F_ZERO) pc_ += si; else pc_++; break;
        case 0x52: if (!(flags_ & F_ZERO)) pc_ += si; else pc_++; break;
        case 0x53: case 0x59: if (flags_ & F_SIGN) pc_ += si; else pc_++; break;
        case 0x54: if (!(flags_ & F_SIGN)) pc_ += si; else pc_++; break;
        case 0x5A: if ((flags_ & F_ZERO) || (flags_ & F_SIGN)) pc_ += si; else pc_++; break;
        case 0x5B: if (!(flags_ & F_ZERO) && !(flags_ & F_SIGN)) pc_ += si; else pc_++; break;
        case 0x5C: if ((flags_ & F_ZERO) || !(flags_ & F_SIGN)) pc_ += si; else pc_++; break;
        case 0x78: {  // VSPLAT of a known scalar
            uint64_t v = scalar_as_t(dtype_, R[ra]);
            size_t es = dtype_size(dtype_);
            for (size_t l = 0; l < 32 / es; ++l) std::memcpy(V_[rd].bytes + l * es, &v, es);
            V_[rd].known = true;
            pc_++;
            break;
        }
        case 0xE0: case 0xE1: case 0xE3: case 0xE4: {
            int st = exec_agg(raw, op - 0xE0);
            if (st) return st;
            pc_++;
            break;
        }
        default:
            set_error(kErrUnsupportedProgram, "opcode 0x%02x at %zu is outside the backend's set", op, pc_);
            return kErrUnsupportedProgram;
        }
    }
    return kOk;
}

int Engine::run_parallel(size_t seg_id, uint32_t threads, uint8_t result_reg) {
    // Engine<T>::RunParallel (engine.hpp:143-175): the segment is cut into
    // `threads` chunks, the program runs on each chunk with a copy of the
    // registers, and the chunks' result registers are added in T.
    clear_error();
    if (threads == 0) threads = std::thread::hardware_concurrency();
    if (threads < 1) threads = 1;
    if (segs_.empty() || seg_id >= segs_.size()) return kOk;
    SegmentRef whole = segs_[seg_id];
    uint64_t total = whole.count;
    uint64_t chunk = (total + threads - 1) / threads;
    size_t es = dtype_size(dtype_);
    uint64_t combined = 0;
    double combined_f = 0.0;
    std::vector<uint32_t> code = code_;
    for (uint32_t t = 0; t < threads; ++t) {
        uint64_t start = static_cast<uint64_t>(t) * chunk;
        if (start >= total) continue;
        uint64_t count = start + chunk > total ? total - start : chunk;
        if (count == 0) continue;
        Engine w(dtype_);
        if (whole.device) w.add_segment_device(static_cast<const char*>(whole.device) + start * es, count);
        else w.add_segment(static_cast<const char*>(whole.host) + start * es, count);
        w.load_program(code.data(), code.size());
        std::memcpy(w.R_, R_, sizeof R_);
        int st = w.run();
        if (st) return st;
        uint64_t r = w.R_[result_reg & 63];
        uint64_t tv = scalar_as_t(dtype_, r);
        switch (dtype_) {
        case F64: combined_f += as_f64(tv); break;
        case F32: combined_f = static_cast<double>(static_cast<float>(combined_f) + as_f32(tv)); break;
        default: combined += tv; break;
        }
    }
    if (dtype_ == F64) R_[result_reg & 63] = f64_bits(combined_f);
    else if (dtype_ == F32) R_[result_reg & 63] = f64_bits(combined_f);
    else R_[result_reg & 63] = set_scalar_t(dtype_, combined);
    return kOk;
}

}  // namespace vx
