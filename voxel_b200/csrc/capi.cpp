// C ABI: engines, instruction encoders, host-side helper objects, errors.
// (Operator entry points live next to their kernels.)
#include <cstdio>
#include <cstring>
#include <string>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <queue>
#include <thread>
#include <vector>

#include "engine.h"
#include "voxel_c.h"
#include "vx_runtime.h"

using vx::Engine;

namespace {

Engine* E(void* e) { return static_cast<Engine*>(e); }
const Engine* E(const void* e) { return static_cast<const Engine*>(e); }

double as_f64(uint64_t b) { double d; std::memcpy(&d, &b, 8); return d; }
uint64_t f64_bits(double d) { uint64_t b; std::memcpy(&b, &d, 8); return b; }

// Instruction::Encode (include/voxel/bytecode/instruction.hpp:65-72)
uint32_t enc(uint8_t op, uint8_t rd, uint8_t ra, uint8_t rb, uint16_t imm) {
    return static_cast<uint32_t>(op) | ((static_cast<uint32_t>(rd) & 0xF) << 8) |
           ((static_cast<uint32_t>(ra) & 0xF) << 12) | ((static_cast<uint32_t>(rb) & 0xF) << 16) |
           ((static_cast<uint32_t>(imm) & 0xFFF) << 20);
}

// Validity bitmap with 1 = null (the reference's voxel::NullBitmap semantics
// as exposed by voxel_null_*; bindings/voxel_c.cpp:150-164).
struct NullBits {
    std::vector<uint64_t> w;
    size_t n;
    explicit NullBits(size_t count) : w((count + 63) / 64, 0), n(count) {}
};

// Host worker pool behind voxel_pool_* (util/thread.hpp:22-110 in the reference).
class Pool {
public:
    explicit Pool(uint32_t n) {
        if (n == 0) n = std::thread::hardware_concurrency();
        if (n == 0) n = 1;
        for (uint32_t i = 0; i < n; ++i) th_.emplace_back([this] { loop(); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    void wait_all() {
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [this] { return q_.empty() && active_ == 0; });
    }
    size_t size() const { return th_.size(); }

private:
    void loop() {
        for (;;) {
            std::function<void()> f;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [this] { return stop_ || !q_.empty(); });
                if (stop_ && q_.empty()) return;
                f = std::move(q_.front());
                q_.pop();
                ++active_;
            }
            f();
            {
                std::lock_guard<std::mutex> lk(mu_);
                --active_;
            }
            done_cv_.notify_all();
        }
    }
    std::vector<std::thread> th_;
    std::queue<std::function<void()>> q_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    int active_ = 0;
    bool stop_ = false;
};

}  // namespace

extern "C" {

// ---- engines ------------------------------------------------------------------

void* voxel_engine_create(int dtype) {
    if (dtype < 0 || dtype > 5) {
        vx::set_error(vx::kErrInvalidArg, "unknown element type %d", dtype);
        return nullptr;
    }
    return new Engine(dtype);
}
void* voxel_engine_create_f64(void) { return new Engine(vx::F64); }
void* voxel_engine_create_f32(void) { return new Engine(vx::F32); }
void* voxel_engine_create_i64(void) { return new Engine(vx::I64); }
void* voxel_engine_create_i32(void) { return new Engine(vx::I32); }
void* voxel_engine_create_u64(void) { return new Engine(vx::U64); }
void* voxel_engine_create_u32(void) { return new Engine(vx::U32); }
void voxel_engine_destroy(void* e) { delete E(e); }
void voxel_engine_destroy_i64(void* e) { delete E(e); }
int voxel_engine_dtype(const void* e) { return E(e)->dtype(); }
size_t voxel_engine_k_lanes(void) { return vx::dtype_lanes(vx::F64); }
size_t voxel_engine_k_lanes_of(const void* e) { return vx::dtype_lanes(E(e)->dtype()); }

size_t voxel_engine_add_segment(void* e, const double* d, size_t n) { return E(e)->add_segment(d, n); }
size_t voxel_engine_add_segment_i64(void* e, const int64_t* d, size_t n) { return E(e)->add_segment(d, n); }
size_t voxel_engine_add_segment_f32(void* e, const float* d, size_t n) { return E(e)->add_segment(d, n); }
size_t voxel_engine_add_segment_i32(void* e, const int32_t* d, size_t n) { return E(e)->add_segment(d, n); }
size_t voxel_engine_add_segment_u32(void* e, const uint32_t* d, size_t n) { return E(e)->add_segment(d, n); }
size_t voxel_engine_add_segment_u64(void* e, const uint64_t* d, size_t n) { return E(e)->add_segment(d, n); }
size_t voxel_engine_add_segment_device(void* e, const void* d, size_t n) { return E(e)->add_segment_device(d, n); }

void voxel_engine_load_program(void* e, const uint32_t* c, size_t n) { E(e)->load_program(c, n); }
void voxel_engine_load_program_i64(void* e, const uint32_t* c, size_t n) { E(e)->load_program(c, n); }

void voxel_engine_run(void* e) { E(e)->run(); }
void voxel_engine_run_i64(void* e) { E(e)->run(); }
int voxel_engine_run_status(void* e) { return E(e)->run(); }
void voxel_engine_run_parallel(void* e, size_t seg, uint32_t threads, uint8_t reg) {
    E(e)->run_parallel(seg, threads, reg);
}
int voxel_engine_run_parallel_status(void* e, size_t seg, uint32_t threads, uint8_t reg) {
    return E(e)->run_parallel(seg, threads, reg);
}

void voxel_engine_set_scalar(void* e, size_t r, uint64_t v) { E(e)->reg(r) = v; }
uint64_t voxel_engine_get_scalar(void* e, size_t r) { return E(e)->reg(r); }
void voxel_engine_set_scalar_f64(void* e, size_t r, double v) { E(e)->reg(r) = f64_bits(v); }
double voxel_engine_get_scalar_f64(void* e, size_t r) { return as_f64(E(e)->reg(r)); }
void voxel_engine_set_scalar_i64(void* e, size_t r, uint64_t v) { E(e)->reg(r) = v; }
uint64_t voxel_engine_get_scalar_i64(void* e, size_t r) { return E(e)->reg(r); }

size_t voxel_engine_explain(void* e, char* buf, size_t cap) {
    const std::string& s = E(e)->explain();
    if (buf && cap) {
        size_t n = s.size() < cap - 1 ? s.size() : cap - 1;
        std::memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return s.size();
}
void voxel_engine_reset(void* e) { E(e)->reset(); }
int voxel_engine_plan(void* e) { return E(e)->plan(); }
double voxel_engine_last_device_ms(const void* e) { return E(e)->last_device_ms(); }

// ---- JIT entry (reference bindings/voxel_c.cpp:80-101) --------------------------
// The reference compiles the fused loop to x86; here the same program is lowered
// and launched as one kernel over the column, with the registers jit_run sets.
double voxel_jit_run(const uint32_t* code, size_t code_len, const double* data, size_t data_len,
                     double threshold) {
    Engine e(vx::F64);
    e.add_segment(data, data_len);
    e.reg(0) = 0;
    e.reg(1) = 0;
    e.reg(2) = data_len;
    e.reg(3) = f64_bits(threshold);
    e.load_program(code, code_len);
    if (e.run() != vx::kOk) return 0.0;
    return as_f64(e.reg(0));
}

// JIT compile (reference bindings/voxel_bindings.cpp:329-340 compiles the
// fused loop to x86 and reports its code size): here "compiled" means the
// program lowers, with the registers jit_run sets, onto one fused GPU kernel
// schedule.  No device work: the lowering is host code.  *schedule_bytes gets
// the size of the lowered schedule (the kernel parameter block).
int voxel_jit_compile(const uint32_t* code, size_t code_len, size_t* schedule_bytes, char* kernel, size_t cap) {
    vx::clear_error();
    static const double probe[64] = {0.0};  // any column: the lowering reads counts, not values
    Engine e(vx::F64);
    e.add_segment(probe, 64);
    e.reg(0) = 0;
    e.reg(1) = 0;
    e.reg(2) = 64;
    e.reg(3) = f64_bits(0.0);
    e.load_program(code, code_len);
    const int st = e.plan();
    if (st) return st;
    if (schedule_bytes) *schedule_bytes = sizeof(vx::ScanParams);
    if (kernel && cap) {
        const std::string& ex = e.explain();
        const size_t k = ex.find("kernel=");
        std::string name = k == std::string::npos ? "" : ex.substr(k + 7);
        while (!name.empty() && (name.back() == '\n' || name.back() == ' ')) name.pop_back();
        const size_t sp = name.find_first_of(" \n");
        if (sp != std::string::npos) name = name.substr(0, sp);
        std::snprintf(kernel, cap, "%s", name.c_str());
    }
    return vx::kOk;
}

// ---- instruction encoders (reference bindings/voxel_c.cpp:106-145) -------------
uint32_t voxel_instr_vload(uint8_t vd, uint8_t ra, uint8_t seg, uint8_t count) {
    return enc(0x70, vd, ra, 0, static_cast<uint16_t>(((seg & 0xF) << 8) | count));
}
uint32_t voxel_instr_vfilter_gt(uint8_t vd, uint8_t va, uint8_t rb) { return enc(0xC5, vd, va, rb, 0); }
uint32_t voxel_instr_vfilter_ge(uint8_t vd, uint8_t va, uint8_t rb) { return enc(0xC6, vd, va, rb, 0); }
uint32_t voxel_instr_vfilter_lt(uint8_t vd, uint8_t va, uint8_t rb) { return enc(0xC3, vd, va, rb, 0); }
uint32_t voxel_instr_vfilter_le(uint8_t vd, uint8_t va, uint8_t rb) { return enc(0xC4, vd, va, rb, 0); }
uint32_t voxel_instr_vsum(uint8_t rd, uint8_t va) { return enc(0xD0, rd, va, 0, 0); }
uint32_t voxel_instr_vred_min(uint8_t rd, uint8_t va) { return enc(0xD5, rd, va, 0, 0); }
uint32_t voxel_instr_vred_max(uint8_t rd, uint8_t va) { return enc(0xD6, rd, va, 0, 0); }
uint32_t voxel_instr_vcount(uint8_t rd, uint8_t va) { return enc(0xD7, rd, va, 0, 0); }
uint32_t voxel_instr_addf(uint8_t rd, uint8_t ra, uint8_t rb) { return enc(0x2A, rd, ra, rb, 0); }
uint32_t voxel_instr_add(uint8_t rd, uint8_t ra, uint8_t rb) { return enc(0x20, rd, ra, rb, 0); }
uint32_t voxel_instr_sub(uint8_t rd, uint8_t ra, uint8_t rb) { return enc(0x21, rd, ra, rb, 0); }
uint32_t voxel_instr_mul(uint8_t rd, uint8_t ra, uint8_t rb) { return enc(0x22, rd, ra, rb, 0); }
uint32_t voxel_instr_mov(uint8_t rd, int16_t imm) { return enc(0x10, rd, 0, 0, static_cast<uint16_t>(imm)); }
uint32_t voxel_instr_movr(uint8_t rd, uint8_t ra) { return enc(0x11, rd, ra, 0, 0); }
uint32_t voxel_instr_cmp(uint8_t ra, uint8_t rb) { return enc(0x40, 0, ra, rb, 0); }
uint32_t voxel_instr_jnz(int16_t off) { return enc(0x52, 0, 0, 0, static_cast<uint16_t>(off)); }
uint32_t voxel_instr_jz(int16_t off) { return enc(0x51, 0, 0, 0, static_cast<uint16_t>(off)); }
uint32_t voxel_instr_jmp(int16_t off) { return enc(0x50, 0, 0, 0, static_cast<uint16_t>(off)); }
uint32_t voxel_instr_halt(void) { return enc(0x01, 0, 0, 0, 0); }

// ---- null bitmap (host object) ---------------------------------------------------
void* voxel_null_create(size_t count) { return new NullBits(count); }
void voxel_null_destroy(void* b) { delete static_cast<NullBits*>(b); }
int voxel_null_is_null(const void* b, size_t row) {
    const NullBits* n = static_cast<const NullBits*>(b);
    if (row >= n->n) return 0;
    return (n->w[row >> 6] >> (row & 63)) & 1;
}
void voxel_null_set_null(void* b, size_t row) {
    NullBits* n = static_cast<NullBits*>(b);
    if (row < n->n) n->w[row >> 6] |= 1ull << (row & 63);
}
void voxel_null_set_valid(void* b, size_t row) {
    NullBits* n = static_cast<NullBits*>(b);
    if (row < n->n) n->w[row >> 6] &= ~(1ull << (row & 63));
}
size_t voxel_null_null_count(const void* b) {
    const NullBits* n = static_cast<const NullBits*>(b);
    size_t c = 0;
    for (uint64_t x : n->w) c += static_cast<size_t>(__builtin_popcountll(x));
    return c;
}
size_t voxel_null_valid_count(const void* b) {
    return static_cast<const NullBits*>(b)->n - voxel_null_null_count(b);
}

// ---- thread pool ---------------------------------------------------------------------
void* voxel_pool_create(uint32_t threads) { return new Pool(threads); }
void voxel_pool_destroy(void* p) { delete static_cast<Pool*>(p); }
void voxel_pool_wait_all(void* p) { static_cast<Pool*>(p)->wait_all(); }
size_t voxel_pool_thread_count(const void* p) { return static_cast<const Pool*>(p)->size(); }

// ---- memory helpers ------------------------------------------------------------------
void* voxel_device_alloc(size_t bytes) {
    vx::clear_error();
    if (vx::ensure_device()) return nullptr;
    return vx::dev_alloc(bytes);
}
void voxel_device_free(void* p) { vx::dev_free(p); }
int voxel_copy_to_device(void* dst, const void* src, size_t bytes, void* stream) {
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : vx::thread_stream();
    int st = vx::h2d(dst, src, bytes, s);
    return st ? st : (stream ? vx::kOk : vx::sync(s));
}
int voxel_copy_to_host(void* dst, const void* src, size_t bytes, void* stream) {
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : vx::thread_stream();
    int st = vx::d2h(dst, src, bytes, s);
    return st ? st : (stream ? vx::kOk : vx::sync(s));
}
int voxel_stream_sync(void* stream) {
    return vx::sync(stream ? static_cast<cudaStream_t>(stream) : vx::thread_stream());
}
int voxel_host_register(void* ptr, size_t bytes) {
    if (vx::ensure_device()) return vx::kErrNoDevice;
    VX_CUDA(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
    return vx::kOk;
}
int voxel_host_unregister(void* ptr) {
    VX_CUDA(cudaHostUnregister(ptr));
    return vx::kOk;
}

// ---- errors --------------------------------------------------------------------------
const char* voxel_last_error(void) { return vx::last_error(); }
int voxel_last_status(void) { return vx::last_status(); }

}  // extern "C"
