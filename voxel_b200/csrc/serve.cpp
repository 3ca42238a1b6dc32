// Serving loop: continuous batching of filter/aggregate programs plus group-by
// and hash-join requests over device-resident columns.
//
// Clients submit requests from any thread; each gets an id and a timestamp.
// Two workers, each with its own CUDA stream, drain the arrival queues in
// arrival order:
//   - the program worker takes every queued program whose working memory fits
//     the free part of the budget (up to max_batch) and runs them as one
//     launch of the batched executor; programs that arrive while a batch runs
//     form the next batch, prepared on the host while the device works on the
//     previous one (two batches in flight, alternating streams);
//   - operator workers (kOpWorkers = 8 threads, one stream each) run group-by
//     and join requests, several at once.
// Both workers admit work by device-memory footprint: a request reserves its
// estimated working memory from a shared budget before it starts and returns
// it when it completes, so a burst never oversubscribes HBM.  The workers run
// concurrently on the device.  Latency = completion time - submission time;
// percentiles are taken over completed requests.
//
// No counterpart in the reference (its closest piece, the streaming engine of
// include/voxel/exec/streaming.hpp, is not on this path).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.h"
#include "join.h"
#include "voxel_c.h"
#include "vx_runtime.h"

namespace vx {

namespace {

using Clock = std::chrono::steady_clock;

enum Kind { kProgram = 0, kGroupBy = 1, kJoin = 2 };

struct Request {
    uint64_t id = 0;
    int kind = kProgram;
    size_t footprint = 0;
    Clock::time_point t_submit, t_start, t_done;  // t_start: admitted to a worker
    int status = kOk;
    bool done = false;
    std::string error;
    // program
    int dtype = 0;
    std::vector<uint32_t> code;
    uint64_t regs_in[64] = {0};
    const void* d_col = nullptr;
    size_t count = 0;
    int want_sel = 0;
    size_t sel_cap = 0;
    uint32_t* d_sel = nullptr;
    uint64_t regs_out[64] = {0};
    uint64_t sel_count = 0;
    int overflow = 0;
    // group-by (keys u32, values f64 on the device; groups sorted by key to host arrays)
    const uint32_t* g_keys = nullptr;
    const double* g_vals = nullptr;
    size_t g_n = 0, g_expected = 0, g_cap = 0;
    uint32_t* o_keys = nullptr;
    double *o_sum = nullptr, *o_min = nullptr, *o_max = nullptr;
    uint64_t* o_count = nullptr;
    uint64_t groups = 0;
    // join (device sides and pair buffers)
    const int64_t* j_build = nullptr;
    const uint64_t* j_payload = nullptr;
    size_t j_nb = 0;
    const int64_t* j_probe = nullptr;
    size_t j_np = 0;
    uint32_t *j_left = nullptr, *j_right = nullptr;
    size_t j_cap = 0;
    uint64_t j_pairs = 0, j_sum = 0, j_all = 0;
};

// working memory a request needs on the device while it runs (estimates)
size_t program_footprint(size_t count) {
    // per work item (4096 groups of >= 4 rows): a 96-byte partial + status
    return 4096 + (count / 16384 + 1) * 112;
}
size_t groupby_footprint(size_t expected, size_t n) {
    size_t cap = 16;
    while (cap < 2 * expected) cap <<= 1;
    return cap * 56 + (expected + 1) * 64 + (n > 0 ? 64 : 0) + 4096;
}
size_t join_footprint(size_t nb, size_t np) { return nb * 64 + probe_scratch_bytes(np) + 4096; }

}  // namespace

class Server {
public:
    Server(size_t budget, uint32_t max_batch) : budget_(budget), max_batch_(max_batch ? max_batch : 4096) {
        prog_thread_ = std::thread([this] { program_loop(); });
        for (int i = 0; i < kOpWorkers; ++i) op_threads_.emplace_back([this] { operator_loop(); });
    }

    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_work_.notify_all();
        cv_done_.notify_all();
        prog_thread_.join();
        for (auto& t : op_threads_) t.join();
    }

    uint64_t submit(std::unique_ptr<Request> r) {
        if (r->footprint > budget_) {
            set_error(kErrCapacity, "request needs %zu bytes of working memory, the budget is %zu", r->footprint,
                      budget_);
            return 0;
        }
        std::lock_guard<std::mutex> lk(mu_);
        r->id = ++next_id_;
        r->t_submit = Clock::now();
        uint64_t id = r->id;
        if (r->kind == kProgram) prog_q_.push_back(r.get());
        else op_q_.push_back(r.get());
        reqs_.emplace(id, std::move(r));
        cv_work_.notify_all();
        return id;
    }

    int wait(uint64_t id, double timeout_s) {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = reqs_.find(id);
        if (it == reqs_.end()) {
            set_error(kErrInvalidArg, "unknown request id %llu", static_cast<unsigned long long>(id));
            return kErrInvalidArg;
        }
        Request* r = it->second.get();
        auto deadline = Clock::now() + std::chrono::duration<double>(timeout_s);
        while (!r->done) {
            if (cv_done_.wait_until(lk, deadline) == std::cv_status::timeout && !r->done) {
                set_error(kErrDeviceTimeout, "request %llu not complete after %.3f s",
                          static_cast<unsigned long long>(id), timeout_s);
                return kErrDeviceTimeout;
            }
        }
        if (r->status) set_error(r->status, "%s", r->error.c_str());
        return r->status;
    }

    // copies the result out and forgets the request
    int result(uint64_t id, uint64_t* regs64, uint64_t* count, uint64_t* aux, double* latency_ms) {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = reqs_.find(id);
        if (it == reqs_.end() || !it->second->done) {
            set_error(kErrInvalidArg, "request %llu unknown or not complete", static_cast<unsigned long long>(id));
            return kErrInvalidArg;
        }
        Request* r = it->second.get();
        int st = r->status;
        if (r->kind == kProgram) {
            if (regs64) std::memcpy(regs64, r->regs_out, sizeof(r->regs_out));
            if (count) *count = r->sel_count;
            if (aux) *aux = static_cast<uint64_t>(r->overflow);
        } else if (r->kind == kGroupBy) {
            if (count) *count = r->groups;
            if (aux) *aux = 0;
        } else {
            if (count) *count = r->j_pairs;
            if (aux) aux[0] = r->j_sum;
        }
        if (latency_ms)
            *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
        if (st) set_error(st, "%s", r->error.c_str());
        reqs_.erase(it);
        return st;
    }

    int stats(uint64_t* completed, double* p50, double* p99, double* mean, uint64_t* peak_bytes) {
        std::lock_guard<std::mutex> lk(mu_);
        std::vector<double> v = lat_;
        if (completed) *completed = v.size();
        if (peak_bytes) *peak_bytes = peak_;
        if (v.empty()) {
            if (p50) *p50 = 0;
            if (p99) *p99 = 0;
            if (mean) *mean = 0;
            return kOk;
        }
        std::sort(v.begin(), v.end());
        auto pct = [&](double q) { return v[std::min(v.size() - 1, static_cast<size_t>(q * (v.size() - 1) + 0.5))]; };
        if (p50) *p50 = pct(0.50);
        if (p99) *p99 = pct(0.99);
        if (mean) {
            double s = 0;
            for (double x : v) s += x;
            *mean = s / v.size();
        }
        return kOk;
    }

    // mean time in the arrival queue and in service, per request kind
    int breakdown(int kind, double* queue_ms, double* service_ms, uint64_t* n) {
        if (kind < 0 || kind > 2) {
            set_error(kErrInvalidArg, "request kind %d outside 0..2", kind);
            return kErrInvalidArg;
        }
        std::lock_guard<std::mutex> lk(mu_);
        const Breakdown& b = by_kind_[kind];
        if (queue_ms) *queue_ms = b.n ? b.queue_ms / b.n : 0.0;
        if (service_ms) *service_ms = b.n ? b.service_ms / b.n : 0.0;
        if (n) *n = b.n;
        return kOk;
    }

    int batch_stats(uint64_t* batches, uint64_t* programs, uint64_t* max_batch, double* build_ms,
                    double* max_build_ms, double* wait_ms) {
        std::lock_guard<std::mutex> lk(mu_);
        if (batches) *batches = bstat_.batches;
        if (programs) *programs = bstat_.programs;
        if (max_batch) *max_batch = bstat_.max_batch;
        if (build_ms) *build_ms = bstat_.build_ms;
        if (max_build_ms) *max_build_ms = bstat_.max_build_ms;
        if (wait_ms) *wait_ms = bstat_.wait_ms;
        return kOk;
    }

    void reset_stats() {
        std::lock_guard<std::mutex> lk(mu_);
        lat_.clear();
        for (auto& b : by_kind_) b = Breakdown{};
        bstat_ = BatchStats{};
        peak_ = in_use_;
    }

private:
    // Takes queued requests (arrival order) whose footprint fits; caller holds mu_.
    std::vector<Request*> admit(std::deque<Request*>& q, size_t max_n) {
        std::vector<Request*> out;
        while (!q.empty() && out.size() < max_n) {
            Request* r = q.front();
            if (in_use_ + r->footprint > budget_) break;  // head of line waits for memory
            in_use_ += r->footprint;
            peak_ = std::max(peak_, in_use_);
            r->t_start = Clock::now();
            out.push_back(r);
            q.pop_front();
        }
        return out;
    }

    void finish(std::vector<Request*>& rs) {
        std::lock_guard<std::mutex> lk(mu_);
        auto now = Clock::now();
        for (Request* r : rs) {
            r->t_done = now;
            r->done = true;
            in_use_ -= r->footprint;
            lat_.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
            Breakdown& b = by_kind_[r->kind];
            b.queue_ms += std::chrono::duration<double, std::milli>(r->t_start - r->t_submit).count();
            b.service_ms += std::chrono::duration<double, std::milli>(r->t_done - r->t_start).count();
            ++b.n;
        }
        cv_done_.notify_all();
        cv_work_.notify_all();  // memory came back: the other worker may admit now
    }

    struct InFlight {
        std::unique_ptr<Batch> batch;
        std::vector<Request*> reqs;
        cudaStream_t stream = nullptr;
    };

    // host time to lower, upload and launch a batch, and its size
    void note_batch(size_t n, Clock::time_point t0) {
        const double ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
        std::lock_guard<std::mutex> lk(mu_);
        ++bstat_.batches;
        bstat_.programs += n;
        bstat_.max_batch = std::max<uint64_t>(bstat_.max_batch, n);
        bstat_.build_ms += ms;
        bstat_.max_build_ms = std::max(bstat_.max_build_ms, ms);
    }

    void complete_batch(InFlight& f) {
        const auto t_wait = Clock::now();
        int st = f.batch->fetch(f.stream);
        {
            const double ms = std::chrono::duration<double, std::milli>(Clock::now() - t_wait).count();
            std::lock_guard<std::mutex> lk(mu_);
            bstat_.wait_ms += ms;
        }
        std::string err = st ? last_error() : "";
        for (size_t i = 0; i < f.reqs.size(); ++i) {
            Request* r = f.reqs[i];
            r->status = st;
            r->error = err;
            if (!st) {
                f.batch->registers(i, r->regs_out);
                r->sel_count = f.batch->out(i).sel_count;
                r->overflow = f.batch->out(i).overflow;
            }
        }
        finish(f.reqs);
        f.batch.reset();
        f.reqs.clear();
    }

    void program_loop() {
        if (ensure_device()) return;
        cudaStream_t streams[2];
        for (auto& s : streams) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        InFlight slot[2];
        int cur = 0;
        for (;;) {
            std::vector<Request*> take;
            {
                std::unique_lock<std::mutex> lk(mu_);
                const bool busy = slot[cur ^ 1].batch != nullptr;
                // with a batch in flight, do not block: finish it instead; when
                // stopping, queued programs still run (waiting for memory if needed)
                while (!busy && (prog_q_.empty() || in_use_ + prog_q_.front()->footprint > budget_)) {
                    if (stop_ && prog_q_.empty()) break;
                    cv_work_.wait(lk);
                }
                if (stop_ && prog_q_.empty() && !busy) break;
                take = admit(prog_q_, max_batch_);
            }
            if (!take.empty()) {
                const auto t_build = Clock::now();
                InFlight& f = slot[cur];
                f.stream = streams[cur];
                f.batch = std::make_unique<Batch>();
                f.reqs = take;
                std::vector<Request*> bad;
                std::vector<Request*> ok;
                for (Request* r : take) {
                    int st = f.batch->add(r->dtype, r->code.data(), r->code.size(), r->regs_in, r->d_col, r->count,
                                          r->want_sel != 0, r->sel_cap, r->d_sel);
                    if (st) {
                        r->status = st;
                        r->error = last_error();
                        bad.push_back(r);
                        // a rejected program leaves the batch: rebuild without it below
                    } else {
                        ok.push_back(r);
                    }
                }
                if (!bad.empty()) {
                    finish(bad);
                    f.batch = std::make_unique<Batch>();
                    for (Request* r : ok)
                        f.batch->add(r->dtype, r->code.data(), r->code.size(), r->regs_in, r->d_col, r->count,
                                     r->want_sel != 0, r->sel_cap, r->d_sel);
                    f.reqs = ok;
                }
                if (f.reqs.empty()) {
                    f.batch.reset();
                } else {
                    int st = f.batch->launch(f.stream, false);
                    note_batch(f.reqs.size(), t_build);
                    if (st) {
                        std::string err = last_error();
                        for (Request* r : f.reqs) {
                            r->status = st;
                            r->error = err;
                        }
                        finish(f.reqs);
                        f.batch.reset();
                        f.reqs.clear();
                    }
                }
            }
            // the other slot's batch has had the device while this one was prepared
            InFlight& prev = slot[cur ^ 1];
            if (prev.batch) complete_batch(prev);
            if (take.empty() && slot[cur].batch) complete_batch(slot[cur]);
            else cur ^= 1;
        }
        for (auto& f : slot)
            if (f.batch) complete_batch(f);
        for (auto& s : streams) cudaStreamDestroy(s);
    }

    void run_groupby(Request* r) {
        void* agg = voxel_agg_create();
        voxel_agg_init(agg, r->g_expected);
        int st = last_status();
        if (!st) st = voxel_agg_accumulate_dev(agg, r->g_keys, r->g_vals, r->g_n, thread_stream());
        if (!st) {
            uint64_t g = voxel_agg_group_count(agg);
            if (g > r->g_cap) {
                st = kErrCapacity;
                set_error(st, "group-by produced %llu groups, output capacity %zu",
                          static_cast<unsigned long long>(g), r->g_cap);
            } else {
                size_t got = voxel_agg_results(agg, r->o_keys, r->o_sum, r->o_min, r->o_max, r->o_count);
                if (got == static_cast<size_t>(-1)) st = last_status() ? last_status() : kErrCuda;
                else r->groups = got;
            }
        }
        voxel_agg_destroy(agg);
        r->status = st;
        if (st) r->error = last_error();
    }

    void run_join(Request* r) {
        DevBuf cs(32);
        int st = cs.p ? kOk : kErrOutOfMemory;
        if (!st)
            st = voxel_hashjoin_i64_dev(r->j_build, r->j_payload, r->j_nb, r->j_probe, r->j_np, r->j_left, r->j_right,
                                        r->j_cap, 1, cs.as<uint64_t>(), thread_stream());
        if (!st) {
            uint64_t h[3] = {0, 0, 0};
            st = d2h(h, cs.p, 24, thread_stream());
            if (!st) st = sync(thread_stream());
            r->j_pairs = h[0];
            r->j_sum = h[1];
            r->j_all = h[2];
        }
        r->status = st;
        if (st) r->error = last_error();
    }

    void operator_loop() {
        if (ensure_device()) return;
        for (;;) {
            std::vector<Request*> take;
            {
                std::unique_lock<std::mutex> lk(mu_);
                while (op_q_.empty() || in_use_ + op_q_.front()->footprint > budget_) {
                    if (stop_ && op_q_.empty()) break;
                    cv_work_.wait(lk);
                }
                if (stop_ && op_q_.empty()) break;
                take = admit(op_q_, 1);
            }
            for (Request* r : take) {
                clear_error();
                if (r->kind == kGroupBy) run_groupby(r);
                else run_join(r);
            }
            finish(take);
        }
    }

    size_t budget_;
    uint32_t max_batch_;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    std::deque<Request*> prog_q_, op_q_;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs_;
    std::vector<double> lat_;
    struct Breakdown {
        double queue_ms = 0, service_ms = 0;
        uint64_t n = 0;
    };
    Breakdown by_kind_[3];
    struct BatchStats {
        uint64_t batches = 0, programs = 0, max_batch = 0;
        double build_ms = 0, max_build_ms = 0, wait_ms = 0;
    };
    BatchStats bstat_;
    uint64_t next_id_ = 0;
    size_t in_use_ = 0, peak_ = 0;
    bool stop_ = false;
    static constexpr int kOpWorkers = 8;
    std::thread prog_thread_;
    std::vector<std::thread> op_threads_;
};

}  // namespace vx

using namespace vx;

extern "C" {

void* voxel_server_create(size_t budget_bytes, uint32_t max_batch) {
    clear_error();
    if (ensure_device()) return nullptr;
    return new Server(budget_bytes, max_batch);
}

void voxel_server_destroy(void* s) { delete static_cast<Server*>(s); }

uint64_t voxel_server_submit_program(void* s, int dtype, const uint32_t* code, size_t len, const uint64_t* regs64,
                                     const void* d_col, size_t count, int want_selection, size_t sel_capacity,
                                     uint32_t* d_sel) {
    clear_error();
    auto r = std::make_unique<Request>();
    r->kind = kProgram;
    r->dtype = dtype;
    r->code.assign(code, code + len);
    std::memcpy(r->regs_in, regs64, sizeof(r->regs_in));
    r->d_col = d_col;
    r->count = count;
    r->want_sel = want_selection;
    r->sel_cap = sel_capacity;
    r->d_sel = d_sel;
    r->footprint = program_footprint(count);
    return static_cast<Server*>(s)->submit(std::move(r));
}

uint64_t voxel_server_submit_groupby(void* s, const uint32_t* d_keys, const double* d_values, size_t n,
                                     size_t expected_groups, size_t out_capacity, uint32_t* out_keys,
                                     double* out_sum, double* out_min, double* out_max, uint64_t* out_count) {
    clear_error();
    auto r = std::make_unique<Request>();
    r->kind = kGroupBy;
    r->g_keys = d_keys;
    r->g_vals = d_values;
    r->g_n = n;
    r->g_expected = expected_groups;
    r->g_cap = out_capacity;
    r->o_keys = out_keys;
    r->o_sum = out_sum;
    r->o_min = out_min;
    r->o_max = out_max;
    r->o_count = out_count;
    r->footprint = groupby_footprint(expected_groups, n);
    return static_cast<Server*>(s)->submit(std::move(r));
}

uint64_t voxel_server_submit_join(void* s, const int64_t* d_build, const uint64_t* d_payload, size_t nb,
                                  const int64_t* d_probe, size_t np, uint32_t* d_left, uint32_t* d_right,
                                  size_t capacity) {
    clear_error();
    auto r = std::make_unique<Request>();
    r->kind = kJoin;
    r->j_build = d_build;
    r->j_payload = d_payload;
    r->j_nb = nb;
    r->j_probe = d_probe;
    r->j_np = np;
    r->j_left = d_left;
    r->j_right = d_right;
    r->j_cap = capacity;
    r->footprint = join_footprint(nb, np);
    return static_cast<Server*>(s)->submit(std::move(r));
}

int voxel_server_wait(void* s, uint64_t id, double timeout_s) {
    clear_error();
    return static_cast<Server*>(s)->wait(id, timeout_s);
}

int voxel_server_result(void* s, uint64_t id, uint64_t* regs64, uint64_t* count, uint64_t* aux,
                        double* latency_ms) {
    clear_error();
    return static_cast<Server*>(s)->result(id, regs64, count, aux, latency_ms);
}

int voxel_server_stats(void* s, uint64_t* completed, double* p50_ms, double* p99_ms, double* mean_ms,
                       uint64_t* peak_bytes) {
    return static_cast<Server*>(s)->stats(completed, p50_ms, p99_ms, mean_ms, peak_bytes);
}

void voxel_server_reset_stats(void* s) { static_cast<Server*>(s)->reset_stats(); }

int voxel_server_batch_stats(void* s, uint64_t* batches, uint64_t* programs, uint64_t* max_batch,
                             double* build_ms, double* max_build_ms, double* wait_ms) {
    clear_error();
    return static_cast<Server*>(s)->batch_stats(batches, programs, max_batch, build_ms, max_build_ms, wait_ms);
}

int voxel_server_breakdown(void* s, int kind, double* queue_ms, double* service_ms, uint64_t* completed) {
    clear_error();
    return static_cast<Server*>(s)->breakdown(kind, queue_ms, service_ms, completed);
}

}  // extern "C"
