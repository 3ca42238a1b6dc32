// Test infrastructure only: a flat C entry layer over the reference VoxelVM's
// own header-only C++ operators, compiled from the reference sources by
// oracle/build_oracle.py into oracle/_ref/libvoxel_ref.so. Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, as the
// checker and as the timed reference CPU path; no product code links it.
//
// Every function forwards to the reference type named in its comment
// (paths are relative to the reference project root).
#include "voxel/voxel.hpp"

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

using namespace voxel;

namespace {

template <typename T>
int engine_run_t(const uint32_t* code, size_t len, const void* const* segs,
                 const size_t* counts, size_t nsegs, const uint64_t* regs_in,
                 uint64_t* regs_out) {
    // include/voxel/exec/engine.hpp:35-81 (AddSegment, LoadProgram, Run)
    auto* e = new Engine<T>();
    for (size_t s = 0; s < nsegs; ++s)
        e->AddSegment(const_cast<T*>(static_cast<const T*>(segs[s])), counts[s]);
    for (size_t r = 0; r < 64; ++r) e->ScalarReg(r) = regs_in[r];
    std::vector<u32> v(code, code + len);
    e->LoadProgram(v);
    e->Run();
    for (size_t r = 0; r < 64; ++r) regs_out[r] = e->ScalarReg(r);
    delete e;
    return 0;
}

template <typename T>
int engine_run_parallel_t(const uint32_t* code, size_t len, const void* const* segs,
                          const size_t* counts, size_t nsegs, const uint64_t* regs_in,
                          size_t seg_id, uint32_t threads, uint8_t result_reg,
                          uint64_t* regs_out) {
    // include/voxel/exec/engine.hpp:143-175 (RunParallel)
    auto* e = new Engine<T>();
    for (size_t s = 0; s < nsegs; ++s)
        e->AddSegment(const_cast<T*>(static_cast<const T*>(segs[s])), counts[s]);
    for (size_t r = 0; r < 64; ++r) e->ScalarReg(r) = regs_in[r];
    std::vector<u32> v(code, code + len);
    e->LoadProgram(v);
    e->RunParallel(seg_id, threads, result_reg);
    for (size_t r = 0; r < 64; ++r) regs_out[r] = e->ScalarReg(r);
    delete e;
    return 0;
}

template <typename T>
size_t vfilter_t(int op, const T* d, size_t n, T a, T b, uint64_t* bitmap) {
    // include/voxel/ops/filter.hpp:42-288 (VectorFilter::Apply*)
    ops::VectorFilter<T> f;
    typename ops::VectorFilter<T>::FilterResult r;
    switch (op) {
    case 0: r = f.ApplyEQ(d, n, a); break;
    case 1: r = f.ApplyNE(d, n, a); break;
    case 2: r = f.ApplyLT(d, n, a); break;
    case 3: r = f.ApplyLE(d, n, a); break;
    case 4: r = f.ApplyGT(d, n, a); break;
    case 5: r = f.ApplyGE(d, n, a); break;
    default: r = f.ApplyBetween(d, n, a, b); break;
    }
    if (!r.Bitmap.empty()) std::memcpy(bitmap, r.Bitmap.data(), r.Bitmap.size() * 8);
    return r.PassCount;
}

template <typename K>
size_t hashagg_t(const K* keys, const double* vals, size_t n, size_t expected, K* okeys,
                 double* osum, double* omin, double* omax, uint64_t* ocount) {
    // include/voxel/ops/aggregate.hpp:159-261 (HashAggregator Init/Accumulate/Finalize)
    Arena arena;
    ops::HashAggregator<K, f64> agg(arena);
    agg.Init(expected);
    agg.Accumulate(keys, vals, n);
    size_t g = agg.GroupCount();
    using St = typename ops::HashAggregator<K, f64>::AggregateState;
    std::vector<St> st(g);
    std::vector<K> ks(g);
    agg.Finalize(ks.data(), st.data(), g);
    for (size_t i = 0; i < g; ++i) {
        okeys[i] = ks[i];
        osum[i] = st[i].Sum;
        omin[i] = st[i].Min;
        omax[i] = st[i].Max;
        ocount[i] = st[i].Count;
    }
    return g;
}

template <typename K>
size_t hashjoin_t(const K* build, size_t nb, const K* probe, size_t np, uint32_t* left,
                  uint32_t* right, size_t maxm, int all) {
    // include/voxel/ops/join.hpp:36-102 (Build, Probe, ProbeAllMatches)
    Arena arena;
    ops::HashJoin<K> j(arena);
    j.Build(build, nb);
    size_t m = 0;
    if (all)
        j.ProbeAllMatches(probe, np, left, right, m, maxm);
    else
        j.Probe(probe, np, left, right, m);
    return m;
}

double now_us() {
    return std::chrono::duration<double, std::micro>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// One chunk of the scan + group-by pipeline composed from reference operators.
struct GroupPipe {
    Arena arena;
    ops::HashAggregator<i32, f64> sumAgg;  // SUM(price*qty), COUNT
    ops::HashAggregator<i32, f64> mmAgg;   // MIN(price), MAX(price)
    GroupPipe() : sumAgg(arena), mmAgg(arena) {}
};

void group_chunk(GroupPipe& p, const encoding::BitPackedEncoding& keyPack,
                 const encoding::DictionaryEncoding<i32>& dict, const double* price,
                 const int32_t* qty, size_t begin, size_t end, double pthr, int32_t qlo,
                 int32_t qhi) {
    size_t n = end - begin;
    if (n == 0) return;
    // 1. key = Dictionary[BitPacked.DecodeBatch] (encoding.hpp:156-167, 411-422)
    std::vector<u32> idx(n);
    keyPack.DecodeBatch(idx.data(), begin, n);
    std::vector<i32> key(n);
    for (size_t i = 0; i < n; ++i) key[i] = dict.Dictionary[idx[i]];
    // 2. predicates (filter.hpp:42-78, 255-288) combined by ColumnFilter (526-547)
    ops::VectorFilter<f64> fp;
    ops::VectorFilter<i32> fq;
    auto rp = fp.ApplyGT(price + begin, n, pthr);
    auto rq = fq.ApplyBetween(qty + begin, n, qlo, qhi);
    ops::ColumnFilter<f64> cf;
    cf.Init(n);
    cf.AndWith(rp.Bitmap.data(), rp.Bitmap.size());
    cf.AndWith(rq.Bitmap.data(), rq.Bitmap.size());
    // 3. selection vector (filter.hpp:378-399)
    ops::SelectionVector<f64> sel;
    cf.BuildSelectionVector(sel);
    // 4. gather + materialised price*qty, then HashAggregator (aggregate.hpp:168-239)
    std::vector<i32> gk(sel.Count);
    std::vector<f64> gv(sel.Count), gp(sel.Count);
    for (size_t i = 0; i < sel.Count; ++i) {
        u32 r = sel.Indices[i];
        gk[i] = key[r];
        volatile double prod = price[begin + r] * static_cast<double>(qty[begin + r]);
        gv[i] = prod;
        gp[i] = price[begin + r];
    }
    p.sumAgg.Accumulate(gk.data(), gv.data(), sel.Count);
    p.mmAgg.Accumulate(gk.data(), gp.data(), sel.Count);
}

}  // namespace

// encoding.hpp:281-354 (DeltaEncoding<T>::Build, DecodeBatch); returns BaseValue's bits
template <typename T>
uint64_t delta_build_t(const T* data, size_t n, T* deltas) {
    encoding::DeltaEncoding<T> e;
    e.Build(data, n);
    if (!e.Deltas.empty()) std::memcpy(deltas, e.Deltas.data(), e.Deltas.size() * sizeof(T));
    return static_cast<uint64_t>(e.BaseValue);
}
template <typename T>
void delta_decode_t(const T* deltas, size_t n, uint64_t base, size_t offset, size_t count, T* out) {
    encoding::DeltaEncoding<T> e;
    e.BaseValue = static_cast<T>(base);
    e.Deltas.assign(deltas, deltas + n);
    e.DecodeBatch(out, offset, count);
}
// join.hpp:216-310 (MergeJoin<TKey>::Join / JoinUnique, SemiJoin, AntiJoin)
template <typename T>
size_t merge_join_t(const T* l, size_t nl, const T* r, size_t nr, uint32_t* lo, uint32_t* ro, int unique) {
    ops::MergeJoin<T> j;
    sz m = 0;
    if (unique) j.JoinUnique(l, nl, r, nr, lo, ro, m);
    else j.Join(l, nl, r, nr, lo, ro, m);
    return m;
}
template <typename T>
size_t semi_join_t(const T* l, size_t nl, const T* r, size_t nr, uint32_t* out, int anti) {
    Arena arena;
    sz m = 0;
    if (anti) {
        ops::AntiJoin<T> j;
        j.Join(l, nl, r, nr, out, m, arena);
    } else {
        ops::SemiJoin<T> j;
        j.Join(l, nl, r, nr, out, m, arena);
    }
    return m;
}

// exec/engine.hpp:176-300 (Engine<T>::WindowDelta / Sum / Mean / StdDev /
// Variance / Quantile and TimeWindowSum, static members)
template <typename T>
size_t window_t(int kind, const T* d, size_t n, T* out, size_t outLen, uint8_t w, double q) {
    switch (kind) {
    case 0: return Engine<T>::WindowDelta(d, n, out, outLen);
    case 1: return Engine<T>::WindowSum(d, n, out, outLen, w);
    case 2: return Engine<T>::WindowMean(d, n, out, outLen, w);
    case 3: return Engine<T>::WindowStdDev(d, n, out, outLen, w);
    case 4: return Engine<T>::WindowVariance(d, n, out, outLen, w);
    default: return Engine<T>::WindowQuantile(d, n, out, outLen, w, q);
    }
}

extern "C" {

int vref_engine_run(int dtype, const uint32_t* code, size_t len, const void* const* segs,
                    const size_t* counts, size_t nsegs, const uint64_t* regs_in,
                    uint64_t* regs_out) {
    switch (dtype) {
    case 0: return engine_run_t<f64>(code, len, segs, counts, nsegs, regs_in, regs_out);
    case 2: return engine_run_t<i64>(code, len, segs, counts, nsegs, regs_in, regs_out);
    case 3: return engine_run_t<i32>(code, len, segs, counts, nsegs, regs_in, regs_out);
    case 4: return engine_run_t<u64>(code, len, segs, counts, nsegs, regs_in, regs_out);
    case 5: return engine_run_t<u32>(code, len, segs, counts, nsegs, regs_in, regs_out);
    default: return -1;  // Engine<f32> does not compile in the reference (engine.hpp:398,406)
    }
}

int vref_engine_run_parallel(int dtype, const uint32_t* code, size_t len,
                             const void* const* segs, const size_t* counts, size_t nsegs,
                             const uint64_t* regs_in, size_t seg_id, uint32_t threads,
                             uint8_t result_reg, uint64_t* regs_out) {
    switch (dtype) {
    case 0: return engine_run_parallel_t<f64>(code, len, segs, counts, nsegs, regs_in, seg_id, threads, result_reg, regs_out);
    case 2: return engine_run_parallel_t<i64>(code, len, segs, counts, nsegs, regs_in, seg_id, threads, result_reg, regs_out);
    case 3: return engine_run_parallel_t<i32>(code, len, segs, counts, nsegs, regs_in, seg_id, threads, result_reg, regs_out);
    case 4: return engine_run_parallel_t<u64>(code, len, segs, counts, nsegs, regs_in, seg_id, threads, result_reg, regs_out);
    case 5: return engine_run_parallel_t<u32>(code, len, segs, counts, nsegs, regs_in, seg_id, threads, result_reg, regs_out);
    default: return -1;
    }
}

// bindings/voxel_c.cpp:80-101 (voxel_jit_run): x86-64 JIT fused filter+sum.
double vref_jit_run(const uint32_t* code, size_t len, const double* data, size_t n,
                    double threshold) {
    auto compiler = codegen::CreateJitCompiler();
    if (!compiler) return 0.0;
    codegen::JitFunction func;
    std::vector<u32> v(code, code + len);
    if (!compiler->Compile(v.data(), v.size(), func) || !func.IsValid()) {
        compiler->Release(func);
        return 0.0;
    }
    RegFile rf;
    rf.Scalar(0) = 0;
    rf.Scalar(1) = 0;
    rf.Scalar(2) = n;
    rf.Scalar(3) = std::bit_cast<u64>(threshold);
    f64* seg = const_cast<f64*>(data);
    u64 cnt = n;
    func.Entry(&rf, &seg, &cnt);
    double r = std::bit_cast<f64>(rf.Scalar(0));
    compiler->Release(func);
    return r;
}

// Median wall time (us) of `runs` executions of the f64 filter+sum program, after
// `warmup` executions: mode 0 = interpreter (Engine<f64>::Run), 1 = JIT entry
// (compiled once), 2 = Engine<f64>::RunParallel on `threads` threads.
// validate.cpp:14-20 is the methodology followed (warm-ups, median).
double vref_time_filter_sum_f64(int mode, const uint32_t* code, size_t len,
                                const double* data, size_t n, double threshold, int warmup,
                                int runs, uint32_t threads, double* result) {
    std::vector<double> t;
    std::vector<u32> v(code, code + len);
    double res = 0;
    if (mode == 1) {
        auto compiler = codegen::CreateJitCompiler();
        if (!compiler) return -1;
        codegen::JitFunction func;
        if (!compiler->Compile(v.data(), v.size(), func) || !func.IsValid()) return -1;
        for (int i = 0; i < warmup + runs; ++i) {
            RegFile rf;
            rf.Scalar(0) = 0; rf.Scalar(1) = 0; rf.Scalar(2) = n;
            rf.Scalar(3) = std::bit_cast<u64>(threshold);
            f64* sb = const_cast<f64*>(data);
            u64 sc = n;
            double t0 = now_us();
            func.Entry(&rf, &sb, &sc);
            double t1 = now_us();
            if (i >= warmup) t.push_back(t1 - t0);
            res = std::bit_cast<f64>(rf.Scalar(0));
        }
        compiler->Release(func);
    } else if (mode == 3) {
        // Engine<f64>::Run on `threads` row chunks at once (each a multiple of
        // kLanes, R2 = its own row count), for programs outside the fast path
        // where RunParallel would loop every worker over all rows; the
        // accumulator R0 is the sum of the chunks' R0.
        const sz kl = Engine<f64>::kLanes;
        const sz per = ((n / threads) / kl) * kl;
        for (int i = 0; i < warmup + runs; ++i) {
            std::vector<Engine<f64>> w(threads);
            std::vector<std::thread> th;
            double t0 = now_us();
            for (u32 k = 0; k < threads; ++k) {
                th.emplace_back([&, k] {
                    const sz start = k * per;
                    const sz cnt = k + 1 == threads ? ((n - start) / kl) * kl : per;
                    Engine<f64>& e = w[k];
                    e.AddSegment(const_cast<double*>(data) + start, cnt);
                    e.ScalarReg(0) = 0; e.ScalarReg(1) = 0; e.ScalarReg(2) = cnt;
                    e.ScalarReg(3) = std::bit_cast<u64>(threshold);
                    e.ScalarReg(4) = kl;
                    for (sz r = 5; r < 16; ++r) e.ScalarReg(r) = 0;
                    e.LoadProgram(v);
                    e.Run();
                });
            }
            for (auto& x : th) x.join();
            double t1 = now_us();
            if (i >= warmup) t.push_back(t1 - t0);
            res = 0;
            for (u32 k = 0; k < threads; ++k) res += std::bit_cast<f64>(w[k].ScalarReg(0));
        }
    } else {
        Engine<f64> e;
        e.AddSegment(const_cast<double*>(data), n);
        for (int i = 0; i < warmup + runs; ++i) {
            e.ScalarReg(0) = 0; e.ScalarReg(1) = 0; e.ScalarReg(2) = n;
            e.ScalarReg(3) = std::bit_cast<u64>(threshold);
            e.ScalarReg(4) = Engine<f64>::kLanes;
            e.LoadProgram(v);
            double t0 = now_us();
            if (mode == 2) e.RunParallel(0, threads, 0); else e.Run();
            double t1 = now_us();
            if (i >= warmup) t.push_back(t1 - t0);
            res = std::bit_cast<f64>(e.ScalarReg(0));
        }
    }
    std::sort(t.begin(), t.end());
    if (result) *result = res;
    return t.empty() ? 0.0 : t[t.size() / 2];
}

size_t vref_vfilter_f64(int op, const double* d, size_t n, double a, double b, uint64_t* bm) { return vfilter_t<f64>(op, d, n, a, b, bm); }
size_t vref_vfilter_f32(int op, const float* d, size_t n, float a, float b, uint64_t* bm) { return vfilter_t<f32>(op, d, n, a, b, bm); }
size_t vref_vfilter_i64(int op, const int64_t* d, size_t n, int64_t a, int64_t b, uint64_t* bm) { return vfilter_t<i64>(op, d, n, a, b, bm); }
size_t vref_vfilter_i32(int op, const int32_t* d, size_t n, int32_t a, int32_t b, uint64_t* bm) { return vfilter_t<i32>(op, d, n, a, b, bm); }
size_t vref_vfilter_u64(int op, const uint64_t* d, size_t n, uint64_t a, uint64_t b, uint64_t* bm) { return vfilter_t<u64>(op, d, n, a, b, bm); }
size_t vref_vfilter_u32(int op, const uint32_t* d, size_t n, uint32_t a, uint32_t b, uint64_t* bm) { return vfilter_t<u32>(op, d, n, a, b, bm); }

// simd/scalar.hpp:214-227 (scalar_filter_gt_f32): values > threshold, compacted in row order
size_t vref_scalar_filter_gt_f32(float* dst, const float* src, float threshold, size_t n) {
    return simd::scalar::scalar_filter_gt_f32(dst, src, threshold, n);
}

// simd/scalar.hpp:229-238 (scalar_sum_f32): 8 f32 lane accumulators, then the tail
float vref_scalar_sum_f32(const float* src, size_t n) { return simd::scalar::scalar_sum_f32(src, n); }

// encoding.hpp:281-354 (DeltaEncoding<T>): the helpers sit before the extern "C" block
uint64_t vref_delta_build_i64(const int64_t* d, size_t n, int64_t* o) { return delta_build_t<i64>(d, n, o); }
uint64_t vref_delta_build_i32(const int32_t* d, size_t n, int32_t* o) { return delta_build_t<i32>(d, n, o); }
uint64_t vref_delta_build_u64(const uint64_t* d, size_t n, uint64_t* o) { return delta_build_t<u64>(d, n, o); }
uint64_t vref_delta_build_u32(const uint32_t* d, size_t n, uint32_t* o) { return delta_build_t<u32>(d, n, o); }
void vref_delta_decode_i64(const int64_t* d, size_t n, uint64_t b, size_t off, size_t c, int64_t* o) { delta_decode_t<i64>(d, n, b, off, c, o); }
void vref_delta_decode_i32(const int32_t* d, size_t n, uint64_t b, size_t off, size_t c, int32_t* o) { delta_decode_t<i32>(d, n, b, off, c, o); }
void vref_delta_decode_u64(const uint64_t* d, size_t n, uint64_t b, size_t off, size_t c, uint64_t* o) { delta_decode_t<u64>(d, n, b, off, c, o); }
void vref_delta_decode_u32(const uint32_t* d, size_t n, uint64_t b, size_t off, size_t c, uint32_t* o) { delta_decode_t<u32>(d, n, b, off, c, o); }

// encoding.hpp:456-521 (FrameOfReferenceEncoding::Build, DecodeBatch)
void vref_for_build_f64(const double* d, size_t n, int32_t* codes, double* base, double* scale) {
    encoding::FrameOfReferenceEncoding e;
    e.Build(d, n);
    if (!e.EncodedValues.empty()) std::memcpy(codes, e.EncodedValues.data(), e.EncodedValues.size() * 4);
    *base = e.BaseValue;
    *scale = e.Scale;
}
void vref_for_decode_f64(const int32_t* codes, size_t n, double base, double scale, size_t offset, size_t count,
                         double* out) {
    encoding::FrameOfReferenceEncoding e;
    e.BaseValue = base;
    e.Scale = scale;
    e.EncodedValues.assign(codes, codes + n);
    e.DecodeBatch(out, offset, count);
}

size_t vref_merge_join_i64(const int64_t* l, size_t nl, const int64_t* r, size_t nr, uint32_t* lo, uint32_t* ro, int u) { return merge_join_t<i64>(l, nl, r, nr, lo, ro, u); }
size_t vref_merge_join_i32(const int32_t* l, size_t nl, const int32_t* r, size_t nr, uint32_t* lo, uint32_t* ro, int u) { return merge_join_t<i32>(l, nl, r, nr, lo, ro, u); }
size_t vref_merge_join_u64(const uint64_t* l, size_t nl, const uint64_t* r, size_t nr, uint32_t* lo, uint32_t* ro, int u) { return merge_join_t<u64>(l, nl, r, nr, lo, ro, u); }
size_t vref_merge_join_u32(const uint32_t* l, size_t nl, const uint32_t* r, size_t nr, uint32_t* lo, uint32_t* ro, int u) { return merge_join_t<u32>(l, nl, r, nr, lo, ro, u); }
size_t vref_semi_join_i64(const int64_t* l, size_t nl, const int64_t* r, size_t nr, uint32_t* o, int a) { return semi_join_t<i64>(l, nl, r, nr, o, a); }
size_t vref_semi_join_i32(const int32_t* l, size_t nl, const int32_t* r, size_t nr, uint32_t* o, int a) { return semi_join_t<i32>(l, nl, r, nr, o, a); }
size_t vref_semi_join_u64(const uint64_t* l, size_t nl, const uint64_t* r, size_t nr, uint32_t* o, int a) { return semi_join_t<u64>(l, nl, r, nr, o, a); }
size_t vref_semi_join_u32(const uint32_t* l, size_t nl, const uint32_t* r, size_t nr, uint32_t* o, int a) { return semi_join_t<u32>(l, nl, r, nr, o, a); }

size_t vref_window_f64(int k, const double* d, size_t n, double* o, size_t ol, uint8_t w, double q) { return window_t<f64>(k, d, n, o, ol, w, q); }
size_t vref_window_i64(int k, const int64_t* d, size_t n, int64_t* o, size_t ol, uint8_t w, double q) { return window_t<i64>(k, d, n, o, ol, w, q); }
size_t vref_window_i32(int k, const int32_t* d, size_t n, int32_t* o, size_t ol, uint8_t w, double q) { return window_t<i32>(k, d, n, o, ol, w, q); }
size_t vref_window_u64(int k, const uint64_t* d, size_t n, uint64_t* o, size_t ol, uint8_t w, double q) { return window_t<u64>(k, d, n, o, ol, w, q); }
size_t vref_window_u32(int k, const uint32_t* d, size_t n, uint32_t* o, size_t ol, uint8_t w, double q) { return window_t<u32>(k, d, n, o, ol, w, q); }
size_t vref_time_window_sum_f64(const int64_t* ts, const double* v, size_t n, int64_t st, int64_t dur, double* o, size_t ol) { return Engine<f64>::TimeWindowSum(ts, v, n, st, dur, o, ol); }
size_t vref_time_window_sum_i64(const int64_t* ts, const int64_t* v, size_t n, int64_t st, int64_t dur, int64_t* o, size_t ol) { return Engine<i64>::TimeWindowSum(ts, v, n, st, dur, o, ol); }
size_t vref_time_window_sum_i32(const int64_t* ts, const int32_t* v, size_t n, int64_t st, int64_t dur, int32_t* o, size_t ol) { return Engine<i32>::TimeWindowSum(ts, v, n, st, dur, o, ol); }
size_t vref_time_window_sum_u64(const int64_t* ts, const uint64_t* v, size_t n, int64_t st, int64_t dur, uint64_t* o, size_t ol) { return Engine<u64>::TimeWindowSum(ts, v, n, st, dur, o, ol); }
size_t vref_time_window_sum_u32(const int64_t* ts, const uint32_t* v, size_t n, int64_t st, int64_t dur, uint32_t* o, size_t ol) { return Engine<u32>::TimeWindowSum(ts, v, n, st, dur, o, ol); }

// filter.hpp:378-399 (SelectionVector::BuildFromBitmap)
size_t vref_selection_from_bitmap(const uint64_t* bm, size_t rows, uint32_t* out) {
    ops::SelectionVector<f64> s;
    s.BuildFromBitmap(bm, rows);
    if (s.Count) std::memcpy(out, s.Indices.data(), s.Count * 4);
    return s.Count;
}

// filter.hpp:526-547 (ColumnFilter::Init + AndWith)
size_t vref_column_filter_and(const uint64_t* const* bms, size_t nbm, size_t rows, uint64_t* out) {
    ops::ColumnFilter<f64> cf;
    cf.Init(rows);
    size_t words = (rows + 63) / 64;
    for (size_t i = 0; i < nbm; ++i) cf.AndWith(bms[i], words);
    if (words) std::memcpy(out, cf.GetBitmap().data(), words * 8);
    return cf.GetActiveCount();
}

// encoding.hpp:370-395 (BitPackedEncoding::Build); returns the bit width.
uint32_t vref_bitpack_build(const uint32_t* data, size_t n, uint64_t* words_out, size_t cap_words, size_t* nwords) {
    encoding::BitPackedEncoding e;
    e.Build(data, n);
    *nwords = e.PackedData.size();
    if (e.PackedData.size() <= cap_words && !e.PackedData.empty())
        std::memcpy(words_out, e.PackedData.data(), e.PackedData.size() * 8);
    return e.BitWidth;
}

// encoding.hpp:397-422 (BitPackedEncoding::Decode / DecodeBatch)
void vref_bitpack_decode(const uint64_t* words, size_t nwords, uint32_t width, size_t value_count, size_t offset, size_t count, uint32_t* out) {
    encoding::BitPackedEncoding e;
    e.BitWidth = width;
    e.PackedData.assign(words, words + nwords);
    e.ValueCount = value_count;
    e.DecodeBatch(out, offset, count);
}

// encoding.hpp:113-150 (DictionaryEncoding::Build); returns the cardinality.
size_t vref_dict_build_i32(const int32_t* data, size_t n, int32_t* dict_out, uint32_t* idx_out) {
    encoding::DictionaryEncoding<i32> d;
    d.Build(data, n);
    if (!d.Dictionary.empty()) std::memcpy(dict_out, d.Dictionary.data(), d.Dictionary.size() * 4);
    if (!d.Indices.empty()) std::memcpy(idx_out, d.Indices.data(), d.Indices.size() * 4);
    return d.Dictionary.size();
}
size_t vref_dict_build_f64(const double* data, size_t n, double* dict_out, uint32_t* idx_out) {
    encoding::DictionaryEncoding<f64> d;
    d.Build(data, n);
    if (!d.Dictionary.empty()) std::memcpy(dict_out, d.Dictionary.data(), d.Dictionary.size() * 8);
    if (!d.Indices.empty()) std::memcpy(idx_out, d.Indices.data(), d.Indices.size() * 4);
    return d.Dictionary.size();
}

// encoding.hpp:156-167 (DictionaryEncoding::DecodeBatch)
void vref_dict_decode_i32(const int32_t* dict, size_t card, const uint32_t* idx, size_t n, size_t offset, size_t count, int32_t* out) {
    encoding::DictionaryEncoding<i32> d;
    d.Dictionary.assign(dict, dict + card);
    d.Indices.assign(idx, idx + n);
    d.DecodeBatch(out, offset, count);
}
void vref_dict_decode_f64(const double* dict, size_t card, const uint32_t* idx, size_t n, size_t offset, size_t count, double* out) {
    encoding::DictionaryEncoding<f64> d;
    d.Dictionary.assign(dict, dict + card);
    d.Indices.assign(idx, idx + n);
    d.DecodeBatch(out, offset, count);
}

// encoding.hpp:202-220 (RLEEncoding::Build); returns the run count.
size_t vref_rle_build_i64(const int64_t* data, size_t n, int64_t* values_out, uint32_t* runs_out) {
    encoding::RLEEncoding<i64> r;
    r.Build(data, n);
    if (!r.Values.empty()) {
        std::memcpy(values_out, r.Values.data(), r.Values.size() * 8);
        std::memcpy(runs_out, r.RunLengths.data(), r.RunLengths.size() * 4);
    }
    return r.Values.size();
}
size_t vref_rle_build_f64(const double* data, size_t n, double* values_out, uint32_t* runs_out) {
    encoding::RLEEncoding<f64> r;
    r.Build(data, n);
    if (!r.Values.empty()) {
        std::memcpy(values_out, r.Values.data(), r.Values.size() * 8);
        std::memcpy(runs_out, r.RunLengths.data(), r.RunLengths.size() * 4);
    }
    return r.Values.size();
}

// encoding.hpp:231-257 (RLEEncoding::DecodeBatch)
void vref_rle_decode_i64(const int64_t* values, const uint32_t* runs, size_t nruns, size_t offset, size_t count, int64_t* out) {
    encoding::RLEEncoding<i64> r;
    r.Values.assign(values, values + nruns);
    r.RunLengths.assign(runs, runs + nruns);
    r.DecodeBatch(out, offset, count);
}
void vref_rle_decode_f64(const double* values, const uint32_t* runs, size_t nruns, size_t offset, size_t count, double* out) {
    encoding::RLEEncoding<f64> r;
    r.Values.assign(values, values + nruns);
    r.RunLengths.assign(runs, runs + nruns);
    r.DecodeBatch(out, offset, count);
}

size_t vref_hashagg_i32_f64(const int32_t* keys, const double* vals, size_t n, size_t expected, int32_t* okeys, double* osum, double* omin, double* omax, uint64_t* ocount) {
    return hashagg_t<i32>(keys, vals, n, expected, okeys, osum, omin, omax, ocount);
}
size_t vref_hashagg_u32_f64(const uint32_t* keys, const double* vals, size_t n, size_t expected, uint32_t* okeys, double* osum, double* omin, double* omax, uint64_t* ocount) {
    return hashagg_t<u32>(keys, vals, n, expected, okeys, osum, omin, omax, ocount);
}
size_t vref_hashagg_i64_f64(const int64_t* keys, const double* vals, size_t n, size_t expected, int64_t* okeys, double* osum, double* omin, double* omax, uint64_t* ocount) {
    return hashagg_t<i64>(keys, vals, n, expected, okeys, osum, omin, omax, ocount);
}

// aggregate.hpp:665-706 (GroupedAggregator over pre-sorted keys)
size_t vref_grouped_agg_i32_f64(const int32_t* keys, const double* vals, size_t n, int32_t* okeys, double* osum, double* omin, double* omax, uint64_t* ocount) {
    Arena arena;
    ops::GroupedAggregator<i32, f64> g(arena);
    g.AccumulateSorted(keys, vals, n);
    std::vector<f64> avg(n ? n : 1);
    std::vector<sz> cnt(n ? n : 1);
    sz gc = 0;
    g.FinalizeGroups(okeys, osum, omin, omax, cnt.data(), avg.data(), gc);
    for (sz i = 0; i < gc; ++i) ocount[i] = cnt[i];
    return gc;
}

// sort.hpp:83-160 (RadixSort<u64>::Sort with a u32 payload)
void vref_radix_sort_u64(uint64_t* keys, uint32_t* idx, size_t n) {
    ops::RadixSort<u64> s;
    s.Sort(keys, idx, n);
}
void vref_radix_sort_u32(uint32_t* keys, uint32_t* idx, size_t n) {
    ops::RadixSort<u32> s;
    s.Sort(keys, idx, n);
}
void vref_radix_sort_i64(int64_t* keys, uint32_t* idx, size_t n) {
    ops::RadixSort<i64> s;
    s.Sort(keys, idx, n);
}
void vref_radix_sort_i32(int32_t* keys, uint32_t* idx, size_t n) {
    ops::RadixSort<i32> s;
    s.Sort(keys, idx, n);
}

// sort.hpp:504-541 (SortOperator, stable merge sort on f64) and 490-502 (TopKSelect)
void vref_sort_ascending_f64(const double* d, size_t n, uint32_t* idx) {
    Segment<f64> seg(const_cast<double*>(d), n);
    ops::SortOperator::SortAscending(seg, idx);
}
void vref_sort_descending_f64(const double* d, size_t n, uint32_t* idx) {
    Segment<f64> seg(const_cast<double*>(d), n);
    ops::SortOperator::SortDescending(seg, idx);
}
void vref_topk_f64(const double* d, size_t n, size_t k, double* out, int largest) {
    ops::TopKSelect(d, n, k, out, largest != 0);
}

size_t vref_hashjoin_i64(const int64_t* b, size_t nb, const int64_t* p, size_t np, uint32_t* l, uint32_t* r, size_t maxm, int all) {
    return hashjoin_t<i64>(b, nb, p, np, l, r, maxm, all);
}
size_t vref_hashjoin_u32(const uint32_t* b, size_t nb, const uint32_t* p, size_t np, uint32_t* l, uint32_t* r, size_t maxm, int all) {
    return hashjoin_t<u32>(b, nb, p, np, l, r, maxm, all);
}
size_t vref_hashjoin_i32(const int32_t* b, size_t nb, const int32_t* p, size_t np, uint32_t* l, uint32_t* r, size_t maxm, int all) {
    return hashjoin_t<i32>(b, nb, p, np, l, r, maxm, all);
}

// Scan + group-by composed from the reference operators over rows [0, n):
// key = dict[unpack(keyPacked)], WHERE price > pthr AND qty BETWEEN qlo AND qhi,
// GROUP BY key: SUM(price*qty), COUNT, MIN(price), MAX(price). Row chunks run on
// `threads` std::threads (chunk boundaries on 64-row multiples) and are combined
// with HashAggregator::Merge (aggregate.hpp:243-248). Outputs are in the merged
// table's slot order; returns the group count. *elapsed_us gets the wall time.
size_t vref_scan_groupby(const uint64_t* keyPacked, size_t nwords, uint32_t width,
                         const int32_t* dict, size_t card, const double* price,
                         const int32_t* qty, size_t n, double pthr, int32_t qlo, int32_t qhi,
                         int threads, int32_t* okeys, double* osum, double* omin, double* omax,
                         uint64_t* ocount, double* elapsed_us) {
    encoding::BitPackedEncoding keyPack;
    keyPack.BitWidth = width;
    keyPack.PackedData.assign(keyPacked, keyPacked + nwords);
    keyPack.ValueCount = n;
    encoding::DictionaryEncoding<i32> d;
    d.Dictionary.assign(dict, dict + card);
    if (threads < 1) threads = 1;
    double t0 = now_us();
    std::vector<GroupPipe*> pipes(threads);
    for (int t = 0; t < threads; ++t) {
        pipes[t] = new GroupPipe();
        pipes[t]->sumAgg.Init(card);
        pipes[t]->mmAgg.Init(card);
    }
    size_t chunk = ((n + threads - 1) / threads + 63) / 64 * 64;
    std::vector<std::thread> ths;
    for (int t = 0; t < threads; ++t) {
        size_t b = std::min(n, (size_t)t * chunk), e = std::min(n, b + chunk);
        ths.emplace_back([&, t, b, e] { group_chunk(*pipes[t], keyPack, d, price, qty, b, e, pthr, qlo, qhi); });
    }
    for (auto& th : ths) th.join();
    for (int t = 1; t < threads; ++t) {
        pipes[0]->sumAgg.Merge(pipes[t]->sumAgg);
        pipes[0]->mmAgg.Merge(pipes[t]->mmAgg);
    }
    double t1 = now_us();
    if (elapsed_us) *elapsed_us = t1 - t0;
    size_t g = pipes[0]->sumAgg.GroupCount();
    using St = ops::HashAggregator<i32, f64>::AggregateState;
    std::vector<St> st(g);
    std::vector<i32> ks(g);
    pipes[0]->sumAgg.Finalize(ks.data(), st.data(), g);
    for (size_t i = 0; i < g; ++i) {
        okeys[i] = ks[i];
        osum[i] = st[i].Sum;
        ocount[i] = st[i].Count;
        auto* mm = pipes[0]->mmAgg.Lookup(ks[i]);
        omin[i] = mm ? mm->Min : 0.0;
        omax[i] = mm ? mm->Max : 0.0;
    }
    for (auto* p : pipes) delete p;
    return g;
}

}  // extern "C"
