// voxel_py: the reference's Python module surface (bindings/voxel_bindings.cpp:
// 25-396), implemented over this backend's C ABI (include/voxel_c.h).  Class,
// method and argument names follow the reference so its Python callers run
// unchanged; the work runs on the GPU.  Engines for f32 / i32 / u64 / u32 and
// the HashAggregator's results() are additions.  The reference's window
// functions, mmap / chunked readers, streaming engine, thread pool, profiler
// and JIT introspection are not on this backend's path and are not bound.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstdint>
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "voxel_c.h"

namespace py = pybind11;

namespace {

[[noreturn]] void fail(const char* what) {
    const char* e = voxel_last_error();
    throw std::runtime_error(std::string(what) + ": " + (e && *e ? e : "unknown error"));
}

uint64_t f64_bits(double v) {
    uint64_t b;
    std::memcpy(&b, &v, 8);
    return b;
}
double bits_f64(uint64_t b) {
    double v;
    std::memcpy(&v, &b, 8);
    return v;
}

// 32-bit instruction [op:8][rd:4][ra:4][rb:4][imm12:12] (bytecode/instruction.hpp:64-79)
uint32_t enc(uint8_t op, uint8_t rd = 0, uint8_t ra = 0, uint8_t rb = 0, uint16_t imm = 0) {
    return static_cast<uint32_t>(op) | ((rd & 0xFu) << 8) | ((ra & 0xFu) << 12) | ((rb & 0xFu) << 16) |
           ((static_cast<uint32_t>(imm) & 0xFFFu) << 20);
}

// opcode numbers (bytecode/opcodes.hpp)
enum Op : uint8_t {
    NOP = 0x00, HALT = 0x01, MOV = 0x10, MOVR = 0x11, ADD = 0x20, SUB = 0x21, MUL = 0x22, ADDF = 0x2A, CMP = 0x40,
    JMP = 0x50, JZ = 0x51, JNZ = 0x52, JLE = 0x5A, JGE = 0x5C, VLOAD = 0x70, VSTORE = 0x71, VADD = 0x80,
    VSUB = 0x81, VMUL = 0x82, VMIN = 0x87, VMAX = 0x88, VFILTER = 0xC0, VFILTER_GT = 0xC5, VFILTER_GE = 0xC6,
    VSUM = 0xD0, VRED_MIN = 0xD5, VRED_MAX = 0xD6, VCOUNT = 0xD7,
};

struct Instruction {
    uint32_t raw = 0;
};

// core/types.hpp:32-54
enum class DataType : uint32_t {
    Null = 0, Bool = 1, Int8 = 2, Int16 = 3, Int32 = 4, Int64 = 5, Uint8 = 6, Uint16 = 7, Uint32 = 8, Uint64 = 9,
    Float32 = 10, Float64 = 11, Decimal128 = 14, String = 20, Binary = 21, Date = 30, Timestamp = 32,
};

struct VectorFilterF64 {};

// One engine per element type; add_segment borrows the array (kept alive here).
struct PyEngine {
    void* h = nullptr;
    int dtype;
    std::vector<py::object> keep;
    explicit PyEngine(int dt) : dtype(dt) {
        h = voxel_engine_create(dt);
        if (!h) fail("voxel_engine_create");
    }
    ~PyEngine() {
        if (h) voxel_engine_destroy(h);
    }
    PyEngine(const PyEngine&) = delete;
    PyEngine& operator=(const PyEngine&) = delete;

    template <typename T>
    size_t add_segment(py::array_t<T, py::array::c_style | py::array::forcecast> arr) {
        keep.push_back(arr);  // borrowed, as the reference's add_segment: read at run time
        switch (dtype) {
        case 0: return voxel_engine_add_segment(h, reinterpret_cast<const double*>(arr.data()), arr.size());
        case 2: return voxel_engine_add_segment_i64(h, reinterpret_cast<const int64_t*>(arr.data()), arr.size());
        case 1: return voxel_engine_add_segment_f32(h, reinterpret_cast<const float*>(arr.data()), arr.size());
        case 3: return voxel_engine_add_segment_i32(h, reinterpret_cast<const int32_t*>(arr.data()), arr.size());
        case 4: return voxel_engine_add_segment_u64(h, reinterpret_cast<const uint64_t*>(arr.data()), arr.size());
        default: return voxel_engine_add_segment_u32(h, reinterpret_cast<const uint32_t*>(arr.data()), arr.size());
        }
    }
    void load_program(const std::vector<uint32_t>& code) { voxel_engine_load_program(h, code.data(), code.size()); }
    void run() {
        if (voxel_engine_run_status(h)) fail("run");
    }
    void run_parallel(size_t seg, uint32_t threads, uint8_t reg) {
        if (voxel_engine_run_parallel_status(h, seg, threads, reg)) fail("run_parallel");
    }
    uint64_t get_scalar(size_t i) { return voxel_engine_get_scalar(h, i); }
    void set_scalar(size_t i, uint64_t v) { voxel_engine_set_scalar(h, i, v); }
};

template <int DT, typename T>
struct EngineT : PyEngine {
    EngineT() : PyEngine(DT) {}
};

struct NullBitmap {
    void* h;
    size_t n;
    explicit NullBitmap(size_t count) : h(voxel_null_create(count)), n(count) {}
    ~NullBitmap() { voxel_null_destroy(h); }
};

struct Arena {
    size_t block_size;
    explicit Arena(size_t b) : block_size(b) {}
};

struct HashAggregator {
    void* h;
    explicit HashAggregator(Arena&) : h(voxel_agg_create()) {}
    ~HashAggregator() { voxel_agg_destroy(h); }
};

struct HashJoin {
    std::vector<int64_t> build;
    explicit HashJoin(Arena&) {}
};

struct DictionaryEncodingF64 {
    void* h = voxel_dict_create();
    size_t n = 0;
    ~DictionaryEncodingF64() { voxel_dict_destroy(h); }
};

struct SegmentF64 {
    py::array_t<double, py::array::c_style | py::array::forcecast> arr;  // borrowed, like Segment<f64>
    size_t n = 0;
};

struct RLEEncodingF64 {
    std::vector<double> values;
    std::vector<uint32_t> runs;
    size_t n = 0;
};

template <typename E, typename T>
void bind_engine(py::module_& m, const char* name, const char* get_typed, bool f64_scalars = false) {
    auto c = py::class_<E>(m, name)
                 .def(py::init<>())
                 .def("add_segment", &PyEngine::add_segment<T>, py::arg("data"))
                 .def("load_program", &PyEngine::load_program, py::arg("code"))
                 .def("run", &PyEngine::run)
                 .def("run_parallel", &PyEngine::run_parallel, py::arg("seg_id"), py::arg("threads") = 0,
                      py::arg("result_reg") = 0)
                 .def("get_scalar", &PyEngine::get_scalar)
                 .def("set_scalar", &PyEngine::set_scalar)
                 // a read-only class property, as Engine<T>::kLanes is bound in the reference
                 // (voxel_bindings.cpp:126): EngineF64.k_lanes and engine.k_lanes are both 4
                 .def_property_readonly_static("k_lanes", [](py::object) { return 32 / sizeof(T); });
    if (f64_scalars) {
        c.def("get_scalar_f64", [](E& e, size_t i) { return voxel_engine_get_scalar_f64(e.h, i); });
        c.def("set_scalar_f64", [](E& e, size_t i, double v) { voxel_engine_set_scalar_f64(e.h, i, v); });
        // window functions (reference bindings/voxel_bindings.cpp:127-171): results written into `out`
        using F64Arr = py::array_t<double, py::array::c_style | py::array::forcecast>;
        using OutArr = py::array_t<double, py::array::c_style>;
        auto win = [](int kind, F64Arr data, OutArr out, uint8_t w, double q) {
            return voxel_window(0, kind, data.data(), static_cast<size_t>(data.size()), out.mutable_data(),
                                static_cast<size_t>(out.size()), w, q);
        };
        c.def("window_delta", [win](E&, F64Arr d, OutArr o) { return win(0, d, o, 2, 0.0); }, py::arg("data"),
              py::arg("out"));
        c.def("window_sum", [win](E&, F64Arr d, OutArr o, uint8_t w) { return win(1, d, o, w, 0.0); },
              py::arg("data"), py::arg("out"), py::arg("window"));
        c.def("window_mean", [win](E&, F64Arr d, OutArr o, uint8_t w) { return win(2, d, o, w, 0.0); },
              py::arg("data"), py::arg("out"), py::arg("window"));
        c.def("window_stddev", [win](E&, F64Arr d, OutArr o, uint8_t w) { return win(3, d, o, w, 0.0); },
              py::arg("data"), py::arg("out"), py::arg("window"));
        c.def("window_variance", [win](E&, F64Arr d, OutArr o, uint8_t w) { return win(4, d, o, w, 0.0); },
              py::arg("data"), py::arg("out"), py::arg("window"));
        c.def("window_quantile",
              [win](E&, F64Arr d, OutArr o, uint8_t w, double q) { return win(5, d, o, w, q); }, py::arg("data"),
              py::arg("out"), py::arg("window"), py::arg("quantile"));
        c.def("time_window_sum",
              [](E&, py::array_t<int64_t, py::array::c_style | py::array::forcecast> ts, F64Arr v, int64_t start,
                 int64_t dur, OutArr out) {
                  const size_t cnt = std::min<size_t>(static_cast<size_t>(ts.size()), static_cast<size_t>(v.size()));
                  return voxel_time_window_sum(0, ts.data(), v.data(), cnt, start, dur, out.mutable_data(),
                                               static_cast<size_t>(out.size()));
              },
              py::arg("timestamps"), py::arg("values"), py::arg("start_time"), py::arg("duration_sec"),
              py::arg("out"));
    }
    if (get_typed) {
        c.def(get_typed, [](E& e, size_t i) {
            uint64_t b = voxel_engine_get_scalar(e.h, i);
            T v;
            if constexpr (sizeof(T) == 8) std::memcpy(&v, &b, 8);
            else v = static_cast<T>(b);
            return v;
        });
    }
}

}  // namespace

PYBIND11_MODULE(voxel_py, m) {
    m.doc() = "VoxelVM Python bindings on the B200 backend (columnar filter / aggregate path on the GPU)";

    py::enum_<DataType>(m, "DataType")
        .value("Null", DataType::Null).value("Bool", DataType::Bool).value("Int8", DataType::Int8)
        .value("Int16", DataType::Int16).value("Int32", DataType::Int32).value("Int64", DataType::Int64)
        .value("Uint8", DataType::Uint8).value("Uint16", DataType::Uint16).value("Uint32", DataType::Uint32)
        .value("Uint64", DataType::Uint64).value("Float32", DataType::Float32).value("Float64", DataType::Float64)
        .value("Decimal128", DataType::Decimal128).value("String", DataType::String)
        .value("Binary", DataType::Binary).value("Date", DataType::Date).value("Timestamp", DataType::Timestamp)
        .export_values();

    py::enum_<Op>(m, "Opcode")
        .value("NOP", NOP).value("HALT", HALT).value("MOV", MOV).value("ADD", ADD).value("SUB", SUB)
        .value("MUL", MUL).value("CMP", CMP).value("JMP", JMP).value("JZ", JZ).value("JNZ", JNZ)
        .value("VLOAD", VLOAD).value("VSTORE", VSTORE).value("VADD", VADD).value("VFILTER_GT", VFILTER_GT)
        .value("VSUM", VSUM).value("ADDF", ADDF)
        .export_values();

    m.attr("CMP_EQ") = 0;
    m.attr("CMP_NE") = 1;
    m.attr("CMP_LT") = 2;
    m.attr("CMP_LE") = 3;
    m.attr("CMP_GT") = 4;
    m.attr("CMP_GE") = 5;

    py::class_<Instruction>(m, "Instruction")
        .def(py::init<>())
        .def_property("raw", [](const Instruction& i) { return i.raw; }, [](Instruction& i, uint32_t v) { i.raw = v; })
        .def("op", [](const Instruction& i) { return static_cast<uint8_t>(i.raw & 0xFF); })
        .def("rd", [](const Instruction& i) { return static_cast<uint8_t>((i.raw >> 8) & 0xF); })
        .def("ra", [](const Instruction& i) { return static_cast<uint8_t>((i.raw >> 12) & 0xF); })
        .def("rb", [](const Instruction& i) { return static_cast<uint8_t>((i.raw >> 16) & 0xF); })
        .def("imm12", [](const Instruction& i) { return static_cast<uint16_t>((i.raw >> 20) & 0xFFF); })
        .def_static("nop", []() { return Instruction{enc(NOP)}; })
        .def_static("halt", []() { return Instruction{enc(HALT)}; })
        .def_static("mov", [](uint8_t rd, int16_t imm) { return Instruction{enc(MOV, rd, 0, 0, static_cast<uint16_t>(imm))}; })
        .def_static("movr", [](uint8_t rd, uint8_t ra) { return Instruction{enc(MOVR, rd, ra)}; })
        .def_static("add", [](uint8_t rd, uint8_t ra, uint8_t rb) { return Instruction{enc(ADD, rd, ra, rb)}; })
        .def_static("sub", [](uint8_t rd, uint8_t ra, uint8_t rb) { return Instruction{enc(SUB, rd, ra, rb)}; })
        .def_static("mul", [](uint8_t rd, uint8_t ra, uint8_t rb) { return Instruction{enc(MUL, rd, ra, rb)}; })
        .def_static("addf", [](uint8_t rd, uint8_t ra, uint8_t rb) { return Instruction{enc(ADDF, rd, ra, rb)}; })
        .def_static("cmp", [](uint8_t ra, uint8_t rb) { return Instruction{enc(CMP, 0, ra, rb)}; })
        .def_static("jmp", [](int16_t o) { return Instruction{enc(JMP, 0, 0, 0, static_cast<uint16_t>(o))}; })
        .def_static("jz", [](int16_t o) { return Instruction{enc(JZ, 0, 0, 0, static_cast<uint16_t>(o))}; })
        .def_static("jnz", [](int16_t o) { return Instruction{enc(JNZ, 0, 0, 0, static_cast<uint16_t>(o))}; })
        .def_static("jle", [](int16_t o) { return Instruction{enc(JLE, 0, 0, 0, static_cast<uint16_t>(o))}; })
        .def_static("jge", [](int16_t o) { return Instruction{enc(JGE, 0, 0, 0, static_cast<uint16_t>(o))}; })
        .def_static("vload", [](uint8_t vd, uint8_t ra, uint8_t seg, uint8_t count) {
            return Instruction{enc(VLOAD, vd, ra, 0, static_cast<uint16_t>(((seg & 0xF) << 8) | count))};
        })
        .def_static("vstore", [](uint8_t vs, uint8_t ra, uint8_t seg, uint8_t count) {
            return Instruction{enc(VSTORE, vs, ra, 0, static_cast<uint16_t>(((seg & 0xF) << 8) | count))};
        })
        .def_static("vadd", [](uint8_t vd, uint8_t va, uint8_t vb) { return Instruction{enc(VADD, vd, va, vb)}; })
        .def_static("vsub", [](uint8_t vd, uint8_t va, uint8_t vb) { return Instruction{enc(VSUB, vd, va, vb)}; })
        .def_static("vmul", [](uint8_t vd, uint8_t va, uint8_t vb) { return Instruction{enc(VMUL, vd, va, vb)}; })
        .def_static("vmin", [](uint8_t vd, uint8_t va, uint8_t vb) { return Instruction{enc(VMIN, vd, va, vb)}; })
        .def_static("vmax", [](uint8_t vd, uint8_t va, uint8_t vb) { return Instruction{enc(VMAX, vd, va, vb)}; })
        .def_static("vfilter", [](uint8_t vd, uint8_t va, uint8_t rb, uint8_t mode) {
            return Instruction{enc(VFILTER, vd, va, rb, mode & 0x7)};
        })
        .def_static("vfilter_gt", [](uint8_t vd, uint8_t va, uint8_t rb) { return Instruction{enc(VFILTER_GT, vd, va, rb)}; })
        .def_static("vfilter_ge", [](uint8_t vd, uint8_t va, uint8_t rb) { return Instruction{enc(VFILTER_GE, vd, va, rb)}; })
        .def_static("vsum", [](uint8_t rd, uint8_t va) { return Instruction{enc(VSUM, rd, va)}; })
        .def_static("vred_min", [](uint8_t rd, uint8_t va) { return Instruction{enc(VRED_MIN, rd, va)}; })
        .def_static("vred_max", [](uint8_t rd, uint8_t va) { return Instruction{enc(VRED_MAX, rd, va)}; })
        .def_static("vcount", [](uint8_t rd, uint8_t va) { return Instruction{enc(VCOUNT, rd, va)}; });

    bind_engine<EngineT<0, double>, double>(m, "EngineF64", nullptr, true);
    bind_engine<EngineT<2, int64_t>, int64_t>(m, "EngineI64", "get_scalar_i64");
    bind_engine<EngineT<1, float>, float>(m, "EngineF32", nullptr, true);
    bind_engine<EngineT<3, int32_t>, int32_t>(m, "EngineI32", nullptr);
    bind_engine<EngineT<4, uint64_t>, uint64_t>(m, "EngineU64", nullptr);
    bind_engine<EngineT<5, uint32_t>, uint32_t>(m, "EngineU32", nullptr);

    py::class_<NullBitmap>(m, "NullBitmap")
        .def(py::init<size_t>())
        .def("is_null", [](NullBitmap& b, size_t r) { return voxel_null_is_null(b.h, r) != 0; })
        .def("set_null", [](NullBitmap& b, size_t r) { voxel_null_set_null(b.h, r); })
        .def("set_valid", [](NullBitmap& b, size_t r) { voxel_null_set_valid(b.h, r); })
        .def("null_count", [](NullBitmap& b) { return voxel_null_null_count(b.h); })
        .def("valid_count", [](NullBitmap& b) { return voxel_null_valid_count(b.h); })
        .def("set_all_valid", [](NullBitmap& b) { for (size_t r = 0; r < b.n; ++r) voxel_null_set_valid(b.h, r); })
        .def("set_all_null", [](NullBitmap& b) { for (size_t r = 0; r < b.n; ++r) voxel_null_set_null(b.h, r); });

    py::class_<DictionaryEncodingF64>(m, "DictionaryEncodingF64")
        .def(py::init<>())
        .def("build", [](DictionaryEncodingF64& d, py::array_t<double, py::array::c_style | py::array::forcecast> a) {
            voxel_dict_build(d.h, a.data(), a.size());
            if (voxel_last_status()) fail("DictionaryEncodingF64.build");
            d.n = a.size();
        })
        .def_property_readonly("dictionary", [](DictionaryEncodingF64& d) {
            py::array_t<double> out(voxel_dict_cardinality(d.h));
            voxel_dict_values(d.h, out.mutable_data());
            return out;
        })
        .def_property_readonly("memory_usage",
                               [](DictionaryEncodingF64& d) { return voxel_dict_cardinality(d.h) * 8 + d.n * 4; })
        .def("decode_batch", [](DictionaryEncodingF64& d, size_t offset, size_t count) {
            py::array_t<double> out(count);
            voxel_dict_decode_batch(d.h, out.mutable_data(), offset, count);
            if (voxel_last_status()) fail("DictionaryEncodingF64.decode_batch");
            return out;
        });

    py::class_<RLEEncodingF64>(m, "RLEEncodingF64")
        .def(py::init<>())
        .def("build", [](RLEEncodingF64& r, py::array_t<double, py::array::c_style | py::array::forcecast> a) {
            r.values.clear();
            r.runs.clear();
            r.n = a.size();
            const double* p = a.data();
            for (size_t i = 0; i < r.n;) {  // runs of bit-identical values (encoding.hpp:202-225)
                size_t j = i + 1;
                while (j < r.n && std::memcmp(&p[j], &p[i], 8) == 0 && j - i < 0xFFFFFFFFu) ++j;
                r.values.push_back(p[i]);
                r.runs.push_back(static_cast<uint32_t>(j - i));
                i = j;
            }
        })
        .def_property_readonly("memory_usage", [](RLEEncodingF64& r) { return r.values.size() * 8 + r.runs.size() * 4; })
        .def("decode_batch", [](RLEEncodingF64& r, size_t offset, size_t count) {
            py::array_t<double> out(count);
            if (voxel_rle_decode_i64(reinterpret_cast<const int64_t*>(r.values.data()), r.runs.data(), r.runs.size(),
                                     offset, count, reinterpret_cast<int64_t*>(out.mutable_data())))
                fail("RLEEncodingF64.decode_batch");
            return out;
        });

    py::class_<Arena>(m, "Arena").def(py::init<size_t>(), py::arg("block_size") = 65536);

    py::class_<HashAggregator>(m, "HashAggregator")
        .def(py::init<Arena&>(), py::keep_alive<1, 2>())
        .def("init", [](HashAggregator& a, size_t expected) { voxel_agg_init(a.h, expected); })
        .def("accumulate", [](HashAggregator& a, py::array_t<uint32_t, py::array::c_style | py::array::forcecast> k,
                              py::array_t<double, py::array::c_style | py::array::forcecast> v) {
            size_t n = std::min<size_t>(k.size(), v.size());
            voxel_agg_accumulate(a.h, k.data(), v.data(), n);
            if (voxel_last_status()) fail("HashAggregator.accumulate");
        })
        .def("group_count", [](HashAggregator& a) { return voxel_agg_group_count(a.h); })
        .def("results", [](HashAggregator& a) {
            size_t g = voxel_agg_group_count(a.h);
            py::array_t<uint32_t> k(g);
            py::array_t<double> s(g), mn(g), mx(g);
            py::array_t<uint64_t> c(g);
            if (voxel_agg_results(a.h, k.mutable_data(), s.mutable_data(), mn.mutable_data(), mx.mutable_data(),
                                  c.mutable_data()) == static_cast<size_t>(-1))
                fail("HashAggregator.results");
            return py::make_tuple(k, s, mn, mx, c);
        });

    m.def("sort_ascending", [](py::array_t<double, py::array::c_style | py::array::forcecast> a) {
        py::array_t<uint32_t> idx(a.size());
        voxel_sort_ascending(a.data(), a.size(), idx.mutable_data());
        if (voxel_last_status()) fail("sort_ascending");
        return idx;
    });
    m.def("topk_select", [](py::array_t<double, py::array::c_style | py::array::forcecast> a, size_t k, bool largest) {
        py::array_t<double> out(k);
        voxel_topk(a.data(), a.size(), k, out.mutable_data(), largest ? 1 : 0);
        if (voxel_last_status()) fail("topk_select");
        return out;
    });

    py::class_<HashJoin>(m, "HashJoin")
        .def(py::init<Arena&>(), py::keep_alive<1, 2>())
        .def("build", [](HashJoin& j, py::array_t<uint32_t, py::array::c_style | py::array::forcecast> keys) {
            j.build.assign(keys.data(), keys.data() + keys.size());
        })
        .def("contains", [](HashJoin& j, uint32_t key) {
            int64_t p = key;
            uint32_t l = 0, r = 0;
            size_t m = voxel_hashjoin_i64(j.build.data(), j.build.size(), &p, 1, &l, &r, 1, 0);
            if (m == static_cast<size_t>(-1)) fail("HashJoin.contains");
            return m > 0;
        })
        .def("probe", [](HashJoin& j, py::array_t<uint32_t, py::array::c_style | py::array::forcecast> pk) {
            size_t n = pk.size();
            std::vector<int64_t> p(pk.data(), pk.data() + n);
            std::vector<uint32_t> l(n), r(n);
            size_t m = voxel_hashjoin_i64(j.build.data(), j.build.size(), p.data(), n, l.data(), r.data(), n, 0);
            if (m == static_cast<size_t>(-1)) fail("HashJoin.probe");
            return py::make_tuple(py::array_t<uint32_t>(m, l.data()), py::array_t<uint32_t>(m, r.data()), m);
        });

    py::class_<VectorFilterF64>(m, "VectorFilterF64")
        .def(py::init<>())
        .def("apply_gt", [](VectorFilterF64&, py::array_t<double, py::array::c_style | py::array::forcecast> a,
                            double threshold) {
            size_t n = a.size();
            py::array_t<uint64_t> bm((n + 63) / 64);
            size_t c = voxel_vfilter(0, 4, a.data(), n, f64_bits(threshold), 0, bm.mutable_data());
            if (c == static_cast<size_t>(-1)) fail("VectorFilterF64.apply_gt");
            return py::make_tuple(bm, c);
        });

    // fused filter+sum over one f64 column: R0 = R1 = 0, R2 = total_count,
    // R3 = threshold; returns R0 (the reference raises when it cannot compile)
    m.def("jit_run", [](const std::vector<uint32_t>& code,
                        py::array_t<double, py::array::c_style | py::array::forcecast> data, double threshold,
                        size_t total_count) {
        void* e = voxel_engine_create_f64();
        if (!e) fail("jit_run");
        voxel_engine_add_segment(e, data.data(), data.size());
        voxel_engine_set_scalar(e, 0, 0);
        voxel_engine_set_scalar(e, 1, 0);
        voxel_engine_set_scalar(e, 2, total_count);
        voxel_engine_set_scalar(e, 3, f64_bits(threshold));
        voxel_engine_load_program(e, code.data(), code.size());
        int st = voxel_engine_run_status(e);
        double r = bits_f64(voxel_engine_get_scalar(e, 0));
        voxel_engine_destroy(e);
        if (st) fail("JIT compilation failed");
        return r;
    }, py::arg("code"), py::arg("data"), py::arg("threshold"), py::arg("total_count"));

    // reference bindings/voxel_bindings.cpp:329-340: {"compiled": bool, "code_size", "code_ptr"}; the
    // compiled form here is the lowered GPU kernel schedule (no host code pointer: 0), named in "kernel"
    m.def("jit_compile", [](const std::vector<uint32_t>& code) {
        size_t bytes = 0;
        char kernel[32] = {0};
        if (voxel_jit_compile(code.data(), code.size(), &bytes, kernel, sizeof(kernel)) != 0)
            return py::dict(py::arg("compiled") = false);
        return py::dict(py::arg("compiled") = true, py::arg("code_size") = bytes, py::arg("code_ptr") = 0,
                        py::arg("kernel") = std::string(kernel));
    }, py::arg("code"));

    // reference bindings/voxel_bindings.cpp:97-103: a view of an f64 buffer
    py::class_<SegmentF64>(m, "SegmentF64")
        .def(py::init<>())
        .def(py::init([](py::array_t<double, py::array::c_style | py::array::forcecast> a, size_t n) {
                 SegmentF64 s;
                 s.arr = a;
                 s.n = std::min<size_t>(n, static_cast<size_t>(a.size()));
                 return s;
             }),
             py::arg("data"), py::arg("count"))
        .def(py::init([](py::array_t<double, py::array::c_style | py::array::forcecast> a) {
                 SegmentF64 s;
                 s.arr = a;
                 s.n = static_cast<size_t>(a.size());
                 return s;
             }),
             py::arg("data"))
        .def("__getitem__", [](const SegmentF64& s, size_t i) {
            if (i >= s.n) throw py::index_error("segment index out of range");
            return s.arr.data()[i];
        })
        .def("__len__", [](const SegmentF64& s) { return s.n; })
        .def_property_readonly("size", [](const SegmentF64& s) { return s.n; });

    m.attr("__version__") = "1.0.0";
}
