"""Engine parity on the GPU: every program runs through the C ABI
(voxel_engine_*) on the CUDA backend and must reproduce the reference
interpreter's registers - bit-exact for integers, counts, min/max and
offsets; f64 sums within 1e-12 relative (FP64 compensated accumulation);
f32 columns within 1e-6 of the restatement."""
import struct

import numpy as np
import pytest

import inputs
import oracle
from voxel_b200 import bytecode as bc
from voxel_b200 import capi
from voxel_b200 import templates as T
from voxel_b200.engine import Engine, VoxelError

pytestmark = pytest.mark.gpu

F64_RTOL = 1e-12
F32_RTOL = 1e-6


def f64(b):
    return struct.unpack("<d", struct.pack("<Q", b & 0xFFFFFFFFFFFFFFFF))[0]


def float_acc_regs(code):
    """Registers the program accumulates with ADDF (or the fused fast path)."""
    regs = set()
    for c in code:
        if c & 0xFF == 0x2A and ((c >> 8) & 0xF) in (((c >> 12) & 0xF), ((c >> 16) & 0xF)):
            regs.add((c >> 8) & 0xF)
    return regs


def run_gpu(dtype, code, arrays, regs):
    e = Engine(dtype)
    for a in arrays:
        e.add_segment(a)
    for i, v in enumerate(regs):
        e.set_scalar(i, v)
    e.load_program(code)
    e.run()
    return e.registers(16), e


def assert_regs(dtype, code, got, want, rtol):
    facc = float_acc_regs(code) if dtype in (0, 1) else set()
    for r in range(16):
        if got[r] == want[r]:
            continue
        if dtype in (0, 1) and f64(got[r]) != f64(got[r]) and f64(want[r]) != f64(want[r]):
            continue  # both NaN: the payload of a NaN register is not part of the result
        assert r in facc, f"R{r}: got {got[r]:#x} want {want[r]:#x}"
        g, w = f64(got[r]), f64(want[r])
        if g != g and w != w:
            continue  # both NaN: a NaN sum's payload is not part of the result
        assert abs(g - w) <= rtol * max(abs(w), 1e-300), f"R{r}: {g!r} vs {w!r}"


def test_known_answers(golden):
    for case in golden["kat"]:
        dt = case["dtype"]
        arrays = [np.asarray(d, dtype=T.NP[dt]) for d in case["data"]]
        got, _ = run_gpu(dt, case["code"], arrays, case["regs"])
        assert_regs(dt, case["code"], got, case["expect"], F64_RTOL)
    # c_test.cpp: the fused fast path returns exactly 26.0
    got, _ = run_gpu(0, golden["kat"][2]["code"], [np.arange(1, 9, dtype=np.float64)], golden["kat"][2]["regs"])
    assert f64(got[0]) == 26.0


def test_golden_programs(golden):
    for case in golden["programs"]:
        dt, n = case["dtype"], case["n"]
        col = inputs.column(dt, n, case["seed"])
        got, _ = run_gpu(dt, case["code"], [col], case["regs"])
        assert_regs(dt, case["code"], got, case["expect"], F64_RTOL)


def test_config1_ground_truth(golden):
    c = golden["config1"]
    x = inputs.mt_uniform(c["seed"], c["n"])
    regs = [0, 0, c["n"], T.reg_image(0, 500.0), 4]
    got, e = run_gpu(0, bc.filter_sum_program(), [x], regs)
    assert e.explain().startswith("fast")
    assert got[1] == 1_000_000
    s = f64(got[0])
    assert abs(s - f64(c["sum_bits"])) <= F64_RTOL * s
    assert abs(s - 375538740.218) < 1e-3  # docs/Benchmarks.md:7
    got, e = run_gpu(0, bc.filter_sum_count_program(), [x], regs + [0, 0])
    assert got[6] == 500720
    # the SUM + COUNT program runs on the fused filter+sum kernel with its count, same sum
    assert "kernel=fsum" in e.explain()
    assert abs(f64(got[0]) - f64(c["sum_bits"])) <= F64_RTOL * s
    # jit_run entry point (voxel_c.cpp:80-101)
    code = np.asarray(bc.filter_sum_program(), np.uint32)
    j = capi.lib().voxel_jit_run(code.ctypes.data, code.size, x.ctypes.data, x.size, 500.0)
    assert abs(j - s) <= F64_RTOL * s


def test_f32_programs_against_reference_filters_and_restatement():
    """f32 programs (no reference engine exists for f32): every register as
    the restatement's, and the aggregates pinned to the rows the reference's
    own VectorFilter<f32> + ColumnFilter select (COUNT, MIN, MAX exact; SUM
    within 1e-6 relative)."""
    rng = np.random.default_rng(11)
    for n in (8, 64, 1000, 4096, 65536, 1 << 20):
        col = T.make_column(T.F32, n, rng)
        for agg in T.AGGS:
            prog = T.random_program(T.F32, rng, agg=agg)
            regs = prog.registers(n)
            st, want, _ = oracle.engine_run_port(T.F32, prog.code, [col], regs)
            assert st == 0
            got, _ = run_gpu(T.F32, prog.code, [col], regs)
            assert_regs(T.F32, prog.code, got, want[:16], F32_RTOL)
            ref = oracle.f32_program_expect(prog.preds, [agg], col)[agg]
            v = T.image_value(T.F32, got[0]) if agg != "COUNT" else got[0]
            if agg == "SUM":
                assert abs(v - ref) <= F32_RTOL * abs(ref) + 1e-30, (v, ref)
            else:
                assert v == ref, (agg, v, ref)
        aggs = ["SUM", "COUNT", "MIN", "MAX"]
        base = T.random_program(T.F32, rng, npreds=int(rng.integers(1, 5)))
        prog = T.build_multi(T.F32, base.preds, aggs)
        got, _ = run_gpu(T.F32, prog.code, [col], prog.registers(n))
        ref = oracle.f32_program_expect(base.preds, aggs, col)
        assert got[T.MULTI_ACC["COUNT"]] == ref["COUNT"]
        assert T.image_value(T.F32, got[T.MULTI_ACC["MIN"]]) == ref["MIN"]
        assert T.image_value(T.F32, got[T.MULTI_ACC["MAX"]]) == ref["MAX"]
        s = T.image_value(T.F32, got[T.MULTI_ACC["SUM"]])
        assert abs(s - ref["SUM"]) <= F32_RTOL * abs(ref["SUM"]) + 1e-30
        # fused fast path on f32 (f64 accumulation)
        code = bc.filter_sum_program()
        regs = [0, 0, n, T.reg_image(T.F32, 500.0), 8]
        st, want, fast = oracle.engine_run_port(T.F32, code, [col], regs)
        assert fast == 1
        got, _ = run_gpu(T.F32, code, [col], regs)
        assert abs(f64(got[0]) - f64(want[0])) <= F32_RTOL * abs(f64(want[0])) + 1e-30
        assert got[1] == want[1]


def test_templates_match_sql_and_interpreter():
    rng = np.random.default_rng(12)
    for dt in range(6):
        for agg in T.AGGS:
            n = 8 * int(rng.integers(1, 4000))
            col = T.make_column(dt, n, rng)
            prog = T.random_program(dt, rng, agg=agg)
            got, _ = run_gpu(dt, prog.code, [col], prog.registers(n))
            sql = T.sql_reference(prog, col)
            v = got[0] if agg == "COUNT" else T.image_value(dt, got[0])
            if agg == "SUM" and dt in (0, 1):
                assert abs(v - sql) <= (F64_RTOL if dt == 0 else F32_RTOL) * max(abs(sql), 1.0)
            elif agg in ("MIN", "MAX") and dt == T.F32:
                assert v == float(np.float32(sql)) or v == sql
            else:
                assert v == sql, (dt, agg)


def test_edge_sizes_and_offsets():
    rng = np.random.default_rng(13)
    for dt in (0, 2, 3, 5):
        kl = T.K_LANES[dt]
        for n in (0, 1, kl - 1, kl, kl + 1, 255, 256, 257, 1 << 16, (1 << 16) + 3):
            col = T.make_column(dt, n, rng)
            thr = T.reg_image(dt, 500 if dt else 500.0)
            for off0 in (0, 1, kl, 3 * kl + 1):
                regs = [0, off0, n, thr, kl]
                code = bc.filter_sum_program()
                want = oracle.engine_run_ref(dt, code, [col], regs)
                got, _ = run_gpu(dt, code, [col], regs)
                assert_regs(dt, code, got, want[:16], F64_RTOL)


def test_large_column_properties():
    """Full-size property: sum over a 2^27-row column equals the sum of the
    per-chunk sums of the same program (linearity), and the count is exact."""
    rng = np.random.default_rng(14)
    n = 1 << 27
    x = (rng.random(n) * 1000.0)
    thr = T.reg_image(0, 500.0)
    got, e = run_gpu(0, bc.filter_sum_count_program(), [x], [0, 0, n, thr, 4, 0, 0])
    cnt = int((x > 500.0).sum())
    assert got[6] == cnt
    total = f64(got[0])
    parts = 0.0
    for k in range(4):
        sl = x[k * (n // 4):(k + 1) * (n // 4)]
        g, _ = run_gpu(0, bc.filter_sum_program(), [sl], [0, 0, sl.size, thr, 4])
        parts += f64(g[0])
    assert abs(total - parts) <= F64_RTOL * total
    exact = float(np.sum(x[x > 500.0], dtype=np.float64))
    assert abs(total - exact) <= 1e-10 * total


def test_run_parallel_matches_reference():
    rng = np.random.default_rng(15)
    n = 100_003
    x = rng.random(n) * 1000.0
    code = bc.filter_sum_program()
    regs = [0, 0, n, T.reg_image(0, 500.0), 4]
    e = Engine(0)
    e.add_segment(x)
    for i, v in enumerate(regs):
        e.set_scalar(i, v)
    e.load_program(code)
    e.run_parallel(0, 7, 0)
    if oracle.have_ref():
        rin = np.array(regs + [0] * (64 - len(regs)), np.uint64)
        rout = np.zeros(64, np.uint64)
        ptrs, counts = oracle._segs([x])
        c = np.asarray(code, np.uint32)
        oracle.ref().vref_engine_run_parallel(0, c.ctypes.data, c.size, ptrs, counts, 1, rin.ctypes.data, 0, 7, 0,
                                              rout.ctypes.data)
        want = f64(int(rout[0]))
    else:
        chunk = (n + 6) // 7
        want = sum(float(np.sum([v for v in x[t * chunk:t * chunk + (min(chunk, n - t * chunk) // 4) * 4] if v > 500]))
                   for t in range(7))
    got = e.get_scalar_f64(0)
    assert abs(got - want) <= F64_RTOL * want


def test_segment_aggregates(golden):
    """AGG_SUM / AGG_COUNT / AGG_MIN / AGG_MAX over a segment (engine.hpp:499-569)."""
    rng = np.random.default_rng(16)
    for dt in (0, 2, 3):
        col = T.make_column(dt, 10_000, rng)
        code = [bc.agg("SUM", 0, 0, 1), bc.agg("COUNT", 1, 0, 1), bc.agg("MIN", 2, 0, 1), bc.agg("MAX", 3, 0, 1),
                bc.halt()]
        regs = [0, 17, 0, 0]
        st, want, _ = oracle.engine_run_port(dt, code, [col], regs)
        got, _ = run_gpu(dt, code, [col], regs)
        for r in (1, 2, 3):
            assert got[r] == want[r], (dt, r)
        if dt == 0:
            assert abs(f64(got[0]) - f64(want[0])) <= F64_RTOL * f64(want[0])
        else:
            assert got[0] == want[0]


def test_unsupported_program_fails_loudly():
    e = Engine(0)
    e.add_segment(np.zeros(8))
    e.load_program([bc.vload(0, 1, 0), bc.enc(0x80, 6, 6, 0), bc.add(1, 1, 4), bc.cmp(1, 2), bc.jnz(-4), bc.halt()])
    e.set_scalar(2, 8)
    e.set_scalar(4, 4)
    with pytest.raises(VoxelError) as ei:
        e.run()
    assert ei.value.status == 2


def test_multi_reduction_programs_against_reference():
    """Programs with one predicate set and 2-4 aggregates (SUM, COUNT, MIN,
    MAX of the same filter) run on the multi-reduction range kernel and give
    the reference interpreter's registers (f32: the restatement's)."""
    rng = np.random.default_rng(21)
    combos = (["SUM", "COUNT"], ["SUM", "COUNT", "MIN", "MAX"], ["MIN", "MAX"], ["COUNT", "MAX", "SUM"],
              ["MAX", "COUNT"])
    for dt in range(6):
        for aggs in combos:
            for n in (8, 8 * int(rng.integers(2, 600)), 1 << 16, (1 << 20) + 8 * 37):
                base = T.random_program(dt, rng, npreds=int(rng.integers(1, 5)))
                prog = T.build_multi(dt, base.preds, aggs)
                col = T.make_column(dt, n, rng)
                regs = prog.registers(n)
                if dt == T.F32:
                    st, want, _ = oracle.engine_run_port(dt, prog.code, [col], regs)
                    assert st == 0
                else:
                    want = oracle.engine_run_ref(dt, prog.code, [col], regs)
                got, e = run_gpu(dt, prog.code, [col], regs)
                assert "kernel=mrange" in e.explain(), e.explain()
                assert_regs(dt, prog.code, got, want[:16], F32_RTOL if dt == T.F32 else F64_RTOL)


def test_filter_sum_count_all_compares_against_reference():
    """`filter x OP t; SUM(x); COUNT` for every element type and compare op,
    with thresholds at zero, inside the data and NaN, over columns holding
    zeros (and NaN for floats): the fused filter+sum kernel with its count
    gives the reference interpreter's registers (f32: the restatement's)."""
    rng = np.random.default_rng(22)
    for dt in range(6):
        kl = T.K_LANES[dt]
        for op in range(6):
            thresholds = [0, 500, 999] + ([-1] if dt in (T.F64, T.F32, T.I64, T.I32) else [])
            if dt in (T.F64, T.F32):
                thresholds.append(float("nan"))
            for thr in thresholds:
                n = kl * int(rng.integers(1, 5000))
                col = T.make_column(dt, n, rng)
                col[rng.random(n) < 0.05] = 0
                if dt in (T.F64, T.F32):
                    col[rng.random(n) < 0.02] = np.nan
                fold = bc.addf(0, 0, 5) if dt in (T.F64, T.F32) else bc.add(0, 0, 5)
                code = [bc.vload(0, 1, 0), bc.vfilter(op, 1, 0, 3), bc.vsum(5, 1), fold, bc.vcount(7, 1),
                        bc.add(6, 6, 7), bc.add(1, 1, 4), bc.cmp(1, 2), bc.jnz(-8), bc.halt()]
                regs = [0, 0, n, T.reg_image(dt, thr), kl, 0, 0]
                if dt == T.F32:
                    st, want, _ = oracle.engine_run_port(dt, code, [col], regs)
                    assert st == 0
                else:
                    want = oracle.engine_run_ref(dt, code, [col], regs)
                got, e = run_gpu(dt, code, [col], regs)
                assert "kernel=fsum" in e.explain(), e.explain()
                assert_regs(dt, code, got, want[:16], F32_RTOL if dt == T.F32 else F64_RTOL)
