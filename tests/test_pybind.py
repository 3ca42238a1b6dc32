"""voxel_py, the pybind module with the reference's Python surface
(bindings/voxel_bindings.cpp): names and encodings on the CPU; every class
run on the GPU against the oracle / numpy."""
import os
import sys

import numpy as np
import pytest

import oracle
from voxel_b200 import bytecode as bc

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "voxel_b200", "lib")
sys.path.insert(0, LIB)
V = pytest.importorskip("voxel_py")


def test_module_surface_and_encoders():
    for name in ("EngineF64", "EngineI64", "EngineF32", "EngineI32", "EngineU64", "EngineU32", "Instruction",
                 "NullBitmap", "DictionaryEncodingF64", "RLEEncodingF64", "VectorFilterF64", "Arena",
                 "HashAggregator", "HashJoin", "sort_ascending", "topk_select", "jit_run", "DataType", "Opcode"):
        assert hasattr(V, name), name
    assert (V.CMP_EQ, V.CMP_NE, V.CMP_LT, V.CMP_LE, V.CMP_GT, V.CMP_GE) == (0, 1, 2, 3, 4, 5)
    assert int(V.DataType.Float64) == 11 and int(V.DataType.Int64) == 5
    I = V.Instruction
    pairs = [(I.vload(0, 1, 0, 0), bc.vload(0, 1, 0)), (I.vfilter_gt(1, 0, 3), bc.vfilter(4, 1, 0, 3)),
             (I.vfilter_ge(1, 0, 3), bc.vfilter(5, 1, 0, 3)), (I.vsum(5, 1), bc.vsum(5, 1)),
             (I.vcount(7, 1), bc.vcount(7, 1)), (I.addf(0, 0, 5), bc.addf(0, 0, 5)), (I.add(1, 1, 4), bc.add(1, 1, 4)),
             (I.sub(1, 1, 4), bc.sub(1, 1, 4)), (I.cmp(1, 2), bc.cmp(1, 2)), (I.jnz(-6), bc.jnz(-6)),
             (I.mov(3, -5), bc.mov(3, -5)), (I.movr(3, 4), bc.movr(3, 4)), (I.halt(), bc.halt())]
    for a, b in pairs:
        assert a.raw == b
    x = I.jnz(-6)
    assert x.op() == 0x52 and x.imm12() == 0xFFA and I.vload(2, 1, 3, 7).imm12() == (3 << 8) | 7
    assert V.EngineF64.k_lanes == 4 and V.EngineU32.k_lanes == 8 and V.EngineF64().k_lanes == 4


@pytest.mark.gpu
def test_engine_and_jit_match_reference_golden(golden):
    c = golden["config1"]
    data = np.empty(c["n"])
    from voxel_b200 import capi

    capi.datagen().vgen_uniform_f64_mt(c["seed"], c["n"], 0.0, 1000.0, data.ctypes.data)
    e = V.EngineF64()
    assert e.add_segment(data) == 0
    e.set_scalar(2, c["n"])
    e.set_scalar_f64(3, c["threshold"])
    e.set_scalar(4, 4)
    e.load_program(bc.filter_sum_program())
    e.run()
    got = e.get_scalar_f64(0)
    want = np.array([c["sum_bits"]], np.uint64).view(np.float64)[0]
    assert abs(got - want) <= 1e-12 * abs(want) and e.get_scalar(1) == c["offset"]
    j = V.jit_run(bc.filter_sum_program(), data, c["threshold"], c["n"])
    assert abs(j - want) <= 1e-12 * abs(want)
    ei = V.EngineI64()
    col = np.arange(1, 1001, dtype=np.int64)
    ei.add_segment(col)
    code = [bc.vload(0, 1, 0), bc.vsum(5, 0), bc.add(0, 0, 5), bc.add(1, 1, 4), bc.cmp(1, 2), bc.jnz(-5), bc.halt()]
    ei.set_scalar(2, 1000)
    ei.set_scalar(4, 4)
    ei.load_program(code)
    ei.run()
    st, want, _ = oracle.engine_run_port(2, code, [col], [0, 0, 1000, 0, 4] + [0] * 59)
    assert st == 0 and ei.get_scalar_i64(0) == 500500 == want[0]


@pytest.mark.gpu
def test_operators():
    rng = np.random.default_rng(71)
    x = rng.random(100_003) * 1000
    bm, c = V.VectorFilterF64().apply_gt(x, 500.0)
    want = np.packbits((x > 500.0).astype(np.uint8), bitorder="little")
    assert c == int((x > 500.0).sum())
    assert (bm.view(np.uint8)[:want.size] == want).all()
    idx = V.sort_ascending(x)
    assert (idx == np.argsort(x, kind="stable")).all()
    assert (V.topk_select(x, 10, True) == np.sort(x)[::-1][:10]).all()
    agg = V.HashAggregator(V.Arena())
    agg.init(100)
    k = rng.integers(0, 100, 50_000).astype(np.uint32)
    v = rng.normal(size=50_000)
    agg.accumulate(k, v)
    assert agg.group_count() == np.unique(k).size
    keys, s, mn, mx, cnt = agg.results()
    assert (keys == np.unique(k)).all() and (cnt == np.bincount(k)[keys]).all()
    np.testing.assert_allclose(s, np.bincount(k, weights=v)[keys], rtol=1e-12, atol=1e-9)
    hj = V.HashJoin(V.Arena())
    hj.build(np.array([1, 2, 3, 4], np.uint32))
    left, right, m = hj.probe(np.array([2, 4, 6], np.uint32))
    assert m == 2 and list(left) == [0, 1] and list(right) == [1, 3]  # examples/test_suite.cpp:471-493
    assert hj.contains(3) and not hj.contains(9)
    d = V.DictionaryEncodingF64()
    y = rng.integers(0, 50, 10_000).astype(np.float64)
    d.build(y)
    assert (d.dictionary == np.unique(y)).all() and d.memory_usage == 50 * 8 + 10_000 * 4
    assert (d.decode_batch(100, 500) == y[100:600]).all()
    r = V.RLEEncodingF64()
    z = np.repeat(rng.random(300), rng.integers(1, 9, 300))
    r.build(z)
    assert (r.decode_batch(7, z.size - 7) == z[7:]).all()
    nb = V.NullBitmap(100)
    nb.set_null(5)
    assert nb.is_null(5) and nb.null_count() == 1 and nb.valid_count() == 99
    nb.set_all_null()
    assert nb.null_count() == 100


def test_jit_compile_and_segment_view():
    """jit_compile reports whether a program lowers onto one fused kernel
    (bindings/voxel_bindings.cpp:329-340; host code, no device work), and
    SegmentF64 is a borrowed view of an f64 buffer (97-103)."""
    r = V.jit_compile(bc.filter_sum_program())
    assert r["compiled"] is True and r["code_size"] > 0 and r["kernel"] == "fsum"
    # jit_run sets R0-R3 only: with R4 = 0 the SUM + COUNT loop never advances,
    # and the reference's JIT compiles only the fused filter+sum pattern
    assert V.jit_compile(bc.filter_sum_count_program()) == {"compiled": False}
    bad = [bc.vload(0, 1, 0), bc.enc(0x80, 6, 6, 0), bc.add(1, 1, 4), bc.cmp(1, 2), bc.jnz(-4), bc.halt()]
    assert V.jit_compile(bad) == {"compiled": False}
    x = np.arange(10, dtype=np.float64) * 1.5
    s = V.SegmentF64(x)
    assert len(s) == 10 and s.size == 10 and s[3] == 4.5
    s2 = V.SegmentF64(x, 4)
    assert len(s2) == 4 and s2[3] == 4.5
    with pytest.raises(IndexError):
        s2[4]
    assert len(V.SegmentF64()) == 0
    for name in ("window_delta", "window_sum", "window_mean", "window_stddev", "window_variance",
                 "window_quantile", "time_window_sum"):
        assert hasattr(V.EngineF64, name), name


@pytest.mark.gpu
def test_engine_f64_window_methods_match_reference():
    """EngineF64's window methods (bindings/voxel_bindings.cpp:127-171) give
    the reference's Engine<f64>::Window* outputs bit for bit."""
    if not oracle.have_ref():
        pytest.skip("reference library not built")
    R = oracle.ref()
    rng = np.random.default_rng(5)
    x = np.cumsum(rng.normal(size=100_003))
    e = V.EngineF64()
    for kind, call in ((0, lambda o: e.window_delta(x, o)), (1, lambda o: e.window_sum(x, o, 9)),
                       (2, lambda o: e.window_mean(x, o, 9)), (3, lambda o: e.window_stddev(x, o, 12)),
                       (4, lambda o: e.window_variance(x, o, 12)), (5, lambda o: e.window_quantile(x, o, 30, 0.75))):
        w, q = {0: (2, 0), 1: (9, 0), 2: (9, 0), 3: (12, 0), 4: (12, 0), 5: (30, 0.75)}[kind]
        want = np.zeros(x.size)
        m = R.vref_window_f64(kind, x.ctypes.data, x.size, want.ctypes.data, x.size, w, q)
        got = np.zeros(x.size)
        assert call(got) == m
        assert (got[:m].view(np.uint64) == want[:m].view(np.uint64)).all(), kind
    ts = np.cumsum(rng.integers(0, 3, 5000)).astype(np.int64)
    v = rng.normal(size=5000)
    want = np.zeros(100)
    m = R.vref_time_window_sum_f64(ts.ctypes.data, v.ctypes.data, 5000, 10, 37, want.ctypes.data, 100)
    got = np.zeros(100)
    assert e.time_window_sum(ts, v, 10, 37, got) == m
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)
