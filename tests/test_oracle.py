"""The oracle (CPU restatement) pinned against the reference's golden vectors.

golden.json was produced by running the reference VoxelVM's own interpreter,
JIT and operators (tests/golden/make_golden.py); here the plain-C restatement
in oracle/ must reproduce every one of those outputs.  When the compiled
reference is present (oracle/_ref), random cases are also cross-checked live.
"""
import hashlib
import struct

import numpy as np
import pytest

import inputs
import oracle
from voxel_b200 import bytecode as bc
from voxel_b200 import templates as T


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def f64(bits):
    return struct.unpack("<d", struct.pack("<Q", bits))[0]


def test_known_answers(golden):
    for case in golden["kat"]:
        dt = case["dtype"]
        arrays = [np.asarray(d, dtype=T.NP[dt]) for d in case["data"]]
        st, regs, _ = oracle.engine_run_port(dt, case["code"], arrays, case["regs"])
        assert st == 0
        assert regs[:16] == case["expect"], case["name"]
    # test_suite.cpp:283 / 319 and c_test.cpp:34 values
    assert f64(golden["kat"][0]["expect"][0]) == 26.0
    assert golden["kat"][1]["expect"][0] == 90
    assert f64(golden["kat"][2]["expect"][0]) == 26.0


def test_config1_ground_truth(golden):
    c = golden["config1"]
    x = inputs.mt_uniform(c["seed"], c["n"])
    assert digest(x[:1000]) == c["data_digest"]
    regs = [0, 0, c["n"], T.reg_image(T.F64, c["threshold"]), 4]
    st, r, fast = oracle.engine_run_port(0, bc.filter_sum_program(), [x], regs)
    assert st == 0 and fast == 1
    assert r[0] == c["sum_bits"] == 0x41B662443437BE79  # published: 375,538,740.218
    assert abs(f64(r[0]) - 375538740.218) < 1e-3
    st, r2, fast2 = oracle.engine_run_port(0, bc.filter_sum_count_program(), [x], regs + [0, 0])
    assert st == 0 and fast2 == 0
    assert r2[6] == c["count"] == 500720  # docs/Benchmarks.md:7
    assert r2[0] == c["count_sum_bits"]


def test_program_cases(golden):
    for case in golden["programs"]:
        dt, n = case["dtype"], case["n"]
        col = inputs.column(dt, n, case["seed"])
        st, regs, _ = oracle.engine_run_port(dt, case["code"], [col], case["regs"])
        assert st == 0, case
        assert regs[:16] == case["expect"], (case["kind"], dt, n)


def test_vfilter_and_selection(golden):
    ops = golden["ops"]
    k = ops["vfilter_kat"]
    d = np.asarray(k["data"])
    bm = np.zeros(1, np.uint64)
    cnt = oracle.port().vo_vfilter(0, 4, d.ctypes.data, d.size, T.reg_image(T.F64, 4.0), 0, bm.ctypes.data)
    assert cnt == k["count"] == 4 and int(bm[0]) == k["bitmap"]
    for c in ops["vfilter"]:
        dt, n = c["dtype"], c["n"]
        col = inputs.column(dt, n, c["seed"])
        words = (n + 63) // 64
        bm = np.zeros(max(words, 1), np.uint64)
        a = struct.unpack("<I", struct.pack("<f", c["a"]))[0] if dt == 1 else T.reg_image(dt, c["a"])
        b = struct.unpack("<I", struct.pack("<f", c["b"]))[0] if dt == 1 else T.reg_image(dt, c["b"])
        cnt = oracle.port().vo_vfilter(dt, c["op"], col.ctypes.data, n, a, b, bm.ctypes.data)
        assert cnt == c["count"] and digest(bm[:words]) == c["digest"], c
    for c in ops["selection"]:
        bmp = inputs.bitmap(c["n"], c["seed"])
        out = np.zeros(max(c["n"], 1), np.uint32)
        cnt = oracle.port().vo_selection_from_bitmap(bmp.ctypes.data, c["n"], out.ctypes.data)
        assert cnt == c["count"] and digest(out[:cnt]) == c["digest"]


def test_encodings(golden):
    ops = golden["ops"]
    P = oracle.port()
    for c in ops["bitpack"]:
        v = inputs.u32_values(c["n"], c["maxv"], c["seed"])
        w = P.vo_bitpack_width(v.ctypes.data, v.size)
        assert w == c["width"]
        words = np.zeros(c["nwords"] + 1, np.uint64)
        nw = P.vo_bitpack_build(v.ctypes.data, v.size, w, words.ctypes.data)
        assert nw == c["nwords"] and digest(words[:nw]) == c["words_digest"]
        out = np.zeros(v.size, np.uint32)
        P.vo_bitpack_decode(words.ctypes.data, nw, w, v.size, 0, v.size, out.ctypes.data)
        assert (out == v).all()
    for c in ops["dict"]:
        v = inputs.i32_values(c["n"], c["card"], c["seed"])
        d = np.zeros(v.size, np.int32)
        idx = np.zeros(v.size, np.uint32)
        k = P.vo_dict_build_i32(v.ctypes.data, v.size, d.ctypes.data, idx.ctypes.data)
        assert k == c["cardinality"] and digest(d[:k]) == c["dict_digest"] and digest(idx) == c["idx_digest"]
    for c in ops["rle"]:
        v = inputs.rle_i64(c["n"], c["seed"])
        vals = np.zeros(v.size, np.int64)
        runs = np.zeros(v.size, np.uint32)
        k = P.vo_rle_build_i64(v.ctypes.data, v.size, vals.ctypes.data, runs.ctypes.data)
        assert k == c["runs"] and digest(vals[:k]) == c["values_digest"] and digest(runs[:k]) == c["runs_digest"]
        for dcase in c["decodes"]:
            out = np.zeros(dcase["count"], np.int64)
            P.vo_rle_decode_i64(vals.ctypes.data, runs.ctypes.data, k, dcase["offset"], dcase["count"],
                                out.ctypes.data)
            assert digest(out) == dcase["digest"]


def test_groupby(golden):
    ops = golden["ops"]
    kat = ops["hashagg_kat"]
    k, s, mn, mx, c = oracle.groupby_port(np.asarray(kat["keys"], np.int32), np.asarray(kat["values"]))
    g = kat["groups"]
    assert k.tolist() == g["keys"] and s.tolist() == g["sum"] and c.tolist() == g["count"] == [3, 2]
    for case in ops["hashagg"]:
        keys, vals = inputs.group_input(case["n"], case["card"], case["seed"])
        k, s, mn, mx, c = oracle.groupby_port(keys, vals)
        g = case["groups"]
        assert k.tolist() == g["keys"] and c.tolist() == g["count"]
        assert mn.tolist() == g["min"] and mx.tolist() == g["max"]
        assert s.tolist() == g["sum"]  # same row-order sequential sum: bit-identical


def test_radix_sort(golden):
    for c in golden["ops"]["radix"]:
        k = inputs.sort_keys(c["dtype"], c["n"], c["seed"])
        idx = np.arange(c["n"], dtype=np.uint32)
        oracle.port().vo_radix_sort(c["dtype"], k.ctypes.data, idx.ctypes.data, c["n"])
        assert digest(k) == c["keys_digest"] and digest(idx) == c["idx_digest"], c


def test_hashjoin(golden):
    for c in golden["ops"]["hashjoin"]:
        if c["seed"] == 0:
            b = np.array([1, 2, 3, 4], np.int64)
            p = np.array([2, 4, 6], np.int64)
        else:
            b, p = inputs.join_input(c["nb"], c["np"], c["dup"], c["seed"])
        cap = c["np"] * (8 if c["dup"] else 1) + 8
        l = np.zeros(cap, np.uint32)
        r = np.zeros(cap, np.uint32)
        m = oracle.port().vo_hashjoin_i64(b.ctypes.data, b.size, p.ctypes.data, p.size, l.ctypes.data,
                                          r.ctypes.data, cap, c["all"])
        assert m == c["matches"] and digest(l[:m], r[:m]) == c["digest"], c
    kat = golden["ops"]["hashjoin"][0]
    assert kat["left"] == [0, 1] and kat["right"] == [1, 3]  # test_suite.cpp:471-493


def test_scan_groupby(golden):
    for c in golden["ops"]["scan_groupby"]:
        d = inputs.config2(c["n"], c["seed"])
        k, s, mn, mx, cnt = oracle.scan_groupby_port(d["packed"], d["width"], d["dict"], d["price"], d["qty"],
                                                      20.0, 10, 50)
        assert k.size == c["groups"] and digest(k) == c["keys_digest"] and digest(cnt) == c["count_digest"]
        assert digest(mn) == c["min_digest"] and digest(mx) == c["max_digest"]
        np.testing.assert_allclose(s, c["sums"], rtol=1e-12)


@pytest.mark.skipif(not oracle.have_ref(), reason="compiled reference not present")
def test_restatement_matches_reference_live():
    rng = np.random.default_rng(99)
    for dt in (0, 2, 3, 4, 5):
        for _ in range(6):
            n = int(rng.integers(1, 300)) * T.K_LANES[dt]
            col = T.make_column(dt, n, rng)
            prog = T.random_program(dt, rng)
            regs = prog.registers(n)
            st, mine, _ = oracle.engine_run_port(dt, prog.code, [col], regs)
            assert st == 0
            assert mine == oracle.engine_run_ref(dt, prog.code, [col], regs)


def test_f32_restatement_pinned_to_reference_filters():
    """f32 has no reference engine (Engine<f32> does not compile), so the
    restated f32 programs are pinned to the reference's own f32 operators:
    rows selected by VectorFilter<f32> + ColumnFilter give COUNT exactly,
    MIN / MAX exactly and SUM within 1e-6; for `x > t` the selected values
    equal the reference's scalar_filter_gt_f32 compaction."""
    if not oracle.have_ref():
        pytest.skip("reference library not built")
    rng = np.random.default_rng(31)
    for n in (8, 64, 1000, 8 * 4093):
        col = T.make_column(T.F32, n, rng)
        for aggs in (["SUM"], ["COUNT"], ["MIN"], ["MAX"], ["SUM", "COUNT", "MIN", "MAX"]):
            base = T.random_program(T.F32, rng, npreds=int(rng.integers(1, 5)))
            prog = T.build_multi(T.F32, base.preds, aggs) if len(aggs) > 1 else T.build(T.F32, base.preds, aggs[0])
            st, got, _ = oracle.engine_run_port(T.F32, prog.code, [col], prog.registers(n))
            assert st == 0
            want = oracle.f32_program_expect(base.preds, aggs, col)
            for a in aggs:
                reg = T.MULTI_ACC[a] if len(aggs) > 1 else 0
                v = T.image_value(T.F32, got[reg]) if a != "COUNT" else got[reg]
                if a == "SUM":
                    assert abs(v - want[a]) <= 1e-6 * abs(want[a]) + 1e-30, (a, v, want[a])
                else:
                    assert v == want[a], (a, v, want[a])
        sel = oracle.f32_selection_ref([(4, 500.0)], col)
        assert (col[sel] == oracle.f32_filter_gt_ref(col, 500.0)).all()


def test_codec_restatement_against_reference(golden):
    """The restated delta and frame-of-reference decoders reproduce the
    reference's DeltaEncoding / FrameOfReferenceEncoding outputs (golden
    fixtures, and the live reference build at random offsets)."""
    import ctypes as C

    P = oracle.port()
    np_t = {2: np.int64, 3: np.int32, 4: np.uint64, 5: np.uint32}
    for case in golden["codecs"]["delta"]:
        dt, n = case["dtype"], case["n"]
        w = 8 if dt in (2, 4) else 4
        data = inputs.codec_ints(np_t[dt], n, case["seed"])
        deltas = np.zeros(max(n, 1), np_t[dt])
        P.vo_delta_build(w, data.ctypes.data, n, deltas.ctypes.data)
        assert hashlib.sha256(deltas[:n].tobytes()).hexdigest() == case["deltas_digest"]
        for d in case["decodes"]:
            out = np.zeros(max(d["count"], 1), np_t[dt])
            P.vo_delta_decode(w, deltas.ctypes.data, n, case["base"], d["offset"], d["count"], out.ctypes.data)
            assert hashlib.sha256(out[:d["count"]].tobytes()).hexdigest() == d["digest"]
    for case in golden["codecs"]["frame_of_reference"]:
        n = case["n"]
        if not oracle.have_ref():
            break
        x = inputs.codec_f64(n, case["seed"])
        codes = np.zeros(max(n, 1), np.int32)
        base, scale = C.c_double(), C.c_double()
        oracle.ref().vref_for_build_f64(x.ctypes.data, n, codes.ctypes.data, C.byref(base), C.byref(scale))
        for d in case["decodes"]:
            m = max(0, min(d["count"], n - d["offset"]))
            out = np.zeros(max(m, 1))
            P.vo_for_decode_f64(codes.ctypes.data, n, base.value, scale.value, d["offset"], d["count"],
                                out.ctypes.data)
            assert hashlib.sha256(out[:m].tobytes()).hexdigest() == d["digest"]


def test_join_family_restatement_against_reference(golden):
    """The restated merge / semi / anti joins reproduce the reference's
    MergeJoin (Join, JoinUnique), SemiJoin and AntiJoin outputs (i64 keys;
    the other key types share the algorithm)."""
    P = oracle.port()
    for case in golden["joins"]:
        if case["dtype"] != 2:
            continue
        lk, rk = inputs.merge_join_input(np.int64, case["nl"], case["nr"], case["dup"], case["seed"])
        for unique in (0, 1):
            want = case[f"merge{unique}"]
            cap = max(1, want["matches"])
            lo = np.zeros(cap, np.uint32)
            ro = np.zeros(cap, np.uint32)
            m = P.vo_merge_join_i64(lk.ctypes.data, lk.size, rk.ctypes.data, rk.size, lo.ctypes.data,
                                    ro.ctypes.data, cap, unique)
            assert m == want["matches"]
            assert hashlib.sha256(lo[:m].tobytes() + ro[:m].tobytes()).hexdigest() == want["digest"]
        ls = inputs.shuffled(lk, case["seed"])
        for anti in (0, 1):
            want = case[f"semi{anti}"]
            o = np.zeros(max(ls.size, 1), np.uint32)
            m = P.vo_semi_join_i64(ls.ctypes.data, ls.size, rk.ctypes.data, rk.size, o.ctypes.data, anti)
            assert m == want["matches"] and hashlib.sha256(o[:m].tobytes()).hexdigest() == want["digest"]


def test_window_restatement_against_reference(golden):
    """The restated f64 window functions reproduce the reference's
    Engine<f64>::Window* outputs bit for bit, and TimeWindowSum's buckets."""
    P = oracle.port()
    for c in golden["windows"]["windows"]:
        if c["dtype"] != 0:
            continue
        x = inputs.window_values(0, c["n"], c["seed"])
        o = np.zeros(max(c["out_len"], 1))
        m = P.vo_window_f64(c["kind"], x.ctypes.data, c["n"], o.ctypes.data, c["out_len"], c["window"], c["q"])
        assert m == c["written"], c
        assert hashlib.sha256(o[:m].tobytes()).hexdigest() == c["digest"], c
    for c in golden["windows"]["time_windows"]:
        if c["dtype"] != 0:
            continue
        ts, v = inputs.time_window_input(0, c["n"], c["seed"])
        o = inputs.window_values(0, c["out_len"], c["seed"] + 1)[: c["out_len"]].copy()
        assert hashlib.sha256(o.tobytes()).hexdigest() == c["init_digest"]
        m = P.vo_time_window_sum_f64(ts.ctypes.data, v.ctypes.data, c["n"], c["start"], c["duration"],
                                     o.ctypes.data, c["out_len"])
        assert m == c["returned"]
        for i, val in c["changed"]:
            assert o[i] == val
