"""The remaining reference C ABI operators on the GPU: HashAggregator object,
one-shot and sort-based group-by, SortOperator index sorts, TopK and the f64
dictionary, each against the reference's known answers and the oracle."""
import math

import numpy as np
import pytest

import inputs
import oracle
from voxel_b200 import capi

pytestmark = pytest.mark.gpu
FAIL = (1 << 64) - 1


def test_agg_object_c_test_kat():
    L = capi.lib()
    keys = np.array([0, 1, 0, 1, 0], np.uint32)
    vals = np.array([10, 20, 30, 40, 50], np.float64)
    a = L.voxel_agg_create()
    L.voxel_agg_init(a, 10)
    L.voxel_agg_accumulate(a, keys.ctypes.data, vals.ctypes.data, 5)
    assert L.voxel_agg_group_count(a) == 2  # c_test.cpp:48-55
    k = np.zeros(2, np.uint32)
    s, mn, mx = (np.zeros(2) for _ in range(3))
    c = np.zeros(2, np.uint64)
    assert L.voxel_agg_results(a, k.ctypes.data, s.ctypes.data, mn.ctypes.data, mx.ctypes.data, c.ctypes.data) == 2
    assert k.tolist() == [0, 1] and s.tolist() == [90.0, 60.0] and c.tolist() == [3, 2]  # test_suite.cpp:432-452
    assert mn.tolist() == [10.0, 20.0] and mx.tolist() == [50.0, 40.0]
    # accumulate is incremental, and growing past the initial capacity keeps every group
    rng = np.random.default_rng(31)
    k2 = rng.integers(0, 5000, size=200_000).astype(np.uint32)
    v2 = rng.random(200_000) * 100
    L.voxel_agg_accumulate(a, k2.ctypes.data, v2.ctypes.data, k2.size)
    allk = np.concatenate([keys, k2])
    assert L.voxel_agg_group_count(a) == np.unique(allk).size
    L.voxel_agg_destroy(a)


def test_groupby_against_reference(golden):
    L = capi.lib()
    for case in golden["ops"]["hashagg"]:
        keys, vals = inputs.group_input(case["n"], case["card"], case["seed"])
        g = case["groups"]
        ng = len(g["keys"])
        ok = np.zeros(ng, np.int32)
        s, mn, mx = (np.zeros(ng) for _ in range(3))
        c = np.zeros(ng, np.uint64)
        got = L.voxel_groupby_i32_f64(keys.ctypes.data, vals.ctypes.data, keys.size, 16, ok.ctypes.data, s.ctypes.data,
                                      mn.ctypes.data, mx.ctypes.data, c.ctypes.data)
        assert got == ng, capi.last_error()
        assert ok.tolist() == g["keys"] and c.tolist() == g["count"]
        assert mn.tolist() == g["min"] and mx.tolist() == g["max"]
        np.testing.assert_allclose(s, g["sum"], rtol=1e-12, atol=0)
        # sort-based plan over the same rows, pre-sorted by key (stable)
        order = np.argsort(keys, kind="stable")
        sk, sv = np.ascontiguousarray(keys[order]), np.ascontiguousarray(vals[order])
        got2 = L.voxel_grouped_sorted_i32_f64(sk.ctypes.data, sv.ctypes.data, sk.size, ok.ctypes.data, s.ctypes.data,
                                              mn.ctypes.data, mx.ctypes.data, c.ctypes.data)
        assert got2 == ng and ok.tolist() == g["keys"] and c.tolist() == g["count"]
        np.testing.assert_allclose(s, g["sum"], rtol=1e-12, atol=0)


def test_groupby_high_cardinality():
    L = capi.lib()
    rng = np.random.default_rng(32)
    n, card = 2_000_000, 1_000_000
    w = np.arange(1, card + 1, dtype=np.float64) ** -1.0
    cdf = np.cumsum(w / w.sum())
    keys = (np.searchsorted(cdf, rng.random(n), side="right") * 37 - 10**7).astype(np.int32)
    vals = rng.random(n) * 1000
    want = oracle.groupby_port(keys, vals)
    ng = want[0].size
    ok = np.zeros(ng, np.int32)
    s, mn, mx = (np.zeros(ng) for _ in range(3))
    c = np.zeros(ng, np.uint64)
    got = L.voxel_groupby_i32_f64(keys.ctypes.data, vals.ctypes.data, n, 1000, ok.ctypes.data, s.ctypes.data,
                                  mn.ctypes.data, mx.ctypes.data, c.ctypes.data)
    assert got == ng and (ok == want[0]).all() and (c == want[4]).all()
    assert (mn == want[2]).all() and (mx == want[3]).all()
    np.testing.assert_allclose(s, want[1], rtol=1e-12, atol=0)


def test_groupby_large_table_mixed_signs_exact():
    """Tables above 2,048 slots accumulate with 192-bit global atomics whose
    returned old values carry into the next word: values of both signs over
    many binades give the correctly rounded group sums, and the oracle's
    keys, counts, min and max, whether the table grew from a small size hint
    or was sized up front."""
    L = capi.lib()
    rng = np.random.default_rng(34)
    n, card = 1_500_000, 200_000
    keys = (rng.integers(0, card, n) * 7 - 700_000).astype(np.int32)
    vals = rng.standard_normal(n) * np.exp(rng.uniform(-20, 20, n))
    want = oracle.groupby_port(keys, vals)
    ng = want[0].size
    order = np.argsort(keys, kind="stable")
    cuts = np.searchsorted(keys[order], want[0], side="left").tolist() + [n]
    sv = vals[order]
    exact = np.array([math.fsum(sv[cuts[g]:cuts[g + 1]]) for g in range(ng)])
    for hint in (16, card):  # grown from a small table, and sized up front
        ok = np.zeros(ng, np.int32)
        s, mn, mx = (np.zeros(ng) for _ in range(3))
        c = np.zeros(ng, np.uint64)
        got = L.voxel_groupby_i32_f64(keys.ctypes.data, vals.ctypes.data, n, hint, ok.ctypes.data, s.ctypes.data,
                                      mn.ctypes.data, mx.ctypes.data, c.ctypes.data)
        assert got == ng, capi.last_error()
        assert (ok == want[0]).all() and (c == want[4]).all()
        assert (mn == want[2]).all() and (mx == want[3]).all()
        np.testing.assert_allclose(s, exact, rtol=1e-14, atol=1e-300)


def test_sort_and_topk(golden):
    L = capi.lib()
    kat = golden["ops"]["sort_kat"]
    d = np.asarray(kat["data"])
    idx = np.zeros(d.size, np.uint32)
    L.voxel_sort_ascending(d.ctypes.data, d.size, idx.ctypes.data)
    assert idx.tolist() == kat["indices"] == [1, 3, 0, 2, 4]  # c_test.cpp:66-68
    t = np.asarray(kat["topk_data"])
    top = np.zeros(3)
    L.voxel_topk(t.ctypes.data, t.size, 3, top.ctypes.data, 1)
    assert top.tolist() == kat["top3"] == [9.0, 6.0, 5.0]  # c_test.cpp:74-76
    rng = np.random.default_rng(33)
    x = np.round(rng.random(300_001) * 1000, 1)  # many ties: stability matters
    x[::7] = -x[::7]
    x[5] = -0.0
    for desc, fn in ((0, L.voxel_sort_ascending), (1, L.voxel_sort_descending)):
        out = np.zeros(x.size, np.uint32)
        fn(x.ctypes.data, x.size, out.ctypes.data)
        if oracle.have_ref():
            want = np.zeros(x.size, np.uint32)
            f = oracle.ref().vref_sort_descending_f64 if desc else oracle.ref().vref_sort_ascending_f64
            f(x.ctypes.data, x.size, want.ctypes.data)
        else:
            want = np.argsort(-x if desc else x, kind="stable").astype(np.uint32)
        assert (out == want).all()
    k = 1000
    top = np.zeros(k)
    L.voxel_topk(x.ctypes.data, x.size, k, top.ctypes.data, 0)
    assert (top == np.sort(x)[:k]).all()


def test_dictionary_f64(golden):
    L = capi.lib()
    d = L.voxel_dict_create()
    data = np.array([1.0, 2.0, 1.0, 2.0, 3.0])
    L.voxel_dict_build(d, data.ctypes.data, 5)
    assert L.voxel_dict_cardinality(d) == 3  # test_suite.cpp:376-389
    out = np.zeros(5)
    L.voxel_dict_decode_batch(d, out.ctypes.data, 0, 5)
    assert (out == data).all()
    # zeros (both signs), negative values, NaNs and integer-valued doubles
    z = np.array([0.0, -0.0, 3.0, -2.0, 0.0, np.nan, 3.0, -2.0, np.nan, 1e-310, 1e-310, -np.inf, np.inf, 0.0])
    z = np.concatenate([z, np.arange(50.0)[np.random.default_rng(35).integers(0, 50, 10_000)]])
    L.voxel_dict_build(d, z.ctypes.data, z.size)
    fin = z[~np.isnan(z)]
    want = np.unique(np.where(fin == 0.0, 0.0, fin)).size + int(np.isnan(z).sum())  # each NaN its own entry
    assert L.voxel_dict_cardinality(d) == want
    out = np.zeros(z.size)
    L.voxel_dict_decode_batch(d, out.ctypes.data, 0, z.size)
    assert ((out == z) | (np.isnan(out) & np.isnan(z))).all()
    rng = np.random.default_rng(34)
    pool = rng.random(777) * 1e6
    x = pool[rng.integers(0, pool.size, 100_000)]
    L.voxel_dict_build(d, x.ctypes.data, x.size)
    card = L.voxel_dict_cardinality(d)
    vals = np.zeros(card)
    L.voxel_dict_values(d, vals.ctypes.data)
    if oracle.have_ref():
        rd = np.zeros(x.size)
        ri = np.zeros(x.size, np.uint32)
        rc = oracle.ref().vref_dict_build_f64(x.ctypes.data, x.size, rd.ctypes.data, ri.ctypes.data)
        assert rc == card and (vals == rd[:rc]).all()
    else:
        assert (vals == np.unique(x)).all()
    out = np.zeros(5000)
    L.voxel_dict_decode_batch(d, out.ctypes.data, 1234, 5000)
    assert (out == x[1234:6234]).all()
    L.voxel_dict_destroy(d)
