"""Full-size parity: the workloads at their full sizes against the reference's
own outputs on the same seeded inputs (tests/golden/fullsize.json, written by
tests/golden/make_fullsize.py from the reference build).

* scan + group-by, 2^25 rows: keys, counts and min/max bit-exact, sums within
  1e-12 relative of HashAggregator's row-order sums;
* radix sort, 2^28 u64 keys + u32 row ids: keys and stable permutation
  bit-exact (SHA-256);
* hash join, 2^24 build x 2^29 probe: match count, payload sum and every
  (probe, build) pair in probe order bit-exact (SHA-256);
* the config-1 program over 2^28 rows: COUNT exact, SUM within 1e-12.
"""
import struct

import numpy as np
import pytest

import fullsize
from voxel_b200 import bytecode as bc
from voxel_b200 import capi
from voxel_b200 import templates as T
from voxel_b200.engine import Engine

pytestmark = pytest.mark.gpu
FS = fullsize.load()
FAIL = (1 << 64) - 1


def need(name):
    if name not in FS:
        pytest.skip(f"tests/golden/fullsize.json has no '{name}' entry (run tests/golden/make_fullsize.py)")
    return FS[name]


def f64(b):
    return struct.unpack("<d", struct.pack("<Q", b & 0xFFFFFFFFFFFFFFFF))[0]


def test_config2_full_size_against_reference():
    want = need("config2")
    d = fullsize.config2_input(want["n"], want["seed"])
    L = capi.lib()
    card = d["dict"].size
    ok = np.zeros(card, np.int32)
    s, mn, mx = (np.zeros(card) for _ in range(3))
    c = np.zeros(card, np.uint64)
    g = L.voxel_scan_groupby(d["packed"].ctypes.data, d["packed"].size, d["width"], d["dict"].ctypes.data, card,
                             d["price"].ctypes.data, d["qty"].ctypes.data, d["n"], fullsize.PTHR, fullsize.QLO,
                             fullsize.QHI, ok.ctypes.data, s.ctypes.data, mn.ctypes.data, mx.ctypes.data,
                             c.ctypes.data)
    assert g == want["groups"], capi.last_error()
    assert fullsize.sha(ok[:g]) == want["keys_sha"]
    assert fullsize.sha(c[:g]) == want["count_sha"]
    assert fullsize.sha(mn[:g]) == want["min_sha"] and fullsize.sha(mx[:g]) == want["max_sha"]
    np.testing.assert_allclose(s[:g], np.asarray(want["sums"]), rtol=1e-12, atol=0)


def test_radix_sort_full_size_against_reference():
    want = need("sort")
    keys = fullsize.sort_input(want["n"], want["seed"])
    idx = np.arange(keys.size, dtype=np.uint32)
    L = capi.lib()
    assert L.voxel_radix_sort(T.U64, keys.ctypes.data, idx.ctypes.data, keys.size) == 0, capi.last_error()
    assert fullsize.sha(keys) == want["keys_sha"]
    assert fullsize.sha(idx) == want["idx_sha"]


def test_hashjoin_full_size_against_reference():
    want = need("join")
    build, probe = fullsize.join_input(want["build"], want["probe"], want["seed_build"], want["seed_probe"])
    left = np.empty(probe.size, np.uint32)
    right = np.empty(probe.size, np.uint32)
    L = capi.lib()
    m = L.voxel_hashjoin_i64(build.ctypes.data, build.size, probe.ctypes.data, probe.size, left.ctypes.data,
                             right.ctypes.data, probe.size, 1)
    assert m != FAIL, capi.last_error()
    assert m == want["matches"]
    assert int(right[:m].astype(np.uint64).sum(dtype=np.uint64)) == want["payload_sum"]
    assert fullsize.sha(left[:m], right[:m]) == want["pairs_sha"]


def test_config1_program_full_size_against_reference():
    want = need("config1")
    x = fullsize.config1_input(want["n"], want["seed"])
    n = x.size
    e = Engine(T.F64)
    e.add_segment(x)
    for i, v in enumerate([0, 0, n, T.reg_image(T.F64, 500.0), 4, 0, 0]):
        e.set_scalar(i, v)
    e.load_program(bc.filter_sum_count_program())
    e.run()
    assert "kernel=fsum" in e.explain()
    assert e.get_scalar(6) == want["sum_count_r6"]
    w = f64(want["sum_count_r0"])
    assert abs(e.get_scalar_f64(0) - w) <= 1e-12 * abs(w)
    e2 = Engine(T.F64)
    e2.add_segment(x)
    for i, v in enumerate([0, 0, n, T.reg_image(T.F64, 500.0), 4]):
        e2.set_scalar(i, v)
    e2.load_program(bc.filter_sum_program())
    e2.run()
    assert e2.get_scalar(1) == want["sum_only_r1"]
    w = f64(want["sum_only_r0"])
    assert abs(e2.get_scalar_f64(0) - w) <= 1e-12 * abs(w)
