"""The Python front end (voxel_b200/frontend: voxel_query, voxel_sql) on the
GPU against the reference's own query builder (bindings/voxel_query.py) run
on the reference's voxel_py (tests/golden/frontend.json): sums within 1e-12,
counts (as the reference returns them: the integer's bits read as a double),
min / max, sort indices, top-k values and group counts exact.  voxel_sql's
statements compile onto the same queries."""
import json
import os
import struct
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "voxel_b200", "frontend"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import make_frontend_golden as G  # noqa: E402  (input builders only)
import voxel_query as vq  # noqa: E402
import voxel_sql as vsql  # noqa: E402
from voxel_b200.engine import VoxelError  # noqa: E402

pytestmark = pytest.mark.gpu
with open(os.path.join(ROOT, "tests", "golden", "frontend.json")) as f:
    FIX = json.load(f)


def f64(bits):
    return struct.unpack("<d", struct.pack("<Q", bits))[0]


def check(got, want, name):
    if "f64_bits" in want:
        w = f64(want["f64_bits"])
        if got == w:
            return
        # sums: the reference adds row groups in order, the GPU compensated
        assert abs(got - w) <= 1e-12 * abs(w), (name, got, w)
    elif "int" in want:
        assert int(got) == want["int"], name
    else:
        a = np.ascontiguousarray(got)
        assert str(a.dtype) == want["dtype"] and a.size == want["size"], name
        import hashlib
        assert hashlib.sha256(a.tobytes()).hexdigest() == want["digest"], name


def test_query_builder_matches_reference():
    for c in FIX["cases"]:
        x = G.column(c["kind"], c["n"], c["seed"])
        keys = G.keys_for(c["n"], c["seed"])
        chain = [(m, tuple(a)) for m, a in c["chain"]]
        check(G.run_case(vq, chain, x, keys), c["result"], c["name"])
    x = G.column("plain", 4000, 13)
    h = FIX["helpers"]
    check(vq.filter_and_sum(x, 500.0), h["filter_and_sum"], "filter_and_sum")
    check(vq.filter_and_count(x, 500.0), h["filter_and_count"], "filter_and_count")
    check(vq.group_sum(x, G.keys_for(4000, 13)), h["group_sum"], "group_sum")
    check(vq.from_list([1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0, 8.0]).filter_gt(2.5).sum().run(), h["from_list_sum"],
          "from_list")


def test_query_builder_quirks_are_kept():
    x = G.column("plain", 4000, 14)
    c = vq.from_numpy(x).filter_gt(500).count().run()
    assert struct.unpack("<Q", struct.pack("<d", c))[0] == int((x > 500).sum())  # bits of the count
    assert vq.from_numpy(x).min().run() == 0.0  # integer compare from R0 = 0.0
    with pytest.raises(VoxelError):
        vq.from_numpy(x).filter_gt(1).sum().count().run()  # the reference's second loop never ends
    with pytest.raises(VoxelError):
        vq.from_numpy(x[:10]).sum().run()  # 10 rows: the offset never equals the total


def test_sql_statements_compile_onto_the_queries():
    x = G.column("plain", 4000, 13)
    h = FIX["helpers"]
    check(vsql.execute("SELECT SUM(price) FROM t WHERE price > 500", x), h["filter_and_sum"], "sql sum")
    check(vsql.execute("select count(*) from trades where price > 500.0;", {"trades": x}), h["filter_and_count"],
          "sql count")
    # only the last comparison applies, as in the query builder
    a = vsql.execute("SELECT SUM(v) FROM t WHERE v > 100 AND v < 600", x)
    assert a == vq.from_numpy(x).filter_lt(600).sum().run()
    assert vsql.execute("SELECT MAX(v) FROM t", x) == vq.from_numpy(x).max().run()
    idx = vsql.execute("SELECT v FROM t ORDER BY v DESC", x)
    assert (idx == vq.from_numpy(x).sort().run()).all()
    top = vsql.execute("SELECT v FROM t LIMIT 4", x)
    assert (top == np.sort(x)[::-1][:4]).all()
    assert vsql.execute("SELECT SUM(v) FROM (SELECT v FROM t LIMIT 8)", x) == pytest.approx(np.sort(x)[-8:].sum(),
                                                                                            rel=1e-12)
    with pytest.raises(VoxelError):
        vsql.execute("SELECT AVG(v) FROM t", x)  # SUM then COUNT: the reference's second loop never ends


def test_sql_group_by_on_the_gpu(tmp_path):
    x = G.column("plain", 40_000, 15)
    k = G.keys_for(40_000, 15)
    r = vsql.execute("SELECT SUM(v) FROM t WHERE v > 200 AND v <= 900 GROUP BY k", {"t": x, "k": k})
    m = (x > 200) & (x <= 900)
    assert r == {"groups": int(np.unique(k[m]).size), "function": "sum"}
    # OR is taken as AND, as the reference's mask builder does
    r = vsql.execute("SELECT COUNT(v) FROM t WHERE v < 100 OR v > 900 GROUP BY k", {"t": x, "k": k})
    assert r == {"groups": int(np.unique(k[(x < 100) & (x > 900)]).size), "function": "count"}
    ints = np.floor(x / 100.0)
    r = vsql.execute("SELECT MIN(v) FROM t WHERE v = 3 GROUP BY k", {"t": ints, "k": k})
    assert r == {"groups": int(np.unique(k[np.abs(ints - 3) < 1e-10]).size), "function": "min"}
    r = vsql.execute("SELECT SUM(v) FROM t GROUP BY nothere", {"t": x[:1000]})
    assert r == {"groups": 1000, "function": "sum"}  # no key column: row numbers
    p = tmp_path / "data.csv"
    p.write_text("price\n" + "\n".join(f"{v:.17g}" for v in x[:4000]) + "\nbad\n")
    got = vsql.execute(f"SELECT SUM(price) FROM '{p}' WHERE price > 500")
    assert got == pytest.approx(vq.filter_and_sum(np.array(x[:4000]), 500.0), rel=1e-12)
