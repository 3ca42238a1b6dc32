"""Serving loop: every request's result is the same run alone (submitted and
awaited one at a time) and run inside a concurrent mix of programs, group-bys
and joins under a tight working-memory budget; and each equals the direct
(non-served) entry points.  Requests larger than the whole budget are refused
with VOXEL_ECAPACITY."""
import numpy as np
import pytest
import torch

from voxel_b200 import capi
from voxel_b200 import templates as T
from voxel_b200.serve import Server, ServerError

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def make_requests(rng):
    progs = []
    for i in range(48):
        dt = i % 6
        kl = T.K_LANES[dt]
        n = max(kl, int(2 ** rng.uniform(8, 20)) // kl * kl)
        col = torch.from_numpy(T.make_column(dt, n, rng)).to(DEV)
        progs.append((T.random_program(dt, rng), col))
    groups = []
    for ng in (10, 1000, 50_000):
        n = ng * 8
        keys = torch.from_numpy((rng.zipf(1.3, n) % ng).astype(np.uint32)).to(DEV)
        vals = torch.from_numpy(rng.normal(size=n) * 100).to(DEV)
        groups.append((keys, vals, ng))
    joins = []
    for nb in (1000, 200_000):
        b = rng.permutation(np.arange(nb * 3, dtype=np.int64))[:nb]
        p = rng.choice(b, size=nb * 10)
        p[rng.random(p.size) < 0.1] = -1
        payload = torch.arange(nb, dtype=torch.int64, device=DEV)
        joins.append((torch.from_numpy(b).to(DEV), payload, torch.from_numpy(p).to(DEV)))
    return progs, groups, joins


def submit_all(srv, progs, groups, joins, order):
    ids, bufs = [], []
    for kind, i in order:
        if kind == "p":
            prog, col = progs[i]
            sel = torch.full((col.numel(),), -1, dtype=torch.int32, device=DEV)
            bufs.append(sel)
            ids.append((kind, i, srv.submit_program(prog, col, want_selection=True, capacity=col.numel(), dsel=sel),
                        sel))
        elif kind == "g":
            keys, vals, ng = groups[i]
            ids.append((kind, i, srv.submit_groupby(keys, vals, ng, capacity=ng), None))
        else:
            b, pay, p = joins[i]
            left = torch.zeros(p.numel(), dtype=torch.int32, device=DEV)
            right = torch.zeros(p.numel(), dtype=torch.int32, device=DEV)
            ids.append((kind, i, srv.submit_join(b, pay, p, left, right, p.numel()), (left, right)))
    return ids


def collect(srv, ids):
    out = {}
    for kind, i, rid, extra in ids:
        r = srv.result(rid)
        if kind == "p":
            r["selection"] = extra[:r["count"]].cpu().numpy()
        elif kind == "j":
            r["left"] = extra[0][:r["count"]].cpu().numpy()
            r["right"] = extra[1][:r["count"]].cpu().numpy()
        r.pop("latency_ms")
        out[(kind, i)] = r
    return out


def same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        if isinstance(a[k], np.ndarray):
            assert a[k].dtype == b[k].dtype and (a[k].view(np.uint8) == b[k].view(np.uint8)).all(), k
        else:
            assert a[k] == b[k], k


def test_results_identical_alone_and_in_the_mix():
    rng = np.random.default_rng(61)
    progs, groups, joins = make_requests(rng)
    order = [("p", i) for i in range(len(progs))] + [("g", i) for i in range(len(groups))] + \
            [("j", i) for i in range(len(joins))]
    with Server(budget_bytes=64 << 20, max_batch=16) as srv:
        alone = {}
        for item in order:
            alone.update(collect(srv, submit_all(srv, progs, groups, joins, [item])))
        mixed_order = list(order) * 2
        rng.shuffle(mixed_order)
        mixed = collect(srv, submit_all(srv, progs, groups, joins, mixed_order))
        st = srv.stats()
        assert st["completed"] >= len(order) * 3
        assert 0 < st["peak_reserved_bytes"] <= 64 << 20
        assert 0 < st["p50_ms"] <= st["p99_ms"]
    for key, want in alone.items():
        same(mixed[key], want)

    # and both equal the direct entry points
    L = capi.lib()
    for i, (prog, col) in enumerate(progs):
        b = L.voxel_batch_create()
        regs = np.array(prog.registers(col.numel()), np.uint64)
        code = np.asarray(prog.code, np.uint32)
        assert L.voxel_batch_add(b, prog.dtype, code.ctypes.data, code.size, regs.ctypes.data, col.data_ptr(),
                                 col.numel(), 0, 0, None) == 0
        assert L.voxel_batch_launch(b, 0, None) == 0 and L.voxel_batch_fetch(b, None) == 0
        out = np.zeros(64, np.uint64)
        cnt = np.zeros(1, np.uint64)
        L.voxel_batch_result(b, 0, out.ctypes.data, cnt.ctypes.data, None)
        L.voxel_batch_destroy(b)
        assert [int(x) for x in out] == alone[("p", i)]["registers"] and int(cnt[0]) == alone[("p", i)]["count"]
        c = col.cpu().numpy()
        m = np.ones(c.size, bool)
        for q in prog.preds:
            v = np.float32(q.value) if prog.dtype == T.F32 else T.NP[prog.dtype](q.value)
            m &= [np.equal, np.not_equal, np.less, np.less_equal, np.greater, np.greater_equal][q.op](c, v)
        assert (alone[("p", i)]["selection"] == np.flatnonzero(m)).all()
    for i, (keys, vals, ng) in enumerate(groups):
        k = keys.cpu().numpy()
        v = vals.cpu().numpy()
        present = np.unique(k)
        r = alone[("g", i)]
        assert (r["keys"] == present).all()
        assert (r["count"] == np.bincount(k, minlength=ng)[present]).all()
        np.testing.assert_allclose(r["sum"], np.bincount(k, weights=v, minlength=ng)[present], rtol=1e-12,
                                   atol=1e-9)
    for i, (b, pay, p) in enumerate(joins):
        left = torch.zeros(p.numel(), dtype=torch.int32, device=DEV)
        right = torch.zeros(p.numel(), dtype=torch.int32, device=DEV)
        cs = torch.zeros(4, dtype=torch.int64, device=DEV)
        assert L.voxel_hashjoin_i64_dev(b.data_ptr(), pay.data_ptr(), b.numel(), p.data_ptr(), p.numel(),
                                        left.data_ptr(), right.data_ptr(), p.numel(), 1, cs.data_ptr(), None) == 0
        m = int(cs[0])
        r = alone[("j", i)]
        assert r["count"] == m and r["aux"] == int(cs[1])
        assert (r["left"] == left[:m].cpu().numpy()).all() and (r["right"] == right[:m].cpu().numpy()).all()


def test_request_larger_than_budget_is_refused():
    rng = np.random.default_rng(62)
    with Server(budget_bytes=1 << 20, max_batch=8) as srv:
        keys = torch.zeros(100_000, dtype=torch.int32, device=DEV)
        vals = torch.zeros(100_000, dtype=torch.float64, device=DEV)
        with pytest.raises(ServerError, match="budget"):
            srv.submit_groupby(keys, vals, 100_000)
        assert capi.lib().voxel_last_status() == 9  # VOXEL_ECAPACITY
        prog = T.random_program(T.F64, rng)
        col = torch.from_numpy(T.make_column(T.F64, 4096, rng)).to(DEV)
        r = srv.result(srv.submit_program(prog, col))
        assert r["count"] >= 0
