"""Serving loop: every request's result is the same run alone (submitted and
awaited one at a time) and run inside a concurrent mix of programs, group-bys
and joins under a tight working-memory budget; and each equals the reference:
program registers the reference interpreter's (f32: the restatement's, with
its aggregates pinned to the reference's f32 filters), group-by rows
HashAggregator's (keys, counts, min, max exact; sums within 1e-12), join pairs
HashJoin::ProbeAllMatches's in probe order.  Requests larger than the whole
budget are refused with VOXEL_ECAPACITY."""
import struct

import numpy as np
import pytest
import torch

import oracle

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

    # and each equals the reference on the same inputs
    for i, (prog, col) in enumerate(progs):
        c = col.cpu().numpy()
        regs = prog.registers(c.size)
        if prog.dtype == T.F32:
            st, want, _ = oracle.engine_run_port(prog.dtype, prog.code, [c], regs)
            assert st == 0
            ref = oracle.f32_program_expect(prog.preds, [prog.agg], c)[prog.agg]
            got0 = alone[("p", i)]["registers"][0]
            v = T.image_value(T.F32, got0) if prog.agg != "COUNT" else got0
            assert (abs(v - ref) <= 1e-6 * abs(ref) + 1e-30) if prog.agg == "SUM" else v == ref
        else:
            want = oracle.engine_run_ref(prog.dtype, prog.code, [c], regs)
        got = alone[("p", i)]["registers"]
        for r in range(16):
            if got[r] == want[r]:
                continue
            assert prog.dtype in (T.F64, T.F32) and r == 0 and prog.agg == "SUM", (i, r, got[r], want[r])
            g, w = f64(got[r]), f64(want[r])
            assert abs(g - w) <= (1e-6 if prog.dtype == T.F32 else 1e-12) * abs(w), (i, g, w)
        # the selection: the rows the reference's VectorFilter + ColumnFilter pass
        m = np.ones(c.size, bool)
        for q in prog.preds:
            v = np.float32(q.value) if prog.dtype == T.F32 else T.NP[prog.dtype](q.value)
            m &= [np.equal, np.not_equal, np.less, np.less_equal, np.greater, np.greater_equal][q.op](c, v)
        assert (alone[("p", i)]["selection"] == np.flatnonzero(m)).all()
        assert alone[("p", i)]["count"] == int(m.sum())
    L = oracle.ref()
    for i, (keys, vals, ng) in enumerate(groups):
        k = keys.cpu().numpy().astype(np.uint32)
        v = vals.cpu().numpy()
        ok = np.zeros(ng, np.uint32)
        sm, mn, mx = (np.zeros(ng) for _ in range(3))
        cnt = np.zeros(ng, np.uint64)
        g = L.vref_hashagg_u32_f64(k.ctypes.data, v.ctypes.data, k.size, ng, ok.ctypes.data, sm.ctypes.data,
                                   mn.ctypes.data, mx.ctypes.data, cnt.ctypes.data)
        o = np.argsort(ok[:g], kind="stable")
        r = alone[("g", i)]
        assert (r["keys"] == ok[:g][o]).all()
        assert (r["count"] == cnt[:g][o]).all()
        assert (r["min"] == mn[:g][o]).all() and (r["max"] == mx[:g][o]).all()
        np.testing.assert_allclose(r["sum"], sm[:g][o], rtol=1e-12, atol=1e-9)
    for i, (b, pay, p) in enumerate(joins):
        hb = b.cpu().numpy()
        hp = p.cpu().numpy()
        wl = np.zeros(hp.size, np.uint32)
        wr = np.zeros(hp.size, np.uint32)
        m = int(L.vref_hashjoin_i64(hb.ctypes.data, hb.size, hp.ctypes.data, hp.size, wl.ctypes.data,
                                    wr.ctypes.data, hp.size, 1))
        r = alone[("j", i)]
        assert r["count"] == m
        assert (r["left"].view(np.uint32) == wl[:m]).all() and (r["right"].view(np.uint32) == wr[:m]).all()
        assert r["aux"] == int(wr[:m].astype(np.uint64).sum())  # payload = build row id


def f64(b):
    return struct.unpack("<d", struct.pack("<Q", b & 0xFFFFFFFFFFFFFFFF))[0]


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
