"""Learned plan choices (voxel_b200/planner.py) on the GPU: the MLP, trained on
engine-measured labels, sizes the HashAggregator table, picks hash- vs
sort-based GROUP BY and the hash join's build side.  Every plan gives the
same bits -- with the trained model, without a model (the reference's
defaults) and with a deliberately wrong (untrained) model -- and the GROUP BY
rows equal the reference HashAggregator's, the join pairs the reference
HashJoin's.  The q-error of the estimates and the time of each plan are
printed."""
import ctypes as C
import time

import numpy as np
import pytest
import torch

import oracle
from voxel_b200 import estimator as E
from voxel_b200 import planner as P
from voxel_b200 import templates as T

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


@pytest.fixture(scope="module")
def model():
    rng = np.random.default_rng(7)
    cols = []
    g = torch.Generator(device=DEV)
    g.manual_seed(8)
    for i in range(48):
        card = int(2 ** rng.uniform(3, 23))
        n = int(2 ** rng.uniform(18, 22))
        k = torch.randint(0, card, (n,), generator=g, device=DEV, dtype=torch.int64)
        if i % 3 == 2:
            cols.append((T.I64, (k * 7919 - 12345).contiguous()))
        else:
            cols.append((P.U32, k.to(torch.int32).contiguous()))
    X, Y, meta = P.planner_training_set(cols, 24, rng)
    m = E.Model(seed=3)
    m.train(X, Y, epochs=80, batch=256, lr=3e-3, seed=3)
    return m


def groupby_outputs(plan, dk, dv, n, card):
    out = {k: torch.zeros(card, dtype=t, device=DEV) for k, t in
           (("keys", torch.int32), ("sum", torch.float64), ("min", torch.float64), ("max", torch.float64),
            ("count", torch.int64))}
    ptrs = {k: v.data_ptr() for k, v in out.items()}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g = P.run_groupby(plan, dk.data_ptr(), dv.data_ptr(), n, ptrs)
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    return g, {k: v[:g].cpu().numpy() for k, v in out.items()}, secs


def test_groupby_plans_give_identical_bits(model):
    wrong = E.Model(seed=99)  # untrained: estimates unrelated to the data
    rng = np.random.default_rng(11)
    n = 1 << 23
    for card in (200, 60_000, 3_000_000):
        keys = (rng.zipf(1.2, n) % card).astype(np.uint32) if card < 10_000 else rng.integers(0, card, n, np.uint32)
        vals = rng.normal(size=n) * 100
        dk = torch.from_numpy(keys.view(np.int32)).to(DEV)
        dv = torch.from_numpy(vals).to(DEV)
        truth = int(np.unique(keys).size)
        plans = {"model": P.plan_groupby(dk.data_ptr(), n, model),
                 "default": P.plan_groupby(dk.data_ptr(), n, None),
                 "wrong": P.plan_groupby(dk.data_ptr(), n, wrong),
                 "hash-exact": P.GroupByPlan("hash", truth, None, "forced"),
                 "sort": P.GroupByPlan("sort", truth, None, "forced")}
        res, times = {}, {}
        for name, plan in plans.items():
            groupby_outputs(plan, dk, dv, n, truth)  # warm-up (allocations, autotuning)
            g, o, secs = groupby_outputs(plan, dk, dv, n, truth)
            assert g == truth, (name, g, truth)
            res[name], times[name] = o, secs
        base = res["default"]
        for name, o in res.items():
            for k in o:
                assert (o[k].view(np.uint8) == base[k].view(np.uint8)).all(), (card, name, k)
        est = plans["model"].estimated_groups
        q = E.q_error(est, truth)
        print(f"\ngroup-by card {truth}: model est {est:.0f} (q-error {q:.2f}, plan {plans['model'].method}); "
              f"wrong est {plans['wrong'].estimated_groups:.0f}; times ms: " +
              ", ".join(f"{k} {v * 1e3:.2f}" for k, v in times.items()))
        assert q < 4.0, (truth, est)
        if card == 200:  # against the reference HashAggregator on a sample
            m = 1 << 18
            ok = np.zeros(m, np.uint32)
            s, mn, mx = (np.zeros(m) for _ in range(3))
            c = np.zeros(m, np.uint64)
            gg = oracle.ref().vref_hashagg_u32_f64(keys[:m].ctypes.data, vals[:m].ctypes.data, m, 16, ok.ctypes.data,
                                                   s.ctypes.data, mn.ctypes.data, mx.ctypes.data, c.ctypes.data)
            sk = torch.from_numpy(keys[:m].view(np.int32)).to(DEV)
            sv = torch.from_numpy(vals[:m]).to(DEV)
            g2, o2, _ = groupby_outputs(plans["model"], sk, sv, m, int(np.unique(keys[:m]).size))
            order = np.argsort(ok[:gg])
            assert g2 == gg
            assert (o2["keys"].view(np.uint32) == ok[:gg][order]).all()
            assert (o2["count"].view(np.uint64) == c[:gg][order]).all()
            assert (o2["min"] == mn[:gg][order]).all() and (o2["max"] == mx[:gg][order]).all()
            np.testing.assert_allclose(o2["sum"], s[:gg][order], rtol=1e-12, atol=1e-9)


def test_join_build_side_plans_give_the_reference_pairs(model):
    wrong = E.Model(seed=98)
    rng = np.random.default_rng(12)
    nl, nr = 1 << 22, 1 << 22
    right_all = rng.permutation(np.arange(nr, dtype=np.int64) * 3)
    left_all = right_all[rng.integers(0, nr, nl)]
    left_all[rng.random(nl) < 0.2] = -5  # misses
    dl_all = torch.from_numpy(left_all).to(DEV)
    dr_all = torch.from_numpy(right_all).to(DEV)
    cut = int(0.05 * 3 * nr)
    lp = [T.Pred(2, cut)]                    # left keys < 5% of the range: a small side after the filter
    rp = [T.Pred(5, 0.0)]                    # right: every key >= 0
    words = lambda n: (n + 63) // 64  # noqa: E731
    sides = {}
    for name, (d, n, preds) in (("left", (dl_all, nl, lp)), ("right", (dr_all, nr, rp))):
        bms = [torch.zeros(words(n), dtype=torch.int64, device=DEV) for _ in preds]
        band = torch.zeros(words(n), dtype=torch.int64, device=DEV)
        rows = torch.zeros(n, dtype=torch.int32, device=DEV)
        k = P.select_rows(T.I64, d.data_ptr(), n, preds, [b.data_ptr() for b in bms], band.data_ptr(),
                          rows.data_ptr())
        sides[name] = (d[rows[:k].long()].contiguous(), k, rows[:k])
    (dl, kl, rows_l), (dr, kr, rows_r) = sides["left"], sides["right"]
    hl = left_all[left_all < cut]
    hr = right_all[right_all >= 0]
    assert kl == hl.size and kr == hr.size
    cap = kl + 16
    results, times = {}, {}
    plans = {"model": P.plan_join((T.I64, dl_all.data_ptr(), nl, lp), (T.I64, dr_all.data_ptr(), nr, rp), model),
             "default": P.plan_join((T.I64, dl_all.data_ptr(), nl, lp), (T.I64, dr_all.data_ptr(), nr, rp), None),
             "wrong": P.plan_join((T.I64, dl_all.data_ptr(), nl, lp), (T.I64, dr_all.data_ptr(), nr, rp), wrong),
             "left-forced": P.JoinPlan("left", 0, 0, "forced")}
    for name, plan in plans.items():
        lo = torch.zeros(cap, dtype=torch.int32, device=DEV)
        ro = torch.zeros(cap, dtype=torch.int32, device=DEV)
        ta = torch.zeros(cap, dtype=torch.int32, device=DEV)
        tb = torch.zeros(cap, dtype=torch.int32, device=DEV)
        for rep in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            m = P.run_join(plan, dl.data_ptr(), kl, dr.data_ptr(), kr, lo.data_ptr(), ro.data_ptr(), cap,
                           ta.data_ptr(), tb.data_ptr())
            torch.cuda.synchronize()
            times[name] = time.perf_counter() - t0
        results[name] = (lo[:m].cpu().numpy(), ro[:m].cpu().numpy())
    wl = np.zeros(cap, np.uint32)
    wr = np.zeros(cap, np.uint32)
    wm = oracle.ref().vref_hashjoin_i64(hr.ctypes.data, hr.size, hl.ctypes.data, hl.size, wl.ctypes.data,
                                         wr.ctypes.data, cap, 1)
    for name, (a, b) in results.items():
        assert a.size == wm and (a.view(np.uint32) == wl[:wm]).all() and (b.view(np.uint32) == wr[:wm]).all(), name
    ql = E.q_error(plans["model"].estimated_left, kl)
    print(f"\njoin: filtered left {kl} (model est {plans['model'].estimated_left:.0f}, q-error {ql:.2f}), right {kr}; "
          f"model builds {plans['model'].build}, wrong builds {plans['wrong'].build}; times ms: " +
          ", ".join(f"{k} {v * 1e3:.2f}" for k, v in times.items()))
    assert plans["model"].build == "left" and plans["default"].build == "right"
    assert ql < 4.0
