"""Learned estimator: device sketches, exact (engine-measured) labels, the MLP's
forward pass and gradients against the FP64 oracle, and the gain of the
trained network over the histogram + independence estimator it replaces."""
import numpy as np
import pytest
import torch

from oracle import mlp_ref
from voxel_b200 import capi
from voxel_b200 import estimator as E
from voxel_b200 import templates as T

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def test_sketch_matches_numpy():
    rng = np.random.default_rng(51)
    for dt in range(6):
        col = T.make_column(dt, 300_001, rng)
        d = torch.from_numpy(col).to(DEV)
        sk = E.sketch(dt, d.data_ptr(), col.size)
        x = col.astype(np.float64)
        assert sk.n == col.size and sk.min == x.min() and sk.max == x.max()
        w = (x.max() - x.min()) / 64
        b = np.clip(((x - x.min()) / w).astype(np.int64), 0, 63)
        assert (np.frombuffer(bytes(sk.hist), np.uint64) == np.bincount(b, minlength=64)).all()
        true_d = np.unique(col).size
        est = E.hll_estimate(np.frombuffer(bytes(sk.hll), np.uint8))
        assert abs(est - true_d) <= 0.08 * true_d


def test_exact_labels_match_numpy_and_engine():
    L = E._setup()
    rng = np.random.default_rng(52)
    for dt in range(6):
        col = T.make_column(dt, 8 * 20_000, rng)
        d = torch.from_numpy(col).to(DEV)
        progs = [T.random_program(dt, rng, agg="COUNT") for _ in range(40)]
        sets = (E.PredSet * len(progs))(*[E.pred_set(dt, p.preds) for p in progs])
        rows = np.zeros(len(progs), np.uint64)
        dist = np.zeros(len(progs), np.uint64)
        assert L.voxel_exact_labels_dev(dt, d.data_ptr(), col.size, sets, len(progs), rows.ctypes.data,
                                        dist.ctypes.data) == 0, capi.last_error()
        for p, r, dd in zip(progs, rows, dist):
            m = np.ones(col.size, bool)
            for q in p.preds:
                v = np.float32(q.value) if dt == T.F32 else T.NP[dt](q.value)
                m &= [np.equal, np.not_equal, np.less, np.less_equal, np.greater, np.greater_equal][q.op](col, v)
            assert int(r) == int(m.sum()) and int(dd) == np.unique(col[m]).size
        # the engine's own COUNT of the same programs agrees
        b = L.voxel_batch_create()
        for p in progs:
            regs = np.array(p.registers(col.size), np.uint64)
            code = np.asarray(p.code, np.uint32)
            assert L.voxel_batch_add(b, dt, code.ctypes.data, code.size, regs.ctypes.data, d.data_ptr(), col.size, 0,
                                     0, None) == 0
        assert L.voxel_batch_launch(b, 0, None) == 0 and L.voxel_batch_fetch(b, None) == 0
        for i, r in enumerate(rows):
            out = np.zeros(64, np.uint64)
            cnt = np.zeros(1, np.uint64)
            L.voxel_batch_result(b, i, out.ctypes.data, cnt.ctypes.data, None)
            assert int(out[0]) == int(r) == int(cnt[0])
        L.voxel_batch_destroy(b)


def test_mlp_forward_and_gradients_match_oracle():
    L = E._setup()
    m = E.Model(seed=7)
    p = m.params()
    assert p.size == 11586
    rng = np.random.default_rng(53)
    X = rng.random((100, 48)).astype(np.float32)
    Y = rng.normal(size=(100, 2)).astype(np.float32)
    yhat = m.predict(X)
    want, _, _ = mlp_ref.forward(p, X)
    np.testing.assert_allclose(yhat, want, rtol=1e-4, atol=1e-5)
    dx = torch.from_numpy(X).to(DEV)
    dy = torch.from_numpy(Y).to(DEV)
    idx = torch.arange(100, dtype=torch.int32, device=DEV)
    g = np.zeros(11586, np.float32)
    import ctypes as C
    loss = C.c_float(0)
    assert L.voxel_mlp_grad(m.h, dx.data_ptr(), dy.data_ptr(), idx.data_ptr(), 100, g.ctypes.data, C.byref(loss)) == 0
    wl, wg = mlp_ref.loss_and_grad(p, X, Y)
    assert abs(loss.value - wl) <= 1e-4 * abs(wl)
    scale = np.abs(wg).max()
    assert np.abs(g - wg).max() <= 2e-4 * scale


def test_trained_model_beats_histogram_independence():
    rng = np.random.default_rng(54)
    cols = []
    for i in range(180):
        dt = i % 6
        n = int(2 ** rng.uniform(10, 18)) // 8 * 8
        cols.append((dt, torch.from_numpy(T.make_column(dt, n, rng)).to(DEV)))
    X, Y, meta = E.build_training_set(cols, 60, rng)
    ntr = int(0.8 * len(X))
    model = E.Model(seed=3)
    losses = model.train(X[:ntr], Y[:ntr], epochs=25, batch=256, lr=3e-3)
    assert losses[-1] < losses[0]
    pred = model.predict(X[ntr:])
    q_mlp, q_base = [], []
    for y, (n, rows, dist, base, _) in zip(pred, meta[ntr:]):
        er, ed = E.decode(y, n)
        q_mlp.append(E.q_error(er, rows))
        q_base.append(E.q_error(base[0], rows))
    q_mlp, q_base = np.array(q_mlp), np.array(q_base)
    assert np.median(q_mlp) < np.median(q_base)
    assert np.percentile(q_mlp, 90) < np.percentile(q_base, 90)
