"""Learned selectivity / distinct-count estimator (host orchestration).

The column sketches, exact labels, MLP training steps and inference are the
backend's CUDA kernels (voxel_sketch_column_dev, voxel_exact_labels_dev,
voxel_mlp_*).  This module turns a sketch plus a program's predicates into the
48 input features, builds the engine-measured training set, and compares the
model against the estimator it replaces (histogram + independence).

Features (48):
  0-5    element type one-hot
  6      log2(rows + 1) / 32
  7      log2(HLL distinct estimate + 1) / 32
  8-15   the 64-bucket histogram folded into 8 coarse fractions
  16-47  four predicate slots x 8: active, is EQ, is NE, is LT/LE, is GT/GE,
         threshold position in [min, max], histogram CDF at the threshold,
         1 / distinct estimate
Targets (2): ln((selected rows + 1) / (rows + 1)), ln(distinct selected values + 1).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import capi
from . import templates as T

N_FEATURES = 48


class Sketch(C.Structure):
    _fields_ = [("n", C.c_uint64), ("min", C.c_double), ("max", C.c_double), ("hist", C.c_uint64 * 64),
                ("hll", C.c_uint8 * 4096)]


class PredSet(C.Structure):
    _fields_ = [("natoms", C.c_int32), ("op", C.c_int32 * 4), ("pad", C.c_int32), ("thr", C.c_uint64 * 4)]


def _setup():
    L = capi.lib()
    L.voxel_sketch_column_dev.restype = C.c_int
    L.voxel_sketch_column_dev.argtypes = [C.c_int, C.c_void_p, C.c_size_t, C.POINTER(Sketch)]
    L.voxel_exact_labels_dev.restype = C.c_int
    L.voxel_exact_labels_dev.argtypes = [C.c_int, C.c_void_p, C.c_size_t, C.POINTER(PredSet), C.c_uint32,
                                         C.c_void_p, C.c_void_p]
    L.voxel_mlp_param_count.restype = C.c_size_t
    L.voxel_mlp_create.restype = C.c_void_p
    L.voxel_mlp_create.argtypes = [C.c_uint64]
    L.voxel_mlp_destroy.argtypes = [C.c_void_p]
    for f in ("voxel_mlp_set_params", "voxel_mlp_get_params"):
        getattr(L, f).restype = C.c_int
        getattr(L, f).argtypes = [C.c_void_p, C.c_void_p]
    L.voxel_mlp_grad.restype = C.c_int
    L.voxel_mlp_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    L.voxel_mlp_train_step.restype = C.c_int
    L.voxel_mlp_train_step.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_float]
    L.voxel_mlp_infer.restype = C.c_int
    L.voxel_mlp_infer.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]
    return L


def sketch(dtype: int, dcol: int, n: int) -> Sketch:
    L = _setup()
    s = Sketch()
    st = L.voxel_sketch_column_dev(dtype, dcol, n, C.byref(s))
    if st:
        raise RuntimeError(capi.last_error())
    return s


def hll_estimate(regs: np.ndarray) -> float:
    """HyperLogLog cardinality (Flajolet et al. 2007) with the linear-counting
    small-range correction."""
    m = regs.size
    alpha = 0.7213 / (1.0 + 1.079 / m)
    e = alpha * m * m / float(np.sum(np.ldexp(1.0, -regs.astype(np.int64))))
    zeros = int(np.sum(regs == 0))
    if e <= 2.5 * m and zeros:
        e = m * math.log(m / zeros)
    return e


def _cdf(sk: Sketch, hist: np.ndarray, t: float) -> float:
    lo, hi = sk.min, sk.max
    n = max(int(sk.n), 1)
    if hi <= lo:
        return 0.0 if t <= lo else 1.0
    x = (t - lo) / (hi - lo) * 64.0
    if x <= 0:
        return 0.0
    if x >= 64:
        return 1.0
    b = int(x)
    return (float(hist[:b].sum()) + float(hist[b]) * (x - b)) / n


def features(dtype: int, sk: Sketch, preds) -> np.ndarray:
    f = np.zeros(N_FEATURES, np.float32)
    f[dtype] = 1.0
    n = int(sk.n)
    hist = np.frombuffer(bytes(sk.hist), np.uint64).astype(np.float64)
    d = hll_estimate(np.frombuffer(bytes(sk.hll), np.uint8))
    f[6] = math.log2(n + 1) / 32
    f[7] = math.log2(d + 1) / 32
    f[8:16] = hist.reshape(8, 8).sum(axis=1) / max(n, 1)
    span = sk.max - sk.min
    for i, p in enumerate(preds[:4]):
        o = 16 + 8 * i
        f[o] = 1.0
        f[o + 1 + (0 if p.op == 0 else 1 if p.op == 1 else 2 if p.op in (2, 3) else 3)] = 1.0
        t = float(p.value)
        f[o + 5] = np.clip((t - sk.min) / span, -0.1, 1.1) if span > 0 else 0.5
        f[o + 6] = _cdf(sk, hist, t)
        f[o + 7] = 1.0 / max(d, 1.0)
    return f


def baseline_estimate(dtype: int, sk: Sketch, preds):
    """The estimator the model replaces: per-predicate histogram selectivity,
    predicates assumed independent; distinct = HLL * selectivity, capped."""
    n = max(int(sk.n), 1)
    hist = np.frombuffer(bytes(sk.hist), np.uint64).astype(np.float64)
    d = max(hll_estimate(np.frombuffer(bytes(sk.hll), np.uint8)), 1.0)
    sel = 1.0
    for p in preds:
        c = _cdf(sk, hist, float(p.value))
        s = {0: 1.0 / d, 1: 1.0 - 1.0 / d, 2: c, 3: c, 4: 1.0 - c, 5: 1.0 - c}[p.op]
        sel *= min(max(s, 0.0), 1.0)
    rows = sel * n
    return rows, min(d * sel, rows) if rows > 0 else 0.0


def targets(rows: int, n: int, distinct: int):
    return (math.log((rows + 1.0) / (n + 1.0)), math.log(distinct + 1.0))


def decode(y, n: int):
    return (math.exp(float(y[0])) * (n + 1.0) - 1.0, math.exp(float(y[1])) - 1.0)


def q_error(est: float, true: float) -> float:
    e, t = max(est, 0.0) + 1.0, max(true, 0.0) + 1.0
    return max(e / t, t / e)


def pred_set(dtype: int, preds) -> PredSet:
    ps = PredSet()
    ps.natoms = len(preds)
    for i, p in enumerate(preds):
        ps.op[i] = p.op
        if dtype == T.F32:
            ps.thr[i] = int(np.float32(p.value).view(np.uint32))
        else:
            ps.thr[i] = T.reg_image(dtype, p.value)
    return ps


def build_training_set(columns, programs_per_column: int, rng: np.random.Generator):
    """columns: list of (dtype, device tensor); returns X, Y, meta (n, rows, distinct, baseline)."""
    import torch  # noqa: PLC0415

    L = _setup()
    X, Y, meta = [], [], []
    for dtype, dcol in columns:
        n = dcol.numel()
        sk = sketch(dtype, dcol.data_ptr(), n)
        progs = [T.random_program(dtype, rng) for _ in range(programs_per_column)]
        sets = (PredSet * len(progs))(*[pred_set(dtype, p.preds) for p in progs])
        rows = np.zeros(len(progs), np.uint64)
        dist = np.zeros(len(progs), np.uint64)
        st = L.voxel_exact_labels_dev(dtype, dcol.data_ptr(), n, sets, len(progs), rows.ctypes.data, dist.ctypes.data)
        if st:
            raise RuntimeError(capi.last_error())
        for p, r, dd in zip(progs, rows, dist):
            X.append(features(dtype, sk, p.preds))
            Y.append(targets(int(r), n, int(dd)))
            meta.append((n, int(r), int(dd), baseline_estimate(dtype, sk, p.preds), p))
    del torch
    return np.asarray(X, np.float32), np.asarray(Y, np.float32), meta


class Model:
    def __init__(self, seed: int = 1):
        self.L = _setup()
        self.h = self.L.voxel_mlp_create(seed)
        if not self.h:
            raise RuntimeError(capi.last_error())

    def __del__(self):
        try:
            self.L.voxel_mlp_destroy(self.h)
        except Exception:
            pass

    def params(self) -> np.ndarray:
        p = np.zeros(self.L.voxel_mlp_param_count(), np.float32)
        self.L.voxel_mlp_get_params(self.h, p.ctypes.data)
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        self.L.voxel_mlp_set_params(self.h, p.ctypes.data)

    def train(self, X: np.ndarray, Y: np.ndarray, epochs: int = 30, batch: int = 512, lr: float = 2e-3,
              seed: int = 0) -> list:
        import torch  # noqa: PLC0415

        dev = torch.device("cuda", 0)
        dx = torch.from_numpy(np.ascontiguousarray(X)).to(dev)
        dy = torch.from_numpy(np.ascontiguousarray(Y)).to(dev)
        rng = np.random.default_rng(seed)
        losses = []
        n = X.shape[0]
        for ep in range(epochs):
            perm = torch.from_numpy(rng.permutation(n).astype(np.int32)).to(dev)
            for b0 in range(0, n, batch):
                m = min(batch, n - b0)
                idx = perm[b0:b0 + m]
                st = self.L.voxel_mlp_train_step(self.h, dx.data_ptr(), dy.data_ptr(), idx.data_ptr(), m,
                                                 lr * (0.5 if ep >= epochs * 2 // 3 else 1.0))
                if st:
                    raise RuntimeError(capi.last_error())
            losses.append(self.loss(dx, dy))
        torch.cuda.synchronize()
        return losses

    def loss(self, dx, dy) -> float:
        import torch  # noqa: PLC0415

        n = dx.shape[0]
        idx = torch.arange(n, dtype=torch.int32, device=dx.device)
        out = C.c_float(0)
        self.L.voxel_mlp_grad(self.h, dx.data_ptr(), dy.data_ptr(), idx.data_ptr(), n, None, C.byref(out))
        return out.value / n

    def predict(self, X: np.ndarray) -> np.ndarray:
        import torch  # noqa: PLC0415

        dev = torch.device("cuda", 0)
        dx = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(dev)
        dy = torch.zeros((X.shape[0], 2), dtype=torch.float32, device=dev)
        st = self.L.voxel_mlp_infer(self.h, dx.data_ptr(), X.shape[0], dy.data_ptr(), None)
        if st:
            raise RuntimeError(capi.last_error())
        return dy.cpu().numpy()
