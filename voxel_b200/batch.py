"""Batched execution of many bytecode programs with learned output sizing.

Each program is one filter/aggregate loop over one device-resident column.  A
`LearnedBatch` runs all of them in one persistent launch of the batched
executor (`voxel_batch_*`, replayed from a CUDA graph) and also writes each
program's selection vector (the ascending row ids that satisfy all of its
predicates).  Selection buffers are sized from the learned estimator: every
column is sketched once on the device, the MLP predicts each program's
selected-row count, and the buffer gets that estimate times a margin.  The
estimate never changes a result: the executor always reports the exact count,
and a program whose buffer was too small is re-run with a buffer of exactly
that size (count, then write).

`plain_two_pass` is the baseline the batch replaces: one launch per program to
count, then one more to write into an exactly sized buffer.
"""
from __future__ import annotations

from collections.abc import Sequence
from dataclasses import dataclass, field

import numpy as np

from . import capi
from . import estimator as E


class ProgramResult:
    """One program's outputs: its 64 registers after the run, the exact count of
    selected rows and the selection vector (a device int32 view of row ids,
    made on first access)."""

    __slots__ = ("registers", "count", "estimate", "overflowed", "_sel", "_pool", "_off")

    def __init__(self, registers, count, selection=None, estimate=0.0, overflowed=False, pool=None, off=0):
        self.registers = registers
        self.count = count
        self.estimate = estimate
        self.overflowed = overflowed
        self._sel = selection
        self._pool = pool
        self._off = off

    @property
    def selection(self):
        if self._sel is None and self._pool is not None:
            self._sel = self._pool[self._off:self._off + self.count]
        return self._sel

    @selection.setter
    def selection(self, v):
        self._sel = v
        self._pool = None


class BatchResults(Sequence):
    """The results of one batch run, one ProgramResult per program, made on
    access from the host arrays the run fetched (registers, counts, overflow
    flags) and the device selection buffers."""

    def __init__(self, regs, counts, est, overflowed, pool, offs, extra):
        self.registers = regs          # (programs, 64) uint64
        self.counts = counts           # (programs,) uint64
        self._est, self._ovf, self._pool, self._offs, self._extra = est, overflowed, pool, offs, extra
        self._cache = [None] * len(counts)

    def __len__(self):
        return len(self._cache)

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self[k] for k in range(*i.indices(len(self)))]
        r = self._cache[i]
        if r is None:
            pool, off = self._extra.get(i, (self._pool, int(self._offs[i])))
            r = ProgramResult(self.registers[i], int(self.counts[i]), None, float(self._est[i]), bool(self._ovf[i]),
                              pool, off)
            self._cache[i] = r
        return r


def _batch_add(L, b, prog, dcol, n, want, cap, sel_ptr):
    regs = np.array(prog.registers(n), np.uint64)
    code = np.asarray(prog.code, np.uint32)
    st = L.voxel_batch_add(b, prog.dtype, code.ctypes.data, code.size, regs.ctypes.data, dcol.data_ptr(), n, want,
                           cap, sel_ptr)
    if st:
        raise RuntimeError(capi.last_error())


def _batch_out(L, b, i):
    regs = np.zeros(64, np.uint64)
    cnt = np.zeros(1, np.uint64)
    ovf = np.zeros(1, np.int32)
    if L.voxel_batch_result(b, i, regs.ctypes.data, cnt.ctypes.data, ovf.ctypes.data):
        raise RuntimeError(capi.last_error())
    return [int(x) for x in regs], int(cnt[0]), bool(ovf[0])


@dataclass
class LearnedBatch:
    model: "E.Model | None"
    margin: float = 4.0
    slack: int = 1024
    spill_rows: int | None = None  # spill arena rows (None: the library default)
    programs: list = field(default_factory=list)
    columns: list = field(default_factory=list)  # (dtype, device tensor) per program
    sketches: dict = field(default_factory=dict)

    def add(self, program, dcol) -> int:
        self.programs.append(program)
        self.columns.append(dcol)
        return len(self.programs) - 1

    # -- sizing ---------------------------------------------------------------
    def estimates(self) -> np.ndarray:
        """Predicted selected rows per program (sketches are cached per column)."""
        feats = []
        for prog, dcol in zip(self.programs, self.columns):
            key = dcol.data_ptr()
            if key not in self.sketches:
                self.sketches[key] = E.sketch(prog.dtype, dcol.data_ptr(), dcol.numel())
            feats.append(E.features(prog.dtype, self.sketches[key], prog.preds))
        X = np.asarray(feats, np.float32)
        if self.model is None:  # no model: histogram + independence estimate
            return np.array([E.baseline_estimate(p.dtype, self.sketches[c.data_ptr()], p.preds)[0]
                             for p, c in zip(self.programs, self.columns)])
        Y = self.model.predict(X)
        return np.array([E.decode(y, c.numel())[0] for y, c in zip(Y, self.columns)])

    def prepare(self, stream=None):
        """Sizes the buffers and records the batch (one CUDA graph)."""
        import torch  # noqa: PLC0415

        L = capi.lib()
        est = self.estimates()
        caps = [int(min(c.numel(), np.ceil(max(e, 0.0) * self.margin) + self.slack))
                for e, c in zip(est, self.columns)]
        self.est = est
        self.caps = caps
        offs = np.concatenate([[0], np.cumsum(caps)]).astype(np.int64)
        dev = self.columns[0].device
        self.pool = torch.empty(int(offs[-1]) + 1, dtype=torch.int32, device=dev)
        self.offs = offs
        self.b = L.voxel_batch_create()
        if self.spill_rows is not None:
            L.voxel_batch_set_spill_capacity(self.b, int(self.spill_rows))
        base = self.pool.data_ptr()
        for i, (prog, dcol) in enumerate(zip(self.programs, self.columns)):
            _batch_add(L, self.b, prog, dcol, dcol.numel(), 1, caps[i], base + 4 * int(offs[i]))
        self.stream = stream
        return self

    # -- execution ------------------------------------------------------------
    def run(self):
        """One graph launch of every program.  A program whose selection outgrew
        its buffer has the rest in the batch's spill arena and gets an exactly
        sized buffer assembled on the device; only if the arena was full is it
        re-run exactly.  Returns a BatchResults (a sequence of ProgramResult)."""
        import torch  # noqa: PLC0415

        import time  # noqa: PLC0415

        L = capi.lib()
        sh = self.stream.cuda_stream if self.stream is not None else None
        t0 = time.perf_counter()
        if L.voxel_batch_launch(self.b, 1, sh) or L.voxel_batch_fetch(self.b, sh):
            raise RuntimeError(capi.last_error())
        t1 = time.perf_counter()
        n = len(self.programs)
        regs = np.zeros((n, 64), np.uint64)
        cnts = np.zeros(n, np.uint64)
        ovfs = np.zeros(n, np.int32)
        if L.voxel_batch_results_all(self.b, regs.ctypes.data, cnts.ctypes.data, ovfs.ctypes.data):
            raise RuntimeError(capi.last_error())
        redo = np.flatnonzero(ovfs)
        t2 = time.perf_counter()
        extra = {}
        if redo.size:
            # programs whose rows past the estimate-sized buffer all went to the
            # spill arena: assemble buffer + spilled fragments into exact
            # buffers; the rest (arena full) are re-run exactly
            gather = redo[ovfs[redo] == 1]
            rerun = redo[ovfs[redo] != 1]
            for ids, how in ((gather, "gather"), (rerun, "rerun")):
                if not ids.size:
                    continue
                sizes = cnts[ids]
                offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
                pool2 = torch.empty(int(offs[-1]) + 1, dtype=torch.int32, device=self.pool.device)
                idx = ids.astype(np.uint64)
                if how == "gather":
                    st = L.voxel_batch_gather_overflow(self.b, ids.size, idx.ctypes.data, pool2.data_ptr(), sh)
                else:
                    caps = sizes.astype(np.uint64)
                    st = L.voxel_batch_rerun(self.b, ids.size, idx.ctypes.data, caps.ctypes.data, pool2.data_ptr(), sh)
                if st:
                    raise RuntimeError(capi.last_error())
                if how == "rerun":
                    regs2 = np.zeros((n, 64), np.uint64)
                    cnt2 = np.zeros(n, np.uint64)
                    ovf2 = np.zeros(n, np.int32)
                    if L.voxel_batch_results_all(self.b, regs2.ctypes.data, cnt2.ctypes.data, ovf2.ctypes.data):
                        raise RuntimeError(capi.last_error())
                    if ovf2[ids].any() or (cnt2[ids] != sizes).any() or (regs2[ids] != regs[ids]).any():
                        raise RuntimeError("exact re-run disagrees with the batch")
                for k, i in enumerate(ids.tolist()):
                    extra[i] = (pool2, int(offs[k]))  # a view is made on first access
        out = BatchResults(regs, cnts, self.est, ovfs, self.pool, self.offs, extra)
        self.last_timing = {"launch_fetch_ms": (t1 - t0) * 1e3, "results_ms": (t2 - t1) * 1e3,
                            "overflow_ms": (time.perf_counter() - t2) * 1e3, "overflowed": int(redo.size),
                            "reruns": int((ovfs[redo] != 1).sum()) if redo.size else 0}
        return out

    def close(self):
        if getattr(self, "b", None):
            capi.lib().voxel_batch_destroy(self.b)
            self.b = None


def plain_two_pass(programs, columns, stream=None):
    """One launch per program to count, then one to write the selection into an
    exactly sized buffer.  Returns a list of ProgramResult."""
    import torch  # noqa: PLC0415

    L = capi.lib()
    sh = stream.cuda_stream if stream is not None else None
    out = []
    for prog, dcol in zip(programs, columns):
        n = dcol.numel()
        b = L.voxel_batch_create()
        try:
            _batch_add(L, b, prog, dcol, n, 0, 0, None)
            if L.voxel_batch_launch(b, 0, sh) or L.voxel_batch_fetch(b, sh):
                raise RuntimeError(capi.last_error())
            _, cnt, _ = _batch_out(L, b, 0)
        finally:
            L.voxel_batch_destroy(b)
        buf = torch.empty(max(cnt, 1), dtype=torch.int32, device=dcol.device)
        b = L.voxel_batch_create()
        try:
            _batch_add(L, b, prog, dcol, n, 1, cnt, buf.data_ptr())
            if L.voxel_batch_launch(b, 0, sh) or L.voxel_batch_fetch(b, sh):
                raise RuntimeError(capi.last_error())
            regs, cnt2, ovf = _batch_out(L, b, 0)
        finally:
            L.voxel_batch_destroy(b)
        if ovf or cnt2 != cnt:
            raise RuntimeError("write pass disagrees with the count pass")
        out.append(ProgramResult(regs, cnt, buf[:cnt]))
    return out


def train_estimator(columns, runs: int, seed: int = 0, epochs: int = 30, batch: int = 1024, lr: float = 2e-3):
    """Trains the MLP on `runs` engine-measured (exact) selectivities over the
    given (dtype, device column) list.  Returns (model, held-out q-errors of the
    model and of the histogram + independence estimator)."""
    rng = np.random.default_rng(seed)
    per_col = max(1, runs // max(len(columns), 1))
    X, Y, meta = E.build_training_set(columns, per_col, rng)
    n = len(X)
    perm = rng.permutation(n)
    ntr = int(0.9 * n)
    tr, te = perm[:ntr], perm[ntr:]
    model = E.Model(seed=seed + 1)
    model.train(X[tr], Y[tr], epochs=epochs, batch=batch, lr=lr, seed=seed)
    pred = model.predict(X[te])
    q_m, q_b = [], []
    for y, k in zip(pred, te):
        nrows, rows, _, base, _ = meta[k]
        q_m.append(E.q_error(E.decode(y, nrows)[0], rows))
        q_b.append(E.q_error(base[0], rows))
    return model, np.array(q_m), np.array(q_b), n

