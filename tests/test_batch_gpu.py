"""Batched persistent executor: many programs of mixed element types in one
launch (and replayed from a CUDA graph) must reproduce each program run alone
through the engine, the reference interpreter's registers (oracle), and the
exact selection vector; undersized selection buffers are flagged with the
exact count still reported."""
import numpy as np
import pytest
import torch

import oracle
from voxel_b200 import capi
from voxel_b200 import templates as T
from voxel_b200.engine import Engine

pytestmark = pytest.mark.gpu
F64_RTOL = 1e-12


def f64(b):
    return np.array([b], np.uint64).view(np.float64)[0]


def float_acc_regs(code):
    out = set()
    for c in code:
        if c & 0xFF == 0x2A and ((c >> 8) & 0xF) in (((c >> 12) & 0xF), ((c >> 16) & 0xF)):
            out.add((c >> 8) & 0xF)
    return out


def make_batch(progs, cols, caps, want=1, bounds=None):
    """bounds: the loop's row bound per program (default: the column length)."""
    L = capi.lib()
    b = L.voxel_batch_create()
    dev = torch.device("cuda", 0)
    keep = []
    for i, (prog, col, cap) in enumerate(zip(progs, cols, caps)):
        dcol = torch.from_numpy(col).to(dev)
        sel = torch.zeros(max(cap, 1), dtype=torch.int32, device=dev)
        keep += [dcol, sel]
        regs = np.array(prog.registers(bounds[i] if bounds else col.size), np.uint64)
        code = np.asarray(prog.code, np.uint32)
        st = L.voxel_batch_add(b, prog.dtype, code.ctypes.data, code.size, regs.ctypes.data, dcol.data_ptr(), col.size,
                               want, cap, sel.data_ptr())
        assert st == 0, capi.last_error()
    return b, keep


def results(b, i):
    L = capi.lib()
    regs = np.zeros(64, np.uint64)
    cnt = np.zeros(1, np.uint64)
    ovf = np.zeros(1, np.int32)
    assert L.voxel_batch_result(b, i, regs.ctypes.data, cnt.ctypes.data, ovf.ctypes.data) == 0
    return [int(x) for x in regs], int(cnt[0]), int(ovf[0])


def check_regs(dt, code, got, want, rtol=F64_RTOL):
    facc = float_acc_regs(code) if dt in (0, 1) else set()
    for r in range(16):
        if got[r] != want[r]:
            assert r in facc, (dt, r, got[r], want[r])
            g, w = f64(got[r]), f64(want[r])
            assert abs(g - w) <= rtol * max(abs(w), 1e-300)


def test_batch_matches_engine_oracle_and_selection():
    L = capi.lib()
    rng = np.random.default_rng(41)
    progs, cols, masks = [], [], []
    for i in range(96):
        dt = i % 6
        n = int(T.K_LANES[dt] * rng.integers(1, 3000))
        col = T.make_column(dt, n, rng)
        prog = T.random_program(dt, rng)
        progs.append(prog)
        cols.append(col)
        m = np.ones(n, bool)
        for p in prog.preds:
            v = np.float32(p.value) if dt == T.F32 else T.NP[dt](p.value)
            m &= [np.equal, np.not_equal, np.less, np.less_equal, np.greater, np.greater_equal][p.op](col, v)
        masks.append(m)
    caps = [int(m.sum()) for m in masks]
    b, keep = make_batch(progs, cols, caps)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    for use_graph in (0, 1, 1):
        assert L.voxel_batch_launch(b, use_graph, stream.cuda_stream) == 0, capi.last_error()
        assert L.voxel_batch_fetch(b, stream.cuda_stream) == 0, capi.last_error()
        for i, (prog, col, m) in enumerate(zip(progs, cols, masks)):
            regs, cnt, ovf = results(b, i)
            assert cnt == int(m.sum()) and ovf == 0
            sel = keep[2 * i + 1][:cnt].cpu().numpy().astype(np.int64)
            assert (sel == np.flatnonzero(m)).all()
            e = Engine(prog.dtype)
            e.add_segment(col)
            for r, v in enumerate(prog.registers(col.size)):
                e.set_scalar(r, v)
            e.load_program(prog.code)
            e.run()
            check_regs(prog.dtype, prog.code, regs, e.registers(16))
            if prog.dtype != T.F32 and col.size <= 4000:
                want = oracle.engine_run_ref(prog.dtype, prog.code, [col], prog.registers(col.size))
                check_regs(prog.dtype, prog.code, regs, want)
    L.voxel_batch_destroy(b)


def test_batch_overflow_is_flagged_with_exact_count():
    L = capi.lib()
    rng = np.random.default_rng(42)
    col = T.make_column(T.I32, 80_000, rng)
    prog = T.build(T.I32, [T.Pred(2, 500)], "COUNT")  # ~50% of rows
    want = int((col < 500).sum())
    b, keep = make_batch([prog], [col], [want // 3])
    assert L.voxel_batch_launch(b, 1, None) == 0 and L.voxel_batch_fetch(b, None) == 0
    regs, cnt, ovf = results(b, 0)
    assert ovf == 1 and cnt == want and regs[0] == want
    sel = keep[1][: want // 3].cpu().numpy().astype(np.int64)
    assert (sel == np.flatnonzero(col < 500)[: want // 3]).all()
    # the rows past the buffer are in the spill arena: the exact selection
    pool = torch.zeros(want, dtype=torch.int32, device=torch.device("cuda", 0))
    progs = np.zeros(1, np.uint64)
    assert L.voxel_batch_gather_overflow(b, 1, progs.ctypes.data, pool.data_ptr(), None) == 0, capi.last_error()
    assert (pool.cpu().numpy().astype(np.int64) == np.flatnonzero(col < 500)).all()
    L.voxel_batch_destroy(b)


def test_batch_large_columns_properties():
    """Two 2^26-row columns plus small ones in one launch: results equal the
    single-program kernels (integers bit-exact, f64 within 1e-12)."""
    L = capi.lib()
    rng = np.random.default_rng(43)
    progs, cols = [], []
    for dt, n in ((T.F64, 1 << 26), (T.U32, 1 << 26), (T.I64, 1000), (T.F32, 8 * 12345)):
        cols.append(T.make_column(dt, n, rng))
        progs.append(T.random_program(dt, rng, selectivity=0.3))
    b, keep = make_batch(progs, cols, [0] * len(cols), want=0)
    assert L.voxel_batch_launch(b, 1, None) == 0 and L.voxel_batch_fetch(b, None) == 0
    for i, (prog, col) in enumerate(zip(progs, cols)):
        regs, cnt, ovf = results(b, i)
        e = Engine(prog.dtype)
        e.add_segment(col)
        for r, v in enumerate(prog.registers(col.size)):
            e.set_scalar(r, v)
        e.load_program(prog.code)
        e.run()
        check_regs(prog.dtype, prog.code, regs, e.registers(16))
    L.voxel_batch_destroy(b)


def _specials(dt):
    if dt in (T.F64, T.F32):
        fi = np.finfo(T.NP[dt])
        return [np.nan, np.inf, -np.inf, 0.0, -0.0, float(fi.smallest_subnormal), -float(fi.smallest_subnormal),
                float(fi.tiny), float(fi.max), float(fi.min), 1.0, -1.0, 2.5, -7.25]
    ii = np.iinfo(T.NP[dt])
    return [int(ii.min), int(ii.min) + 1, int(ii.max) - 1, int(ii.max), 0, 1, 2, 7] + ([-1, -7] if ii.min < 0 else [])


def test_batch_range_form_edge_cases():
    """Programs the executor rewrites as lo <= x <= hi (plus excluded values):
    NaN / +-0 / +-inf / subnormal data and thresholds, thresholds at the type's
    extremes (x < lowest, x > highest), empty intervals and repeated or NaN
    exclusions give the same count, selection vector and registers as the
    single-program engine.  Ragged columns run their loop to the next whole
    group, so the last group's lanes past the column are zero padding (counted
    by the reductions, never selected)."""
    L = capi.lib()
    rng = np.random.default_rng(44)
    progs, cols, masks, bounds = [], [], [], []
    for dt in range(6):
        sp = _specials(dt)
        flt = dt in (T.F64, T.F32)
        for k in range(24):
            kl = T.K_LANES[dt]
            n = int(kl * rng.integers(40, 400) + (k % kl))  # ragged tails too
            extra = ([float(v) for v in rng.uniform(-10, 10, 8)] if flt else
                     [int(v) for v in rng.integers(-10 if dt in (T.I64, T.I32) else 0, 10, 8)])
            vals = np.array(sp + extra, dtype=object)
            col = np.array(list(rng.choice(vals, n)), dtype=T.NP[dt])
            npred = int(rng.integers(1, 5))
            preds = [T.Pred(int(rng.integers(0, 6)), rng.choice(vals)) for _ in range(npred)]
            if k % 6 == 0:  # an empty interval
                t = rng.choice(vals)
                preds = [T.Pred(5, t), T.Pred(2, t)]
            if k % 6 == 1 and npred < 4:  # a repeated exclusion
                preds += [T.Pred(1, preds[0].value)]
            prog = T.build(dt, preds, T.AGGS[k % 4])
            m = np.ones(n, bool)
            with np.errstate(invalid="ignore", over="ignore"):
                for p in preds:
                    v = np.float32(p.value) if dt == T.F32 else T.NP[dt](p.value)
                    m &= [np.equal, np.not_equal, np.less, np.less_equal, np.greater, np.greater_equal][p.op](col, v)
            progs.append(prog)
            cols.append(col)
            masks.append(m)
            bounds.append(-(-n // kl) * kl)
    caps = [int(m.sum()) for m in masks]
    b, keep = make_batch(progs, cols, caps, bounds=bounds)
    forms = [L.voxel_batch_form(b, i) for i in range(len(progs))]
    assert sum(f > 0 for f in forms) >= len(progs) * 3 // 4  # most take the range form
    assert L.voxel_batch_launch(b, 1, None) == 0 and L.voxel_batch_fetch(b, None) == 0, capi.last_error()
    for i, (prog, col, m) in enumerate(zip(progs, cols, masks)):
        regs, cnt, ovf = results(b, i)
        assert cnt == int(m.sum()) and ovf == 0, (i, forms[i], prog.preds)
        sel = keep[2 * i + 1][:cnt].cpu().numpy().astype(np.int64)
        assert (sel == np.flatnonzero(m)).all(), (i, forms[i], prog.preds)
        e = Engine(prog.dtype)
        e.add_segment(col)
        for r, v in enumerate(prog.registers(bounds[i])):
            e.set_scalar(r, v)
        e.load_program(prog.code)
        e.run()
        # the single-program engine takes the same range form, so the reference
        # interpreter (the restated one for f32, which has no reference engine)
        # is the independent check for both
        if prog.dtype == T.F32:
            st_, oracle_regs, _ = oracle.engine_run_port(prog.dtype, prog.code, [col], prog.registers(bounds[i]))
            assert st_ == 0
        else:
            oracle_regs = oracle.engine_run_ref(prog.dtype, prog.code, [col], prog.registers(bounds[i]))
        facc = float_acc_regs(prog.code) if prog.dtype in (0, 1) else set()
        for want in (e.registers(16), oracle_regs[:16]):
            for r in range(16):
                if regs[r] != want[r]:
                    g, w = f64(regs[r]), f64(want[r])
                    assert r in facc and ((np.isnan(g) and np.isnan(w)) or abs(g - w) <= F64_RTOL * max(abs(w), 1e-300)), \
                        (i, forms[i], prog.preds, prog.agg, r, regs[r], want[r])
    L.voxel_batch_destroy(b)


@pytest.mark.parametrize("margin,slack,spill", [(4.0, 1024, None), (0.0, 0, None), (0.0, 0, 1000)])
def test_learned_batch_run_matches_plain_two_pass(margin, slack, spill):
    """LearnedBatch.run (graph launch, bulk results; a program whose estimated
    buffer was too small gets its rows past the buffer from the spill arena,
    or is re-run exactly when the arena is full) equals one exact two-pass
    launch per program: registers, counts and selection vectors.  With no
    margin every program with a selected row overflows; with a 1000-row arena
    most of those are re-run."""
    from voxel_b200 import batch as B

    rng = np.random.default_rng(45)
    dev = torch.device("cuda", 0)
    progs, cols = [], []
    for i in range(60):
        dt = i % 6
        n = int(T.K_LANES[dt] * rng.integers(1, 20000))
        progs.append(T.random_program(dt, rng))
        cols.append(torch.from_numpy(T.make_column(dt, n, rng)).to(dev))
    stream = torch.cuda.Stream(dev)
    lb = B.LearnedBatch(None, margin=margin, slack=slack, spill_rows=spill)
    for p, c in zip(progs, cols):
        lb.add(p, c)
    lb.prepare(stream)
    plain = B.plain_two_pass(progs, cols, stream)
    for _ in range(2):
        res = lb.run()
        assert len(res) == len(progs)
        if margin == 0.0:
            assert lb.last_timing["overflowed"] == sum(r.count > 0 for r in plain)
            if spill is None:
                assert lb.last_timing["reruns"] == 0
            else:
                assert lb.last_timing["reruns"] > 0
        for a, b in zip(res, plain):
            assert np.array_equal(np.asarray(a.registers, np.uint64), np.asarray(b.registers, np.uint64))
            assert a.count == b.count and torch.equal(a.selection, b.selection)
    lb.close()


def _sum_count_program(dt, p0, p1):
    """Two reductions in one loop over the conjunction of two atoms: SUM into
    r0, COUNT into r3 (the interpreted several-reduction class)."""
    from voxel_b200 import bytecode as bc

    kl = T.K_LANES[dt]
    code = [bc.vsplat(8, 8), bc.vsplat(9, 9), bc.vsplat(12, 12)]
    head = len(code)
    code += [bc.vload(0, 1, 0), bc.vcmp(p0.op, 4, 0, 8), bc.vcmp(p1.op, 5, 0, 9), bc.vand(4, 4, 5),
             bc.vand(6, 4, 0), bc.vsum(5, 6), bc.addf(0, 0, 5) if dt in (T.F64, T.F32) else bc.add(0, 0, 5),
             bc.vand(7, 4, 12), bc.vcount(10, 7), bc.add(3, 3, 10), bc.add(1, 1, 4), bc.cmp(1, 2)]
    code.append(bc.jnz(head - len(code)))
    code.append(bc.halt())
    regs = {0: 0, 1: 0, 3: 0, 4: kl, 8: T.reg_image(dt, p0.value), 9: T.reg_image(dt, p1.value),
            12: T.reg_image(dt, 1)}
    return T.Program(dt, [p0, p1], "SUM", code, regs, 0)


def test_batch_interpreted_classes_with_spill():
    """Programs without a range form (two reductions in one loop, NE-only
    predicates, three NE atoms) run on the interpreted class kernels: counts,
    selection vectors (through buffers a third of the size, the rest from the
    spill arena) and registers equal numpy and the reference interpreter."""
    L = capi.lib()
    rng = np.random.default_rng(46)
    progs, cols, masks = [], [], []
    for i in range(36):
        dt = i % 6
        n = int(T.K_LANES[dt] * rng.integers(200, 30000))
        col = T.make_column(dt, n, rng)
        a, b, c = (float(x) for x in rng.uniform(0, 1000, 3))
        if dt not in (T.F64, T.F32):
            a, b, c = (float(int(x)) for x in (a, b, c))
        kind = i // 6 % 3
        if kind == 0:
            prog = _sum_count_program(dt, T.Pred(5, min(a, b)), T.Pred(2, max(a, b)))
        elif kind == 1:
            prog = T.build(dt, [T.Pred(1, a), T.Pred(1, b)], T.AGGS[i % 4])
        else:
            prog = T.build(dt, [T.Pred(4, min(a, b)), T.Pred(1, a), T.Pred(1, b), T.Pred(1, c)], T.AGGS[i % 4])
        m = np.ones(n, bool)
        for p in prog.preds:
            v = np.float32(p.value) if dt == T.F32 else T.NP[dt](p.value)
            m &= [np.equal, np.not_equal, np.less, np.less_equal, np.greater, np.greater_equal][p.op](col, v)
        progs.append(prog)
        cols.append(col)
        masks.append(m)
    caps = [int(m.sum()) // 3 for m in masks]
    b, keep = make_batch(progs, cols, caps)
    forms = [L.voxel_batch_form(b, i) for i in range(len(progs))]
    assert all(f == 0 for f in forms)  # none has a range form
    assert L.voxel_batch_launch(b, 1, None) == 0 and L.voxel_batch_fetch(b, None) == 0, capi.last_error()
    over = []
    for i, (prog, col, m) in enumerate(zip(progs, cols, masks)):
        regs, cnt, ovf = results(b, i)
        assert cnt == int(m.sum()), i
        if cnt > caps[i]:
            assert ovf == 1, i
            over.append(i)
        if prog.dtype == T.F32:
            st_, want, _ = oracle.engine_run_port(prog.dtype, prog.code, [col], prog.registers(col.size))
            assert st_ == 0
        else:
            want = oracle.engine_run_ref(prog.dtype, prog.code, [col], prog.registers(col.size))
        check_regs(prog.dtype, prog.code, regs, want)
    sizes = [int(masks[i].sum()) for i in over]
    pool = torch.zeros(max(sum(sizes), 1), dtype=torch.int32, device=torch.device("cuda", 0))
    ids = np.asarray(over, np.uint64)
    assert L.voxel_batch_gather_overflow(b, len(over), ids.ctypes.data, pool.data_ptr(), None) == 0, capi.last_error()
    got = pool.cpu().numpy().astype(np.int64)
    off = 0
    for i, sz in zip(over, sizes):
        assert (got[off:off + sz] == np.flatnonzero(masks[i])).all(), i
        off += sz
    L.voxel_batch_destroy(b)
