"""Generate tests/golden/golden.json from the reference VoxelVM itself.

Runs the reference's own interpreter, JIT and operators (compiled from its
sources by oracle/build_oracle.py into oracle/_ref) on small seeded inputs and
records their outputs.  Inputs are either stored inline or regenerated from a
numpy PCG64 seed (tests/golden/inputs.py), so the fixture stays small.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import ctypes as C

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import oracle  # noqa: E402
from oracle import build_oracle  # noqa: E402
from voxel_b200 import bytecode as bc  # noqa: E402
from voxel_b200 import templates as T  # noqa: E402
import inputs  # noqa: E402

OUT = os.path.join(HERE, "golden.json")


def f64b(x: float) -> int:
    return T.reg_image(T.F64, x)


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def run_ref(dtype, code, arrays, regs):
    return oracle.engine_run_ref(dtype, code, arrays, regs)


def kat_cases():
    out = []
    # examples/test_suite.cpp:254-285 (Engine / f64, Tier-0 because of the leading MOV)
    code = [bc.mov(4, 4), bc.vload(0, 1, 0), bc.vfilter_gt(1, 0, 3), bc.vsum(5, 1), bc.addf(0, 0, 5),
            bc.add(1, 1, 4), bc.cmp(1, 2), bc.jnz(-6), bc.halt()]
    data = [1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0, 8.0]
    regs = [0, 0, 8, f64b(4.0)]
    out.append(dict(name="test_suite_engine_f64", dtype=0, code=code, data=[data], regs=regs,
                    expect=run_ref(0, code, [np.array(data)], regs)[:16]))
    # examples/test_suite.cpp:290-321 (Engine / i64)
    code = [bc.mov(4, 4), bc.vload(0, 1, 0), bc.vfilter_gt(1, 0, 3), bc.vsum(5, 1), bc.add(0, 0, 5),
            bc.add(1, 1, 4), bc.cmp(1, 2), bc.jnz(-6), bc.halt()]
    data = [10, 20, 30, 40]
    regs = [0, 0, 4, 15]
    out.append(dict(name="test_suite_engine_i64", dtype=2, code=code, data=[data], regs=regs,
                    expect=run_ref(2, code, [np.array(data, np.int64)], regs)[:16]))
    # examples/c_test.cpp:14-36 (fused fast path, 26.0); note ADD's rb is kLanes
    code = [bc.vload(0, 1, 0), bc.vfilter_gt(1, 0, 3), bc.vsum(5, 1), bc.addf(0, 0, 5), bc.add(1, 1, 4),
            bc.cmp(1, 2), bc.jnz(-6), bc.halt()]
    regs = [0, 0, 8, f64b(4.0)]
    out.append(dict(name="c_test_interpreter", dtype=0, code=code, data=[[1.0, 2, 3, 4, 5, 6, 7, 8]], regs=regs,
                    expect=run_ref(0, code, [np.arange(1, 9, dtype=np.float64)], regs)[:16]))
    return out


def program_cases():
    cases = []
    rng = np.random.default_rng(7001)
    sizes = [0, 1, 3, 4, 5, 7, 8, 9, 16, 63, 64, 65, 1000, 1003, 4096, 20000]
    for dtype in (0, 2, 3, 4, 5):
        kl = T.K_LANES[dtype]
        for n in sizes:
            seed = int(rng.integers(1 << 31))
            col = inputs.column(dtype, n, seed)
            # fused fast path (any size: the tail is dropped)
            thr = T.reg_image(dtype, 500 if dtype else 500.0)
            for cmp_op in (4, 2, 0):
                code = bc.filter_sum_program(0, cmp_op)
                regs = [0, 0, n, thr, kl]
                cases.append(dict(kind="fast", dtype=dtype, n=n, seed=seed, code=code, regs=regs,
                                  expect=run_ref(dtype, code, [col], regs)[:16]))
            if n % kl:
                continue  # the CMP/JNZ loops below only terminate on whole groups
            if n == 0:
                continue
            code = bc.filter_sum_count_program(0, 4)
            regs = [0, 0, n, thr, kl, 0, 0]
            if dtype != 0:
                code = [c if (c & 0xFF) != 0x2A else bc.add(0, 0, 5) for c in code]
            cases.append(dict(kind="count", dtype=dtype, n=n, seed=seed, code=code, regs=regs,
                              expect=run_ref(dtype, code, [col], regs)[:16]))
            for t in range(3):
                prog = T.random_program(dtype, rng)
                regs = prog.registers(n)
                cases.append(dict(kind="template", dtype=dtype, n=n, seed=seed, code=prog.code, regs=regs,
                                  agg=prog.agg, expect=run_ref(dtype, prog.code, [col], regs)[:16]))
    # chained VFILTERs with VCOUNT, VRED_MIN over filtered lanes, ragged JL loop
    for dtype in (0, 2, 3):
        kl = T.K_LANES[dtype]
        for n in (8, 64, 1003, 4096):
            seed = int(rng.integers(1 << 31))
            col = inputs.column(dtype, n, seed)
            t1, t2 = T.reg_image(dtype, 200 if dtype else 200.0), T.reg_image(dtype, 700 if dtype else 700.0)
            code = [bc.vload(0, 1, 0), bc.vfilter(4, 1, 0, 3, 1), bc.vfilter(2, 2, 1, 6, 2), bc.vsum(5, 2),
                    bc.addf(0, 0, 5) if dtype == 0 else bc.add(0, 0, 5), bc.vcount(7, 2), bc.add(8, 8, 7),
                    bc.vred_min(9, 2), bc.smin(10, 10, 9), bc.vred_max(11, 2), bc.smax(12, 12, 11),
                    bc.add(1, 1, 4), bc.cmp(1, 2), bc.jl(-13), bc.halt()]
            regs = [0, 0, n, t1, kl, 0, t2, 0, 0, 0, 0x7FFFFFFFFFFFFFFF, 0, 0]
            cases.append(dict(kind="chained", dtype=dtype, n=n, seed=seed, code=code, regs=regs,
                              expect=run_ref(dtype, code, [col], regs)[:16]))
    return cases


def config1():
    n = 1_000_000
    x = inputs.mt_uniform(42, n)
    code = bc.filter_sum_program()
    regs = [0, 0, n, f64b(500.0), 4]
    r = run_ref(0, code, [x], regs)
    code2 = bc.filter_sum_count_program()
    r2 = run_ref(0, code2, [x], [0, 0, n, f64b(500.0), 4, 0, 0])
    c = np.array(code, np.uint32)
    j = oracle.ref().vref_jit_run(c.ctypes.data, c.size, x.ctypes.data, n, 500.0)
    return dict(n=n, seed=42, threshold=500.0, sum_bits=r[0], offset=r[1], count=r2[6], count_sum_bits=r2[0],
                jit_bits=f64b(j), data_digest=digest(x[:1000]))


def op_cases():
    L = oracle.ref()
    ops = {}
    # filter.hpp KAT (test_suite.cpp:410-427)
    d = np.array([1.0, 3.0, 5.0, 7.0, 2.0, 4.0, 6.0, 8.0])
    bm = np.zeros(1, np.uint64)
    pc = L.vref_vfilter_f64(4, d.ctypes.data, 8, 4.0, 0.0, bm.ctypes.data)
    ops["vfilter_kat"] = dict(data=d.tolist(), threshold=4.0, bitmap=int(bm[0]), count=int(pc))
    # random filters per type and op, small sizes
    rng = np.random.default_rng(7002)
    fl = []
    for dtype, name in ((0, "f64"), (1, "f32"), (2, "i64"), (3, "i32"), (4, "u64"), (5, "u32")):
        for n in (0, 1, 63, 64, 65, 1000, 4097):
            seed = int(rng.integers(1 << 31))
            col = inputs.column(dtype, n, seed)
            for op in range(7):
                a, b = (300, 600) if dtype >= 2 else (300.0, 600.0)
                words = (n + 63) // 64
                bm = np.zeros(max(words, 1), np.uint64)
                f = getattr(L, f"vref_vfilter_{name}")
                cnt = f(op, col.ctypes.data, n, a, b, bm.ctypes.data)
                fl.append(dict(dtype=dtype, n=n, seed=seed, op=op, a=a, b=b, count=int(cnt),
                               digest=digest(bm[:words])))
    ops["vfilter"] = fl
    # selection vector from a bitmap
    sv = []
    for n in (0, 1, 64, 100, 5000):
        seed = int(rng.integers(1 << 31))
        bmp = inputs.bitmap(n, seed)
        out = np.zeros(max(n, 1), np.uint32)
        c = L.vref_selection_from_bitmap(bmp.ctypes.data, n, out.ctypes.data)
        sv.append(dict(n=n, seed=seed, count=int(c), digest=digest(out[:c])))
    ops["selection"] = sv
    # bit packing + dictionary + RLE round trips (test_suite.cpp:376-405)
    bp = []
    for n, maxv in ((1, 1), (100, 1000), (1000, 1023), (4099, 7), (3000, 2**31)):
        seed = int(rng.integers(1 << 31))
        v = inputs.u32_values(n, maxv, seed)
        words = np.zeros((n * 32 + 63) // 64 + 1, np.uint64)
        nw = C_size()
        w = L.vref_bitpack_build(v.ctypes.data, n, words.ctypes.data, words.size, nw)
        out = np.zeros(n, np.uint32)
        L.vref_bitpack_decode(words.ctypes.data, nw.value, w, n, 0, n, out.ctypes.data)
        bp.append(dict(n=n, maxv=maxv, seed=seed, width=int(w), nwords=int(nw.value),
                       words_digest=digest(words[:nw.value]), decode_ok=bool((out == v).all())))
    ops["bitpack"] = bp
    dc = []
    for n, card in ((5, 3), (1000, 50), (4096, 1000)):
        seed = int(rng.integers(1 << 31))
        v = inputs.i32_values(n, card, seed)
        dic = np.zeros(n, np.int32)
        idx = np.zeros(n, np.uint32)
        k = L.vref_dict_build_i32(v.ctypes.data, n, dic.ctypes.data, idx.ctypes.data)
        dc.append(dict(n=n, card=card, seed=seed, cardinality=int(k), dict_digest=digest(dic[:k]),
                       idx_digest=digest(idx)))
    ops["dict"] = dc
    rl = []
    for n in (1, 6, 1000, 5000):
        seed = int(rng.integers(1 << 31))
        v = inputs.rle_i64(n, seed)
        vals = np.zeros(n, np.int64)
        runs = np.zeros(n, np.uint32)
        k = L.vref_rle_build_i64(v.ctypes.data, n, vals.ctypes.data, runs.ctypes.data)
        dec = []
        for off, cnt in ((0, n), (n // 3, n // 2), (max(n - 3, 0), 10)):
            out = np.zeros(cnt, np.int64)
            L.vref_rle_decode_i64(vals.ctypes.data, runs.ctypes.data, k, off, cnt, out.ctypes.data)
            dec.append(dict(offset=off, count=cnt, digest=digest(out)))
        rl.append(dict(n=n, seed=seed, runs=int(k), values_digest=digest(vals[:k]), runs_digest=digest(runs[:k]),
                       decodes=dec))
    ops["rle"] = rl
    # HashAggregator KAT (test_suite.cpp:432-452) via i32 keys / f64 values
    keys = np.array([0, 1, 0, 1, 0], np.int32)
    vals = np.array([10, 20, 30, 40, 50], np.float64)
    g = agg_ref(keys, vals)
    ops["hashagg_kat"] = dict(keys=keys.tolist(), values=vals.tolist(), groups=g)
    ga = []
    for n, card in ((100, 10), (5000, 1000), (20000, 37)):
        seed = int(rng.integers(1 << 31))
        k, v = inputs.group_input(n, card, seed)
        ga.append(dict(n=n, card=card, seed=seed, groups=agg_ref(k, v)))
    ops["hashagg"] = ga
    # radix sort u64 + u32 payload
    rs = []
    for dtype, name in ((4, "u64"), (5, "u32"), (2, "i64"), (3, "i32")):
        for n in (0, 1, 2, 1000, 5000):
            seed = int(rng.integers(1 << 31))
            k = inputs.sort_keys(dtype, n, seed)
            idx = np.arange(n, dtype=np.uint32)
            getattr(L, f"vref_radix_sort_{name}")(k.ctypes.data, idx.ctypes.data, n)
            rs.append(dict(dtype=dtype, n=n, seed=seed, keys_digest=digest(k), idx_digest=digest(idx)))
    ops["radix"] = rs
    # hash join (test_suite.cpp:471-493 KAT + random with duplicates)
    hj = []
    for nb, np_, dup, seed_all in ((4, 3, False, None), (1000, 5000, False, 1), (500, 3000, True, 2)):
        if seed_all is None:
            b = np.array([1, 2, 3, 4], np.int64)
            p = np.array([2, 4, 6], np.int64)
            seed = 0
        else:
            seed = int(rng.integers(1 << 31))
            b, p = inputs.join_input(nb, np_, dup, seed)
        for all_ in (0, 1):
            cap = np_ * (8 if dup else 1) + 8
            l = np.zeros(cap, np.uint32)
            r = np.zeros(cap, np.uint32)
            m = L.vref_hashjoin_i64(b.ctypes.data, nb, p.ctypes.data, np_, l.ctypes.data, r.ctypes.data, cap, all_)
            hj.append(dict(nb=nb, np=np_, dup=dup, seed=seed, all=all_, matches=int(m),
                           left=l[:m].tolist() if m <= 16 else None, right=r[:m].tolist() if m <= 16 else None,
                           digest=digest(l[:m], r[:m])))
    ops["hashjoin"] = hj
    # sort / topk KAT (c_test.cpp:58-76)
    s = np.array([3.0, 1, 4, 1, 5])
    idx = np.zeros(5, np.uint32)
    L.vref_sort_ascending_f64(s.ctypes.data, 5, idx.ctypes.data)
    tk = np.array([3.0, 1, 4, 1, 5, 9, 2, 6])
    top = np.zeros(3)
    L.vref_topk_f64(tk.ctypes.data, 8, 3, top.ctypes.data, 1)
    ops["sort_kat"] = dict(data=s.tolist(), indices=idx.tolist(), topk_data=tk.tolist(), top3=top.tolist())
    # scan + group-by (config-2 shape, small)
    sg = []
    for n in (1000, 50000):
        seed = int(rng.integers(1 << 31))
        c2 = inputs.config2(n, seed)
        k, sm, mn, mx, cnt, _ = oracle.scan_groupby_ref(c2["packed"], c2["width"], c2["dict"], c2["price"],
                                                         c2["qty"], 20.0, 10, 50, threads=1)
        sg.append(dict(n=n, seed=seed, groups=int(k.size), keys_digest=digest(k), count_digest=digest(cnt),
                       min_digest=digest(mn), max_digest=digest(mx), sums=[float(v) for v in sm]))
    ops["scan_groupby"] = sg
    return ops


def codec_cases():
    """DeltaEncoding<T> and FrameOfReferenceEncoding run by the reference."""
    L = oracle.ref()
    rng = np.random.default_rng(9101)
    delta = []
    for name, dt, npt in (("i64", 2, np.int64), ("i32", 3, np.int32), ("u64", 4, np.uint64), ("u32", 5, np.uint32)):
        for n in (0, 1, 7, 2048, 2049, 50_000):
            seed = int(rng.integers(1 << 31))
            data = inputs.codec_ints(npt, n, seed)
            deltas = np.zeros(max(n, 1), npt)
            base = int(getattr(L, f"vref_delta_build_{name}")(data.ctypes.data, n, deltas.ctypes.data))
            decs = []
            for off, cnt in ((0, n), (0, n + 5), (n // 3, n // 2), (max(n - 1, 0), 4), (n + 2, 3), (5, 0)):
                out = np.zeros(max(cnt, 1), npt)
                getattr(L, f"vref_delta_decode_{name}")(deltas.ctypes.data, n, base, off, cnt, out.ctypes.data)
                decs.append(dict(offset=off, count=cnt, digest=digest(out[:cnt])))
            delta.append(dict(dtype=dt, n=n, seed=seed, base=base, deltas_digest=digest(deltas[:n]), decodes=decs))
    fr = []
    for n in (0, 1, 5, 4096, 100_001):
        seed = int(rng.integers(1 << 31))
        x = inputs.codec_f64(n, seed)
        codes = np.zeros(max(n, 1), np.int32)
        base, scale = C.c_double(), C.c_double()
        L.vref_for_build_f64(x.ctypes.data, n, codes.ctypes.data, C.byref(base), C.byref(scale))
        decs = []
        for off, cnt in ((0, n), (n // 2, n), (n + 1, 2)):
            out = np.zeros(max(cnt, 1))
            L.vref_for_decode_f64(codes.ctypes.data, n, base.value, scale.value, off, cnt, out.ctypes.data)
            m = max(0, min(cnt, n - off))
            decs.append(dict(offset=off, count=cnt, digest=digest(out[:m])))
        fr.append(dict(n=n, seed=seed, base=base.value, scale=scale.value, codes_digest=digest(codes[:n]),
                       decodes=decs))
    return dict(delta=delta, frame_of_reference=fr)


def join_family_cases():
    """MergeJoin (Join, JoinUnique), SemiJoin and AntiJoin run by the reference."""
    L = oracle.ref()
    rng = np.random.default_rng(9201)
    out = []
    for name, dt, npt in (("i64", 2, np.int64), ("i32", 3, np.int32), ("u64", 4, np.uint64), ("u32", 5, np.uint32)):
        for nl, nr, dup in ((0, 5, 1), (5, 0, 1), (1, 1, 1), (300, 200, 1), (2000, 1500, 4), (40_000, 30_000, 3)):
            seed = int(rng.integers(1 << 31))
            lk, rk = inputs.merge_join_input(npt, nl, nr, dup, seed)
            case = dict(dtype=dt, nl=nl, nr=nr, dup=dup, seed=seed)
            for unique in (0, 1):
                cap = max(1, nl * min(max(nr, 1), dup * 4))
                lo = np.zeros(cap, np.uint32)
                ro = np.zeros(cap, np.uint32)
                m = int(getattr(L, f"vref_merge_join_{name}")(lk.ctypes.data, nl, rk.ctypes.data, nr, lo.ctypes.data,
                                                             ro.ctypes.data, unique))
                assert m <= cap
                case[f"merge{unique}"] = dict(matches=m, digest=digest(lo[:m], ro[:m]))
            for anti in (0, 1):
                o = np.zeros(max(nl, 1), np.uint32)
                # the semi / anti joins assume no order: shuffle the left side for them
                ls = inputs.shuffled(lk, seed)
                m = int(getattr(L, f"vref_semi_join_{name}")(ls.ctypes.data, nl, rk.ctypes.data, nr, o.ctypes.data,
                                                            anti))
                case[f"semi{anti}"] = dict(matches=m, digest=digest(o[:m]))
            out.append(case)
    return out


def window_cases():
    """Engine<T>::Window* and TimeWindowSum run by the reference."""
    L = oracle.ref()
    rng = np.random.default_rng(9301)
    out = []
    for name, dt in (("f64", 0), ("i64", 2), ("i32", 3), ("u64", 4), ("u32", 5)):
        for n in (0, 1, 3, 9, 1000, 70_001):
            seed = int(rng.integers(1 << 31))
            x = inputs.window_values(dt, n, seed)
            for kind in range(6):
                for w, q in ((1, 0.5), (2, 0.0), (3, 1.0), (8, 0.25), (37, 0.9), (255, 0.5)):
                    if kind == 0 and w != 2:
                        continue
                    for out_len in (n, max(n // 3, 1)):
                        o = np.zeros(max(out_len, 1), x.dtype)
                        m = int(getattr(L, f"vref_window_{name}")(kind, x.ctypes.data, n, o.ctypes.data, out_len, w,
                                                                 q))
                        out.append(dict(dtype=dt, n=n, seed=seed, kind=kind, window=w, q=q, out_len=out_len,
                                        written=m, digest=digest(o[:m])))
    tw = []
    for name, dt in (("f64", 0), ("i64", 2), ("i32", 3), ("u64", 4), ("u32", 5)):
        for n, dur, start in ((0, 10, 0), (100, 7, 3), (5000, 60, -100), (50_000, 1, 0)):
            seed = int(rng.integers(1 << 31))
            ts, v = inputs.time_window_input(dt, n, seed)
            for out_len in (1, 64, 10_000):
                if dt == 0 and n * out_len > 100_000_000:
                    continue  # f64 buckets are stored as values: keep the fixture small
                o = np.zeros(out_len, v.dtype)
                o[:] = inputs.window_values(dt, out_len, seed + 1)[:out_len] if out_len else o
                o0 = o.copy()
                m = int(getattr(L, f"vref_time_window_sum_{name}")(ts.ctypes.data, v.ctypes.data, n, start, dur,
                                                                  o.ctypes.data, out_len))
                changed = np.flatnonzero(o != o0) if dt == 0 else np.zeros(0, np.int64)
                tw.append(dict(dtype=dt, n=n, seed=seed, start=start, duration=dur, out_len=out_len, returned=m,
                               changed=[[int(i), float(o[i])] for i in changed] if dt == 0 else None,
                               digest=digest(o) if dt != 0 else None, init_digest=digest(o0)))
    return dict(windows=out, time_windows=tw)


def C_size():
    import ctypes
    return ctypes.c_size_t(0)


def agg_ref(keys, vals):
    L = oracle.ref()
    n = keys.size
    ok = np.zeros(max(n, 1), np.int32)
    s, mn, mx = (np.zeros(max(n, 1)) for _ in range(3))
    c = np.zeros(max(n, 1), np.uint64)
    g = L.vref_hashagg_i32_f64(keys.ctypes.data, vals.ctypes.data, n, 16, ok.ctypes.data, s.ctypes.data,
                               mn.ctypes.data, mx.ctypes.data, c.ctypes.data)
    o = np.argsort(ok[:g], kind="stable")
    return dict(keys=ok[:g][o].tolist(), sum=s[:g][o].tolist(), min=mn[:g][o].tolist(), max=mx[:g][o].tolist(),
                count=[int(x) for x in c[:g][o]])


def main():
    build_oracle.build()
    if not oracle.have_ref():
        raise SystemExit("the reference library is required to generate golden vectors")
    doc = dict(source="reference VoxelVM operators compiled by oracle/build_oracle.py",
               kat=kat_cases(), config1=config1(), programs=program_cases(), ops=op_cases(),
               codecs=codec_cases(), joins=join_family_cases(), windows=window_cases())
    with open(OUT, "w") as f:
        json.dump(doc, f, separators=(",", ":"))
    print(f"wrote {OUT}: {len(doc['programs'])} program cases, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()
