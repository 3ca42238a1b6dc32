"""Operator kernels on the GPU against the oracle: VectorFilter / selection
vectors, decoders, radix sort and hash join.  Small cases reproduce the
reference's own outputs (golden fixtures); large cases check size-independent
properties (round trips, sortedness + stability, counts, pair order)."""
import hashlib
import struct

import numpy as np
import pytest

import inputs
import oracle
from voxel_b200 import capi, encode
from voxel_b200 import templates as T

pytestmark = pytest.mark.gpu
FAIL = (1 << 64) - 1


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def bits(dt, v):
    if dt == T.F32:
        return struct.unpack("<I", struct.pack("<f", v))[0]
    return T.reg_image(dt, v)


def vfilter(dt, op, col, a, b):
    n = col.size
    bm = np.zeros(max((n + 63) // 64, 1), np.uint64)
    c = capi.lib().voxel_vfilter(dt, op, col.ctypes.data, n, bits(dt, a), bits(dt, b), bm.ctypes.data)
    assert c != FAIL, capi.last_error()
    return c, bm[: (n + 63) // 64]


def test_vfilter_golden(golden):
    k = golden["ops"]["vfilter_kat"]
    c, bm = vfilter(T.F64, 4, np.asarray(k["data"]), 4.0, 0.0)
    assert c == 4 and int(bm[0]) == k["bitmap"]  # bits 2,3,6,7 (test_suite.cpp:410-427)
    for case in golden["ops"]["vfilter"]:
        col = inputs.column(case["dtype"], case["n"], case["seed"])
        c, bm = vfilter(case["dtype"], case["op"], col, case["a"], case["b"])
        assert c == case["count"] and digest(bm) == case["digest"], case


def test_vfilter_full_size():
    rng = np.random.default_rng(21)
    n = (1 << 25) + 17
    for dt in (T.F64, T.I32):
        col = T.make_column(dt, n, rng)
        c, bm = vfilter(dt, 6, col, 10, 50) if dt == T.I32 else vfilter(dt, 4, col, 20.0, 0.0)
        m = (col >= 10) & (col <= 50) if dt == T.I32 else col > 20.0
        assert c == int(m.sum())
        want = np.packbits(m, bitorder="little")
        got = bm.view(np.uint8)[: want.size]
        assert (got == want).all()


def test_vfilter_four_byte_types_ragged_and_misaligned():
    """4-byte columns against numpy's predicate for every comparison, at ragged
    sizes around the 256-row warp step, with device pointers at and off the
    16-byte boundary; nothing is written past the last bitmap word."""
    import torch

    L = capi.lib()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(23)
    ops = {0: np.equal, 1: np.not_equal, 2: np.less, 3: np.less_equal, 4: np.greater, 5: np.greater_equal}
    for dt, npt, tt in ((T.I32, np.int32, torch.int32), (T.U32, np.uint32, torch.int32), (T.F32, np.float32, torch.float32)):
        for n in (1, 3, 63, 64, 65, 511, 512, 513, 4097, 100_003):
            host = rng.integers(0, 40, n + 4).astype(npt)
            buf = torch.from_numpy(host.view(np.int32) if npt is np.uint32 else host).to(dev)
            for shift in (0, 1, 3):
                col = host[shift:shift + n]
                for op in range(7):
                    a, b = npt(12), npt(30)
                    m = (col >= a) & (col <= b) if op == 6 else ops[op](col, a)
                    words = (n + 63) // 64
                    bm = torch.zeros(words + 1, dtype=torch.int64, device=dev)
                    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
                    st = L.voxel_vfilter_dev(dt, op, buf.data_ptr() + 4 * shift, n, bits(dt, a), bits(dt, b), bm.data_ptr(),
                                             cnt.data_ptr(), None)
                    assert st == 0, capi.last_error()
                    torch.cuda.synchronize()
                    want = np.packbits(m, bitorder="little")
                    got = bm.cpu().numpy().view(np.uint8)[: want.size]
                    assert (got == want).all() and int(cnt.item()) == int(m.sum()), (dt, n, shift, op)
                    assert int(bm[words].item()) == 0  # nothing written past the last word


def test_selection_and_bitmap_and(golden):
    L = capi.lib()
    for case in golden["ops"]["selection"]:
        bm = inputs.bitmap(case["n"], case["seed"])
        out = np.zeros(max(case["n"], 1), np.uint32)
        c = L.voxel_selection_from_bitmap(bm.ctypes.data, case["n"], out.ctypes.data)
        assert c == case["count"] and digest(out[:c]) == case["digest"]
    rng = np.random.default_rng(22)
    for n in (1, 63, 64, 65, 1000, 65536 * 3 + 5, 1 << 25):
        a = inputs.bitmap(n, int(rng.integers(1 << 30)))
        b = inputs.bitmap(n, int(rng.integers(1 << 30)))
        words = (n + 63) // 64
        out = np.zeros(words, np.uint64)
        arr = (C_ptrs := (__import__("ctypes").c_void_p * 2)(a.ctypes.data, b.ctypes.data))
        c = L.voxel_bitmap_and(arr, 2, n, out.ctypes.data)
        want = np.zeros(words, np.uint64)
        wc = oracle.port().vo_bitmap_and(arr, 2, n, want.ctypes.data)
        assert c == wc and (out == want).all()
        sel = np.zeros(max(int(c), 1), np.uint32)
        cs = L.voxel_selection_from_bitmap(out.ctypes.data, n, sel.ctypes.data)
        assert cs == c
        ref = np.zeros(max(n, 1), np.uint32)
        rc = oracle.port().vo_selection_from_bitmap(want.ctypes.data, n, ref.ctypes.data)
        assert rc == cs and (sel[:cs] == ref[:rc]).all()
        del C_ptrs


def test_bitpack_decode_device_alignments():
    """Whole 4096-value tiles decode four values per thread into 16-byte
    stores when the output is 16-byte aligned, the per-value path otherwise:
    both equal the input for widths 1..32, with offsets and ragged tails, and
    through a dictionary."""
    import torch

    L = capi.lib()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(24)
    for w in (1, 3, 10, 17, 31, 32):
        for n in (4096, 3 * 4096 + 77, 40_001):
            v = rng.integers(0, (1 << w) - 1, n, dtype=np.uint64, endpoint=True).astype(np.uint32)
            words = encode.bitpack(v, w)
            dw = torch.from_numpy(words.view(np.int64)).to(dev)
            for off in (0, 4096, 5):
                if off >= n:
                    continue
                for oshift in (0, 1):
                    out = torch.zeros(n + 8, dtype=torch.int32, device=dev)
                    st = L.voxel_bitpack_decode_dev(dw.data_ptr(), words.size, w, n, off, n - off,
                                                    out.data_ptr() + 4 * oshift, None)
                    assert st == 0, capi.last_error()
                    got = out.cpu().numpy().view(np.uint32)[oshift:oshift + n - off]
                    assert (got == v[off:]).all(), (w, n, off, oshift)
    dct = np.arange(1000, dtype=np.int32) * 7 - 3000
    v = rng.integers(0, 1000, 9000).astype(np.uint32)
    words = encode.bitpack(v, 10)
    dw = torch.from_numpy(words.view(np.int64)).to(dev)
    dd = torch.from_numpy(dct).to(dev)
    for oshift in (0, 1):
        out = torch.zeros(9000 + 8, dtype=torch.int32, device=dev)
        st = L.voxel_dict_bitpack_decode_i32_dev(dw.data_ptr(), words.size, 10, dd.data_ptr(), dct.size, v.size, 0,
                                                 v.size, out.data_ptr() + 4 * oshift, None)
        assert st == 0, capi.last_error()
        assert (out.cpu().numpy()[oshift:oshift + 9000] == dct[v]).all()


def test_decoders_golden_and_round_trip(golden):
    L = capi.lib()
    for case in golden["ops"]["bitpack"]:
        v = inputs.u32_values(case["n"], case["maxv"], case["seed"])
        w = encode.bit_width(v)
        words = encode.bitpack(v, w)
        assert w == case["width"] and words.size == case["nwords"] and digest(words) == case["words_digest"]
        out = np.zeros(v.size, np.uint32)
        assert L.voxel_bitpack_decode(words.ctypes.data, words.size, w, v.size, 0, v.size, out.ctypes.data) == 0
        assert (out == v).all()
        if v.size > 10:  # offset window, past-the-end count clipped like DecodeBatch
            out2 = np.zeros(v.size, np.uint32)
            off = v.size // 3
            assert L.voxel_bitpack_decode(words.ctypes.data, words.size, w, v.size, off, v.size, out2.ctypes.data) == 0
            assert (out2[: v.size - off] == v[off:]).all()
    for case in golden["ops"]["rle"]:
        v = inputs.rle_i64(case["n"], case["seed"])
        vals, runs = encode.rle_build(v)
        assert vals.size == case["runs"] and digest(vals) == case["values_digest"]
        for dc in case["decodes"]:
            out = np.zeros(dc["count"], np.int64)
            assert L.voxel_rle_decode_i64(vals.ctypes.data, runs.ctypes.data, vals.size, dc["offset"], dc["count"],
                                          out.ctypes.data) == 0
            assert digest(out) == dc["digest"], dc
    # dictionary + bit-packed key column of the scan workload, full size
    d = inputs.config2(1 << 25, 2002)
    out = np.zeros(d["n"], np.int32)
    assert L.voxel_dict_bitpack_decode_i32(d["packed"].ctypes.data, d["packed"].size, d["width"], d["dict"].ctypes.data,
                                           d["dict"].size, d["n"], 0, d["n"], out.ctypes.data) == 0
    assert (out == d["key"]).all()
    o2 = np.zeros(1000, np.int32)
    assert L.voxel_dict_decode(T.I32, d["dict"].ctypes.data, d["dict"].size, d["idx"].ctypes.data, d["n"], 12345, 1000,
                               o2.ctypes.data) == 0
    assert (o2 == d["key"][12345:13345]).all()
    # ts column: strictly increasing, runs of 1..64, RLE round trip at full size
    ts = inputs.rle_i64(1 << 25, 2004)
    vals, runs = encode.rle_build(ts)
    out = np.zeros(ts.size + 100, np.int64)
    assert L.voxel_rle_decode_i64(vals.ctypes.data, runs.ctypes.data, vals.size, 0, out.size, out.ctypes.data) == 0
    assert (out[: ts.size] == ts).all() and (out[ts.size:] == 0).all()


def test_radix_sort_golden_and_properties(golden):
    L = capi.lib()
    for case in golden["ops"]["radix"]:
        k = inputs.sort_keys(case["dtype"], case["n"], case["seed"])
        idx = np.arange(case["n"], dtype=np.uint32)
        assert L.voxel_radix_sort(case["dtype"], k.ctypes.data, idx.ctypes.data, case["n"]) == 0, capi.last_error()
        assert digest(k) == case["keys_digest"] and digest(idx) == case["idx_digest"], case
    rng = np.random.default_rng(23)
    for dt, n in ((T.U64, 1 << 24), (T.I64, (1 << 22) + 3), (T.U32, (1 << 23) + 1), (T.I32, 100_001)):
        k0 = inputs.sort_keys(dt, n, int(rng.integers(1 << 30)))
        k = k0.copy()
        idx = np.arange(n, dtype=np.uint32)
        assert L.voxel_radix_sort(dt, k.ctypes.data, idx.ctypes.data, n) == 0, capi.last_error()
        order = np.argsort(k0, kind="stable")  # stable ascending = the reference's permutation
        assert (idx == order).all() and (k == k0[order]).all()


def test_radix_sort_skips_constant_digit_passes():
    """Keys narrower than their type (row ids in u64, small signed values,
    constant high bytes) skip the passes whose digit is the same for every key;
    odd and even numbers of remaining passes, and no pass at all, still give
    numpy's stable permutation."""
    L = capi.lib()
    rng = np.random.default_rng(29)
    n = (1 << 20) + 9
    cases = [
        (T.U64, rng.integers(0, 1 << 20, n, dtype=np.uint64)),                # 3 passes of 8
        (T.U64, rng.integers(0, 1 << 16, n, dtype=np.uint64) << np.uint64(8)),  # 2 passes, digit 0 constant
        (T.I64, rng.integers(-1000, 1000, n).astype(np.int64)),               # sign byte and low bytes
        (T.I64, rng.integers(5, 300, n).astype(np.int64)),                    # non-negative only
        (T.U32, (rng.integers(0, 1 << 8, n, dtype=np.uint32) << np.uint32(24)) | np.uint32(0x00ABCD00)),  # 1 pass
        (T.I32, np.full(n, -7, np.int32)),                                    # every pass skipped
        (T.U32, rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)),  # all passes
    ]
    for dt, k0 in cases:
        k = k0.copy()
        idx = np.arange(n, dtype=np.uint32)
        assert L.voxel_radix_sort(dt, k.ctypes.data, idx.ctypes.data, n) == 0, capi.last_error()
        order = np.argsort(k0, kind="stable")
        assert (idx == order).all() and (k == k0[order]).all(), (dt, k0[:4])


def test_autotuner_times_and_caches_radix_and_scan(tmp_path):
    """First calls of a shape time the candidate configurations, cache the
    fastest per (GPU, family, element type, log2 size) and still return the
    exact result; later calls read the cache."""
    import json

    L = capi.lib()
    path = tmp_path / "tune.json"
    L.voxel_tune_set_cache_path(str(path).encode())
    try:
        L.voxel_tune_enable(1)
        L.voxel_tune_clear()
        n = (1 << 20) + 7
        k0 = inputs.sort_keys(T.U64, n, 77)
        for _ in range(2):
            k = k0.copy()
            idx = np.arange(n, dtype=np.uint32)
            assert L.voxel_radix_sort(T.U64, k.ctypes.data, idx.ctypes.data, n) == 0, capi.last_error()
            order = np.argsort(k0, kind="stable")
            assert (idx == order).all() and (k == k0[order]).all()
        assert L.voxel_tune_lookup(b"radix_onesweep", T.U64, n) in (0, 1)
        assert L.voxel_tune_lookup(b"radix_onesweep", T.U32, n) == -1
        d = inputs.config2(1 << 20, 78)
        card = d["dict"].size
        w = oracle.scan_groupby_port(d["packed"], d["width"], d["dict"], d["price"], d["qty"], 20.0, 10, 50)
        assert L.voxel_scan_groupby_tune(-1) == 0
        for _ in range(2):
            ok = np.zeros(card, np.int32)
            s, mn, mx = (np.zeros(card) for _ in range(3))
            c = np.zeros(card, np.uint64)
            g = L.voxel_scan_groupby(d["packed"].ctypes.data, d["packed"].size, d["width"], d["dict"].ctypes.data,
                                     card, d["price"].ctypes.data, d["qty"].ctypes.data, d["price"].size, 20.0, 10,
                                     50, ok.ctypes.data, s.ctypes.data, mn.ctypes.data, mx.ctypes.data, c.ctypes.data)
            assert g == w[0].size, capi.last_error()
            assert (ok[:g] == w[0]).all() and (c[:g] == w[4]).all() and (mn[:g] == w[2]).all()
            np.testing.assert_allclose(s[:g], w[1], rtol=1e-12, atol=0)
        fam = "scan_groupby_v3_card%d" % (card.bit_length() - 1)
        assert L.voxel_tune_lookup(fam.encode(), T.F64, d["price"].size) in (0, 1, 2, 3, 4, 5)
        entries = json.loads(path.read_text())
        assert {e.split("|")[1] for e in entries} == {"radix_onesweep", fam}
        # tuning off: nothing new is timed or cached
        L.voxel_tune_enable(0)
        k = inputs.sort_keys(T.U32, n, 79)
        idx = np.arange(n, dtype=np.uint32)
        assert L.voxel_radix_sort(T.U32, k.ctypes.data, idx.ctypes.data, n) == 0
        assert L.voxel_tune_lookup(b"radix_onesweep", T.U32, n) == -1
    finally:
        L.voxel_tune_enable(1)
        L.voxel_tune_set_cache_path(None)


def test_hashjoin_golden_and_properties(golden):
    L = capi.lib()
    for case in golden["ops"]["hashjoin"]:
        if case["seed"] == 0:
            b = np.array([1, 2, 3, 4], np.int64)
            p = np.array([2, 4, 6], np.int64)
        else:
            b, p = inputs.join_input(case["nb"], case["np"], case["dup"], case["seed"])
        cap = case["np"] * (8 if case["dup"] else 1) + 8
        l = np.zeros(cap, np.uint32)
        r = np.zeros(cap, np.uint32)
        m = L.voxel_hashjoin_i64(b.ctypes.data, b.size, p.ctypes.data, p.size, l.ctypes.data, r.ctypes.data, cap,
                                 case["all"])
        assert m == case["matches"] and digest(l[:m], r[:m]) == case["digest"], case
    rng = np.random.default_rng(24)
    for nb, np_, dup in ((1 << 20, 1 << 23, False), (50_000, 400_000, True)):
        b, p = inputs.join_input(nb, np_, dup, int(rng.integers(1 << 30)))
        cap = np_ * (16 if dup else 1)
        l = np.zeros(cap, np.uint32)
        r = np.zeros(cap, np.uint32)
        m = L.voxel_hashjoin_i64(b.ctypes.data, b.size, p.ctypes.data, p.size, l.ctypes.data, r.ctypes.data, cap, 1)
        assert m != FAIL, capi.last_error()
        wl = np.zeros(cap, np.uint32)
        wr = np.zeros(cap, np.uint32)
        wm = oracle.port().vo_hashjoin_i64(b.ctypes.data, b.size, p.ctypes.data, p.size, wl.ctypes.data,
                                           wr.ctypes.data, cap, 1)
        assert m == wm and (l[:m] == wl[:m]).all() and (r[:m] == wr[:m]).all()
        assert (np.diff(l[:m].astype(np.int64)) >= 0).all() and (b[r[:m]] == p[l[:m]]).all()
    # capped probe: the first max_matches pairs in probe order
    b, p = inputs.join_input(1000, 5000, False, 77)
    l = np.zeros(100, np.uint32)
    r = np.zeros(100, np.uint32)
    m = L.voxel_hashjoin_i64(b.ctypes.data, b.size, p.ctypes.data, p.size, l.ctypes.data, r.ctypes.data, 100, 1)
    wl = np.zeros(100, np.uint32)
    wr = np.zeros(100, np.uint32)
    wm = oracle.port().vo_hashjoin_i64(b.ctypes.data, b.size, p.ctypes.data, p.size, wl.ctypes.data, wr.ctypes.data,
                                       100, 1)
    assert m == wm == 100 and (l == wl).all() and (r == wr).all()


def test_bitmap_and_many_bitmaps():
    """AND of 1 to 70 bitmaps: pointer lists passed by value (up to 16), held
    in shared memory (up to 64) and read from the device table beyond, on the
    host and device entry points, against the oracle."""
    import ctypes

    import torch

    L = capi.lib()
    rng = np.random.default_rng(23)
    n = 100_003
    words = (n + 63) // 64
    dev = torch.device("cuda", 0)
    for nbm in (1, 5, 16, 17, 64, 70):
        bms = []
        for _ in range(nbm):
            bits = rng.random(n) < 0.985
            raw = np.packbits(bits, bitorder="little")
            raw = np.concatenate([raw, np.zeros(words * 8 - raw.size, np.uint8)])
            bms.append(raw.view(np.uint64).copy())
        hp = (ctypes.c_void_p * nbm)(*[b.ctypes.data for b in bms])
        out = np.zeros(words, np.uint64)
        c = L.voxel_bitmap_and(hp, nbm, n, out.ctypes.data)
        want = np.zeros(words, np.uint64)
        wc = oracle.port().vo_bitmap_and(hp, nbm, n, want.ctypes.data)
        assert c == wc and (out == want).all(), nbm
        dts = [torch.from_numpy(b.view(np.int64)).to(dev) for b in bms]
        dp = (ctypes.c_void_p * nbm)(*[t.data_ptr() for t in dts])
        dout = torch.zeros(words, dtype=torch.int64, device=dev)
        dcnt = torch.zeros(1, dtype=torch.int64, device=dev)
        assert L.voxel_bitmap_and_dev(ctypes.addressof(dp), nbm, n, dout.data_ptr(), dcnt.data_ptr(), None) == 0
        torch.cuda.synchronize()
        assert int(dcnt.item()) == wc and (dout.cpu().numpy().view(np.uint64) == want).all(), nbm


def test_device_entry_points_equal_host_ones():
    """The device-pointer variants (bitmap AND, dictionary decoders) give the
    host entry points' results; an index outside the dictionary is an error."""
    import ctypes

    import torch

    L = capi.lib()
    dev = torch.device("cuda", 0)
    n = 1_000_003
    a, b = inputs.bitmap(n, 31), inputs.bitmap(n, 32)
    words = (n + 63) // 64
    host_ptrs = (ctypes.c_void_p * 2)(a.ctypes.data, b.ctypes.data)
    want = np.zeros(words, np.uint64)
    wc = L.voxel_bitmap_and(host_ptrs, 2, n, want.ctypes.data)
    da, db = torch.from_numpy(a.view(np.int64)).to(dev), torch.from_numpy(b.view(np.int64)).to(dev)
    dout = torch.zeros(words, dtype=torch.int64, device=dev)
    dcnt = torch.zeros(1, dtype=torch.int64, device=dev)
    dptrs = (ctypes.c_void_p * 2)(da.data_ptr(), db.data_ptr())
    assert L.voxel_bitmap_and_dev(ctypes.addressof(dptrs), 2, n, dout.data_ptr(), dcnt.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert int(dcnt.item()) == wc and (dout.cpu().numpy().view(np.uint64) == want).all()
    d = inputs.config2(1 << 20, 2003)
    pw, dd = torch.from_numpy(d["packed"].view(np.int64)).to(dev), torch.from_numpy(d["dict"]).to(dev)
    o = torch.zeros(d["n"], dtype=torch.int32, device=dev)
    assert L.voxel_dict_bitpack_decode_i32_dev(pw.data_ptr(), d["packed"].size, d["width"], dd.data_ptr(),
                                               d["dict"].size, d["n"], 0, d["n"], o.data_ptr(), None) == 0
    assert (o.cpu().numpy() == d["key"]).all()
    idx = torch.from_numpy(d["idx"].astype(np.int32)).to(dev)
    o2 = torch.zeros(d["n"], dtype=torch.int32, device=dev)
    assert L.voxel_dict_decode_dev(T.I32, dd.data_ptr(), d["dict"].size, idx.data_ptr(), d["n"], o2.data_ptr(),
                                   None) == 0
    assert (o2.cpu().numpy() == d["key"]).all()
    bad = idx.clone()
    bad[777] = d["dict"].size  # one index past the dictionary
    st = L.voxel_dict_decode_dev(T.I32, dd.data_ptr(), d["dict"].size, bad.data_ptr(), d["n"], o2.data_ptr(), None)
    assert st == 1  # VOXEL_EINVAL


def test_rle_decode_zero_length_runs_and_windows():
    """RLE decode with empty runs mixed in (a run of 0 rows covers nothing) and
    windows that start and end inside runs, across the expand kernel's tiles
    (and past the last row, which decodes to 0), against numpy's repeat."""
    L = capi.lib()
    rng = np.random.default_rng(61)
    nruns = 50_000
    runs = rng.integers(0, 6, nruns).astype(np.uint32)  # about 1 in 6 runs is empty
    vals = rng.integers(-(1 << 40), 1 << 40, nruns).astype(np.int64)
    full = np.repeat(vals, runs.astype(np.int64))
    for off, cnt in ((0, full.size), (1, 5000), (2047, 4099), (12345, 60000), (full.size - 10, 30), (5, full.size)):
        out = np.full(cnt, 7, np.int64)
        assert L.voxel_rle_decode_i64(vals.ctypes.data, runs.ctypes.data, nruns, off, cnt, out.ctypes.data) == 0
        want = np.zeros(cnt, np.int64)
        part = full[off:off + cnt]
        want[:part.size] = part
        assert (out == want).all(), (off, cnt)
