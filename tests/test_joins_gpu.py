"""Merge, semi and anti joins on the GPU against the reference's MergeJoin
(Join, JoinUnique), SemiJoin and AntiJoin (include/voxel/ops/join.hpp:216-310):
the golden fixtures for every key type, the live reference build at 2^22
rows, and at 2^26 left rows the size-independent properties (pairs in
left-major order with equal keys, semi + anti = every left row)."""
import hashlib

import numpy as np
import pytest
import torch

import inputs
import oracle
from voxel_b200 import capi

pytestmark = pytest.mark.gpu
NP = {2: np.int64, 3: np.int32, 4: np.uint64, 5: np.uint32}
NAME = {2: "i64", 3: "i32", 4: "u64", 5: "u32"}
FAIL = (1 << 64) - 1


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def merge(dt, lk, rk, cap, unique):
    lo = np.zeros(max(cap, 1), np.uint32)
    ro = np.zeros(max(cap, 1), np.uint32)
    m = capi.lib().voxel_merge_join(dt, lk.ctypes.data, lk.size, rk.ctypes.data, rk.size, lo.ctypes.data,
                                    ro.ctypes.data, cap, unique)
    assert m != FAIL, capi.last_error()
    return lo[:m], ro[:m]


def semi(dt, lk, rk, anti):
    o = np.zeros(max(lk.size, 1), np.uint32)
    m = capi.lib().voxel_semi_join(dt, lk.ctypes.data, lk.size, rk.ctypes.data, rk.size, o.ctypes.data, anti)
    assert m != FAIL, capi.last_error()
    return o[:m]


def test_join_family_golden(golden):
    for case in golden["joins"]:
        dt = case["dtype"]
        lk, rk = inputs.merge_join_input(NP[dt], case["nl"], case["nr"], case["dup"], case["seed"])
        for unique in (0, 1):
            want = case[f"merge{unique}"]
            lo, ro = merge(dt, lk, rk, want["matches"] + 3, unique)
            assert lo.size == want["matches"] and digest(lo, ro) == want["digest"], (dt, unique, case["nl"])
        ls = inputs.shuffled(lk, case["seed"])
        for anti in (0, 1):
            want = case[f"semi{anti}"]
            o = semi(dt, ls, rk, anti)
            assert o.size == want["matches"] and digest(o) == want["digest"], (dt, anti, case["nl"])


def test_join_family_against_live_reference():
    if not oracle.have_ref():
        pytest.skip("reference library not built")
    R = oracle.ref()
    for dt, dup in ((2, 3), (3, 1), (5, 6)):
        lk, rk = inputs.merge_join_input(NP[dt], 1 << 22, 3 << 20, dup, 100 + dt)
        for unique in (0, 1):
            cap = lk.size * (dup * 2 if not unique else 1) + 16
            wl = np.zeros(cap, np.uint32)
            wr = np.zeros(cap, np.uint32)
            m = getattr(R, f"vref_merge_join_{NAME[dt]}")(lk.ctypes.data, lk.size, rk.ctypes.data, rk.size, wl.ctypes.data,
                                                 wr.ctypes.data, unique)
            lo, ro = merge(dt, lk, rk, cap, unique)
            assert lo.size == m and (lo == wl[:m]).all() and (ro == wr[:m]).all(), (dt, unique)
        ls = inputs.shuffled(lk, 7)
        for anti in (0, 1):
            w = np.zeros(ls.size, np.uint32)
            m = getattr(R, f"vref_semi_join_{NAME[dt]}")(ls.ctypes.data, ls.size, rk.ctypes.data, rk.size, w.ctypes.data, anti)
            o = semi(dt, ls, rk, anti)
            assert o.size == m and (o == w[:m]).all(), (dt, anti)


def test_join_family_large_properties_and_cap():
    dev = torch.device("cuda", 0)
    L = capi.lib()
    lk, rk = inputs.merge_join_input(np.int64, 1 << 26, 1 << 25, 2, 555)
    dl, dr = torch.from_numpy(lk).to(dev), torch.from_numpy(rk).to(dev)
    cap = lk.size * 4
    lo = torch.zeros(cap, dtype=torch.int32, device=dev)
    ro = torch.zeros(cap, dtype=torch.int32, device=dev)
    c2 = torch.zeros(2, dtype=torch.int64, device=dev)
    assert L.voxel_merge_join_dev(2, dl.data_ptr(), lk.size, dr.data_ptr(), rk.size, lo.data_ptr(), ro.data_ptr(),
                                  cap, 0, c2.data_ptr(), None) == 0, capi.last_error()
    m = int(c2[0])
    assert m == int(c2[1]) and m > 0
    li = lo[:m].long()
    ri = ro[:m].long()
    assert torch.equal(dl[li], dr[ri])
    key = li * (1 << 26) + ri  # left-major, right ascending, no repeats
    assert bool((key[1:] > key[:-1]).all())
    # every match: per left row the number of equal right keys
    cnt = torch.searchsorted(dr, dl, right=True) - torch.searchsorted(dr, dl)
    assert int(cnt.sum()) == m
    # capped: the first max_matches pairs, the total still reported
    assert L.voxel_merge_join_dev(2, dl.data_ptr(), lk.size, dr.data_ptr(), rk.size, lo.data_ptr(), ro.data_ptr(),
                                  1000, 0, c2.data_ptr(), None) == 0
    assert int(c2[0]) == 1000 and int(c2[1]) == m and torch.equal(lo[:1000].long(), li[:1000])
    # semi + anti partition the left rows
    ls = torch.from_numpy(inputs.shuffled(lk, 9)).to(dev)
    out_s = torch.zeros(lk.size, dtype=torch.int32, device=dev)
    out_a = torch.zeros(lk.size, dtype=torch.int32, device=dev)
    cs = torch.zeros(1, dtype=torch.int64, device=dev)
    ca = torch.zeros(1, dtype=torch.int64, device=dev)
    assert L.voxel_semi_join_dev(2, ls.data_ptr(), lk.size, dr.data_ptr(), rk.size, out_s.data_ptr(), 0,
                                 cs.data_ptr(), None) == 0
    assert L.voxel_semi_join_dev(2, ls.data_ptr(), lk.size, dr.data_ptr(), rk.size, out_a.data_ptr(), 1,
                                 ca.data_ptr(), None) == 0
    ns, na = int(cs[0]), int(ca[0])
    assert ns + na == lk.size
    both = torch.cat([out_s[:ns], out_a[:na]]).long()
    assert torch.equal(torch.sort(both).values, torch.arange(lk.size, device=dev))
    hit = torch.isin(ls, dr)
    assert torch.equal(torch.nonzero(hit).flatten(), out_s[:ns].long())
