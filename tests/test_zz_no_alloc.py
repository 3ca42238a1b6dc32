"""voxel_scan_groupby_noalloc_dev (fixed in-library scratch, allocates nothing)
against voxel_scan_groupby_dev on the same device inputs: bit-identical outputs
on two calls in a row, across a change of dictionary size, and the size limit
of its scratch.  Collected last so it also runs after every other GPU test."""
import ctypes as C

import numpy as np
import pytest
import torch

import inputs
from voxel_b200 import capi

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)
MAX_GROUPS = 4096


def _device_case(n, seed, card):
    d = inputs.config2(n, seed, card=card)
    t = {k: torch.from_numpy(np.ascontiguousarray(d[k])).to(DEV) for k in ("packed", "dict", "price", "qty")}
    return d, t


def _outputs(card):
    return dict(keys=torch.zeros(card, dtype=torch.int32, device=DEV),
                sum=torch.zeros(card, dtype=torch.float64, device=DEV),
                min=torch.zeros(card, dtype=torch.float64, device=DEV),
                max=torch.zeros(card, dtype=torch.float64, device=DEV),
                count=torch.zeros(card, dtype=torch.int64, device=DEV),
                ngroups=torch.zeros(1, dtype=torch.int64, device=DEV))


def _call(noalloc, d, t, pthr=20.0, qlo=10, qhi=50, card=None, want_status=0):
    L = capi.lib()
    card = d["dict"].size if card is None else card
    o = _outputs(max(card, 1))
    args = [t["packed"].data_ptr(), t["packed"].numel(), d["width"], t["dict"].data_ptr(), card,
            t["price"].data_ptr(), t["qty"].data_ptr(), t["price"].numel(), pthr, qlo, qhi,
            o["keys"].data_ptr(), o["sum"].data_ptr(), o["min"].data_ptr(), o["max"].data_ptr(),
            o["count"].data_ptr(), o["ngroups"].data_ptr()]
    if noalloc:
        status = torch.zeros(4, dtype=torch.int32, device=DEV)
        st = L.voxel_scan_groupby_noalloc_dev(*args, status.data_ptr(), None)
    else:
        st = L.voxel_scan_groupby_dev(*args, None)
    if st:
        return st, None
    torch.cuda.synchronize()
    if noalloc:
        assert int(status[0]) == want_status
    g = int(o["ngroups"][0])
    return 0, {k: v[:g].cpu().numpy() for k, v in o.items() if k != "ngroups"}


def _same(a, b):
    assert a["keys"].size == b["keys"].size
    for k in ("keys", "count"):
        assert (a[k] == b[k]).all()
    for k in ("sum", "min", "max"):
        assert (a[k].view(np.uint64) == b[k].view(np.uint64)).all()


def test_noalloc_matches_dev_on_two_calls_in_a_row():
    for n, seed, card in ((1 << 20, 11, MAX_GROUPS), (300_001, 12, 37), (4096, 13, 1)):
        d, t = _device_case(n, seed, card)
        st, want = _call(False, d, t)
        assert st == 0, capi.last_error()
        for _ in range(2):
            st, got = _call(True, d, t)
            assert st == 0, capi.last_error()
            _same(got, want)


def test_noalloc_other_predicates():
    d, t = _device_case(200_000, 14, 900)
    for pthr, qlo, qhi in ((-1.0, 0, 1000), (1e9, 10, 50), (20.0, 50, 10)):
        st, want = _call(False, d, t, pthr, qlo, qhi)
        assert st == 0
        st, got = _call(True, d, t, pthr, qlo, qhi)
        assert st == 0, capi.last_error()
        _same(got, want)


def test_noalloc_rejects_dictionary_beyond_its_scratch():
    d, t = _device_case(10_000, 15, 100)
    st, _ = _call(True, d, t, card=MAX_GROUPS + 1)
    assert st == 1 and "4096" in capi.last_error()
    # nothing was launched: the next call is still correct
    st, want = _call(False, d, t)
    st2, got = _call(True, d, t)
    assert st == 0 and st2 == 0
    _same(got, want)


def test_noalloc_table_recovers_after_flagged_calls():
    """A call that flags a key outside the dictionary (status bit 2) or a
    product that is not finite (bit 1) still leaves the shared table at rest:
    the next valid call is bit-identical to the allocating entry point."""
    L = capi.lib()
    d, t = _device_case(200_000, 16, 300)
    st, want = _call(False, d, t)
    assert st == 0, capi.last_error()
    # a dictionary shorter than the packed indices need
    st, _ = _call(True, d, t, card=150, want_status=2)
    assert st == 0
    assert L.voxel_scan_groupby_status_code(2) == 1 and "dictionary" in capi.last_error()
    st, got = _call(True, d, t)
    assert st == 0, capi.last_error()
    _same(got, want)
    # an infinite price (with a qty in range) passes the predicate and makes a
    # non-finite product
    bad = t["price"].clone()
    bad[1234] = float("inf")
    badq = t["qty"].clone()
    badq[1234] = 20
    tb = dict(t, price=bad, qty=badq)
    st, _ = _call(True, d, tb, want_status=1)
    assert st == 0
    assert L.voxel_scan_groupby_status_code(1) == 7
    st, got = _call(True, d, t)
    assert st == 0, capi.last_error()
    _same(got, want)
