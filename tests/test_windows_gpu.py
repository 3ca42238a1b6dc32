"""Window functions on the GPU against the reference's Engine<T>::Window*
and TimeWindowSum (include/voxel/exec/engine.hpp:176-300): every golden case
bit-exact (each window is evaluated in the reference's operation order), the
live reference at 2^22 rows, and TimeWindowSum's f64 buckets within 1e-12."""
import hashlib

import numpy as np
import pytest
import torch

import inputs
import oracle
from voxel_b200 import capi

pytestmark = pytest.mark.gpu
NAME = {0: "f64", 2: "i64", 3: "i32", 4: "u64", 5: "u32"}


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def test_windows_golden(golden):
    L = capi.lib()
    for c in golden["windows"]["windows"]:
        x = inputs.window_values(c["dtype"], c["n"], c["seed"])
        o = np.zeros(max(c["out_len"], 1), x.dtype)
        m = L.voxel_window(c["dtype"], c["kind"], x.ctypes.data, c["n"], o.ctypes.data, c["out_len"], c["window"],
                           c["q"])
        assert m == c["written"], (c, capi.last_error())
        assert digest(o[:m]) == c["digest"], c


def test_time_window_sum_golden(golden):
    L = capi.lib()
    for c in golden["windows"]["time_windows"]:
        dt = c["dtype"]
        ts, v = inputs.time_window_input(dt, c["n"], c["seed"])
        o = inputs.window_values(dt, c["out_len"], c["seed"] + 1)[: c["out_len"]].copy()
        m = L.voxel_time_window_sum(dt, ts.ctypes.data, v.ctypes.data, c["n"], c["start"], c["duration"],
                                    o.ctypes.data, c["out_len"])
        assert m == c["returned"], c
        if dt == 0:
            o0 = inputs.window_values(0, c["out_len"], c["seed"] + 1)[: c["out_len"]]
            changed = dict((i, val) for i, val in c["changed"])
            for i in range(c["out_len"]):
                want = changed.get(i, o0[i])
                assert abs(o[i] - want) <= 1e-12 * max(abs(want), 1.0), (i, o[i], want)
        else:
            assert digest(o) == c["digest"], c


def test_windows_against_live_reference_large():
    if not oracle.have_ref():
        pytest.skip("reference library not built")
    L = capi.lib()
    R = oracle.ref()
    n = (1 << 22) + 13
    for dt in (0, 2, 3):
        x = inputs.window_values(dt, n, 300 + dt)
        # windows of at most 16 inputs take the register-tiled kernels, longer ones the shared-memory ones
        for kind, w, q in ((1, 16, 0), (1, 17, 0), (2, 5, 0), (3, 32, 0), (3, 16, 0), (4, 7, 0), (4, 2, 0),
                           (5, 21, 0.37), (5, 16, 0.5), (5, 9, 0.0), (5, 2, 1.0), (5, 13, 0.81), (0, 2, 0)):
            want = np.zeros(n, x.dtype)
            m = getattr(R, f"vref_window_{NAME[dt]}")(kind, x.ctypes.data, n, want.ctypes.data, n, w, q)
            got = np.zeros(n, x.dtype)
            g = L.voxel_window(dt, kind, x.ctypes.data, n, got.ctypes.data, n, w, q)
            assert g == m and (got[:m].view(np.uint8) == want[:m].view(np.uint8)).all(), (dt, kind, w, q)


def test_time_window_sum_device_full_size():
    """2^27 rows into 2^16 buckets on the device against the reference."""
    if not oracle.have_ref():
        pytest.skip("reference library not built")
    n, nb = 1 << 27, 1 << 16
    ts, v = inputs.time_window_input(2, n, 77)
    want = np.zeros(nb, np.int64)
    m = oracle.ref().vref_time_window_sum_i64(ts.ctypes.data, v.ctypes.data, n, 0, 2048, want.ctypes.data, nb)
    dev = torch.device("cuda", 0)
    dts, dv = torch.from_numpy(ts).to(dev), torch.from_numpy(v).to(dev)
    out = torch.zeros(nb, dtype=torch.int64, device=dev)
    import ctypes as C
    got_n = C.c_size_t(0)
    assert capi.lib().voxel_time_window_sum_dev(2, dts.data_ptr(), dv.data_ptr(), n, 0, 2048, out.data_ptr(), nb,
                                                C.byref(got_n), None) == 0, capi.last_error()
    assert got_n.value == m
    assert (out.cpu().numpy() == want).all()
