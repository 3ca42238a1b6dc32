"""Delta and frame-of-reference codecs on the GPU against the reference's
DeltaEncoding<T> / FrameOfReferenceEncoding (encoding.hpp:281-354, 456-521):
the golden fixtures the reference produced, the live reference build at
larger sizes, and full-size round trips (2^28 rows) against numpy."""
import ctypes as C
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


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def test_delta_golden(golden):
    L = capi.lib()
    for case in golden["codecs"]["delta"]:
        dt, n = case["dtype"], case["n"]
        data = inputs.codec_ints(NP[dt], n, case["seed"])
        deltas = np.zeros(max(n, 1), NP[dt])
        assert L.voxel_delta_encode(dt, data.ctypes.data, n, deltas.ctypes.data) == 0, capi.last_error()
        assert digest(deltas[:n]) == case["deltas_digest"], (dt, n)
        for d in case["decodes"]:
            off, cnt = d["offset"], d["count"]
            out = np.zeros(max(cnt, 1), NP[dt])
            assert L.voxel_delta_decode(dt, deltas.ctypes.data, n, case["base"], off, cnt, out.ctypes.data) == 0
            assert digest(out[:cnt]) == d["digest"], (dt, n, off, cnt)


def test_frame_of_reference_golden(golden):
    L = capi.lib()
    for case in golden["codecs"]["frame_of_reference"]:
        n = case["n"]
        x = inputs.codec_f64(n, case["seed"])
        codes = np.zeros(max(n, 1), np.int32)
        base, scale = C.c_double(), C.c_double()
        assert L.voxel_for_encode_f64(x.ctypes.data, n, codes.ctypes.data, C.byref(base), C.byref(scale)) == 0
        assert digest(codes[:n]) == case["codes_digest"] and base.value == case["base"]
        assert scale.value == case["scale"]
        for d in case["decodes"]:
            off, cnt = d["offset"], d["count"]
            m = max(0, min(cnt, n - off))
            out = np.zeros(max(m, 1))
            assert L.voxel_for_decode_f64(codes.ctypes.data, n, base.value, scale.value, off, cnt,
                                          out.ctypes.data) == 0
            assert digest(out[:m]) == d["digest"], (n, off, cnt)


def test_delta_against_live_reference_with_wraps():
    """Larger columns with wrapping sums, odd offsets and a nonzero base."""
    if not oracle.have_ref():
        pytest.skip("reference library not built")
    L = capi.lib()
    R = oracle.ref()
    rng = np.random.default_rng(91)
    for dt in (2, 3, 4, 5):
        n = 3_000_017
        deltas = rng.integers(0, np.iinfo(NP[dt]).max, size=n, dtype=NP[dt], endpoint=True)
        base = int(rng.integers(0, 1 << 62))
        for off, cnt in ((0, n), (12_345, 2_000_000), (n - 5, 100)):
            want = np.zeros(cnt, NP[dt])
            getattr(R, f"vref_delta_decode_{NAME[dt]}")(deltas.ctypes.data, n, base, off, cnt, want.ctypes.data)
            got = np.zeros(cnt, NP[dt])
            assert L.voxel_delta_decode(dt, deltas.ctypes.data, n, base, off, cnt, got.ctypes.data) == 0
            m = min(cnt, n - off)
            assert (got[:m] == want[:m]).all(), (dt, off, cnt)


def test_codecs_full_size_round_trip_on_device():
    """2^28-row columns on the device: delta encode -> decode is the identity
    (and the decode equals numpy's wrapping cumsum of the deltas); FOR decode
    equals base + code * scale rounded per operation."""
    L = capi.lib()
    dev = torch.device("cuda", 0)
    n = 1 << 28
    g = torch.Generator(device=dev)
    g.manual_seed(92)
    x = torch.randint(-(1 << 40), 1 << 40, (n,), dtype=torch.int64, device=dev, generator=g)
    d = torch.empty_like(x)
    y = torch.empty_like(x)
    assert L.voxel_delta_encode_dev(2, x.data_ptr(), n, d.data_ptr(), None) == 0
    assert L.voxel_delta_decode_dev(2, d.data_ptr(), n, 0, 0, n, y.data_ptr(), None) == 0, capi.last_error()
    torch.cuda.synchronize()
    assert torch.equal(x, y)
    assert torch.equal(torch.cumsum(d, 0), y)  # int64 cumsum wraps like the decode
    del x, d, y
    code = torch.randint(-(1 << 31), 1 << 31, (n,), dtype=torch.int32, device=dev, generator=g)
    out = torch.empty(n, dtype=torch.float64, device=dev)
    base, scale = -12.5, 3.0e-7
    assert L.voxel_for_decode_f64_dev(code.data_ptr(), n, base, scale, 0, n, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    sample = torch.randint(0, n, (1 << 20,), device=dev, generator=g)
    c = code[sample].cpu().numpy().astype(np.float64)
    want = base + (c * scale)  # numpy: one rounding per operation
    assert (out[sample].cpu().numpy() == want).all()


def test_delta_decode_device_alignments():
    """The streaming decode (16-byte aligned deltas) and the plain one
    (misaligned deltas) against numpy's wrapping cumsum, with outputs at
    aligned and misaligned addresses and offsets that do and do not fall on a
    16-byte boundary, across tile boundaries (32 KB tiles) and ragged tails."""
    L = capi.lib()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(93)
    for dt, tdt in ((2, torch.int64), (3, torch.int32)):
        es = 8 if dt == 2 else 4
        for n in (1, 5, 4095, 4096, 4097, 8193, 1_000_003):
            host = rng.integers(np.iinfo(NP[dt]).min, np.iinfo(NP[dt]).max, size=n + 4, dtype=NP[dt])
            buf = torch.from_numpy(host).to(dev)
            base = int(rng.integers(0, 1 << 30))
            for shift in (0, 1):  # deltas at the buffer start (aligned) or one element in (misaligned)
                src = host[shift:shift + n]
                want = (np.cumsum(src.astype(NP[dt]), dtype=NP[dt]) + NP[dt](base)).astype(NP[dt])
                for off in (0, 1, 2, 3):
                    if off >= n:
                        continue
                    for oshift in (0, 1):
                        out = torch.zeros(n + 4, dtype=tdt, device=dev)
                        st = L.voxel_delta_decode_dev(dt, buf.data_ptr() + shift * es, n, base, off, n - off,
                                                      out.data_ptr() + oshift * es, None)
                        assert st == 0, capi.last_error()
                        got = out.cpu().numpy()[oshift:oshift + n - off]
                        assert (got == want[off:]).all(), (dt, n, shift, off, oshift)
