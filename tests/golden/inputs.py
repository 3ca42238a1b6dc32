"""Deterministic input generators shared by the golden-vector script and tests.

All generators use numpy's PCG64 (stable across numpy versions for the calls
used here), except mt_uniform, which reproduces the reference's own
std::mt19937_64 + uniform_real_distribution column (examples/validate.cpp:22-25)
through the backend's C++ data generator.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from voxel_b200 import templates as T  # noqa: E402


def column(dtype: int, n: int, seed: int) -> np.ndarray:
    return T.make_column(dtype, n, np.random.default_rng(seed))


def mt_uniform(seed: int, n: int, lo: float = 0.0, hi: float = 1000.0) -> np.ndarray:
    from voxel_b200 import capi

    x = np.empty(n, np.float64)
    capi.datagen().vgen_uniform_f64_mt(seed, n, lo, hi, x.ctypes.data)
    return x


def bitmap(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    words = max((n + 63) // 64, 1)
    bm = rng.integers(0, 2**63, size=words, dtype=np.int64).astype(np.uint64)
    bm ^= rng.integers(0, 2, size=words, dtype=np.int64).astype(np.uint64) << np.uint64(63)
    if n % 64:
        bm[-1] &= np.uint64((1 << (n % 64)) - 1)
    if n == 0:
        bm[:] = 0
    return bm


def u32_values(n: int, maxv: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = rng.integers(0, maxv, size=n, dtype=np.int64).astype(np.uint32)
    if n:
        v[0] = np.uint32(maxv - 1)
    return v


def i32_values(n: int, card: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    pool = rng.integers(-(2**31), 2**31, size=card, dtype=np.int64).astype(np.int32)
    return pool[rng.integers(0, card, size=n)]


def rle_i64(n: int, seed: int) -> np.ndarray:
    """Strictly increasing run values, runs of 1..64 (the ts column's shape)."""
    rng = np.random.default_rng(seed)
    out = np.empty(n, np.int64)
    i, v = 0, int(rng.integers(0, 1000))
    while i < n:
        r = int(rng.integers(1, 65))
        out[i:i + r] = v
        i += r
        v += int(rng.integers(1, 6))
    return out


def group_input(n: int, card: int, seed: int):
    rng = np.random.default_rng(seed)
    keys = rng.integers(0, card, size=n).astype(np.int32) * 7 - 100
    vals = rng.random(n) * 100.0
    return keys, vals


def sort_keys(dtype: int, n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    if dtype == T.U64:
        k = rng.integers(0, 2**63, size=n, dtype=np.int64).astype(np.uint64) * np.uint64(2)
        k += rng.integers(0, 2, size=n, dtype=np.int64).astype(np.uint64)
        if n > 4:
            k[: n // 4] = k[n // 2: n // 2 + n // 4]  # duplicates exercise stability
        return k
    if dtype == T.U32:
        k = rng.integers(0, 2**32, size=n, dtype=np.int64).astype(np.uint32)
    elif dtype == T.I64:
        k = rng.integers(-(2**62), 2**62, size=n, dtype=np.int64)
    else:
        k = rng.integers(-(2**31), 2**31, size=n, dtype=np.int64).astype(np.int32)
    if n > 4:
        k[: n // 4] = k[n // 2: n // 2 + n // 4]
    return k


def join_input(nb: int, np_: int, dup: bool, seed: int):
    rng = np.random.default_rng(seed)
    if dup:
        pool = rng.integers(-(2**40), 2**40, size=max(nb // 4, 1), dtype=np.int64)
        b = pool[rng.integers(0, pool.size, size=nb)]
    else:
        b = rng.permutation(rng.integers(-(2**40), 2**40, size=nb * 2, dtype=np.int64))
        b = np.unique(b)[:nb]
        b = rng.permutation(b)
    hit = rng.random(np_) < 0.9
    p = np.where(hit, b[rng.integers(0, b.size, size=np_)], rng.integers(2**41, 2**42, size=np_, dtype=np.int64))
    return b.astype(np.int64), p.astype(np.int64)


def zipf_alias_keys(n: int, card: int, s: float, rng: np.random.Generator) -> np.ndarray:
    """Ranks 0..card-1 drawn with P(k) ~ (k+1)^-s (inverse-CDF on the exact pmf)."""
    w = np.arange(1, card + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w / w.sum())
    cdf[-1] = 1.0
    return np.searchsorted(cdf, rng.random(n), side="right").astype(np.int64)


def config2(n: int, seed: int, card: int = 1000) -> dict:
    """The scan + group-by columns: key i32 Zipf(1.1) over `card` values,
    dictionary-encoded and bit-packed; price LogNormal(3,1); qty U[1,100];
    ts strictly increasing in runs of 1-64 (RLE)."""
    from voxel_b200 import encode

    rng = np.random.default_rng(seed)
    if card <= 100_000:
        values = np.sort(rng.choice(np.arange(-50000, 50000, dtype=np.int64), size=card, replace=False)).astype(np.int32)
    else:  # large dictionaries: distinct i32 values over the whole range
        values = np.unique(rng.integers(-(2**31), 2**31 - 1, size=card + card // 4 + 16, dtype=np.int64))
        values = np.sort(rng.permutation(values)[:card]).astype(np.int32)
    rank = zipf_alias_keys(n, card, 1.1, rng)
    perm = rng.permutation(card)
    code = perm[rank]                      # position of each row's key in the sorted value list
    key = values[code]
    price = rng.lognormal(3.0, 1.0, n)
    qty = rng.integers(1, 101, size=n).astype(np.int32)
    # the reference dictionary: sorted unique values present, u32 indices into it
    present = np.bincount(code, minlength=card) > 0
    remap = (np.cumsum(present) - 1).astype(np.uint32)
    dict_ = values[present]
    idx = remap[code]
    width = encode.bit_width(idx)
    packed = encode.bitpack(idx, width)
    return dict(n=n, key=key, dict=dict_, idx=idx, width=width, packed=packed, price=price, qty=qty)


def codec_ints(npt, n: int, seed: int) -> np.ndarray:
    """A mostly increasing integer column with negative steps and wraps (the
    delta codec's inputs): a random walk of steps in [-1000, 100000)."""
    rng = np.random.default_rng(seed)
    steps = rng.integers(-1000, 100_000, size=n, dtype=np.int64)
    start = int(rng.integers(-(2**40), 2**40))
    info = np.iinfo(npt)
    walk = (start + np.cumsum(steps)).astype(object) if n else np.zeros(0, object)
    mod = 1 << info.bits
    vals = [(int(v) % mod) for v in walk]
    out = np.array(vals, dtype=np.uint64 if info.bits == 64 else np.uint32)
    return out.view(npt) if out.size else np.zeros(0, npt)


def codec_f64(n: int, seed: int) -> np.ndarray:
    """A price-like f64 column for the frame-of-reference codec."""
    rng = np.random.default_rng(seed)
    return rng.lognormal(3.0, 1.0, n) - 10.0


def merge_join_input(npt, nl: int, nr: int, dup: int, seed: int):
    """Sorted left / right key columns of one integer type with runs of equal
    keys (up to `dup` copies) and keys on one side only."""
    rng = np.random.default_rng(seed)
    info = np.iinfo(npt)
    lo = max(int(info.min), -(2**40))
    hi = min(int(info.max), 2**40)
    pool = np.unique(rng.integers(lo, hi, size=max(nl, nr) // 2 + 8, dtype=np.int64))

    def side(n):
        if n == 0:
            return np.zeros(0, npt)
        k = pool[rng.integers(0, pool.size, size=n)]
        k = np.repeat(k, rng.integers(1, dup + 1, size=n))[:n]
        return np.sort(k).astype(npt)

    return side(nl), side(nr)


def shuffled(a: np.ndarray, seed: int) -> np.ndarray:
    """A seeded permutation of `a` (the semi / anti joins' unordered left side)."""
    return np.random.default_rng(seed + 1).permutation(a) if a.size else a


WINDOW_NP = {0: np.float64, 2: np.int64, 3: np.int32, 4: np.uint64, 5: np.uint32}


def window_values(dtype: int, n: int, seed: int) -> np.ndarray:
    """A noisy trend with repeats (ties for the quantile), per element type."""
    rng = np.random.default_rng(seed)
    base = np.cumsum(rng.normal(0.0, 3.0, n)) + rng.integers(0, 5, n) * 0.5
    if dtype == 0:
        return base.astype(np.float64)
    v = np.round(base * 1000).astype(np.int64)
    if dtype in (4, 5):
        v = np.abs(v)
    return v.astype(WINDOW_NP[dtype])


def time_window_input(dtype: int, n: int, seed: int):
    """Non-decreasing i64 timestamps (steps 0-3) and values of the element type."""
    rng = np.random.default_rng(seed)
    ts = np.cumsum(rng.integers(0, 4, n)).astype(np.int64) - 50
    return ts, window_values(dtype, n, seed + 7)
