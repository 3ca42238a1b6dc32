"""Host-side column encoders (the data generator's side of the formats).

The layouts are the reference's (include/voxel/data/encoding.hpp):
dictionary = sorted unique values + u32 indices (113-150); bit-packed =
value i at bit i*w of little-endian u64 words, LSB first, straddling into the
next word (370-395, 439-449); RLE = (value, u32 run length) pairs (202-220).
Decoding is the backend's job; encoding happens once, when data is generated.
"""
from __future__ import annotations

import numpy as np


def dict_build_i32(values: np.ndarray):
    d, idx = np.unique(values, return_inverse=True)
    return d.astype(values.dtype), idx.astype(np.uint32)


def bit_width(idx: np.ndarray) -> int:
    m = int(idx.max()) if idx.size else 0
    return max(1, m.bit_length())


def bitpack(idx: np.ndarray, w: int) -> np.ndarray:
    n = idx.size
    nwords = (n * w + 63) // 64
    blocks = (n + 63) // 64
    v = np.zeros(blocks * 64, np.uint64)
    v[:n] = idx.astype(np.uint64) & np.uint64((1 << w) - 1)
    v = v.reshape(blocks, 64)
    out = np.zeros((blocks, w + 1), np.uint64)
    for j in range(64):
        bit = j * w
        word, sh = bit // 64, bit % 64
        out[:, word] |= v[:, j] << np.uint64(sh)
        if sh + w > 64:
            out[:, word + 1] |= v[:, j] >> np.uint64(64 - sh)
    return np.ascontiguousarray(out[:, :w]).reshape(-1)[:nwords].copy()


def rle_build(values: np.ndarray):
    if values.size == 0:
        return values[:0].copy(), np.zeros(0, np.uint32)
    starts = np.flatnonzero(np.concatenate(([True], values[1:] != values[:-1])))
    runs = np.diff(np.concatenate((starts, [values.size]))).astype(np.uint32)
    return values[starts].copy(), runs
