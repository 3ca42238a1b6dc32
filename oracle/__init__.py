"""The oracle: CPU checkers for the CUDA backend (test infrastructure only).

``port()`` is the plain-C restatement (``oracle/voxel_oracle.c``);
``ref()`` is the reference VoxelVM's own operators compiled from its sources
(``oracle/ref_driver.cpp``, present when the reference tree was available at
build time).  Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline use this package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build_oracle

vp, sz = C.c_void_p, C.c_size_t
u8, u32, u64, i32, i64, dbl = C.c_uint8, C.c_uint32, C.c_uint64, C.c_int32, C.c_int64, C.c_double

_port = None
_ref = None


class AggState(C.Structure):
    _fields_ = [("init", C.c_int32), ("count", C.c_uint64), ("sum_f64", C.c_double),
                ("sum_i64", C.c_int64), ("min_bits", C.c_uint64), ("max_bits", C.c_uint64)]


def port() -> C.CDLL:
    global _port
    if _port is None:
        path = build_oracle.ORACLE_SO
        if not os.path.exists(path):
            build_oracle.build_restatement()
        L = C.CDLL(path)
        L.vo_engine_run.restype = C.c_int
        L.vo_engine_run.argtypes = [C.c_int, vp, sz, vp, vp, sz, vp, vp, u64, C.POINTER(C.c_int)]
        L.vo_vfilter.restype = sz
        L.vo_vfilter.argtypes = [C.c_int, C.c_int, vp, sz, u64, u64, vp]
        L.vo_selection_from_bitmap.restype = sz
        L.vo_selection_from_bitmap.argtypes = [vp, sz, vp]
        L.vo_bitmap_and.restype = sz
        L.vo_bitmap_and.argtypes = [vp, sz, sz, vp]
        L.vo_bitpack_width.restype = u32
        L.vo_bitpack_width.argtypes = [vp, sz]
        L.vo_bitpack_build.restype = sz
        L.vo_bitpack_build.argtypes = [vp, sz, u32, vp]
        L.vo_bitpack_decode.restype = None
        L.vo_bitpack_decode.argtypes = [vp, sz, u32, sz, sz, sz, vp]
        L.vo_dict_build_i32.restype = sz
        L.vo_dict_build_i32.argtypes = [vp, sz, vp, vp]
        L.vo_dict_decode_i32.restype = None
        L.vo_dict_decode_i32.argtypes = [vp, sz, vp, sz, sz, sz, vp]
        L.vo_window_f64.restype = sz
        L.vo_window_f64.argtypes = [C.c_int, vp, sz, vp, sz, C.c_uint, dbl]
        L.vo_time_window_sum_f64.restype = sz
        L.vo_time_window_sum_f64.argtypes = [vp, vp, sz, i64, i64, vp, sz]
        L.vo_merge_join_i64.restype = sz
        L.vo_merge_join_i64.argtypes = [vp, sz, vp, sz, vp, vp, sz, C.c_int]
        L.vo_semi_join_i64.restype = sz
        L.vo_semi_join_i64.argtypes = [vp, sz, vp, sz, vp, C.c_int]
        L.vo_delta_build.restype = None
        L.vo_delta_build.argtypes = [C.c_int, vp, sz, vp]
        L.vo_delta_decode.restype = None
        L.vo_delta_decode.argtypes = [C.c_int, vp, sz, u64, sz, sz, vp]
        L.vo_for_decode_f64.restype = None
        L.vo_for_decode_f64.argtypes = [vp, sz, dbl, dbl, sz, sz, vp]
        L.vo_rle_build_i64.restype = sz
        L.vo_rle_build_i64.argtypes = [vp, sz, vp, vp]
        L.vo_rle_decode_i64.restype = None
        L.vo_rle_decode_i64.argtypes = [vp, vp, sz, sz, sz, vp]
        L.vo_groupby_i32_f64.restype = sz
        L.vo_groupby_i32_f64.argtypes = [vp, vp, sz, vp, vp, vp, vp, vp]
        L.vo_radix_sort.restype = None
        L.vo_radix_sort.argtypes = [C.c_int, vp, vp, sz]
        L.vo_hashjoin_i64.restype = sz
        L.vo_hashjoin_i64.argtypes = [vp, sz, vp, sz, vp, vp, sz, C.c_int]
        L.vo_scan_groupby.restype = sz
        L.vo_scan_groupby.argtypes = [vp, sz, u32, vp, sz, vp, vp, sz, dbl, i32, i32, vp, vp, vp, vp, vp]
        _port = L
    return _port


def have_ref() -> bool:
    return os.path.exists(build_oracle.REF_SO)


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        if not have_ref():
            raise RuntimeError("reference library oracle/_ref/libvoxel_ref.so is not built")
        L = C.CDLL(build_oracle.REF_SO)
        L.vref_engine_run.restype = C.c_int
        L.vref_engine_run.argtypes = [C.c_int, vp, sz, vp, vp, sz, vp, vp]
        L.vref_engine_run_parallel.restype = C.c_int
        L.vref_engine_run_parallel.argtypes = [C.c_int, vp, sz, vp, vp, sz, vp, sz, u32, u8, vp]
        L.vref_jit_run.restype = dbl
        L.vref_jit_run.argtypes = [vp, sz, vp, sz, dbl]
        L.vref_time_filter_sum_f64.restype = dbl
        L.vref_time_filter_sum_f64.argtypes = [C.c_int, vp, sz, vp, sz, dbl, C.c_int, C.c_int, u32, C.POINTER(dbl)]
        for t, ct in (("f64", dbl), ("f32", C.c_float), ("i64", i64), ("i32", i32), ("u64", u64), ("u32", u32)):
            f = getattr(L, f"vref_vfilter_{t}")
            f.restype = sz
            f.argtypes = [C.c_int, vp, sz, ct, ct, vp]
        L.vref_selection_from_bitmap.restype = sz
        L.vref_selection_from_bitmap.argtypes = [vp, sz, vp]
        L.vref_column_filter_and.restype = sz
        L.vref_column_filter_and.argtypes = [vp, sz, sz, vp]
        L.vref_bitpack_build.restype = u32
        L.vref_bitpack_build.argtypes = [vp, sz, vp, sz, C.POINTER(sz)]
        L.vref_bitpack_decode.restype = None
        L.vref_bitpack_decode.argtypes = [vp, sz, u32, sz, sz, sz, vp]
        L.vref_dict_build_i32.restype = sz
        L.vref_dict_build_i32.argtypes = [vp, sz, vp, vp]
        L.vref_dict_build_f64.restype = sz
        L.vref_dict_build_f64.argtypes = [vp, sz, vp, vp]
        L.vref_dict_decode_i32.restype = None
        L.vref_dict_decode_i32.argtypes = [vp, sz, vp, sz, sz, sz, vp]
        L.vref_dict_decode_f64.restype = None
        L.vref_dict_decode_f64.argtypes = [vp, sz, vp, sz, sz, sz, vp]
        L.vref_rle_build_i64.restype = sz
        L.vref_rle_build_i64.argtypes = [vp, sz, vp, vp]
        L.vref_rle_decode_i64.restype = None
        L.vref_rle_decode_i64.argtypes = [vp, vp, sz, sz, sz, vp]
        for k in ("i32", "u32", "i64"):
            f = getattr(L, f"vref_hashagg_{k}_f64")
            f.restype = sz
            f.argtypes = [vp, vp, sz, sz, vp, vp, vp, vp, vp]
        L.vref_grouped_agg_i32_f64.restype = sz
        L.vref_grouped_agg_i32_f64.argtypes = [vp, vp, sz, vp, vp, vp, vp, vp]
        for k in ("u64", "u32", "i64", "i32"):
            f = getattr(L, f"vref_radix_sort_{k}")
            f.restype = None
            f.argtypes = [vp, vp, sz]
        L.vref_sort_ascending_f64.restype = None
        L.vref_sort_ascending_f64.argtypes = [vp, sz, vp]
        L.vref_sort_descending_f64.restype = None
        L.vref_sort_descending_f64.argtypes = [vp, sz, vp]
        L.vref_topk_f64.restype = None
        L.vref_topk_f64.argtypes = [vp, sz, sz, vp, C.c_int]
        for k in ("i64", "u32", "i32"):
            f = getattr(L, f"vref_hashjoin_{k}")
            f.restype = sz
            f.argtypes = [vp, sz, vp, sz, vp, vp, sz, C.c_int]
        for t in ("i64", "i32", "u64", "u32"):
            f = getattr(L, f"vref_delta_build_{t}")
            f.restype = u64
            f.argtypes = [vp, sz, vp]
            f = getattr(L, f"vref_delta_decode_{t}")
            f.restype = None
            f.argtypes = [vp, sz, u64, sz, sz, vp]
        L.vref_for_build_f64.restype = None
        L.vref_for_build_f64.argtypes = [vp, sz, vp, C.POINTER(dbl), C.POINTER(dbl)]
        L.vref_for_decode_f64.restype = None
        L.vref_for_decode_f64.argtypes = [vp, sz, dbl, dbl, sz, sz, vp]
        for t in ("i64", "i32", "u64", "u32"):
            f = getattr(L, f"vref_merge_join_{t}")
            f.restype = sz
            f.argtypes = [vp, sz, vp, sz, vp, vp, C.c_int]
            f = getattr(L, f"vref_semi_join_{t}")
            f.restype = sz
            f.argtypes = [vp, sz, vp, sz, vp, C.c_int]
        for t in ("f64", "i64", "i32", "u64", "u32"):
            f = getattr(L, f"vref_window_{t}")
            f.restype = sz
            f.argtypes = [C.c_int, vp, sz, vp, sz, C.c_uint8, dbl]
            f = getattr(L, f"vref_time_window_sum_{t}")
            f.restype = sz
            f.argtypes = [vp, vp, sz, i64, i64, vp, sz]
        L.vref_scalar_filter_gt_f32.restype = sz
        L.vref_scalar_filter_gt_f32.argtypes = [vp, vp, C.c_float, sz]
        L.vref_scalar_sum_f32.restype = C.c_float
        L.vref_scalar_sum_f32.argtypes = [vp, sz]
        L.vref_scan_groupby.restype = sz
        L.vref_scan_groupby.argtypes = [vp, sz, u32, vp, sz, vp, vp, sz, dbl, i32, i32, C.c_int,
                                        vp, vp, vp, vp, vp, C.POINTER(dbl)]
        _ref = L
    return _ref


# ---- convenience wrappers ------------------------------------------------------

def _segs(arrays):
    ptrs = (C.c_void_p * max(1, len(arrays)))(*[a.ctypes.data for a in arrays])
    counts = (C.c_size_t * max(1, len(arrays)))(*[a.size for a in arrays])
    return ptrs, counts


def engine_run_port(dtype: int, code, arrays, regs, agg=None, max_steps=1 << 34):
    """Restated interpreter: returns (status, regs_out list, fast_path flag)."""
    code = np.asarray(code, dtype=np.uint32)
    r = np.array([x & 0xFFFFFFFFFFFFFFFF for x in regs] + [0] * (64 - len(regs)), dtype=np.uint64)
    ptrs, counts = _segs(arrays)
    fp = C.c_int(0)
    st = port().vo_engine_run(dtype, code.ctypes.data, code.size, ptrs, counts, len(arrays),
                              r.ctypes.data, C.cast(agg, vp) if agg is not None else None, max_steps, C.byref(fp))
    return st, [int(x) for x in r], fp.value


def engine_run_ref(dtype: int, code, arrays, regs):
    """The reference Engine<T>::Run itself; returns the 64 registers."""
    code = np.asarray(code, dtype=np.uint32)
    rin = np.array([x & 0xFFFFFFFFFFFFFFFF for x in regs] + [0] * (64 - len(regs)), dtype=np.uint64)
    rout = np.zeros(64, dtype=np.uint64)
    ptrs, counts = _segs(arrays)
    st = ref().vref_engine_run(dtype, code.ctypes.data, code.size, ptrs, counts, len(arrays),
                               rin.ctypes.data, rout.ctypes.data)
    if st:
        raise RuntimeError(f"reference engine has no dtype {dtype}")
    return [int(x) for x in rout]


def groupby_port(keys: np.ndarray, vals: np.ndarray):
    n = keys.size
    ok, s, mn, mx = (np.zeros(max(n, 1), t) for t in (np.int32, np.float64, np.float64, np.float64))
    c = np.zeros(max(n, 1), np.uint64)
    g = port().vo_groupby_i32_f64(keys.ctypes.data, vals.ctypes.data, n, ok.ctypes.data, s.ctypes.data,
                                  mn.ctypes.data, mx.ctypes.data, c.ctypes.data)
    return ok[:g], s[:g], mn[:g], mx[:g], c[:g]


def scan_groupby_port(packed, width, dict_, price, qty, pthr, qlo, qhi):
    card = dict_.size
    ok, s, mn, mx = (np.zeros(max(card, 1), t) for t in (np.int32, np.float64, np.float64, np.float64))
    c = np.zeros(max(card, 1), np.uint64)
    g = port().vo_scan_groupby(packed.ctypes.data, packed.size, width, dict_.ctypes.data, card,
                               price.ctypes.data, qty.ctypes.data, price.size, pthr, qlo, qhi,
                               ok.ctypes.data, s.ctypes.data, mn.ctypes.data, mx.ctypes.data, c.ctypes.data)
    return ok[:g], s[:g], mn[:g], mx[:g], c[:g]


def scan_groupby_ref(packed, width, dict_, price, qty, pthr, qlo, qhi, threads=1):
    """Reference operators composed (sorted by key on return); also returns seconds."""
    card = dict_.size
    ok, s, mn, mx = (np.zeros(max(card, 1), t) for t in (np.int32, np.float64, np.float64, np.float64))
    c = np.zeros(max(card, 1), np.uint64)
    us = C.c_double(0)
    g = ref().vref_scan_groupby(packed.ctypes.data, packed.size, width, dict_.ctypes.data, card,
                                price.ctypes.data, qty.ctypes.data, price.size, pthr, qlo, qhi, threads,
                                ok.ctypes.data, s.ctypes.data, mn.ctypes.data, mx.ctypes.data, c.ctypes.data,
                                C.byref(us))
    o = np.argsort(ok[:g], kind="stable")
    return ok[:g][o], s[:g][o], mn[:g][o], mx[:g][o], c[:g][o], us.value * 1e-6


def f32_selection_ref(preds, col):
    """The rows an f32 program's conjunctive predicates select, decided by the
    reference's own operators: VectorFilter<f32>::Apply* per predicate
    (filter.hpp:42-288) and ColumnFilter::AndWith (526-547), then
    SelectionVector::BuildFromBitmap (378-399).  preds: (op, value) pairs,
    op 0 EQ .. 5 GE.  Returns the ascending row ids."""
    L = ref()
    col = np.ascontiguousarray(col, dtype=np.float32)
    n = col.size
    words = max((n + 63) // 64, 1)
    bms = []
    for op, v in preds:
        bm = np.zeros(words, np.uint64)
        L.vref_vfilter_f32(op, col.ctypes.data, n, float(np.float32(v)), 0.0, bm.ctypes.data)
        bms.append(bm)
    ptrs = (C.c_void_p * len(bms))(*[b.ctypes.data for b in bms])
    out = np.zeros(words, np.uint64)
    L.vref_column_filter_and(ptrs, len(bms), n, out.ctypes.data)
    sel = np.zeros(max(n, 1), np.uint32)
    k = L.vref_selection_from_bitmap(out.ctypes.data, n, sel.ctypes.data)
    return sel[:k]


def f32_filter_gt_ref(col, threshold):
    """simd/scalar.hpp:214-227: the values > threshold in row order."""
    col = np.ascontiguousarray(col, dtype=np.float32)
    out = np.zeros(max(col.size, 1), np.float32)
    k = ref().vref_scalar_filter_gt_f32(out.ctypes.data, col.ctypes.data, float(np.float32(threshold)), col.size)
    return out[:k]


def f32_program_expect(preds, aggs, col):
    """Expected results of an f32 filter/aggregate program whose rows are
    selected by the reference's VectorFilter<f32> + ColumnFilter: COUNT is the
    number of selected rows, SUM their exact sum (the programs accumulate in
    f64; compare within 1e-6 relative), MIN / MAX the extreme selected value or
    the template's sentinel when nothing is selected."""
    import math

    from voxel_b200 import templates as T

    sel = f32_selection_ref([(p.op, p.value) for p in preds], col)
    vals = np.asarray(col, np.float32)[sel]
    out = {}
    for a in aggs:
        if a == "COUNT":
            out[a] = int(sel.size)
        elif a == "SUM":
            out[a] = math.fsum(vals.astype(np.float64))
        elif vals.size == 0:
            out[a] = float(T.sentinel(T.F32, a))
        else:
            out[a] = float(vals.min() if a == "MIN" else vals.max())
    return out
