"""Query builder with the interface of VoxelVM's Python front end
(reference bindings/voxel_query.py), executed on the B200 backend.

    import voxel_query as vq          # with voxel_b200/frontend on sys.path
    vq.from_numpy(data).filter_gt(500.0).sum().run()

Each call emits the same bytecode the reference's builder emits (same
registers: R0 accumulator, R1 offset, R2 total, R3 threshold, R4 lanes; the
same loop shapes, bindings/voxel_query.py:79-139), so results are the
reference's, including its quirks, which are kept deliberately:

* only the last filter_* call applies (each one overwrites R3 and the compare);
* count() returns the integer count's bits read as a double, because run()
  resets the integer-result flag before reading the result (voxel_query.py:
  108, 162);
* min() / max() fold with CMP + JLE / JGE, an integer compare of the f64 bit
  patterns, starting from R0 = 0.0 (voxel_query.py:116-139): min() of positive
  data is 0.0, and negative values order backwards;
* two aggregates in one query run two loops back to back; the second never
  reaches its exit (the reference spins): here it raises VoxelError.

The loops lower onto fused GPU kernels (voxel_b200.engine.Engine);
group_by, sort and topk run the GPU HashAggregator, sort and top-k operators
through the C ABI (voxel_agg_*, voxel_sort_ascending, voxel_topk).
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(os.path.dirname(_HERE))
if _ROOT not in sys.path:
    sys.path.insert(0, _ROOT)

from voxel_b200 import bytecode as _bc  # noqa: E402
from voxel_b200 import capi as _capi  # noqa: E402
from voxel_b200.engine import Engine as _Engine  # noqa: E402

# compare codes (voxel_py CMP_*)
CMP_EQ, CMP_NE, CMP_LT, CMP_LE, CMP_GT, CMP_GE = 0, 1, 2, 3, 4, 5
_F64 = 0


class Query:
    def __init__(self):
        self._engine = None
        self._seg_id = 0
        self._code = []
        self._result_reg = 0
        self._reg_counter = 5  # R0-R4 reserved: acc, offset, total, threshold, lanes
        self._offset_reg = 1
        self._total_reg = 2
        self._thresh_reg = 3
        self._acc_reg = 0
        self._lane_reg = 4
        self._vec_counter = 0

    def _emit(self, raw: int):
        self._code.append(raw)

    def _alloc_reg(self):
        r = self._reg_counter
        self._reg_counter += 1
        return r

    def _filter(self, threshold, cmp):
        self._engine.set_scalar_f64(self._thresh_reg, float(threshold))
        self._has_filter = True
        self._filter_cmp = cmp
        return self

    def filter_gt(self, threshold):
        """Keep rows where value > threshold."""
        return self._filter(threshold, CMP_GT)

    def filter_ge(self, threshold):
        return self._filter(threshold, CMP_GE)

    def filter_eq(self, threshold):
        return self._filter(threshold, CMP_EQ)

    def filter_ne(self, threshold):
        return self._filter(threshold, CMP_NE)

    def filter_lt(self, threshold):
        return self._filter(threshold, CMP_LT)

    def filter_le(self, threshold):
        return self._filter(threshold, CMP_LE)

    def _emit_loop_body(self):
        """VLOAD [+ VFILTER]; returns the vector register holding the lanes."""
        self._emit(_bc.vload(0, self._offset_reg, self._seg_id))
        if getattr(self, "_has_filter", False):
            self._emit(_bc.vfilter(getattr(self, "_filter_cmp", CMP_GT), 1, 0, self._thresh_reg))
            return 1
        return 0

    def _loop_tail(self, back):
        lanes = self._engine.k_lanes
        self._emit(_bc.add(self._offset_reg, self._offset_reg, lanes))
        self._emit(_bc.cmp(self._offset_reg, self._total_reg))
        self._emit(_bc.jnz(back))

    def sum(self):
        r5 = self._alloc_reg()
        vr = self._emit_loop_body()
        self._emit(_bc.vsum(r5, vr))
        self._emit(_bc.addf(self._acc_reg, self._acc_reg, r5))
        self._loop_tail(-6)
        return self

    def count(self):
        r5 = self._alloc_reg()
        vr = self._emit_loop_body()
        self._emit(_bc.vcount(r5, vr))
        self._emit(_bc.add(self._acc_reg, self._acc_reg, r5))
        self._loop_tail(-6)
        self._result_is_int = True
        return self

    def min(self):
        r5 = self._alloc_reg()
        vr = self._emit_loop_body()
        self._emit(_bc.vred_min(r5, vr))
        self._emit(_bc.cmp(self._acc_reg, r5))
        self._emit(_bc.jle(2))
        self._emit(_bc.movr(self._acc_reg, r5))
        self._loop_tail(-8)
        return self

    def max(self):
        r5 = self._alloc_reg()
        vr = self._emit_loop_body()
        self._emit(_bc.vred_max(r5, vr))
        self._emit(_bc.cmp(self._acc_reg, r5))
        self._emit(_bc.jge(2))
        self._emit(_bc.movr(self._acc_reg, r5))
        self._loop_tail(-8)
        return self

    def sort(self, ascending=True):
        """Sort indices of the column (run() returns them; the GPU sort operator)."""
        self._sort_ascending = ascending
        return self

    def topk(self, k, largest=True):
        """Top-k values of the column (the GPU top-k operator)."""
        self._topk = k
        self._topk_largest = largest
        return self

    def group_by(self, group_keys):
        """Group by a u32 key column (run() returns the number of groups)."""
        self._group_keys = group_keys
        return self

    def run(self):
        """Compile and execute the query on the GPU; returns the result."""
        lanes = self._engine.k_lanes
        self._engine.set_scalar_f64(self._acc_reg, 0.0)
        self._engine.set_scalar(self._offset_reg, 0)
        self._engine.set_scalar(self._total_reg, self._total_count)
        self._result_is_int = False  # as the reference does: count()'s flag is lost here
        self._code.insert(0, _bc.mov(self._lane_reg, lanes))
        if len(self._code) == 1:
            self.sum()
        self._emit(_bc.halt())
        self._engine.load_program(self._code)
        self._engine.run()
        L = _capi.lib()
        if hasattr(self, "_group_keys"):
            keys = np.ascontiguousarray(self._group_keys, dtype=np.uint32)
            data = np.ascontiguousarray(self._data, dtype=np.float64)
            agg = L.voxel_agg_create()
            try:
                L.voxel_agg_init(agg, 128)
                L.voxel_agg_accumulate(agg, keys.ctypes.data, data.ctypes.data, min(keys.size, data.size))
                return int(L.voxel_agg_group_count(agg))
            finally:
                L.voxel_agg_destroy(agg)
        if hasattr(self, "_sort_ascending"):
            data = np.ascontiguousarray(self._data, dtype=np.float64)
            idx = np.zeros(data.size, np.uint32)
            L.voxel_sort_ascending(data.ctypes.data, data.size, idx.ctypes.data)
            return idx
        if hasattr(self, "_topk"):
            data = np.ascontiguousarray(self._data, dtype=np.float64)
            out = np.zeros(int(self._topk), np.float64)
            L.voxel_topk(data.ctypes.data, data.size, int(self._topk), out.ctypes.data, 1 if self._topk_largest else 0)
            return out
        if getattr(self, "_result_is_int", False):
            return self._engine.get_scalar(self._acc_reg)
        return self._engine.get_scalar_f64(self._acc_reg)


def from_numpy(data: np.ndarray) -> Query:
    """A query over an f64 column (other dtypes are converted, as the reference does)."""
    if data.dtype != np.float64:
        data = data.astype(np.float64)
    q = Query()
    q._engine = _Engine(_F64)
    q._data = data
    q._seg_id = q._engine.add_segment(data)
    q._total_count = len(data)
    return q


def from_list(values) -> Query:
    return from_numpy(np.array(values, dtype=np.float64))


def filter_and_sum(data, threshold):
    """One-shot filter + sum (the fused fast path)."""
    return from_numpy(data).filter_gt(threshold).sum().run()


def filter_and_count(data, threshold):
    """One-shot filter + count (returns the reference's reinterpreted result)."""
    return from_numpy(data).filter_gt(threshold).count().run()


def group_sum(data, groups):
    """Group by `groups` and sum: returns the number of groups (as the reference)."""
    q = from_numpy(data)
    q._group_keys = np.array(groups, dtype=np.uint32)
    return q.group_by(q._group_keys).run()
