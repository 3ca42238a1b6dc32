"""Plan choices from the learned estimator: the HashAggregator table size,
hash- vs sort-based GROUP BY, and the hash join's build side.

The estimator is the FP32 MLP of voxel_b200/estimator.py (its forward pass is
a CUDA kernel): from a column's device sketch (min / max, 64-bucket histogram,
HyperLogLog registers) and a predicate set it predicts the selected rows and
the distinct selected values.  Here those estimates pick plans:

* GROUP BY: the expected group count sizes the table the way
  HashAggregator::Init(expected) does (reference include/voxel/ops/
  aggregate.hpp:159-166: nextpow2(2 * expected) slots), and above
  `SORT_ABOVE` estimated groups the sort-based GroupedAggregator plan
  (aggregate.hpp:665-706, over radix-sorted keys) replaces the hash table.
* JOIN: the side with fewer estimated rows after its filters is built
  (HashJoin::Build, join.hpp:36-48); when that is the left side the pairs are
  re-ordered into the reference's order (left rows ascending, each one's
  matches newest first), so the pair list is the same either way.

Results never depend on the model: a table sized too small grows by
doubling (the exact path), both GROUP BY plans sum the same fixed-point
integers (bit-identical outputs), and the join's pair list is re-ordered to
the reference's.  Without a model the planner takes the reference's defaults
(HashAggregator::Init(128) as the Python front end sizes it, hash plan, the
right side built).  Each plan keeps its estimate, so callers can report the
q-error against the exact counts the run measures.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import capi
from . import estimator as E
from . import templates as T

DEFAULT_EXPECTED_GROUPS = 128  # bindings/voxel_query.py:173 (HashAggregator.init(128))
SORT_ABOVE = 1 << 20           # estimated groups above which the sort-based plan is taken
U32 = 5
I64 = 2


@dataclass
class GroupByPlan:
    method: str                 # "hash" or "sort"
    expected_groups: int        # the table size hint (hash plan)
    estimated_groups: float | None
    source: str                 # "model" or "default"


@dataclass
class JoinPlan:
    build: str                  # "right" (the reference's) or "left"
    estimated_left: float
    estimated_right: float
    source: str


def _all_rows_pred(sk: E.Sketch):
    # x >= min: every row, a predicate set inside the model's training domain
    return [T.Pred(5, float(sk.min))]


def estimate(dtype: int, dcol: int, n: int, preds, model) -> tuple[float, float]:
    """(selected rows, distinct selected values) the model predicts for a
    device column and a conjunctive predicate list (empty: every row)."""
    sk = E.sketch(dtype, dcol, n)
    preds = list(preds) if preds else _all_rows_pred(sk)
    f = E.features(dtype, sk, preds)
    y = model.predict(f[None, :])[0]
    rows, distinct = E.decode(y, n)
    return min(max(rows, 0.0), float(n)), min(max(distinct, 1.0), float(max(n, 1)))


def plan_groupby(dkeys: int, n: int, model=None, sort_above: int = SORT_ABOVE) -> GroupByPlan:
    """A plan for GROUP BY over a device column of u32 keys."""
    if model is None or n == 0:
        return GroupByPlan("hash", DEFAULT_EXPECTED_GROUPS, None, "default")
    _, d = estimate(U32, dkeys, n, None, model)
    method = "sort" if d > sort_above else "hash"
    return GroupByPlan(method, int(math.ceil(d * 1.25)) + 1, d, "model")


def run_groupby(plan: GroupByPlan, dkeys: int, dvals: int, n: int, out: dict, stream=None) -> int:
    """Runs the plan; `out` holds device pointers keys / sum / min / max /
    count with room for every group.  Returns the group count."""
    ng = C.c_uint64(0)
    st = capi.lib().voxel_groupby_u32_f64_dev(dkeys, dvals, n, plan.expected_groups, 1 if plan.method == "sort" else 0,
                                              out["keys"], out["sum"], out["min"], out["max"], out["count"],
                                              C.byref(ng), stream)
    if st:
        raise RuntimeError(capi.last_error())
    return int(ng.value)


def plan_join(left, right, model=None) -> JoinPlan:
    """left / right: (dtype, device column, rows, predicate list) of the two
    join sides before their filters.  Builds on the side with fewer
    estimated rows after the filters (the right side without a model)."""
    if model is None:
        return JoinPlan("right", float(left[2]), float(right[2]), "default")
    el = estimate(left[0], left[1], left[2], left[3], model)[0] if left[3] else float(left[2])
    er = estimate(right[0], right[1], right[2], right[3], model)[0] if right[3] else float(right[2])
    return JoinPlan("left" if el < er else "right", el, er, "model")


def select_rows(dtype: int, dcol: int, n: int, preds, d_bitmaps, d_bitmap_and, d_rows, stream=None) -> int:
    """Row ids (ascending, u32) of a device column passing a conjunctive
    predicate list, on the GPU: VectorFilter per predicate, ColumnFilter AND,
    SelectionVector.  d_bitmaps: one device bitmap per predicate
    (ceil(n/64) words each); returns the count."""
    L = capi.lib()
    import torch  # noqa: PLC0415  (device scratch for the counts)

    cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
    ptrs = []
    for p, bm in zip(preds, d_bitmaps):
        thr = T.reg_image(dtype, p.value) if dtype != T.F32 else int(np.float32(p.value).view(np.uint32))
        if L.voxel_vfilter_dev(dtype, p.op, dcol, n, thr, 0, bm, cnt.data_ptr(), stream):
            raise RuntimeError(capi.last_error())
        ptrs.append(bm)
    arr = (C.c_void_p * len(ptrs))(*ptrs)
    if L.voxel_bitmap_and_dev(arr, len(ptrs), n, d_bitmap_and, cnt.data_ptr(), stream):
        raise RuntimeError(capi.last_error())
    if L.voxel_selection_from_bitmap_dev(d_bitmap_and, n, d_rows, cnt.data_ptr() + 8, stream):
        raise RuntimeError(capi.last_error())
    return int(cnt[1].item())


def run_join(plan: JoinPlan, dl: int, nl: int, dr: int, nr: int, d_left_out: int, d_right_out: int, cap: int,
             d_tmp_a: int, d_tmp_b: int, stream=None) -> int:
    """Inner hash join of two device i64 key columns: the pairs (left row,
    right row) of HashJoin::Build(right) + ProbeAllMatches(left), in that
    order whichever side the plan builds.  d_tmp_a / d_tmp_b: u32 scratch of
    `cap` entries for the swapped plan.  Returns the pair count."""
    import torch  # noqa: PLC0415

    L = capi.lib()
    cs = torch.zeros(4, dtype=torch.int64, device="cuda")
    if plan.build == "right":
        if L.voxel_hashjoin_i64_dev(dr, None, nr, dl, nl, d_left_out, d_right_out, cap, 1, cs.data_ptr(), stream):
            raise RuntimeError(capi.last_error())
        return int(cs[0].item())
    # built on the left: (right row, left row) pairs in right-row order, re-ordered
    if L.voxel_hashjoin_i64_dev(dl, None, nl, dr, nr, d_tmp_a, d_tmp_b, cap, 1, cs.data_ptr(), stream):
        raise RuntimeError(capi.last_error())
    m = int(cs[0].item())
    if L.voxel_join_pairs_swap_order_dev(d_tmp_a, d_tmp_b, m, d_left_out, d_right_out, stream):
        raise RuntimeError(capi.last_error())
    return m


def planner_training_set(columns, per_column: int, rng: np.random.Generator):
    """Engine-measured training samples for the plan estimates: per device
    column (dtype, tensor), `per_column` predicate sets with thresholds spread
    over the column's range, plus the all-rows set (x >= min), labelled with
    the exact selected rows and distinct selected values
    (voxel_exact_labels_dev)."""
    L = E._setup()
    X, Y, meta = [], [], []
    for dtype, dcol in columns:
        n = dcol.numel()
        sk = E.sketch(dtype, dcol.data_ptr(), n)
        lo, hi = float(sk.min), float(sk.max)
        sets = [_all_rows_pred(sk)]
        for _ in range(per_column - 1):
            a, b = sorted(rng.uniform(lo, hi, 2))
            if dtype not in (T.F64, T.F32):
                a, b = math.floor(a), math.ceil(b)
            k = int(rng.integers(0, 3))
            sets.append([T.Pred(5, a)] if k == 0 else [T.Pred(2, b)] if k == 1 else [T.Pred(5, a), T.Pred(2, b)])
        ps = (E.PredSet * len(sets))(*[E.pred_set(dtype, p) for p in sets])
        rows = np.zeros(len(sets), np.uint64)
        dist = np.zeros(len(sets), np.uint64)
        if L.voxel_exact_labels_dev(dtype, dcol.data_ptr(), n, ps, len(sets), rows.ctypes.data, dist.ctypes.data):
            raise RuntimeError(capi.last_error())
        for p, r, d in zip(sets, rows, dist):
            X.append(E.features(dtype, sk, p))
            Y.append(E.targets(int(r), n, int(d)))
            meta.append((n, int(r), int(d)))
    return np.asarray(X, np.float32), np.asarray(Y, np.float32), meta
