"""Generate tests/golden/frontend.json from the reference's Python query
builder (bindings/voxel_query.py) running on the reference's own voxel_py
module (bindings/voxel_bindings.cpp, compiled by
oracle/build_oracle.build_reference_py into oracle/_ref/refpy).

Each case is a chain of builder calls on a seeded f64 column whose length is
a multiple of the 4 lanes (the reference's loops only terminate then); the
recorded result is the double's bits, an index or value array's digest, or an
integer.  Queries whose reference loop never ends (two aggregates, row counts
that are not a multiple of the lanes) are not run here: they spin in the
reference.

    python tests/golden/make_frontend_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build_oracle  # noqa: E402

OUT = os.path.join(HERE, "frontend.json")

# (name, column transform, chain of (method, args))
CASES = [
    ("sum_gt", "plain", [("filter_gt", (500.0,)), ("sum", ())]),
    ("sum_ge", "plain", [("filter_ge", (250.5,)), ("sum", ())]),
    ("sum_lt", "plain", [("filter_lt", (100.0,)), ("sum", ())]),
    ("sum_le", "shifted", [("filter_le", (-3.0,)), ("sum", ())]),
    ("sum_eq", "ints", [("filter_eq", (7.0,)), ("sum", ())]),
    ("sum_ne", "ints", [("filter_ne", (7.0,)), ("sum", ())]),
    ("sum_all", "plain", [("sum", ())]),
    ("default_sum", "plain", []),
    ("count_gt", "plain", [("filter_gt", (500.0,)), ("count", ())]),
    ("count_all", "withzeros", [("count", ())]),
    ("min_all", "plain", [("min", ())]),
    ("max_all", "plain", [("max", ())]),
    ("min_lt_negative", "shifted", [("filter_lt", (0.0,)), ("min", ())]),
    ("max_gt", "shifted", [("filter_gt", (100.0,)), ("max", ())]),
    ("max_negative", "negative", [("max", ())]),
    ("last_filter_wins", "plain", [("filter_gt", (100.0,)), ("filter_lt", (600.0,)), ("sum", ())]),
    ("group_by", "plain", [("group_by", ("keys",))]),
    ("sort", "plain", [("sort", ())]),
    ("sort_desc_flag", "plain", [("sort", (False,))]),
    ("topk_largest", "plain", [("topk", (5, True))]),
    ("topk_smallest", "plain", [("topk", (7, False))]),
]


def column(kind: str, n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    x = rng.random(n) * 1000.0
    if kind == "shifted":
        return x - 500.0
    if kind == "ints":
        return np.floor(x / 50.0)
    if kind == "withzeros":
        x[rng.random(n) < 0.3] = 0.0
        return x
    if kind == "negative":
        return -x - 1.0
    return x


def keys_for(n: int, seed: int) -> np.ndarray:
    return (np.random.default_rng(seed + 1).zipf(1.5, n) % 97).astype(np.uint32)


def encode(result):
    if isinstance(result, float):
        return {"f64_bits": struct.unpack("<Q", struct.pack("<d", result))[0]}
    if isinstance(result, (int, np.integer)):
        return {"int": int(result)}
    a = np.ascontiguousarray(result)
    return {"dtype": str(a.dtype), "size": int(a.size), "digest": hashlib.sha256(a.tobytes()).hexdigest()}


def run_case(vq, chain, x, keys):
    q = vq.from_numpy(x)
    for method, args in chain:
        args = tuple(keys if a == "keys" else a for a in args)
        q = getattr(q, method)(*args)
    return q.run()


def main():
    build_oracle.build()
    so = build_oracle.build_reference_py()
    if so is None:
        raise SystemExit("the reference's pybind module could not be built")
    sys.path.insert(0, os.path.dirname(so))
    sys.path.insert(0, os.path.join(build_oracle.reference_root(), "bindings"))
    import voxel_query as vq  # the reference's front end on the reference's voxel_py

    cases = []
    for seed, n in ((11, 4000), (12, 65536)):
        for name, kind, chain in CASES:
            x = column(kind, n, seed)
            keys = keys_for(n, seed)
            cases.append(dict(name=name, kind=kind, n=n, seed=seed, chain=[[m, list(a)] for m, a in chain],
                              result=encode(run_case(vq, chain, x, keys))))
    x = column("plain", 4000, 13)
    extra = dict(filter_and_sum=encode(vq.filter_and_sum(x, 500.0)),
                 filter_and_count=encode(vq.filter_and_count(x, 500.0)),
                 group_sum=encode(vq.group_sum(x, keys_for(4000, 13))),
                 from_list_sum=encode(vq.from_list([1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0, 8.0]).filter_gt(2.5).sum().run()))
    with open(OUT, "w") as f:
        json.dump(dict(source="reference bindings/voxel_query.py on the reference's voxel_py", cases=cases,
                       helpers=extra), f, indent=1)
    print(f"wrote {OUT}: {len(cases)} cases")


if __name__ == "__main__":
    main()
