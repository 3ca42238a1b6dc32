"""Generate tests/golden/fullsize.json: the reference's outputs on the
workloads at their full sizes, kept as digests.

Runs the reference VoxelVM itself (compiled from its sources by
oracle/build_oracle.py into oracle/_ref) once per seed on the same seeded
inputs the GPU tests and bench.py build, and records:

* scan + group-by, 2^25 rows (seed 2001): BitPackedEncoding / DictionaryEncoding
  decode, VectorFilter<f64>::ApplyGT, VectorFilter<i32>::ApplyBetween,
  ColumnFilter::AndWith, SelectionVector and HashAggregator<i32,f64> on one
  thread (row-order sums): group keys, counts, min/max bits (SHA-256) and the
  sums themselves;
* radix sort, 2^28 u64 SplitMix64 keys (seed 3001) with u32 row ids:
  RadixSort<u64>::Sort, SHA-256 of the sorted keys and of the permutation;
* hash join, build 2^24 even SplitMix64 keys (seed 3002, payload = build row),
  probe 2^29 keys (vgen_join_probe_i64, seed 3003: 90% Zipf(0.8) over the
  build keys, 10% odd keys that never match): HashJoin<i64>::Build +
  ProbeAllMatches, the match count, the u64 sum of the matched payloads and
  the SHA-256 of the (probe, build) pair arrays in probe order;
* the config-1 program `filter x > 500; SUM(x); COUNT` (and the SUM-only fast
  path program) over 2^28 f64 U[0,1000) from std::mt19937_64(42):
  Engine<f64>::Run registers R0 and R6.

Needs about 20 GB of host memory and a few minutes.

    python tests/golden/make_fullsize.py [--only config2,sort,join,config1]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import fullsize  # noqa: E402
import oracle  # noqa: E402
from oracle import build_oracle  # noqa: E402

OUT = os.path.join(HERE, "fullsize.json")


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(memoryview(np.ascontiguousarray(a)).cast("B"))
    return h.hexdigest()


def do_config2():
    d = fullsize.config2_input()
    t = time.time()
    k, s, mn, mx, c, _ = oracle.scan_groupby_ref(d["packed"], d["width"], d["dict"], d["price"], d["qty"],
                                                 fullsize.PTHR, fullsize.QLO, fullsize.QHI, threads=1)
    return dict(n=d["n"], seed=fullsize.SEED_CONFIG2, groups=int(k.size), keys_sha=sha(k), count_sha=sha(c),
                min_sha=sha(mn), max_sha=sha(mx), sums=[float(v) for v in s], seconds=time.time() - t)


def do_sort():
    keys = fullsize.sort_input()
    idx = np.arange(keys.size, dtype=np.uint32)
    t = time.time()
    oracle.ref().vref_radix_sort_u64(keys.ctypes.data, idx.ctypes.data, keys.size)
    secs = time.time() - t
    return dict(n=int(keys.size), seed=fullsize.SEED_SORT, keys_sha=sha(keys), idx_sha=sha(idx), seconds=secs)


def do_join():
    build, probe = fullsize.join_input()
    left = np.empty(probe.size, np.uint32)
    right = np.empty(probe.size, np.uint32)
    t = time.time()
    m = oracle.ref().vref_hashjoin_i64(build.ctypes.data, build.size, probe.ctypes.data, probe.size,
                                        left.ctypes.data, right.ctypes.data, probe.size, 1)
    secs = time.time() - t
    m = int(m)
    # payload = build row id, so SUM(payload) over the pairs is the sum of the build indices
    psum = int(right[:m].astype(np.uint64).sum(dtype=np.uint64))
    return dict(build=int(build.size), probe=int(probe.size), seed_build=fullsize.SEED_JOIN_BUILD,
                seed_probe=fullsize.SEED_JOIN_PROBE, matches=m, payload_sum=psum,
                pairs_sha=sha(left[:m], right[:m]), seconds=secs)


def do_config1():
    x = fullsize.config1_input()
    n = x.size
    from voxel_b200 import bytecode as bc
    from voxel_b200 import templates as T

    regs = [0, 0, n, T.reg_image(T.F64, 500.0), 4, 0, 0]
    t = time.time()
    r = oracle.engine_run_ref(T.F64, bc.filter_sum_count_program(), [x], regs)
    r1 = oracle.engine_run_ref(T.F64, bc.filter_sum_program(), [x], regs[:5])
    return dict(n=n, seed=fullsize.SEED_CONFIG1, sum_count_r0=r[0], sum_count_r6=r[6], sum_only_r0=r1[0],
                sum_only_r1=r1[1], seconds=time.time() - t)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="config2,sort,join,config1")
    args = ap.parse_args()
    build_oracle.build()
    if not oracle.have_ref():
        raise SystemExit("the reference library is required to generate the full-size fixtures")
    doc = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            doc = json.load(f)
    doc["source"] = "reference VoxelVM operators compiled by oracle/build_oracle.py, full-size workloads"
    for name, fn in (("config2", do_config2), ("sort", do_sort), ("join", do_join), ("config1", do_config1)):
        if name in args.only.split(","):
            t = time.time()
            doc[name] = fn()
            print(f"{name}: {time.time() - t:.1f} s", flush=True)
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=1)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
