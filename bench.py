#!/usr/bin/env python
"""Benchmark: fused scan + group-by (filter+agg GB/s against the HBM roofline).

Workload (per GPU): 2^25 rows
  key   i32 Zipf(s=1.1) over 1,000 values, dictionary-encoded + bit-packed (10 bits)
  price f64 LogNormal(mu=3, sigma=1)
  qty   i32 Uniform[1,100]
  WHERE price > 20.0 AND qty BETWEEN 10 AND 50
  GROUP BY key: SUM(price*qty) FP64, COUNT, MIN(price), MAX(price)
A step is one pass of the fused kernel over the columns (444.6 MB of encoded
input; inputs are larger than the 126 MB L2, so no flush is needed).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl voxel|reference]

Multi-GPU: one process per GPU (torchrun); each rank scans its own 2^25-row
partition (weak scaling, no data-path collective), time = max over ranks.
`--impl reference` times the reference VoxelVM's own CPU operators (compiled
from its sources into oracle/_ref) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

METRIC = "filter+agg GB/s vs HBM peak"
UNIT = "GB/s"
ROWS = 1 << 25
PTHR, QLO, QHI = 20.0, 10, 50


def algorithmic_bytes(d: dict) -> int:
    """Bytes the scan must read once: packed keys + dictionary + price + qty."""
    return d["packed"].nbytes + d["dict"].nbytes + d["price"].nbytes + d["qty"].nbytes


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """Per-launch DRAM bytes from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", f"{kernel}.md")
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9]+)", txt)
    return int(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload_config(d: dict, world: int) -> dict:
    """The `config` object both arms print."""
    return {"workload": "scan+groupby 2^25 rows/GPU: key i32 zipf(1.1) over 1000, dict+bitpack 10-bit; "
                        "price f64 lognormal(3,1); qty i32 U[1,100]; price>20 AND qty BETWEEN 10 AND 50; "
                        "GROUP BY key SUM(price*qty) COUNT MIN MAX",
            "rows_per_gpu": d["n"], "algorithmic_bytes_per_step": algorithmic_bytes(d),
            "l2": "inputs (444.6 MB) larger than L2 (126 MB); no flush", "parallelism": f"replicas x{world}"}


def make_data(rank: int, rows: int) -> dict:
    import inputs

    return inputs.config2(rows, 2001 + rank)


def cpu_reference(d: dict, threads: int, reps: int, budget_s: float):
    """The reference's operators (oracle/_ref) on the host; returns GB/s, cores, sample."""
    import oracle

    kind = "reference" if oracle.have_ref() else "port"
    nbytes = algorithmic_bytes(d)
    times = []
    t_start = time.perf_counter()
    for _ in range(reps):
        if kind == "reference":
            *_, secs = oracle.scan_groupby_ref(d["packed"], d["width"], d["dict"], d["price"], d["qty"], PTHR, QLO,
                                              QHI, threads=threads)
        else:
            t0 = time.perf_counter()
            oracle.scan_groupby_port(d["packed"], d["width"], d["dict"], d["price"], d["qty"], PTHR, QLO, QHI)
            secs = time.perf_counter() - t0
            threads = 1
        times.append(secs)
        if time.perf_counter() - t_start > budget_s:
            break
    med = statistics.median(times)
    return nbytes / med / 1e9, threads, kind, f"{d['n']} rows x {len(times)} runs (median), full workload"


def run_reference_arm(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    d = make_data(0, args.rows)
    threads = os.cpu_count() or 1
    steps = []
    for _ in range(args.warmup):
        cpu_reference(d, threads, 1, 1e9)
    for _ in range(args.steps):
        gbs, cores, kind, sample = cpu_reference(d, threads, 1, 1e9)
        steps.append(gbs)
    v = statistics.median(steps)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": algorithmic_bytes(d) / v / 1e6,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded numpy PCG64, configs' distributions)",
            "config": workload_config(d, world),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="voxel", choices=["voxel", "reference"])
    ap.add_argument("--rows", type=int, default=ROWS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from voxel_b200 import capi

    L = capi.lib()
    d = make_data(rank, args.rows)
    dev = torch.device("cuda", local)
    t = {k: torch.from_numpy(d[k]).to(dev) for k in ("packed", "dict", "price", "qty")}
    card = d["dict"].size
    out = {"keys": torch.zeros(card, dtype=torch.int32, device=dev),
           "sum": torch.zeros(card, dtype=torch.float64, device=dev),
           "min": torch.zeros(card, dtype=torch.float64, device=dev),
           "max": torch.zeros(card, dtype=torch.float64, device=dev),
           "cnt": torch.zeros(card, dtype=torch.int64, device=dev),
           "ng": torch.zeros(1, dtype=torch.int64, device=dev)}
    # a dedicated stream: kernels and the timing events both go on it
    stream = torch.cuda.Stream(dev)
    sh = stream.cuda_stream

    def step():
        st = L.voxel_scan_groupby_dev(t["packed"].data_ptr(), d["packed"].size, d["width"], t["dict"].data_ptr(),
                                      card, t["price"].data_ptr(), t["qty"].data_ptr(), d["n"], PTHR, QLO, QHI,
                                      out["keys"].data_ptr(), out["sum"].data_ptr(), out["min"].data_ptr(),
                                      out["max"].data_ptr(), out["cnt"].data_ptr(), out["ng"].data_ptr(), sh)
        if st:
            raise RuntimeError(capi.last_error())

    nbytes = algorithmic_bytes(d)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for i in range(args.steps):
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        t1.record(stream)
        torch.cuda.synchronize()
    total_ms = t0.elapsed_time(t1)
    launch_ms = [a.elapsed_time(b) for a, b in ev]
    if dist:
        tt = torch.tensor([total_ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
    ms_per_step = total_ms / args.steps
    value = world * nbytes * args.steps / (total_ms * 1e-3) / 1e9
    kernel_gbs = nbytes / (statistics.mean(launch_ms) * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    traffic = ncu_traffic("scan_groupby_kernel")

    # end to end through the public host entry point: pinned host buffers in,
    # H2D + kernel + D2H of the group rows per step
    host = {k: torch.from_numpy(d[k]).pin_memory() for k in ("packed", "dict", "price", "qty")}
    ho = {"keys": np.zeros(card, np.int32), "sum": np.zeros(card), "min": np.zeros(card), "max": np.zeros(card),
          "cnt": np.zeros(card, np.uint64)}

    def e2e_step():
        g = L.voxel_scan_groupby(host["packed"].data_ptr(), d["packed"].size, d["width"], host["dict"].data_ptr(), card,
                                 host["price"].data_ptr(), host["qty"].data_ptr(), d["n"], PTHR, QLO, QHI,
                                 ho["keys"].ctypes.data, ho["sum"].ctypes.data, ho["min"].ctypes.data,
                                 ho["max"].ctypes.data, ho["cnt"].ctypes.data)
        if g == (1 << 64) - 1:
            raise RuntimeError(capi.last_error())
        return g

    for _ in range(max(2, args.warmup // 2)):
        ng = e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e_steps = max(3, min(args.steps, 10))
    w0 = time.perf_counter()
    for _ in range(e_steps):
        ng = e2e_step()
    e_ms = (time.perf_counter() - w0) * 1e3 / e_steps
    if dist:
        tt = torch.tensor([e_ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e_ms = float(tt.item())
    e2e = {"value": world * nbytes / (e_ms * 1e-3) / 1e9, "unit": UNIT, "h2d_bytes_per_step": nbytes,
           "d2h_bytes_per_step": int(ng) * (4 + 8 * 4) + 8, "ms_per_step": e_ms}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, cores, kind, sample = cpu_reference(d, os.cpu_count() or 1, 3, 20.0)
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
        except Exception as exc:  # the reference library did not travel
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "unavailable", "sample": str(exc)[:120]}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded numpy PCG64, configs' distributions)",
        "config": workload_config(d, world),
        "roofline": {"bound": "hbm", "achieved": kernel_gbs, "peak": peak, "unit": "GB/s",
                     "frac": kernel_gbs / peak, "traffic": traffic, "peak_source": peak_kind,
                     "kernel": "scan_groupby_kernel", "launch_ms_mean": statistics.mean(launch_ms),
                     "frac_of_nominal_8000": kernel_gbs / 8000.0},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clk.summary(),
        "gpu_launches": args.steps,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
