"""The multi-GPU bench path is replicas: each rank scans its own partition and
the job time is the maximum over ranks.  Checked here with two gloo ranks on
the CPU: the reduction the bench uses, the per-rank inputs (distinct seeds,
same shape), and that the reference arm does its work on rank 0 only."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        dev = torch.device("cpu")
        got = bench._max_over_ranks(dist, dev, 10.0 + rank)
        d = bench.make_data(rank, 4096)
        cfg = bench.workload_config(d, world)
        q.put((rank, got, int(d["price"][0] * 1e6), d["n"], cfg["parallelism"]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_time_is_the_max_and_inputs_are_replicas():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert all(r[1] == 11.0 for r in res)                 # max over ranks
    assert res[0][2] != res[1][2] and res[0][3] == res[1][3]  # different seeds, same shape
    assert all(r[4] == "replicas x2" for r in res)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import argparse

    import bench

    called = []
    monkeypatch.setattr(bench, "cpu_reference", lambda *a, **k: called.append(1) or (1.0, 1, "port", "x"))
    args = argparse.Namespace(rows=4096, warmup=1, steps=1)
    bench.run_reference_arm(args, rank=1, world=2)
    assert not called and capsys.readouterr().out == ""
    bench.run_reference_arm(args, rank=0, world=2)
    assert called and '"impl": "reference"' in capsys.readouterr().out
