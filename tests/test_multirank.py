"""The multi-GPU form of the benchmark is one independent replica per rank; its only collective
steps are barriers and the max over ranks of the measured times. Both run here as two gloo ranks
on the CPU."""
from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _rank(rank: int, world: int, port: int, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        times = [3.0, 5.0]  # the slower rank sets the step time
        got = bench.max_over_ranks(times[rank], world, "cpu")
        dist.barrier()
        one = bench.max_over_ranks(7.0, 1, "cpu")  # a single rank reduces nothing
        out.put((rank, got, one))
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 5.0, 7.0), (1, 5.0, 7.0)]


def test_reference_arm_runs_on_rank_zero_only(capsys, monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("RANK", "1")
    args = type("A", (), {"config": "cfg1", "steps": 1, "warmup": 1, "gpus": 2})()
    bench.run_reference(args)
    assert capsys.readouterr().out == ""
