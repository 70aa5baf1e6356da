"""The bench's multi-rank plumbing on CPU: two gloo ranks (127.0.0.1) meet
at its barrier and agree on the maximum of their times, as the replicas of
`bench.py --gpus N` do over NCCL; and under torchrun the reference arm runs
on rank 0 only (other ranks return without work)."""

import os
import socket
import sys
from datetime import timedelta
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, results) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        bench.barrier(world)
        results[rank] = bench.max_over_ranks(1.5 * (rank + 1), world)
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_maximum():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        results = manager.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, results)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        assert dict(results) == {0: 3.0, 1: 3.0}


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("RANK", "1")
    assert bench.run_reference(None) == {}
