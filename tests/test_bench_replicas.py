"""Multi-rank logic of bench.py on CPU: world_size-2 gloo process groups.

The solve does not shard (each GPU runs an independent replica), so the only exchange is
the timing reduction: every rank reports the slowest rank's time. The reference arm runs
on rank 0 alone; other ranks return without output."""
from __future__ import annotations

import io
import os
import sys
from contextlib import redirect_stdout
from pathlib import Path

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _worker(rank: int, world: int, port: int, out: dict) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        got = bench.max_over_ranks(1.5 + rank)  # rank 1 is the slow one
        buf = io.StringIO()
        if rank != 0:
            class Args:
                ref_n, nrhs, steps, warmup, gpus = 64, 4, 1, 0, world
            with redirect_stdout(buf):
                bench.run_reference_arm(Args())
        out[rank] = (got, buf.getvalue())
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_reference_arm_rank_gating():
    port = 29500 + os.getpid() % 2000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0][0] == pytest.approx(2.5) and res[1][0] == pytest.approx(2.5)
    assert res[1][1] == ""  # non-zero ranks print nothing in the reference arm


def test_max_over_ranks_without_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.25) == 3.25
