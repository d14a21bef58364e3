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


def test_reference_arm_line_on_rank_0():
    """The reference arm's JSON line on rank 0 carries the keys the bench contract names, with
    the sample it timed in its config and no host-device bytes."""
    import json
    sys.path.insert(0, str(ROOT))
    import bench
    import oracle
    try:
        oracle.Reference()
    except FileNotFoundError:
        pytest.skip("reference CPU path not built on this machine")

    class Args:
        ref_n, n, nrhs, steps, warmup, gpus = 96, 32768, 4, 2, 1, 1

    buf = io.StringIO()
    os.environ.pop("RANK", None)
    with redirect_stdout(buf):
        bench.run_reference_arm(Args())
    lines = buf.getvalue().strip().splitlines()
    assert len(lines) == 1
    line = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["config"]["n"] == 96 and line["config"]["headline_n"] == 32768
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] == 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
