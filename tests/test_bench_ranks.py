"""The multi-process path of bench.py on the CPU: two ``gloo`` ranks (spawned
processes, rendezvous on 127.0.0.1) reduce their timed regions and success
counts the way the GPU ranks do over NCCL: the whole job's time is the
slowest rank's, its successes the sum over ranks, and every rank gets both."""

from __future__ import annotations

import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime
    import os

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))  # fmt: skip
    try:
        # rank r: timed region 10 (r + 1) ms, 3 + r successes; then the e2e pair
        t, s = bench.rank_totals(dist, 10.0 * (rank + 1), 3 + rank, "cpu")
        t2, s2 = bench.rank_totals(dist, 5.0 - rank, 100 * rank, "cpu")
        Path(out_dir, f"rank{rank}.txt").write_text(f"{t} {s} {t2} {s2}")
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_like_the_gpu_ranks(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        t, s, t2, s2 = Path(tmp_path, f"rank{r}.txt").read_text().split()
        assert float(t) == 20.0 and int(s) == 7          # max time, summed successes
        assert float(t2) == 5.0 and int(s2) == 100


def test_single_process_is_unchanged():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.rank_totals(None, 12.5, 9, "cpu") == (12.5, 9)
