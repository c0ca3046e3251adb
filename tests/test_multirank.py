"""The replica path of bench.py across ranks, on CPU with two gloo ranks: every rank reports the
slowest rank's time and the same whole-job throughput (weak scaling, no data-path collective)."""

from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench

    local_ms = 100.0 + 50.0 * rank  # rank 1 is the slower replica
    dist.barrier()
    total_ms, value = bench.job_throughput(local_ms, steps=4, world=world, dist=dist)
    Path(out_dir, f"rank{rank}.txt").write_text(f"{total_ms} {value}")
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_agree_on_the_slowest_rank(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    results = [tuple(map(float, (tmp_path / f"rank{r}.txt").read_text().split())) for r in range(world)]
    assert results[0] == results[1]
    total_ms, value = results[0]
    assert total_ms == 150.0
    # 2 replicas x 4 blocks x 8 placements in the slowest rank's 150 ms.
    assert value == pytest.approx(2 * 4 * 8 / 0.150)
