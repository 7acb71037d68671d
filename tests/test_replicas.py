"""The multi-GPU path is replicas only (independent rays, images and jobs; no
data-path collective).  bench.py times each replica and reports the slowest
rank: max_over_ranks, run here as two gloo ranks on the CPU."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, values, results):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        assert bench.dist_env() == (rank, world, rank)
        results[rank] = bench.max_over_ranks(values[rank], dist, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        results = m.dict()
        values = [3.25, 7.5]
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, values, results)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert dict(results) == {0: 7.5, 1: 7.5}


def test_single_process_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(2.5) == 2.5
    assert bench.config_dict(256, "mixed", 4, 2, 8)["parallelism"] == "replicas2"
