"""The multi-rank path of bench.py on CPU: world size 2 over gloo. The
photon-mapping path runs as independent replicas (no data-path collective);
the only collectives are the barrier and the max-over-ranks of the step
times, which this checks."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    w, r, lr = bench.dist_env()
    dist = bench.dist_init(w, "gloo")
    dist.barrier()
    got = bench.max_over_ranks(dist, 1.5 + rank, "cpu")  # per-rank step time
    q.put((r, w, got))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 2, 2.5), (1, 2, 2.5)]


def test_single_rank_needs_no_group():
    import bench
    assert bench.max_over_ranks(None, 3.25, "cpu") == 3.25
