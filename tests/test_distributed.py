"""Multi-rank host logic on CPU (gloo, world size 2): the batch sharding and the
max/sum-over-ranks timing the bench reports."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

from mcpdlp.parallel import imbalance, shard_by_nnz

ROOT = Path(__file__).resolve().parent.parent


def test_shard_partitions_every_lp_once():
    sizes = [5, 90, 12, 12, 400, 3, 77, 1000, 8, 250]
    for world in (1, 2, 3, 4):
        shards = shard_by_nnz(sizes, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(sizes)))
        assert len(shards) == world


def test_shard_balance_on_the_uneven_batch():
    import numpy as np
    rng = np.random.default_rng(0)
    m = rng.integers(100, 20001, 256)
    sizes = (m * rng.integers(2, 5, 256) * rng.integers(4, 13, 256)).tolist()
    for world in (2, 4, 8):
        assert imbalance(sizes, shard_by_nnz(sizes, world)) < 1.02


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank: int, world: int, port: int, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "markov-zip1_b200"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    sizes = [10, 20, 30, 40, 55, 60, 5]
    mine = shard_by_nnz(sizes, world)[rank]
    t = torch.tensor([len(mine)], dtype=torch.int64)
    dist.all_reduce(t)
    tmax = bench.max_over_ranks(dist, 1.5 + rank, "cpu")
    tsum = bench.sum_over_ranks(dist, float(sum(sizes[i] for i in mine)), "cpu")
    out.put((rank, int(t.item()), tmax, tsum))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, total, tmax, tsum in got:
        assert total == 7            # every LP solved by exactly one rank
        assert tmax == 2.5           # the slower rank's time
        assert tsum == 220.0         # all ranks' work
