"""Replicas across GPUs: request sharding and the rank bookkeeping, on CPU
with the gloo backend (world size 2) — the same calls bench.py makes under
torchrun with NCCL."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from bh_ringdown_b200 import replicas


def test_shard_is_a_balanced_partition():
    rng = np.random.default_rng(3)
    work = rng.integers(1, 1000, size=57).astype(float)
    for world in (1, 2, 3, 8):
        shards = replicas.shard_requests(work, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(work)))
        loads = [work[s].sum() for s in shards]
        # longest-first greedy: within the largest single item of the mean
        assert max(loads) - min(loads) <= work.max()
        for s in shards:
            assert s == sorted(s)
    assert replicas.shard_requests(work, 4) == replicas.shard_requests(list(work), 4)  # deterministic


def test_request_work_uses_the_solvers_step_count():
    import bh_ringdown_b200 as bhr
    prm = bhr.Params(N=256, M=32, Xmin=-50.0, Xmax=50.0, a=0.5, m=2.0, dt=0.1, T=10.0)
    assert replicas.request_work(prm) == 256 * 32 * 100


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        work = [5.0, 1.0, 4.0, 2.0, 3.0, 9.0]
        mine = replicas.shard_requests(work, world)[rank]
        t = replicas.max_over_ranks(10.0 + rank, dist)
        got = replicas.gather_objects({"rank": rank, "ids": mine}, dist)
        out.put((rank, mine, t, got))
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    ids = sorted(i for _, mine, _, _ in res for i in mine)
    assert ids == list(range(6))                    # the shards partition the requests
    assert all(t == 11.0 for _, _, t, _ in res)     # max over ranks
    for rank, mine, _, got in res:                  # every rank sees every rank's ids
        assert [g["rank"] for g in got] == [0, 1]
        assert got[rank]["ids"] == mine
