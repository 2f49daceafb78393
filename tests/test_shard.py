"""Multi-rank plumbing of the sharded decode on CPU (gloo, world size 2):
disjoint chunk shards per rank, max-over-ranks timing reduction, barrier."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    from shard import Dist, chunk_seeds
    d = Dist("gloo", timeout_s=60)
    d.barrier()
    m = d.max(1.5 + rank)            # each rank's own elapsed time
    seeds = chunk_seeds(d.rank, 64)
    d.barrier()
    d.close()
    q.put((rank, m, seeds[0], seeds[-1]))


def test_two_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert all(m == 2.5 for _, m, _, _ in res)          # MAX over ranks
    assert res[0][2:] == (0, 63) and res[1][2:] == (64, 127)   # disjoint shards


def test_single_rank_is_local():
    from shard import Dist
    d = Dist("gloo")
    assert d.world == 1 and d.max(3.0) == 3.0
    d.close()
