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


def _gpu_worker(rank, world, port, q, tmp):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "matter-compressor_b200"), os.path.join(root, "oracle"),
                    os.path.join(root, "tests", "golden")]
    import numpy as np
    import shapes
    import volumes
    from mcb200 import McLib
    from oracle import Oracle
    from shard import Dist, air_fraction, chunk_seeds
    d = Dist("gloo", timeout_s=120)
    try:
        lib = McLib.product()
        seeds = chunk_seeds(d.rank, 2)
        path = os.path.join(tmp, f"rank{rank}.mca")
        with lib.open(path, 512, 256, 256, 6.0) as a:
            for c, s in enumerate(seeds):
                v = volumes.region(s, (0, 0, 256 * c), (256, 256, 256), air_fraction(c), device="cuda").cpu().numpy()
                assert a.append_par(0, 0, 0, c, v, 6.0) == 0
            offs = [a.chunk_offset(0, 0, 0, c) for c in range(2)]
            d_out = torch.empty(2 * 256 ** 3, dtype=torch.uint8, device="cuda")
            plan = a.plan_chunks(offs, d_out.data_ptr())
            d.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            plan.launch(torch.cuda.current_stream().cuda_stream)
            e1.record()
            torch.cuda.synchronize()
            ms = d.max(e0.elapsed_time(e1))
            d.barrier()
            plan.free()
            got = d_out.cpu().numpy()
        data = open(path, "rb").read()
        orc = Oracle()
        ok = all(np.array_equal(got[c * 256 ** 3:(c + 1) * 256 ** 3],
                                orc.decode_chunk(data[o:o + shapes.blob_len(data, o)])) for c, o in enumerate(offs))
        q.put((rank, ok, ms > 0, seeds))
    finally:
        d.close()


@pytest.mark.gpu
def test_two_ranks_drive_the_library(tmp_path):
    """Two ranks (one process each, gloo for the barrier and the MAX timing
    reduction) decode their own chunk shards through the library on the same
    GPU -- no kernel of one waits on the other -- and each gets the oracle's
    voxels; the reduced time is the same on both ranks."""
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gpu_worker, args=(r, world, port, q, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert all(ok and timed for _, ok, timed, _ in res)
    assert res[0][3] == [0, 1] and res[1][3] == [2, 3]
