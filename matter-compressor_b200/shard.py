"""Multi-GPU plumbing for the chunk-sharded decode: one process per GPU,
torch.distributed for barriers and the max-over-ranks timing reduction.

The decode path shards with no exchange step: rank r owns its own chunks
(independent archives / chunk ranges), so the only collectives are a barrier
around the timed region and one MAX all-reduce of the elapsed time.
"""
import datetime
import os

import torch


class Dist:
    def __init__(self, backend="nccl", timeout_s=120):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.pg = None
        if self.world > 1:
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.pg = dist

    def barrier(self):
        if self.pg:
            if self.backend == "nccl":
                self.pg.barrier(device_ids=[self.local])
            else:
                self.pg.barrier()

    def max(self, x):
        """Max of a float over ranks (the whole-job elapsed time)."""
        if not self.pg:
            return x
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()
            self.pg = None


def chunk_seeds(rank, nchunks):
    """Rank r decodes its own chunks: volume seeds r*n .. r*n+n-1."""
    return [rank * nchunks + c for c in range(nchunks)]


def air_fraction(c):
    """Air fraction of chunk c of a shard: 30 % .. 60 % in 8 steps."""
    return 0.3 + 0.3 * (c % 8) / 7.0
