"""Workload builders for the benchmark configurations beyond batched chunk
decode: the multi-LOD synthetic volume archive (dataloader region reads and
serving) and the serving request trace.

Volume: LOD l of a (nz, ny, nx) volume has extent ceil(dim / 2^l) voxels per
axis (at least one chunk). Every LOD is generated on its own from the seeded
field (volumes.region with one air threshold per LOD), since the content of a
synthetic pyramid does not matter for timing; LOD decimation of real data
is not part of the hot path measured here.

Trace: Poisson arrivals at a given rate; 70 % single 16^3 blocks, 20 % 128^3
regions, 10 % 256^3 chunks; LOD uniform over the pyramid's first levels;
spatial locality Zipf(1.1) over the 128^3 cells of the chosen LOD, ranked by
a fixed seeded permutation.
"""
import math

import numpy as np
import torch

import volumes
from mcb200 import REQ_BLOCK, REQ_CHUNK, REQ_REGION


def lod_chunks(dims, lod):
    """Chunks per axis (z, y, x) of LOD `lod` for a (nz, ny, nx) volume."""
    return tuple(max(1, math.ceil(math.ceil(d / (1 << lod)) / 256)) for d in dims)


def build_volume_archive(lib, path, dims=(1024, 2048, 2048), lods=4, q=6.0, seed=0, air=0.4, group=8,
                         device="cuda"):
    """Archive of a synthetic multi-LOD volume, chunks encoded on the GPU in
    batches of `group`. Returns the open archive and the number of chunks."""
    nz, ny, nx = dims
    a = lib.open(path, nx, ny, nz, q)
    total = 0
    for lod in range(lods):
        cz, cy, cx = lod_chunks(dims, lod)
        ext = (cz * 256, cy * 256, cx * 256)
        cut = volumes.air_threshold(seed + 1000 * lod, air, ext, device)
        coords = [(z, y, x) for z in range(cz) for y in range(cy) for x in range(cx)]
        for g0 in range(0, len(coords), group):
            part = coords[g0:g0 + group]
            vox = [volumes.region(seed + 1000 * lod, (z * 256, y * 256, x * 256), (256, 256, 256), air, air_cut=cut,
                                  device=device).contiguous() for z, y, x in part]
            rc = a.append_chunks(lod, part, [v.data_ptr() for v in vox], q, on_device=True)
            if rc != 0:
                raise RuntimeError(f"append_chunks failed at LOD {lod}")
            del vox
        total += len(coords)
    torch.cuda.synchronize()
    return a, total


class Trace:
    """A seeded serving trace: arrival times and request parameters."""

    KINDS = (REQ_BLOCK, REQ_REGION, REQ_CHUNK)
    NAMES = ("block", "region", "chunk")

    def __init__(self, seed, n, rate, dims, lods=4, mix=(0.7, 0.2, 0.1), zipf=1.1, region=128):
        rng = np.random.default_rng(seed)
        self.arrival_ns = np.cumsum(rng.exponential(1e9 / rate, n)).astype(np.uint64)
        self.kind = rng.choice(3, n, p=list(mix))
        self.lod = rng.integers(0, lods, n)
        self.region = region
        self.req = np.zeros((n, 7), np.int64)   # z, y, x, dz, dy, dx (voxel or block/chunk coordinates)
        perms = []
        for lod in range(lods):
            cz, cy, cx = lod_chunks(dims, lod)
            cells = (cz * 2, cy * 2, cx * 2)   # 128^3 cells
            perms.append((cells, np.random.default_rng(seed * 31 + lod).permutation(cells[0] * cells[1] * cells[2])))
        for i in range(n):
            cells, perm = perms[self.lod[i]]
            ncell = len(perm)
            r = int(rng.zipf(zipf))
            while r > ncell:
                r = int(rng.zipf(zipf))
            c = int(perm[r - 1])
            z0 = (c // (cells[1] * cells[2])) * 128
            y0 = ((c // cells[2]) % cells[1]) * 128
            x0 = (c % cells[2]) * 128
            k = self.kind[i]
            if k == 0:    # a block inside the cell
                b = rng.integers(0, 8, 3)
                self.req[i, :3] = ((z0 >> 4) + b[0], (y0 >> 4) + b[1], (x0 >> 4) + b[2])
            elif k == 1:  # a region at an unaligned offset inside the cell
                o = rng.integers(0, 128, 3)
                self.req[i, :6] = (z0 + o[0], y0 + o[1], x0 + o[2], region, region, region)
            else:         # the chunk holding the cell
                self.req[i, :3] = (z0 >> 8, y0 >> 8, x0 >> 8)

    def __len__(self):
        return len(self.kind)

    def out_bytes(self, i):
        k = self.kind[i]
        return 4096 if k == 0 else (self.region ** 3 if k == 1 else 256 ** 3)
