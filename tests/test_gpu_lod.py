"""LOD pyramid on the device: mc_b200_decimate_dev against the oracle's
decimation, and mc_b200_append_pyramid against the chunk blobs of the
reference's one-shot builder (mc_build) on the same volume."""
import hashlib
import os

import numpy as np
import pytest

import shapes
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_decimate_matches_oracle(gpu, oracle):
    """Odd and even extents, air-heavy and saturated content, two launches in
    a row into the same output buffer."""
    import torch
    rng = np.random.default_rng(4)
    for shape in [(33, 47, 70), (1, 1, 1), (2, 3, 5), (64, 18, 255), (17, 1, 300)]:
        vol = rng.integers(0, 256, shape).astype(np.uint8)
        vol[rng.random(shape) < 0.5] = 0
        vol[rng.random(shape) < 0.05] = 255
        want = oracle.decimate(vol)
        d_src = torch.from_numpy(vol).cuda()
        d_dst = torch.full(want.shape, 0xEE, dtype=torch.uint8, device="cuda")
        for _ in range(2):
            assert gpu.decimate_dev(d_src.data_ptr(), *shape, d_dst.data_ptr()) == 0
            assert np.array_equal(d_dst.cpu().numpy(), want), shape


def test_pyramid_matches_builder(gpu, tmp_path):
    """Every LOD's chunk blobs of the device pyramid == mc_build's digests
    (two qualities); the all-air chunk stays absent."""
    import torch
    g = np.load(os.path.join(GOLDEN, "pyramid.npz"))
    vol = shapes.pyramid_volume()
    nz, ny, nx = vol.shape
    d_vol = torch.from_numpy(vol).cuda()
    levels = shapes.pyramid_levels(nz, ny, nx)
    for q in sorted(set(float(k[0]) for k in g["keys"])):
        want = {tuple(int(v) for v in k[1:]): d for k, d in zip(g["keys"], g["blob_sha"]) if float(k[0]) == q}
        path = str(tmp_path / f"p{q}.mca")
        with gpu.open(path, nx, ny, nz, q) as a:
            rc, nl = a.append_pyramid(d_vol.data_ptr(), nz, ny, nx, q)
            assert rc == 0 and nl == len(levels) == len(g["levels"])
            data = open(path, "rb").read()
            for lod, (dz, dy, dx) in levels:
                for cz in range((dz + 255) // 256):
                    for cy in range((dy + 255) // 256):
                        for cx in range((dx + 255) // 256):
                            co = a.chunk_offset(lod, cz, cy, cx)
                            key = (lod, cz, cy, cx)
                            if key not in want:
                                assert co <= 1, (q, key)
                                continue
                            blob = data[co:co + shapes.blob_len(data, co)]
                            assert hashlib.sha256(blob).hexdigest() == want[key], (q, key)
