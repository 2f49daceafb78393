"""Decode-side deblocking on the device (mc_deblock / mc_b200_deblock_dev)
against the reference's digests and the oracle: golden volumes, random sizes
and qualities, batches, and decoded chunks deblocked where they were decoded."""
import os

import numpy as np
import pytest

import shapes
from conftest import GOLDEN, sha

pytestmark = pytest.mark.gpu
CHUNK = 256 ** 3


def test_golden_volumes_host_dropin(gpu):
    """mc_deblock on host volumes reproduces the reference's output digests."""
    g = np.load(os.path.join(GOLDEN, "deblock.npz"))
    vols = dict(shapes.deblock_volumes())
    for name, q, want in zip(g["names"], g["q"], g["out_sha"]):
        v = vols[str(name)].copy()
        gpu.deblock(v, float(q))
        assert sha(v) == want, (name, q)


def test_random_volumes_batched_on_device(gpu, oracle):
    """A batch of equal-shape device volumes, each == the oracle; air voxels
    stay 0 and the gaps between the volumes are not touched."""
    import torch
    rng = np.random.default_rng(3)
    for nz, ny, nx in [(33, 47, 70), (16, 64, 17), (64, 18, 40), (1, 40, 80), (50, 1, 33)]:
        count = 3
        lv = rng.integers(20, 230, (count, (nz + 15) // 16, (ny + 15) // 16, (nx + 15) // 16))
        vol = np.repeat(np.repeat(np.repeat(lv, 16, 1), 16, 2), 16, 3)[:, :nz, :ny, :nx]
        vol = vol + rng.integers(-5, 6, vol.shape)
        vol[rng.random(vol.shape) < 0.04] = 0
        vol = np.clip(vol, 0, 255).astype(np.uint8)
        stride = nz * ny * nx + 96
        buf = np.full(count * stride, 0xA7, np.uint8)
        for c in range(count):
            buf[c * stride:c * stride + vol[c].size] = vol[c].ravel()
        d = torch.from_numpy(buf).cuda()
        for q in (1.0, 6.0, 20.0):
            d.copy_(torch.from_numpy(buf))
            assert gpu.deblock_dev(d.data_ptr(), count, stride, nz, ny, nx, q) == 0
            got = d.cpu().numpy()
            for c in range(count):
                want = oracle.deblock(vol[c].copy(), q)
                out = got[c * stride:c * stride + vol[c].size].reshape(nz, ny, nx)
                assert np.array_equal(out, want), (nz, ny, nx, q, c)
                assert not out[vol[c] == 0].any()
                assert (got[c * stride + vol[c].size:(c + 1) * stride] == 0xA7).all()


def test_decoded_chunks_deblocked_in_place(gpu, oracle, tmp_path):
    """Chunks decoded into HBM by the batched decode, then deblocked there as
    two separate 256^3 volumes and, read side by side, as one 256 x 256 x 512
    volume, == the oracle's decode followed by the oracle's deblock."""
    import torch
    import volumes
    with gpu.open(str(tmp_path / "d.mca"), 512, 256, 256, 6.0) as a:
        for i in range(2):
            v = volumes.region(31 + i, (0, 0, 256 * i), (256, 256, 256), 0.4, device="cuda").cpu().numpy()
            assert a.append_par(0, 0, 0, i, v, 6.0) == 0
        offs = [a.chunk_offset(0, 0, 0, i) for i in range(2)]
        data = np.fromfile(str(tmp_path / "d.mca"), np.uint8).tobytes()
        dec = [oracle.decode_chunk(data[o:o + shapes.blob_len(data, o)]).reshape(256, 256, 256) for o in offs]
        d_out = torch.empty(2 * CHUNK, dtype=torch.uint8, device="cuda")
        assert a.decode_chunks_dev(offs, d_out.data_ptr()) == 0
        assert gpu.deblock_dev(d_out.data_ptr(), 2, CHUNK, 256, 256, 256, 6.0) == 0
        got = d_out.cpu().numpy()
        for i in range(2):
            assert np.array_equal(got[i * CHUNK:(i + 1) * CHUNK].reshape(256, 256, 256),
                                  oracle.deblock(dec[i].copy(), 6.0)), i
        d_reg = torch.empty(2 * CHUNK, dtype=torch.uint8, device="cuda")
        assert a.read_regions_dev(0, [(0, 0, 0)], 256, 256, 512, d_reg.data_ptr(), 2 * CHUNK) == 0
        assert gpu.deblock_dev(d_reg.data_ptr(), 1, 2 * CHUNK, 256, 256, 512, 6.0) == 0
        whole = np.concatenate(dec, axis=2)
        assert np.array_equal(d_reg.cpu().numpy().reshape(256, 256, 512), oracle.deblock(whole.copy(), 6.0))


def test_bad_arguments_refused(gpu):
    with pytest.raises(RuntimeError):
        gpu.deblock_dev(0, 1, 64, 4, 4, 4, 6.0)
