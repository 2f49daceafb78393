"""Archive verification with the hashing on the device
(mc_b200_verify_archive_dev) against the reference's mc_verify_archive: a
clean archive, tampered blobs and node tables, a device copy at an odd
address, and the HBM mirror of an open archive."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _archive(gpu, path):
    import torch
    import volumes
    with gpu.open(path, 768, 512, 256, 6.0) as a:
        coords = [(0, 0, 0), (0, 0, 1), (0, 1, 2), (0, 1, 0)]
        vox = [volumes.region(40 + i, (0, 256 * c[1], 256 * c[2]), (256, 256, 256), 0.4, device="cuda").contiguous()
               for i, c in enumerate(coords)]
        assert a.append_chunks(0, coords, [v.data_ptr() for v in vox], 6.0, on_device=True) == 0
        small = volumes.region(50, (0, 0, 0), (256, 256, 256), 0.3, device="cuda").contiguous()
        assert a.append_chunks(1, [(0, 0, 0)], [small.data_ptr()], 3.0, ctx_q=3.0, on_device=True) == 0
        torch.cuda.synchronize()
    return np.fromfile(path, np.uint8)


def _dev_verify(gpu, data, shift=0):
    import torch
    d = torch.zeros(data.size + 16, dtype=torch.uint8, device="cuda")
    d[shift:shift + data.size] = torch.from_numpy(data).cuda()
    h = np.ascontiguousarray(data)
    return gpu.L.mc_b200_verify_archive_dev(h.ctypes.data, d.data_ptr() + shift, data.size, 0)


def test_clean_and_tampered(gpu, ref, tmp_path):
    data = _archive(gpu, str(tmp_path / "v.mca"))
    assert ref.L.mc_verify_archive(data.ctypes.data, data.size, 0) == 0
    for shift in (0, 3, 8):
        assert _dev_verify(gpu, data, shift) == 0
    rng = np.random.default_rng(2)
    # tamper bytes anywhere past the header: blob payloads, length tables,
    # fraction maps, stored hashes, node tables
    for t in range(24):
        bad = data.copy()
        for pos in rng.integers(131072, data.size, int(rng.integers(1, 4))):
            bad[pos] ^= int(rng.integers(1, 256))
        want = ref.L.mc_verify_archive(bad.ctypes.data, bad.size, 0)
        assert _dev_verify(gpu, bad, int(t % 8)) == want == gpu.L.mc_verify_archive(bad.ctypes.data, bad.size, 0), t


def test_mirror_of_open_archive(gpu, tmp_path):
    path = str(tmp_path / "m.mca")
    data = _archive(gpu, path)
    with gpu.open(path, 768, 512, 256, 6.0) as a:
        rc, base, n = a.sync_device()
        assert rc == 0 and n == data.size
        assert gpu.L.mc_b200_verify_archive_dev(data.ctypes.data, base, n, 0) == 0
