"""Training-box sampling with the scoring on the device (mc_b200_sample_boxes)
returns the reference's boxes: the strict reference build's
mc_archive_sample_boxes on the same archive file, over box shapes, material
thresholds, seeds, a second LOD and runs that need several scoring batches."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sample_archive(gpu, tmp_path_factory):
    import torch
    import volumes
    path = str(tmp_path_factory.mktemp("smp") / "s.mca")
    with gpu.open(path, 512, 512, 300, 6.0) as a:
        coords = [(0, 0, 0), (0, 0, 1), (0, 1, 1), (1, 0, 0), (1, 1, 1)]
        vox = [volumes.region(70 + i, (256 * c[0], 256 * c[1], 256 * c[2]), (256, 256, 256), 0.4,
                              device="cuda").contiguous() for i, c in enumerate(coords)]
        assert a.append_chunks(0, coords, [v.data_ptr() for v in vox], 6.0, on_device=True) == 0
        l1 = volumes.region(80, (0, 0, 0), (256, 256, 256), 0.3, device="cuda").contiguous()
        assert a.append_chunks(1, [(0, 0, 0)], [l1.data_ptr()], 6.0, on_device=True) == 0
        torch.cuda.synchronize()
    return path


CASES = [(0, 5, 12, (32, 32, 32), 0.5), (0, 9, 8, (17, 40, 9), 0.3), (0, 0, 6, (64, 64, 64), 0.7),
         (0, 3, 4, (300, 20, 20), 0.2), (0, 11, 10, (16, 16, 16), 0.0), (0, 12, 3, (8, 8, 8), 1.5),
         (0, 13, 40, (1, 1, 1), 0.99), (1, 14, 10, (40, 30, 20), 0.4), (0, 15, 5, (600, 8, 8), 0.1)]


def test_boxes_match_reference(gpu, ref, sample_archive):
    with gpu.open(sample_archive, 512, 512, 300, 6.0) as a, ref.open(sample_archive, 512, 512, 300, 6.0) as ra:
        for lod, seed, count, d, mf in CASES:
            want = ra.sample_boxes(lod, seed, count, *d, mf)
            assert a.sample_boxes_dev(lod, seed, count, *d, mf) == want, (lod, seed, d, mf)
            assert a.sample_boxes(lod, seed, count, *d, mf) == want, (lod, seed, d, mf)
