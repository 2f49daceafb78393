"""Direct differential checks of the oracle against the reference's strict
build on inputs beyond the golden set (skipped when that build is absent)."""
import numpy as np

import shapes


def test_random_blocks(oracle, ref):
    rng = np.random.Generator(np.random.PCG64(7))
    for t in range(120):
        kind = t % 4
        if kind == 0:
            vox = rng.integers(0, 256, 4096)
        elif kind == 1:
            vox = np.where(rng.random(4096) < 0.4, 0, rng.integers(40, 220, 4096))
        elif kind == 2:
            z, y, x = np.meshgrid(np.arange(16), np.arange(16), np.arange(16), indexing="ij")
            vox = (128 + 60 * np.sin(x * 0.3 + t) * np.cos(y * 0.2) + rng.normal(0, 6, (16, 16, 16))).ravel()
        else:
            vox = shapes.block_patterns()[t % 10].astype(int) + rng.integers(-3, 4, 4096)
        vox = np.clip(vox, 0, 255).astype(np.uint8)
        q = float([0.5, 1, 2, 3, 6, 9, 12, 24][t % 8])
        tau = [0, 0, 2, 5][t % 4]
        a = ref.enc_block(vox, q, tau)
        assert oracle.enc_block(vox, q, tau) == a, t
        if a:
            assert np.array_equal(oracle.dec_block(a, q), ref.dec_block(a, q)), t


def test_garbage_streams(oracle, ref):
    rng = np.random.Generator(np.random.PCG64(11))
    for t in range(200):
        p = rng.integers(0, 256, int(rng.integers(1, 400)), dtype=np.uint8).tobytes()
        q = float([1, 3, 6, 12][t % 4])
        assert np.array_equal(oracle.dec_block(p, q), ref.dec_block(p, q)), t
