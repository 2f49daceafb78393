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


def test_deblock_random_volumes(oracle, ref):
    """or_deblock == the reference's mc_deblock on seeded blocky volumes of
    random sizes and qualities (the reference's volume is followed by a zero
    plane: its read past the last z face then sees what the oracle assumes)."""
    import ctypes as C
    ref.L.mc_deblock.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float]
    rng = np.random.default_rng(11)
    for t in range(40):
        nz, ny, nx = (int(v) for v in rng.integers(1, 70, 3))
        lv = rng.integers(30, 200, ((nz + 15) // 16, (ny + 15) // 16, (nx + 15) // 16))
        vol = np.repeat(np.repeat(np.repeat(lv, 16, 0), 16, 1), 16, 2)[:nz, :ny, :nx]
        vol = vol + rng.integers(-6, 7, vol.shape)
        vol[rng.random(vol.shape) < 0.05] = 0
        vol = np.clip(vol, 0, 255).astype(np.uint8)
        q = float(rng.choice([0.5, 2.0, 6.0, 10.0, 30.0]))
        buf = np.zeros(vol.size + ny * nx, np.uint8)
        buf[:vol.size] = vol.ravel()
        ref.L.mc_deblock(buf.ctypes.data, nz, ny, nx, q)
        mine = oracle.deblock(vol.copy(), q)
        assert np.array_equal(mine.ravel(), buf[:vol.size]), (nz, ny, nx, q)
