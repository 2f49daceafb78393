"""Deterministic integer-formula inputs for the golden vectors and tests.

Every pattern is computed from index arithmetic only (no RNG streams), so the
same bytes come out on every machine and numpy version.
"""
import numpy as np

_Z, _Y, _X = np.meshgrid(np.arange(16), np.arange(16), np.arange(16), indexing="ij")


def _hash_u8(i, salt):
    h = (i.astype(np.uint64) * np.uint64(2654435761) + np.uint64(salt) * np.uint64(40503)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(15)
    h = (h * np.uint64(2246822519)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(13)
    return (h & np.uint64(0xFF)).astype(np.int64)


def block_patterns():
    """16^3 blocks covering the codec's paths: smooth, textured, noisy, mixed
    air/material, sparse, constant, saturated, single voxel."""
    i = np.arange(4096)
    z, y, x = _Z.ravel(), _Y.ravel(), _X.ravel()
    pats = []
    pats.append(40 + ((x * 7 + y * 3 + z * 5) % 160))                        # sawtooth texture
    pats.append(128 + 60 * np.sin(x * 0.3) * np.cos(y * 0.2) + 20 * np.cos(z * 0.45))   # smooth
    pats.append(_hash_u8(i, 1))                                            # white noise
    r = np.sqrt((x - 8.0) ** 2 + (y - 8.0) ** 2 + (z - 8.0) ** 2)
    pats.append(np.where(r < 6, 120 + (i % 80), 0))                       # ball in air
    pats.append(np.where(_hash_u8(i, 2) < 100, 0, 40 + _hash_u8(i, 3) % 180))   # 40% speckled air
    pats.append(np.full(4096, 77))                                         # constant
    pats.append(np.where((x + y + z) % 2 == 0, 255, 0))                  # checkerboard extremes
    pats.append(np.where(i == 1234, 200, 0))                               # single voxel
    pats.append(100 + 2 * x + 3 * y + 4 * z + (_hash_u8(i, 4) % 13))    # ramp + noise
    pats.append(np.where(z < 8, 30 + (i % 170), 0))                       # half air
    return [np.clip(p, 0, 255).astype(np.uint8) for p in pats]


def frac_pattern(t):
    i = np.arange(4096)
    if t == 0:
        return np.zeros(4096, np.uint8)
    if t == 1:
        return np.full(4096, 15, np.uint8)
    if t == 2:
        return (i % 16).astype(np.uint8)
    if t == 3:
        return (_hash_u8(i, 9) % 16).astype(np.uint8)
    if t == 4:
        return np.where(i < 2048, 15, np.where(i % 7 == 0, 3, 0)).astype(np.uint8)
    return ((i // 64) % 16).astype(np.uint8)


def chunk_source(name):
    """256^3 chunk from a reference-test style formula (z,y,x raster)."""
    z, y, x = np.meshgrid(np.arange(256), np.arange(256), np.arange(256), indexing="ij", sparse=True)
    if name == "ball":        # the reference roundtrip test's ball, q=8 style
        r = np.sqrt((x - 128.0) ** 2 + (y - 128.0) ** 2 + (z - 128.0) ** 2)
        v = 128.0 + 100.0 * np.cos(r * 0.15)
        v = np.clip(v, 1, 255)
        out = np.where(r > 256 * 0.4, 0, np.floor(v))
    elif name == "sphere_tex":  # textured sphere, coarse texture
        d2 = (x - 128) ** 2 + (y - 128) ** 2 + (z - 128) ** 2
        out = np.where(d2 > 120 * 120, 0, 60 + ((x // 4 * 7 + y // 4 * 3 + z // 4 * 5) % 120))
    elif name == "half_air":
        out = np.where(z < 128, 40 + ((x + y + z) % 150), 0) + 0 * (x + y)
    elif name == "air":
        out = np.zeros((256, 256, 256))
    elif name == "waves":
        out = 120 + 50 * np.sin(x * 0.05 + y * 0.03) * np.cos(z * 0.04) + 20 * np.sin(x * 0.2)
        out = out + 0 * (x + y + z)
    else:
        raise KeyError(name)
    return np.ascontiguousarray(np.broadcast_to(np.clip(out, 0, 255), (256, 256, 256)).astype(np.uint8))


def archive_sequence():
    """A fixed append sequence into a 512x256x256 archive (two LOD0 chunks,
    then preset-ladder chunks at reused coordinates, an air chunk)."""
    return [
        {"name": "ball_par_q8", "op": "par", "at": (0, 0, 0), "q": 8.0, "src": "ball"},
        {"name": "waves_par_q3", "op": "par", "at": (0, 0, 1), "q": 3.0, "src": "waves"},
        {"name": "tex_preset4", "op": "ctx", "at": (1, 0, 0), "preset": 4, "src": "sphere_tex"},
        {"name": "half_preset2", "op": "ctx", "at": (1, 1, 1), "preset": 2, "src": "half_air"},
        {"name": "air_ctx", "op": "ctx", "at": (2, 0, 0), "preset": 4, "src": "air"},
        {"name": "air_par", "op": "par", "at": (2, 0, 1), "q": 6.0, "src": "air"},
        {"name": "waves_preset7", "op": "ctx", "at": (3, 3, 3), "preset": 7, "src": "waves"},
    ]


def deblock_volumes():
    """(name, volume) pairs for the deblocking filter: blocky volumes whose
    16-aligned blocks sit at different levels (flat seams that the filter
    smooths, steep ones it keeps), with air holes and air neighbours, at
    sizes that are and are not multiples of 16."""
    out = []
    for k, (nz, ny, nx) in enumerate([(32, 32, 32), (48, 40, 33), (17, 33, 65), (20, 16, 49), (64, 48, 80)]):
        z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        blk = (z // 16) * 7 + (y // 16) * 3 + (x // 16) * 5
        level = 60 + (_hash_u8(blk.ravel(), 10 + k).reshape(blk.shape) % (24 if k % 2 else 120))
        tex = (x * 3 + y * 5 + z * 7 + k) % 9 - 4
        vol = level + tex
        idx = np.arange(vol.size).reshape(vol.shape)
        vol = np.where(_hash_u8(idx, 20 + k) < 12, 0, vol)                   # speckled air
        vol = np.where((x + 2 * y + 3 * z + 5 * k) % 97 < 6, 0, vol)         # air sheets
        vol = np.where(_hash_u8(idx, 30 + k) > 250, 255, vol)                # saturated voxels
        out.append((f"v{k}_{nz}x{ny}x{nx}", np.clip(vol, 0, 255).astype(np.uint8)))
    return out


def pyramid_volume():
    """A 150 x 200 x 1100 (z, y, x) volume for the LOD pyramid: padded to
    256 x 256 x 1280 it has 5 LOD-0 chunks (one all air), 3 at LOD 1 and 2 at
    LOD 2; material with air holes, odd extents on every axis."""
    nz, ny, nx = 150, 200, 1100
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    idx = (z * ny + y) * nx + x
    vol = 40 + ((x * x // 97 + y * 3 + z * 5) % 150) + _hash_u8(idx.ravel(), 7).reshape(idx.shape) % 9
    vol = np.where(((x // 96) + (y // 64) + (z // 48)) % 5 == 0, 0, vol)      # air pockets
    vol = np.where((x >= 768) & (x < 1024), 0, vol)                           # one all-air LOD-0 chunk
    vol = np.where(_hash_u8(idx.ravel(), 8).reshape(idx.shape) < 20, 0, vol)  # speckled air
    return vol.astype(np.uint8)


def pyramid_levels(nz, ny, nx):
    """The reference one-shot builder's LOD loop (src/mc_archive.c:205-220):
    [(lod, (dz, dy, dx))] with the padded extent of each level. LOD 0 is the
    volume padded to multiples of 256; each next level halves (rounding up)
    while any axis of the current level is at least 256 (LOD 1 always
    follows LOD 0), at most 8 levels."""
    pad = lambda n: (n + 255) // 256 * 256
    d = (pad(nz), pad(ny), pad(nx))
    out = []
    for lod in range(8):
        if min(d) < 1 or not (max(d) >= 256 or lod == 0):
            break
        out.append((lod, d))
        if min(v // 2 for v in d) < 1:
            break
        if max(v // 2 for v in d) < 256 and lod >= 1:
            break
        d = tuple((v + 1) // 2 for v in d)
    return out


def pyramid_chunks(vol, decimate):
    """{(lod, cz, cy, cx): 256^3 chunk} of every LOD of the builder's pyramid
    over `vol`, using `decimate` for the 2x steps; all-air chunks left out."""
    levels = pyramid_levels(*vol.shape)
    cur = np.zeros(levels[0][1], np.uint8)
    cur[:vol.shape[0], :vol.shape[1], :vol.shape[2]] = vol
    out = {}
    for i, (lod, (dz, dy, dx)) in enumerate(levels):
        assert cur.shape == (dz, dy, dx)
        for cz in range((dz + 255) // 256):
            for cy in range((dy + 255) // 256):
                for cx in range((dx + 255) // 256):
                    c = np.zeros((256, 256, 256), np.uint8)
                    part = cur[cz * 256:cz * 256 + 256, cy * 256:cy * 256 + 256, cx * 256:cx * 256 + 256]
                    c[:part.shape[0], :part.shape[1], :part.shape[2]] = part
                    if c.any():
                        out[(lod, cz, cy, cx)] = c
        if i + 1 < len(levels):
            cur = decimate(cur)
    return out


def blob_len(data, co):
    """Total length of the chunk blob at file offset co: header, fmap,
    bitmap, one u16 length per present block, payloads."""
    fml = int.from_bytes(data[co + 12:co + 14], "little")
    bm = np.frombuffer(data, np.uint8, 512, co + 14 + fml)
    npres = int(np.unpackbits(bm).sum())
    lens = np.frombuffer(data, np.uint16, npres, co + 14 + fml + 512)
    return 14 + fml + 512 + 2 * npres + int(lens.astype(np.int64).sum())


def priors_tables():
    """A per-volume prior pair (q=1 and q=12 endpoint tables, u16[8][32]) that
    differs from the baked corpus tables in every trained slot, as a volume's
    own training would: probabilities stay inside the coder's usable range
    [48, 4048]. Deterministic integer formula."""
    c, s = np.meshgrid(np.arange(8), np.arange(32), indexing="ij")
    plo = 48 + (c * 613 + s * 389 + 97) % 4001
    phi = 48 + (c * 271 + s * 757 + 1301) % 4001
    return plo.astype(np.uint16), phi.astype(np.uint16)


def priors_sequence():
    """Appends into a 512x256x256 archive that carries the priors_tables()
    blob: a parallel append at q=6, a preset-ladder append (max error) and a
    parallel append at q=1."""
    return [
        {"name": "waves_par_q6", "op": "par", "at": (0, 0, 0), "q": 6.0, "src": "waves"},
        {"name": "tex_preset3", "op": "ctx", "at": (0, 0, 1), "preset": 3, "src": "sphere_tex"},
        {"name": "half_par_q1", "op": "par", "at": (1, 0, 0), "q": 1.0, "src": "half_air"},
    ]
