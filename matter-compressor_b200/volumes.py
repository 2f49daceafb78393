"""Seeded synthetic volumes for the benchmark configurations.

The reference's published numbers come from real scroll CT crops that are not
available here; these volumes stand in for them with the shapes and value
distributions the benchmark configurations name:

  material: 4-octave 3D value noise, base period 32 voxels, mapped to 40..220,
            plus Gaussian noise sigma=6, clipped to u8;
  air:      voxels where an independent 2-octave low-frequency value noise
            (base period 64) falls below its `air_frac` quantile are set to 0.

Value noise is a hash of integer lattice coordinates, so any sub-volume can
be generated on its own (chunk by chunk) and the field is continuous across
chunk borders. Generation runs with torch on the given device; CPU and GPU
results may differ in the last bit of the noise, which does not matter for
parity: every test feeds the same bytes to both codecs it compares.
"""
import torch

_MASK = 0xFFFFFFFF


def _hash(i, j, k, seed):
    h = (i * 73856093) ^ (j * 19349663) ^ (k * 83492791) ^ (seed * 2654435761)
    h = h & _MASK
    h = ((h ^ (h >> 13)) * 1274126177) & _MASK
    h = ((h ^ (h >> 16)) * 2246822519) & _MASK
    h = h ^ (h >> 13)
    return (h & 0xFFFFFF).to(torch.float32) / float(1 << 24)


def _value_noise(origin, shape, period, seed, device):
    """One octave on the lattice of spacing `period`, smoothstep trilinear."""
    axes = []
    for o, n in zip(origin, shape):
        p = (torch.arange(n, device=device, dtype=torch.float64) + o) / period
        i0 = torch.floor(p)
        t = (p - i0).to(torch.float32)
        axes.append((i0.to(torch.int64), t * t * (3 - 2 * t)))
    (z0, tz), (y0, ty), (x0, tx) = axes
    z0, y0, x0 = z0.view(-1, 1, 1), y0.view(1, -1, 1), x0.view(1, 1, -1)
    tz, ty, tx = tz.view(-1, 1, 1), ty.view(1, -1, 1), tx.view(1, 1, -1)
    out = torch.zeros(shape, dtype=torch.float32, device=device)
    for dz in (0, 1):
        wz = tz if dz else 1 - tz
        for dy in (0, 1):
            wy = ty if dy else 1 - ty
            for dx in (0, 1):
                wx = tx if dx else 1 - tx
                out += wz * wy * wx * _hash(z0 + dz, y0 + dy, x0 + dx, seed)
    return out


def fbm(origin, shape, base_period, octaves, seed, device):
    """Sum of octaves (period halves, amplitude halves), normalised to [0,1)."""
    acc = torch.zeros(shape, dtype=torch.float32, device=device)
    amp, norm = 1.0, 0.0
    for o in range(octaves):
        acc += amp * _value_noise(origin, shape, base_period / (2 ** o), seed * 977 + o, device)
        norm += amp
        amp *= 0.5
    return acc / norm


def air_threshold(seed, air_frac, extent, device, samples=1 << 20):
    """The air-noise quantile over a volume of `extent` voxels, estimated on a
    fixed seeded sample of positions (deterministic for a seed)."""
    if air_frac <= 0:
        return -1.0
    g = torch.Generator(device="cpu").manual_seed(seed * 7919 + 17)
    pts = [torch.randint(0, int(e), (samples,), generator=g) for e in extent]
    vals = torch.zeros(samples, dtype=torch.float32)
    amp, norm = 1.0, 0.0
    for o in range(2):
        period = 64.0 / (2 ** o)
        acc = torch.zeros(samples, dtype=torch.float32)
        pos = [(p.to(torch.float64)) / period for p in pts]
        base = [torch.floor(p) for p in pos]
        t = [(p - b).to(torch.float32) for p, b in zip(pos, base)]
        t = [v * v * (3 - 2 * v) for v in t]
        b = [v.to(torch.int64) for v in base]
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    w = (t[0] if dz else 1 - t[0]) * (t[1] if dy else 1 - t[1]) * (t[2] if dx else 1 - t[2])
                    acc += w * _hash(b[0] + dz, b[1] + dy, b[2] + dx, (seed + 100003) * 977 + o)
        vals += amp * acc
        norm += amp
        amp *= 0.5
    vals /= norm
    return float(torch.quantile(vals, air_frac).item())


def region(seed, origin, shape, air_frac=0.4, air_cut=None, device="cpu", noise_sigma=6.0):
    """u8 volume of `shape` (z,y,x) at voxel `origin` of the seeded field.

    air_cut: precomputed air threshold (air_threshold) for multi-chunk volumes;
    when None the quantile is taken over this region itself.
    """
    shape = tuple(int(s) for s in shape)
    mat = fbm(origin, shape, 32.0, 4, seed, device)
    v = 40.0 + 180.0 * mat
    g = torch.Generator(device=device).manual_seed(
        (seed * 1000003 + origin[0] * 7 + origin[1] * 13 + origin[2] * 17) & 0x7FFFFFFF)
    v += noise_sigma * torch.randn(shape, generator=g, device=device, dtype=torch.float32)
    v = v.round_().clamp_(0, 255).to(torch.uint8)
    if air_frac > 0:
        air = fbm(origin, shape, 64.0, 2, seed + 100003, device)
        if air_cut is None:
            flat = air.reshape(-1)
            sub = flat[:: max(1, flat.numel() // (1 << 22))]
            air_cut = float(torch.quantile(sub.float(), air_frac).item())
        v[air < air_cut] = 0
    return v


def chunk(seed, air_frac=0.4, device="cpu"):
    """One 256^3 chunk (the per-chunk generator of the chunk-decode configs)."""
    return region(seed, (0, 0, 0), (256, 256, 256), air_frac=air_frac, device=device)
