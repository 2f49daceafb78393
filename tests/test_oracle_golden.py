"""The oracle (our C restatement) reproduces the reference's golden vectors
byte for byte: block payloads, decoded blocks, corrupt streams, fraction maps,
XXH64, whole-chunk blobs and decoded chunks."""
import os

import numpy as np
import pytest

import shapes
from conftest import GOLDEN, ctx_q, sha


def test_block_encode_decode(oracle, golden_blocks):
    g = golden_blocks
    pats = shapes.block_patterns()
    for i in range(len(g["q"])):
        q, tau, k = float(g["q"][i]), int(g["tau"][i]), int(g["kind"][i])
        want = g["payload"][g["offs"][i]:g["offs"][i + 1]].tobytes()
        got = oracle.enc_block(pats[k], q, tau)
        assert got == want, f"case {i}: pattern {k} q={q} tau={tau}"
        dec = oracle.dec_block(got, ctx_q(q)) if got else np.zeros(4096, np.uint8)
        assert sha(dec) == g["decoded_sha"][i], f"case {i} decode"


def test_max_error_bound(oracle):
    """|err| <= tau on every voxel when coded with a max-error bound
    (the reference's api test: tau bound, air within [0, tau])."""
    for k, vox in enumerate(shapes.block_patterns()):
        for q, tau in [(2.0, 3), (6.0, 8), (0.5, 1), (16.0, 32)]:
            p = oracle.enc_block(vox, q, tau)
            if not p:
                assert not vox.any()
                continue
            d = oracle.dec_block(p, q).astype(int)
            assert np.abs(d - vox.astype(int)).max() <= tau, (k, q, tau)


def test_corrupt_streams(oracle, golden_corrupt):
    g = golden_corrupt
    for i in range(len(g["q"])):
        p = g["payload"][g["offs"][i]:g["offs"][i + 1]].tobytes()
        assert sha(oracle.dec_block(p, float(g["q"][i]))) == g["decoded_sha"][i], f"stream {i}"


def test_fracmap_and_xxh64(oracle, golden_meta):
    g = golden_meta
    for t in range(len(g["frac"])):
        want = g["fmap"][g["fmap_offs"][t]:g["fmap_offs"][t + 1]].tobytes()
        assert oracle.enc_fracmap(g["frac"][t]) == want
        assert np.array_equal(oracle.dec_fracmap(want), g["frac"][t])
    data = g["xx_data"].tobytes()
    for ln, seed, h in g["xx"]:
        assert oracle.xxh64(data[:int(ln)], int(seed)) == int(h)


def test_chunk_blobs(oracle, golden_chunks):
    g = golden_chunks
    steps = shapes.archive_sequence()
    for i, st in enumerate(steps):
        want = g["blobs"][g["offs"][i]:g["offs"][i + 1]].tobytes()
        vox = shapes.chunk_source(st["src"])
        if st["op"] == "par":
            got = oracle.encode_chunk(vox, st["q"], 0)
        else:
            q, tau = [(0.5, 1), (0.5, 2), (1.0, 4), (2.5, 8), (6.0, 16), (16.0, 32), (32.0, 64), (64.0, 128)][st["preset"]]
            got = oracle.encode_chunk(vox, q, tau)
        assert got == want, st["name"]
        if want:
            assert oracle.blob_hash(want) == int.from_bytes(want[4:12], "little")
            assert sha(oracle.decode_chunk(want)) == g["decoded_sha"][i], st["name"]


def test_scan_and_priors(oracle):
    scan = np.zeros(4096, np.uint16)
    oracle.L.or_scan_table(scan.ctypes.data)
    idx = scan.astype(int)
    l1 = (idx >> 8) + ((idx >> 4) & 15) + (idx & 15)
    assert sorted(idx.tolist()) == list(range(4096))
    assert np.all(np.diff(l1) >= 0)
    same = np.diff(l1) == 0
    assert np.all(np.diff(idx)[same] > 0)      # ties in raster order
    lo, hi = oracle.priors_for_q(1.0), oracle.priors_for_q(12.0)
    assert lo[0] == 115 and hi[0] == 456        # SIG slot 0 endpoints
    assert oracle.priors_for_q(0.25)[0] == 115  # q <= 1 uses the q=1 table
    mid = oracle.priors_for_q(3.4641)           # log-midpoint lies between
    assert min(lo[0], hi[0]) <= mid[0] <= max(lo[0], hi[0])


def test_deblock(oracle):
    """The deblocking restatement reproduces mc_deblock's output digests."""
    g = np.load(os.path.join(GOLDEN, "deblock.npz"))
    vols = dict(shapes.deblock_volumes())
    for name, q, want in zip(g["names"], g["q"], g["out_sha"]):
        v = vols[str(name)].copy()
        oracle.deblock(v, float(q))
        assert sha(v) == want, (name, q)


def test_pyramid(oracle):
    """The one-shot builder's LOD pyramid restated with or_decimate and the
    oracle's chunk encoder: every LOD's chunk blobs == mc_build's digests."""
    import hashlib
    g = np.load(os.path.join(GOLDEN, "pyramid.npz"))
    chunks = shapes.pyramid_chunks(shapes.pyramid_volume(), oracle.decimate)
    for q in sorted(set(float(k[0]) for k in g["keys"])):
        want = {tuple(int(v) for v in k[1:]): d for k, d in zip(g["keys"], g["blob_sha"]) if float(k[0]) == q}
        assert set(want) == set(chunks), q
        for key, c in chunks.items():
            blob = oracle.encode_chunk(c.reshape(-1), q, 0, header_q=q)
            assert hashlib.sha256(blob).hexdigest() == want[key], (q, key)


PRESETS = [(0.5, 1), (0.5, 2), (1.0, 4), (2.5, 8), (6.0, 16), (16.0, 32), (32.0, 64), (64.0, 128)]


@pytest.fixture
def golden_priors(oracle):
    g = np.load(os.path.join(GOLDEN, "priors.npz"))
    oracle.set_priors(g["plo"], g["phi"])
    yield g
    oracle.set_priors(None, None)


def test_priors_blocks(oracle, golden_priors):
    """Per-volume priors (src/mc_codec.c:144-167): block payloads and decoded
    blocks under a non-default prior pair match the reference's."""
    g = golden_priors
    pats = shapes.block_patterns()
    differ = 0
    for i in range(len(g["q"])):
        q, tau, k = float(g["q"][i]), int(g["tau"][i]), int(g["kind"][i])
        want = g["payload"][g["offs"][i]:g["offs"][i + 1]].tobytes()
        got = oracle.enc_block(pats[k], q, tau)
        assert got == want, f"case {i}: pattern {k} q={q} tau={tau}"
        dec = oracle.dec_block(got, q) if got else np.zeros(4096, np.uint8)
        assert sha(dec) == g["decoded_sha"][i], f"case {i} decode"
        oracle.set_priors(None, None)
        differ += oracle.enc_block(pats[k], q, tau) != want
        oracle.set_priors(g["plo"], g["phi"])
    assert differ > len(g["q"]) // 2   # the prior pair really changes the bit stream


def test_priors_chunks(oracle, golden_priors):
    """Chunks appended to an archive whose priors were stamped by
    mc_archive_set_priors (src/mc_archive.c:650-662) decode to the reference's
    voxels when the oracle codes them under the same priors."""
    g = golden_priors
    for i, st in enumerate(shapes.priors_sequence()):
        vox = shapes.chunk_source(st["src"])
        q, tau = (st["q"], 0) if st["op"] == "par" else PRESETS[st["preset"]]
        blob = oracle.encode_chunk(vox, q, tau)
        assert sha(oracle.decode_chunk(blob)) == g["chunk_sha"][i], st["name"]
