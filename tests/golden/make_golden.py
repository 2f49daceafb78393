"""Generates the golden vectors in this folder from the REFERENCE's own code.

Runs the reference sources compiled in strict IEEE mode (oracle/_ref/libmcref.so,
built by `make -C oracle ref` from a reference checkout) through their public
C API and records inputs, payload bytes and digests of decoded outputs:

  blocks.npz   block encode (mc_enc_block) / decode (mc_dec_block) vectors over
               block patterns x qualities x max-error bounds, including
               out-of-range qualities;
  corrupt.npz  arbitrary byte strings decoded as payloads (mc_dec_block);
  meta.npz     fraction-map coder and XXH64 vectors;
  chunks.npz   whole-chunk blobs from mc_archive_append_chunk_par /
               _ctx (preset ladder), the decoded chunk's digest, and the
               archive-file digest of a fixed call sequence;
  pyramid.npz  mc_build (the one-shot builder, which box-decimates LODs) on
               shapes.pyramid_volume() at two qualities: the digest of every
               LOD's chunk blobs, keyed by (q, lod, cz, cy, cx);
  deblock.npz  digests of mc_deblock's output on the shapes.deblock_volumes()
               inputs over a set of qualities (the volume is followed by a
               zero plane, so the reference's read past the last z face sees
               zeros);
  priors.npz   per-volume trained priors (shapes.priors_tables()): block
               encode/decode vectors under mc_codec_set_priors, and an archive
               whose prior blob is stamped by mc_archive_set_priors before the
               shapes.priors_sequence() appends -- its file digest and every
               chunk's decoded digest.

Inputs are deterministic integer formulas (shapes.py) so tests regenerate
them exactly. Usage: python tests/golden/make_golden.py
"""
import hashlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "matter-compressor_b200"))
sys.path.insert(0, HERE)
from mcb200 import McLib  # noqa: E402
import shapes  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "libmcref.so")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    ref = McLib(REF, b200=False)
    ref.L.mc_codec_init()

    # ---------------------------------------------------------------- blocks
    cases = []
    qs = [0.5, 1.0, 2.5, 3.0, 6.0, 12.0, 64.0]
    taus = [0, 1, 4, 16]
    for k, vox in enumerate(shapes.block_patterns()):
        for q in qs:
            for tau in taus:
                cases.append((k, q, tau))
    for k in range(3):   # quality sanitiser: NaN / <=0 / >1024 code at q=8
        for q in [0.0, -3.0, float("nan"), 4096.0]:
            cases.append((k, q, 0))
    pats = shapes.block_patterns()
    payloads, decoded_sha, qarr, tarr, kind = [], [], [], [], []
    for k, q, tau in cases:
        p = ref.enc_block(pats[k], q, tau)
        ctxq = q if (q == q and 0 < q <= 1024) else 8.0
        d = ref.dec_block(p, ctxq) if p else np.zeros(4096, np.uint8)
        payloads.append(np.frombuffer(p, np.uint8))
        decoded_sha.append(sha(d))
        qarr.append(q)
        tarr.append(tau)
        kind.append(k)
    offs = np.cumsum([0] + [len(p) for p in payloads]).astype(np.int64)
    np.savez_compressed(os.path.join(HERE, "blocks.npz"), kind=np.array(kind, np.int32), q=np.array(qarr, np.float32),
                        tau=np.array(tarr, np.int32), offs=offs,
                        payload=np.concatenate(payloads) if payloads else np.zeros(0, np.uint8),
                        decoded_sha=np.array(decoded_sha))
    print("blocks:", len(cases), "cases,", int(offs[-1]), "payload bytes")

    # ---------------------------------------------------------------- corrupt
    rng = np.random.Generator(np.random.PCG64(20260101))
    cp, cq, csha = [], [], []
    for t in range(400):
        n = int(rng.integers(0, 240))
        p = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        q = [1.0, 3.0, 6.0, 12.0][t % 4]
        d = ref.dec_block(p, q)
        cp.append(np.frombuffer(p, np.uint8))
        cq.append(q)
        csha.append(sha(d))
    # truncations / bit flips of valid payloads
    for t in range(200):
        k = t % len(pats)
        p = bytearray(ref.enc_block(pats[k], 6.0, 0))
        if not p:
            continue
        mode = t % 3
        if mode == 0:
            p = p[: int(rng.integers(0, len(p)))]
        elif mode == 1:
            i = int(rng.integers(0, len(p)))
            p[i] ^= 1 << int(rng.integers(0, 8))
        else:
            p = p + bytes(rng.integers(0, 256, int(rng.integers(1, 32)), dtype=np.uint8))
        d = ref.dec_block(bytes(p), 6.0)
        cp.append(np.frombuffer(bytes(p), np.uint8))
        cq.append(6.0)
        csha.append(sha(d))
    coffs = np.cumsum([0] + [len(p) for p in cp]).astype(np.int64)
    np.savez_compressed(os.path.join(HERE, "corrupt.npz"), q=np.array(cq, np.float32), offs=coffs,
                        payload=np.concatenate(cp), decoded_sha=np.array(csha))
    print("corrupt:", len(cp), "streams")

    # ---------------------------------------------------------------- fracmap + xxh64
    fr_in, fr_out, fr_offs = [], [], [0]
    for t in range(6):
        fr = shapes.frac_pattern(t)
        out = np.zeros(2112, np.uint8)
        n = ref.L.mc_enc_fracmap(fr.ctypes.data, out.ctypes.data, out.size)
        fr_in.append(fr)
        fr_out.append(out[:n])
        fr_offs.append(fr_offs[-1] + n)
    xx_data = rng.integers(0, 256, 300, dtype=np.uint8)
    xx = []
    for ln in [0, 1, 3, 4, 7, 8, 31, 32, 33, 63, 64, 100, 255, 300]:
        for seed in [0, 1, 0x6D636368756E6B, 0xFFFFFFFFFFFFFFFF]:
            h = ref.L.mc_xxh64(xx_data.ctypes.data, ln, seed)
            xx.append((ln, seed, h))
    np.savez_compressed(os.path.join(HERE, "meta.npz"), frac=np.stack(fr_in), fmap=np.concatenate(fr_out),
                        fmap_offs=np.array(fr_offs, np.int64), xx_data=xx_data,
                        xx=np.array(xx, dtype=np.uint64))
    print("meta: fracmaps + xxh64 vectors")

    # ---------------------------------------------------------------- chunks + archive
    blobs, names, dsha, cos = [], [], [], []
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "golden.mca")
        with ref.open(path, 1024, 1024, 1024, 6.0) as a:
            for step in shapes.archive_sequence():
                vox = shapes.chunk_source(step["src"])
                if step["op"] == "par":
                    rc = a.append_par(0, *step["at"], vox, step["q"])
                else:
                    rc = a.append_ctx(0, *step["at"], vox, 8.0, preset=step["preset"])
                assert rc == 0, step
                co = a.chunk_offset(0, *step["at"])
                names.append(step["name"])
                cos.append(co)
                dsha.append(sha(a.decode_chunk(co)))
            ref.L.mc_archive_set_metadata(a.a, b"golden", 6)
        data = open(path, "rb").read()
        arc_sha = hashlib.sha256(data).hexdigest()
    for co in cos:
        blobs.append(np.frombuffer(data[co:co + shapes.blob_len(data, co)] if co > 1 else b"", np.uint8))
    boffs = np.cumsum([0] + [len(b) for b in blobs]).astype(np.int64)
    np.savez_compressed(os.path.join(HERE, "chunks.npz"), names=np.array(names), offs=boffs,
                        blobs=np.concatenate(blobs), decoded_sha=np.array(dsha), archive_sha=np.array(arc_sha),
                        archive_len=np.array(len(data), np.int64))
    print("chunks:", len(blobs), "blobs,", int(boffs[-1]), "bytes; archive", len(data), "bytes")
    deblock_golden(ref)
    pyramid_golden(ref)
    priors_golden(ref)


PYRAMID_QS = [6.0, 0.25]


def pyramid_golden(ref):
    import ctypes as C

    class Opts(C.Structure):
        _fields_ = [("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("quality", C.c_float),
                    ("metadata", C.c_char_p), ("meta_len", C.c_size_t)]

    class Src(C.Structure):
        _fields_ = [("v", C.c_void_p), ("nz", C.c_int), ("ny", C.c_int), ("nx", C.c_int)]

    orc = C.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    vol = shapes.pyramid_volume()
    nz, ny, nx = vol.shape
    src = Src(vol.ctypes.data, nz, ny, nx)
    ref.L.mc_build.restype = C.c_void_p
    ref.L.mc_build.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_size_t)]
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    keys, digests = [], []
    levels = shapes.pyramid_levels(nz, ny, nx)
    for q in PYRAMID_QS:
        opts = Opts(0, nx, ny, nz, q, None, 0)
        n = C.c_size_t()
        buf = ref.L.mc_build(C.cast(orc.or_voxel_source, C.c_void_p), C.byref(src), C.byref(opts), C.byref(n))
        data = C.string_at(buf, n.value)
        libc.free(buf)
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "p.mca")
            open(path, "wb").write(data)
            with ref.open(path, nx, ny, nz, q) as a:
                for lod, (dz, dy, dx) in levels:
                    for cz in range((dz + 255) // 256):
                        for cy in range((dy + 255) // 256):
                            for cx in range((dx + 255) // 256):
                                co = a.chunk_offset(lod, cz, cy, cx)
                                if co <= 1:
                                    continue
                                keys.append((q, lod, cz, cy, cx))
                                digests.append(hashlib.sha256(data[co:co + shapes.blob_len(data, co)]).hexdigest())
    np.savez_compressed(os.path.join(HERE, "pyramid.npz"), keys=np.array(keys, np.float64), blob_sha=np.array(digests),
                        levels=np.array([lv for lv, _ in levels], np.int32))
    print("pyramid:", len(digests), "blobs over", len(levels), "LODs")


DEBLOCK_QS = [0.5, 1.0, 3.0, 6.0, 12.0, 40.0]


def deblock_golden(ref):
    import ctypes as C
    ref.L.mc_deblock.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float]
    names, qs, digests = [], [], []
    for name, vol in shapes.deblock_volumes():
        nz, ny, nx = vol.shape
        for q in DEBLOCK_QS:
            buf = np.zeros(vol.size + ny * nx, np.uint8)
            buf[:vol.size] = vol.ravel()
            ref.L.mc_deblock(buf.ctypes.data, nz, ny, nx, q)
            names.append(name)
            qs.append(q)
            digests.append(sha(buf[:vol.size]))
    np.savez_compressed(os.path.join(HERE, "deblock.npz"), names=np.array(names), q=np.array(qs, np.float32),
                        out_sha=np.array(digests))
    print("deblock:", len(digests), "cases")


PRIORS_QS = [1.0, 3.0, 6.0, 12.0]
PRIORS_TAUS = [0, 4]


def priors_golden(ref):
    plo, phi = shapes.priors_tables()
    kinds, qs, taus, pays, dsha = [], [], [], [], []
    ref.set_priors(plo, phi)
    try:
        for k, vox in enumerate(shapes.block_patterns()):
            for q in PRIORS_QS:
                for tau in PRIORS_TAUS:
                    p = ref.enc_block(vox, q, tau)
                    kinds.append(k)
                    qs.append(q)
                    taus.append(tau)
                    pays.append(np.frombuffer(p, np.uint8))
                    dsha.append(sha(ref.dec_block(p, q)))
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "priors.mca")
            names, csha = [], []
            with ref.open(path, 512, 256, 256, 6.0) as a:
                assert ref.L.mc_archive_set_priors(a.a, plo.ctypes.data, phi.ctypes.data) == 0
                for step in shapes.priors_sequence():
                    vox = shapes.chunk_source(step["src"])
                    if step["op"] == "par":
                        rc = a.append_par(0, *step["at"], vox, step["q"])
                    else:
                        rc = a.append_ctx(0, *step["at"], vox, 8.0, preset=step["preset"])
                    assert rc == 0, step
                    names.append(step["name"])
                    csha.append(sha(a.decode_chunk(a.chunk_offset(0, *step["at"]))))
            data = open(path, "rb").read()
    finally:
        ref.set_priors(None, None)
    offs = np.cumsum([0] + [len(p) for p in pays]).astype(np.int64)
    np.savez_compressed(os.path.join(HERE, "priors.npz"), plo=plo, phi=phi, kind=np.array(kinds, np.int32),
                        q=np.array(qs, np.float32), tau=np.array(taus, np.int32), offs=offs,
                        payload=np.concatenate(pays), decoded_sha=np.array(dsha), chunk_names=np.array(names),
                        chunk_sha=np.array(csha), archive_sha=np.array(hashlib.sha256(data).hexdigest()),
                        archive_len=np.array(len(data), np.int64))
    print("priors:", len(pays), "blocks,", len(names), "chunks; archive", len(data), "bytes")


if __name__ == "__main__":
    if sys.argv[1:] in (["deblock"], ["pyramid"], ["priors"]):
        r = McLib(REF, b200=False)
        r.L.mc_codec_init()
        {"deblock": deblock_golden, "pyramid": pyramid_golden, "priors": priors_golden}[sys.argv[1]](r)
    else:
        main()
