"""Host-side archive format, no GPU needed: installing the golden blobs with
mc_archive_append_chunk_compressed, index pre-reservation, metadata and air
markers give a file byte-identical to the reference doing the same calls;
verify / hash / fraction-map helpers match the golden vectors."""
import hashlib
import os

import numpy as np
import pytest

import shapes
from conftest import ROOT

LIB = os.path.join(ROOT, "matter-compressor_b200", "libmc_b200.so")


def product_host():
    from mcb200 import McLib
    return McLib(LIB)


def replay(lib, path, g):
    blobs = [g["blobs"][g["offs"][i]:g["offs"][i + 1]] for i in range(len(g["offs"]) - 1)]
    with lib.open(path, 1024, 1024, 1024, 6.0) as a:
        assert lib.L.mc_archive_reserve_index(a.a, 1, 0, 0, 0) == 0
        for i, b in enumerate(blobs):
            at = [(0, 0, 0), (0, 1, 0), (3, 0, 2), (0, 0, 3)][i % 4]
            lod = i % 3
            if b.size:
                rc = lib.L.mc_archive_append_chunk_compressed(a.a, lod, *at, b.ctypes.data, b.size)
                assert rc == 0
        lib.L.mc_archive_set_metadata(a.a, b"host-format", 11)
        offs = [a.chunk_offset(i % 3, *[(0, 0, 0), (0, 1, 0), (3, 0, 2), (0, 0, 3)][i % 4]) for i in range(len(blobs))]
    return open(path, "rb").read(), offs


def test_compressed_append_byte_identical(tmp_path, ref, golden_chunks):
    got, go = replay(product_host(), str(tmp_path / "p.mca"), golden_chunks)
    want, wo = replay(ref, str(tmp_path / "r.mca"), golden_chunks)
    assert go == wo
    assert hashlib.sha256(got).hexdigest() == hashlib.sha256(want).hexdigest()


def test_reopen_appends(tmp_path, golden_chunks):
    lib = product_host()
    g = golden_chunks
    b = g["blobs"][g["offs"][0]:g["offs"][1]]
    path = str(tmp_path / "a.mca")
    with lib.open(path, 512, 512, 512, 6.0) as a:
        assert lib.L.mc_archive_append_chunk_compressed(a.a, 0, 0, 0, 0, b.ctypes.data, b.size) == 0
    with lib.open(path, 512, 512, 512, 6.0) as a:   # reopen keeps appending
        assert lib.L.mc_archive_append_chunk_compressed(a.a, 0, 1, 1, 1, b.ctypes.data, b.size) == 0
        assert a.chunk_offset(0, 0, 0, 0) > 1 and a.chunk_offset(0, 1, 1, 1) > 1
        assert a.chunk_offset(0, 1, 0, 0) == 0
    assert lib.L.mc_archive_open_dims(path.encode(), 256, 512, 512, 6.0) is None   # dims mismatch


def test_verify_and_hash(tmp_path, golden_chunks):
    lib = product_host()
    g = golden_chunks
    data, _ = replay(lib, str(tmp_path / "v.mca"), g)
    arr = np.frombuffer(data, np.uint8).copy()
    assert lib.L.mc_verify_archive(arr.ctypes.data, arr.size, 0) == 0
    for i in range(len(g["offs"]) - 1):
        b = g["blobs"][g["offs"][i]:g["offs"][i + 1]]
        if b.size:
            assert lib.L.mc_chunk_compute_hash(b.ctypes.data, b.size) == int.from_bytes(b[4:12].tobytes(), "little")
    arr[len(arr) - 100] ^= 0x55      # tamper inside the last blob's payloads
    assert lib.L.mc_verify_archive(arr.ctypes.data, arr.size, 0) == 1


def test_fracmap_xxh64(golden_meta):
    lib = product_host()
    g = golden_meta
    for t in range(len(g["frac"])):
        fr = np.ascontiguousarray(g["frac"][t])
        out = np.zeros(2112, np.uint8)
        n = lib.L.mc_enc_fracmap(fr.ctypes.data, out.ctypes.data, out.size)
        assert out[:n].tobytes() == g["fmap"][g["fmap_offs"][t]:g["fmap_offs"][t + 1]].tobytes()
        back = np.zeros(4096, np.uint8)
        lib.L.mc_dec_fracmap(out.ctypes.data, n, back.ctypes.data)
        assert np.array_equal(back, fr)
    data = np.ascontiguousarray(g["xx_data"])
    for ln, seed, h in g["xx"]:
        assert lib.L.mc_xxh64(data.ctypes.data, int(ln), int(seed)) == int(h)


def test_sampler_and_fractions_match_reference(tmp_path, ref, golden_chunks):
    lib = product_host()
    res = []
    for L, name in [(lib, "p"), (ref, "r")]:
        _, _ = replay(L, str(tmp_path / (name + ".mca")), golden_chunks)
        with L.open(str(tmp_path / (name + ".mca")), 1024, 1024, 1024, 6.0) as a:
            boxes = a.sample_boxes(0, 42, 16, 64, 64, 64, 0.3)
            fr = [L.L.mc_archive_block_fraction(a.a, 0, bz, by, bx) for bz in range(0, 64, 7) for by in (0, 5, 17)
                  for bx in (0, 9, 33)]
            pres = [L.L.mc_archive_block_present(a.a, 0, bz, by, bx) for bz in range(0, 64, 7) for by in (0, 5, 17)
                    for bx in (0, 9, 33)]
        res.append((boxes, fr, pres))
    assert res[0] == res[1]


def test_readers_host_side_match_reference(tmp_path, ref, golden_chunks):
    """mc_open / mc_open_streaming (full and partial fetch): chunk resolution
    (absent, present, out-of-range LOD, failed reads), blob length and bytes,
    dims, quality and LOD count == the reference's readers on the same file."""
    from mcb200 import Reader
    path = str(tmp_path / "r.mca")
    data, _ = replay(ref, path, golden_chunks)
    mine_lib = product_host()
    coords = [(lod, cz, cy, cx) for lod in range(-1, 9) for cz in range(4) for cy in range(2) for cx in range(4)]
    for kind in ("flat", "full", "partial"):
        def mk(lib):
            if kind == "flat":
                return Reader(lib, data=data)
            return Reader(lib, path=path, partial=kind == "partial")
        with mk(mine_lib) as m, mk(ref) as r:
            assert m.info() == r.info()
            for c in coords:
                assert m.chunk_offset_chk(*c) == r.chunk_offset_chk(*c), (kind, c)
                co = r.chunk_offset(*c)
                if co > 1:
                    assert m.blob(co) == r.blob(co) == data[co:co + shapes.blob_len(data, co)]
    # a byte source that fails after the header reports err=1, not an absent chunk
    import ctypes as C
    from mcb200 import READ_FN
    hdr = data[:256]

    def read(ud, off, n, dst):
        if off + n > len(hdr):
            return -1
        C.memmove(dst, hdr[off:off + n], n)
        return 0
    cb = READ_FN(read)
    for lib in (mine_lib, ref):
        Reader(lib, data=data).close()   # binds the reader signatures
        r = lib.L.mc_open_streaming(C.cast(cb, C.c_void_p), None, len(data))
        err = C.c_int()
        assert lib.L.mc_chunk_offset_chk(r, 0, 0, 0, 0, C.byref(err)) == 0 and err.value == 1
        assert lib.L.mc_chunk_offset_chk(r, 7, 0, 0, 0, C.byref(err)) == 0 and err.value == 0   # no root
        lib.L.mc_close(r)
