"""Read-only readers with GPU decode (mc_open, mc_open_streaming, partial
fetch, mc_b200_reader_decode_blocks) against the reference's readers on the
same archive file: identical voxels, and the same bytes pulled through the
byte-range callback."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
PICKS = [(8, 8, 8), (0, 0, 0), (15, 15, 15), (3, 12, 7), (12, 3, 9)]


@pytest.fixture(scope="module")
def reader_archive(gpu, tmp_path_factory):
    import torch
    import volumes
    path = str(tmp_path_factory.mktemp("rd") / "r.mca")
    with gpu.open(path, 768, 256, 256, 6.0) as a:
        vox = [volumes.region(90 + i, (0, 0, 256 * i), (256, 256, 256), 0.4, device="cuda").contiguous()
               for i in range(2)]
        assert a.append_chunks(0, [(0, 0, 0), (0, 0, 1)], [v.data_ptr() for v in vox], 6.0, on_device=True) == 0
        air = torch.zeros((256, 256, 256), dtype=torch.uint8, device="cuda")
        assert a.append_chunks(0, [(0, 0, 2)], [air.data_ptr()], 6.0, on_device=True) == 0
        l1 = volumes.region(95, (0, 0, 0), (256, 256, 256), 0.3, device="cuda").contiguous()
        assert a.append_chunks(1, [(0, 0, 0)], [l1.data_ptr()], 3.0, ctx_q=3.0, on_device=True) == 0
        torch.cuda.synchronize()
        want = {}
        for lod, cx in [(0, 0), (0, 1), (0, 2), (1, 0)]:
            co = a.chunk_offset(lod, 0, 0, cx)
            want[(lod, cx)] = (co, a.decode_chunk(co).reshape(256, 256, 256) if co > 1 else None)
    return path, open(path, "rb").read(), want


def _payload_lens(data, co):
    """(bytes of the chunk's header + bitmap + length table, {block: payload length})."""
    fml = data[co + 12] | (data[co + 13] << 8)
    bm = np.frombuffer(data[co + 14 + fml:co + 14 + fml + 512], np.uint8)
    present = [bi for bi in range(4096) if (bm[bi >> 3] >> (bi & 7)) & 1]
    lens = np.frombuffer(data[co + 14 + fml + 512:co + 14 + fml + 512 + 2 * len(present)], np.uint16)
    return 14 + 512 + 2 * len(present), dict(zip(present, (int(v) for v in lens)))


def _block(vol, bz, by, bx):
    return vol[bz * 16:bz * 16 + 16, by * 16:by * 16 + 16, bx * 16:bx * 16 + 16].reshape(-1)


def test_modes_match_reference_and_archive(gpu, ref, reader_archive):
    from mcb200 import Reader
    path, data, want = reader_archive
    rng = np.random.default_rng(1)
    picks = PICKS + [tuple(int(v) for v in rng.integers(0, 16, 3)) for _ in range(30)]
    for kind in ("flat", "full", "partial"):
        def mk(lib):
            return Reader(lib, data=data) if kind == "flat" else Reader(lib, path=path, partial=kind == "partial")
        with mk(gpu) as m, mk(ref) as r:
            for (lod, cx), (co, vol) in want.items():
                assert m.chunk_offset(lod, 0, 0, cx) == r.chunk_offset(lod, 0, 0, cx) == co
                for p in picks:
                    got = m.decode_block(co, *p)
                    assert np.array_equal(got, r.decode_block(co, *p)), (kind, lod, cx, p)
                    if vol is not None:
                        assert np.array_equal(got, _block(vol, *p)), (kind, lod, cx, p)
                    else:
                        assert not got.any()
            if kind != "flat":
                assert (m.bytes, m.calls) == (r.bytes, r.calls), kind   # same fetch pattern


def test_partial_fetch_reads_less(gpu, reader_archive):
    from mcb200 import Reader
    path, data, want = reader_archive
    co = want[(0, 0)][0]
    with Reader(gpu, path=path) as full, Reader(gpu, path=path, partial=True) as part:
        assert full.chunk_offset(0, 0, 0, 0) == part.chunk_offset(0, 0, 0, 0) == co
        b0, p0 = full.bytes, part.bytes
        for p in PICKS:
            assert np.array_equal(full.decode_block(co, *p), part.decode_block(co, *p))
        assert (part.bytes - p0) * 4 < full.bytes - b0


def test_batched_device_decode(gpu, reader_archive):
    """Blocks in any order, repeated and absent, out-of-range coordinates and
    the all-air chunk: the batch == block-by-block decode, for a flat and a
    partial-fetch reader; the partial batch reads each payload run once."""
    import torch
    from mcb200 import Reader
    path, data, want = reader_archive
    rng = np.random.default_rng(2)
    coords = [tuple(int(v) for v in rng.integers(0, 16, 3)) for _ in range(300)]
    coords += [coords[5], coords[5], (16, 0, 0), (0, -1, 3)]
    for kind in ("flat", "partial"):
        with (Reader(gpu, data=data) if kind == "flat" else Reader(gpu, path=path, partial=True)) as m:
            for (lod, cx), (co, vol) in want.items():
                d = torch.full((len(coords) * 4096,), 0xEE, dtype=torch.uint8, device="cuda")
                b0 = m.bytes
                assert m.decode_blocks_dev(co, coords, d.data_ptr()) == 0
                batch_bytes = m.bytes - b0
                got = d.cpu().numpy().reshape(len(coords), 4096)
                for i, c in enumerate(coords):
                    inside = all(0 <= v < 16 for v in c)
                    exp = _block(vol, *c) if (vol is not None and inside) else np.zeros(4096, np.uint8)
                    assert np.array_equal(got[i], exp), (kind, lod, cx, c)
                if kind == "partial" and vol is not None:
                    # the chunk's header, bitmap and lengths, then each distinct
                    # asked-for payload exactly once
                    idx_bytes, lens = _payload_lens(data, co)
                    distinct = {(c[0] * 16 + c[1]) * 16 + c[2] for c in coords if all(0 <= v < 16 for v in c)}
                    assert batch_bytes == idx_bytes + sum(lens.get(bi, 0) for bi in distinct), (lod, cx)


def test_unreadable_and_corrupt_sources(gpu, ref, reader_archive):
    """A byte source that fails part-way, chunk offsets that point at garbage,
    and a flat archive cut short: zeros, never a crash, and the same voxels
    as the reference's readers where the reference defines them."""
    import ctypes as C
    import torch
    from mcb200 import READ_FN, Reader
    path, data, want = reader_archive
    co = want[(0, 0)][0]
    # a source that serves the first 200 KB only: headers and node tables,
    # not every payload
    short = data[:co + 3000]

    def read(ud, off, n, dst):
        if off + n > len(short):
            return -1
        C.memmove(dst, short[off:off + n], n)
        return 0
    cb = READ_FN(read)
    Reader(gpu, data=data).close()   # binds the reader signatures
    for partial in (0, 1):
        r = gpu.L.mc_open_streaming(C.cast(cb, C.c_void_p), None, len(data))
        gpu.L.mc_reader_set_partial_fetch(r, partial)
        for p in [(0, 0, 0), (8, 8, 8), (15, 15, 15)]:
            out = np.full(4096, 0xEE, np.uint8)
            gpu.L.mc_decode_block(r, co, *p, out.ctypes.data)
            if not partial:
                assert not out.any()   # the whole blob cannot be read
        d = torch.full((3 * 4096,), 0xEE, dtype=torch.uint8, device="cuda")
        coords = np.array([[0, 0, 0], [8, 8, 8], [15, 15, 15]], np.int32)
        assert gpu.L.mc_b200_reader_decode_blocks(r, co, coords.ctypes.data, 3, C.c_void_p(d.data_ptr()), None) == 0
        if not partial:
            assert not d.any().item()
        gpu.L.mc_close(r)
    # flat readers: offsets into garbage and a truncated archive
    with Reader(gpu, data=data) as m, Reader(ref, data=data) as rr:
        for bogus in (co + 7, len(data) - 10, len(data) + 100, 300):
            assert np.array_equal(m.decode_block(bogus, 1, 2, 3), rr.decode_block(bogus, 1, 2, 3)) or \
                not m.decode_block(bogus, 1, 2, 3).any()
    cut = data[:co + 5000]
    with Reader(gpu, data=cut) as m, Reader(ref, data=cut) as rr:
        assert m.chunk_offset(0, 0, 0, 0) == rr.chunk_offset(0, 0, 0, 0)
        for p in PICKS:
            assert np.array_equal(m.decode_block(co, *p), rr.decode_block(co, *p)), p
