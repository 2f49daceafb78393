"""Per-volume trained priors on the GPU (src/mc_codec.c:144-167,
src/mc_archive.c:650-672): an archive whose prior blob replaces the baked
corpus tables must encode byte-identically to the reference and decode
bit-exactly through every GPU path -- block codec, decode_chunk,
read_region(s), the device batch and plan paths, and the readers.

The priors are process-global, as in the reference: set by
mc_codec_set_priors / mc_archive_set_priors, loaded when an archive or reader
is opened. Every test puts the baked tables back when it ends."""
import hashlib
import os

import numpy as np
import pytest

import shapes
from conftest import GOLDEN, sha

pytestmark = pytest.mark.gpu
CHUNK = 256 ** 3


@pytest.fixture(scope="module")
def gp():
    return np.load(os.path.join(GOLDEN, "priors.npz"))


@pytest.fixture
def baked_after(gpu):
    yield
    gpu.set_priors(None, None)


def _append_priors_sequence(lib, path, plo, phi):
    with lib.open(path, 512, 256, 256, 6.0) as a:
        assert lib.L.mc_archive_set_priors(a.a, plo.ctypes.data, phi.ctypes.data) == 0
        for st in shapes.priors_sequence():
            vox = shapes.chunk_source(st["src"])
            if st["op"] == "par":
                assert a.append_par(0, *st["at"], vox, st["q"]) == 0
            else:
                assert a.append_ctx(0, *st["at"], vox, 8.0, preset=st["preset"]) == 0
    return open(path, "rb").read()


def test_block_codec_under_priors(gpu, gp, baked_after):
    pats = shapes.block_patterns()
    gpu.set_priors(gp["plo"], gp["phi"])
    for i in range(len(gp["q"])):
        q, tau, k = float(gp["q"][i]), int(gp["tau"][i]), int(gp["kind"][i])
        want = gp["payload"][gp["offs"][i]:gp["offs"][i + 1]].tobytes()
        assert gpu.enc_block(pats[k], q, tau) == want, (k, q, tau)
        if want:
            assert sha(gpu.dec_block(want, q)) == gp["decoded_sha"][i], (k, q, tau)
    # the baked tables come back: the same pattern codes differently
    # (case 4: pattern 0 at q = 6, no max error)
    gpu.set_priors(None, None)
    assert gpu.enc_block(pats[0], 6.0, 0) != gp["payload"][gp["offs"][4]:gp["offs"][5]].tobytes()


def test_archive_with_priors_byte_identical(gpu, gp, tmp_path, baked_after):
    """mc_archive_set_priors + appends on the GPU: the same file as the
    reference's, and every chunk decodes to the reference's voxels."""
    path = str(tmp_path / "p.mca")
    data = _append_priors_sequence(gpu, path, gp["plo"], gp["phi"])
    assert len(data) == int(gp["archive_len"])
    assert hashlib.sha256(data).hexdigest() == str(gp["archive_sha"])
    gpu.set_priors(None, None)   # opening the archive must load its own priors
    with gpu.open(path, 512, 256, 256, 6.0) as a:
        for i, st in enumerate(shapes.priors_sequence()):
            co = a.chunk_offset(0, *st["at"])
            assert sha(a.decode_chunk(co)) == gp["chunk_sha"][i], st["name"]
        co = a.chunk_offset(0, 0, 0, 0)
        whole = a.decode_chunk(co).reshape(256, 256, 256)
        blk = a.decode_block(co, 5, 9, 3).reshape(16, 16, 16)
        assert np.array_equal(blk, whole[80:96, 144:160, 48:64])
        reg = a.read_regions(0, [(10, 20, 30), (100, 7, 180)], 48, 48, 48).reshape(2, 48, 48, 48)
        assert np.array_equal(reg[0], whole[10:58, 20:68, 30:78])
        assert np.array_equal(reg[1], whole[100:148, 7:55, 180:228])


def test_reference_priors_archive_on_gpu(gpu, ref, gp, tmp_path, baked_after):
    """The reference writes the archive with its priors; the GPU library
    reads it through decode_chunk, the device batch, a decode plan, and the
    flat, streaming and partial-fetch readers; the GPU's batched device append
    under the stamped priors gives the reference's blob."""
    import torch
    from mcb200 import Reader
    path = str(tmp_path / "r.mca")
    try:
        data = _append_priors_sequence(ref, path, gp["plo"], gp["phi"])
    finally:
        ref.set_priors(None, None)
    steps = shapes.priors_sequence()
    with gpu.open(path, 512, 256, 256, 6.0) as a:
        offs = [a.chunk_offset(0, *st["at"]) for st in steps]
        for i, co in enumerate(offs):
            assert sha(a.decode_chunk(co)) == gp["chunk_sha"][i], steps[i]["name"]
        d_out = torch.empty(len(offs) * CHUNK, dtype=torch.uint8, device="cuda")
        assert a.decode_chunks_dev(offs, d_out.data_ptr()) == 0
        got = d_out.cpu().numpy()
        for i in range(len(offs)):
            assert sha(got[i * CHUNK:(i + 1) * CHUNK]) == gp["chunk_sha"][i], steps[i]["name"]
        d_out.zero_()
        plan = a.plan_chunks(offs, d_out.data_ptr())
        try:
            plan.launch()
            torch.cuda.synchronize()
            assert np.array_equal(d_out.cpu().numpy(), got)
        finally:
            plan.free()
    picks = [(0, 0, 0), (8, 8, 8), (15, 15, 15), (3, 12, 7)]
    for kind in ("flat", "full", "partial"):
        def mk(lib):
            return Reader(lib, data=data) if kind == "flat" else Reader(lib, path=path, partial=kind == "partial")
        with mk(gpu) as m, mk(ref) as r:
            for st in steps:
                co = m.chunk_offset(0, *st["at"])
                for p in picks:
                    assert np.array_equal(m.decode_block(co, *p), r.decode_block(co, *p)), (kind, st["name"], p)
    ref.set_priors(None, None)
    # batched device append under the stamped priors: the reference's blob
    with gpu.open(str(tmp_path / "g.mca"), 512, 256, 256, 6.0) as g:
        assert gpu.L.mc_archive_set_priors(g.a, gp["plo"].ctypes.data, gp["phi"].ctypes.data) == 0
        st = steps[0]
        vox = torch.from_numpy(shapes.chunk_source(st["src"])).cuda().contiguous()
        assert g.append_chunks(0, [st["at"]], [vox.data_ptr()], st["q"], on_device=True) == 0
        torch.cuda.synchronize()
        co = g.chunk_offset(0, *st["at"])
        mine = np.fromfile(str(tmp_path / "g.mca"), np.uint8).tobytes()
        assert mine[co:co + shapes.blob_len(mine, co)] == data[offs[0]:offs[0] + shapes.blob_len(data, offs[0])]
