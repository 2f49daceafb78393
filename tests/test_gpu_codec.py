"""GPU parity through the C ABI: the CUDA codec against the golden vectors
(reference output), the oracle and -- where shipped -- the reference build.
Integer/byte results must be bit-exact."""
import hashlib
import os

import numpy as np
import pytest

import shapes
from conftest import ctx_q, sha

pytestmark = pytest.mark.gpu
CHUNK = 256 ** 3
PRESETS = [(0.5, 1), (0.5, 2), (1.0, 4), (2.5, 8), (6.0, 16), (16.0, 32), (32.0, 64), (64.0, 128)]


def test_block_decode_golden(gpu, golden_blocks):
    g = golden_blocks
    for i in range(len(g["q"])):
        p = g["payload"][g["offs"][i]:g["offs"][i + 1]].tobytes()
        if not p:
            continue
        assert sha(gpu.dec_block(p, ctx_q(float(g["q"][i])))) == g["decoded_sha"][i], f"case {i}"


def test_block_encode_golden(gpu, golden_blocks):
    g = golden_blocks
    pats = shapes.block_patterns()
    for i in range(len(g["q"])):
        want = g["payload"][g["offs"][i]:g["offs"][i + 1]].tobytes()
        got = gpu.enc_block(pats[int(g["kind"][i])], float(g["q"][i]), int(g["tau"][i]))
        assert got == want, f"case {i}: kind {int(g['kind'][i])} q={float(g['q'][i])} tau={int(g['tau'][i])}"


def test_runtime_device_is_callers(gpu):
    """The library's runtime sits on the caller's current device."""
    import torch
    assert gpu.L.mc_b200_device() == torch.cuda.current_device()


def test_corrupt_streams_golden(gpu, golden_corrupt):
    g = golden_corrupt
    for i in range(len(g["q"])):
        p = g["payload"][g["offs"][i]:g["offs"][i + 1]].tobytes()
        assert sha(gpu.dec_block(p, float(g["q"][i]))) == g["decoded_sha"][i], f"stream {i}"
    assert gpu.L.mc_b200_last_bad_blocks() == 0


def _blob_of(payloads, q):
    """A chunk blob whose blocks 0..n-1 carry the given payloads (no fracmap,
    hash 0: the decode reads neither)."""
    bm = np.zeros(512, np.uint8)
    for i in range(len(payloads)):
        bm[i >> 3] |= 1 << (i & 7)
    lens = np.asarray([len(p) for p in payloads], np.uint16)
    head = np.float32(q).tobytes() + bytes(8) + np.uint16(0).tobytes()
    return np.frombuffer(head + bm.tobytes() + lens.tobytes() + b"".join(payloads), np.uint8)


def test_corrupt_streams_every_entropy_kernel(gpu, golden_corrupt):
    """The corrupt-stream corpus decoded as blocks of chunk blobs by each way
    of running the entropy stage: one block per lane of a warp, every block on
    a single thread, and the longest eighth on single threads with the rest on
    lanes. Every block equals the reference's decode of its stream."""
    import ctypes as C
    g = golden_corrupt
    groups = {}
    for i in range(len(g["q"])):
        groups.setdefault(float(g["q"][i]), []).append(i)
    blobs, want = [], []
    for q, idx in sorted(groups.items()):
        blobs.append(_blob_of([g["payload"][g["offs"][i]:g["offs"][i + 1]].tobytes() for i in idx], q))
        want.append([str(g["decoded_sha"][i]) for i in idx])
    ptrs = (C.c_void_p * len(blobs))(*[b.ctypes.data for b in blobs])
    lens = np.asarray([b.size for b in blobs], np.uint64)
    try:
        for share in (0, 1, 8):
            assert gpu.L.mc_b200_set_entropy_solo(share) == 0
            out = np.zeros(len(blobs) * CHUNK, np.uint8)
            assert gpu.L.mc_b200_decode_chunk_blobs(C.cast(ptrs, C.c_void_p), lens.ctypes.data, len(blobs),
                                                    out.ctypes.data, CHUNK) == 0
            for c, shas in enumerate(want):
                vol = out[c * CHUNK:(c + 1) * CHUNK].reshape(256, 256, 256)
                for bi, h in enumerate(shas):
                    bz, by, bx = bi >> 8, (bi >> 4) & 15, bi & 15
                    blk = np.ascontiguousarray(vol[bz * 16:bz * 16 + 16, by * 16:by * 16 + 16, bx * 16:bx * 16 + 16])
                    assert sha(blk) == h, (share, c, bi)
    finally:
        gpu.L.mc_b200_set_entropy_solo(-1)


def test_chunk_blobs_decode_golden(gpu, golden_chunks):
    from mcb200 import decode_chunk_blobs
    g = golden_chunks
    blobs = [g["blobs"][g["offs"][i]:g["offs"][i + 1]] for i in range(len(g["offs"]) - 1)]
    out = decode_chunk_blobs(gpu, [b if b.size else None for b in blobs] if False else blobs)
    for i in range(len(blobs)):
        assert sha(out[i * CHUNK:(i + 1) * CHUNK]) == g["decoded_sha"][i], g["names"][i]


def test_chunk_blobs_pipeline(gpu, golden_chunks):
    """More blobs than the pipeline has slots (18 groups of up to 2 over 8
    slots, so slots are reused), a missing blob, and a padded output stride:
    every chunk still matches."""
    import ctypes as C
    g = golden_chunks
    blobs = [g["blobs"][g["offs"][i]:g["offs"][i + 1]] for i in range(len(g["offs"]) - 1)]
    want = [str(s) for s in g["decoded_sha"]]
    seq = [(i * 5) % len(blobs) for i in range(35)]
    arrs = [blobs[i] for i in seq]
    ptrs = (C.c_void_p * len(arrs))(*[(a.ctypes.data if a.size else None) for a in arrs])
    lens = np.asarray([a.size for a in arrs], np.uint64)
    stride = CHUNK + 4096
    out = np.full(len(arrs) * stride, 0x5A, np.uint8)
    rc = gpu.L.mc_b200_decode_chunk_blobs(C.cast(ptrs, C.c_void_p), lens.ctypes.data, len(arrs), out.ctypes.data,
                                          stride)
    assert rc == 0
    for j, i in enumerate(seq):
        assert sha(out[j * stride:j * stride + CHUNK]) == want[i], (j, g["names"][i])
        assert np.all(out[j * stride + CHUNK:(j + 1) * stride] == 0x5A)
    assert gpu.L.mc_b200_last_bad_blocks() == 0


def _append_sequence(lib, path):
    offs = []
    with lib.open(path, 1024, 1024, 1024, 6.0) as a:
        for st in shapes.archive_sequence():
            vox = shapes.chunk_source(st["src"])
            if st["op"] == "par":
                assert a.append_par(0, *st["at"], vox, st["q"]) == 0
            else:
                assert a.append_ctx(0, *st["at"], vox, 8.0, preset=st["preset"]) == 0
            offs.append(a.chunk_offset(0, *st["at"]))
        lib.L.mc_archive_set_metadata(a.a, b"golden", 6)
    return open(path, "rb").read(), offs


def test_archive_byte_identical(gpu, golden_chunks, tmp_path):
    data, offs = _append_sequence(gpu, str(tmp_path / "g.mca"))
    g = golden_chunks
    assert len(data) == int(g["archive_len"])
    assert hashlib.sha256(data).hexdigest() == str(g["archive_sha"])


def test_host_output_calls_from_threads(gpu, golden_chunks, tmp_path):
    """Four host threads decode the archive's chunks into their own pageable
    buffers at the same time, three rounds each: every thread has its own
    stream and pinned bounce buffers, and all of them share one pool of host
    copy threads. Every chunk matches its golden digest."""
    import threading
    g = golden_chunks
    path = str(tmp_path / "t.mca")
    _, offs = _append_sequence(gpu, path)
    errors = []
    with gpu.open(path, 1024, 1024, 1024, 6.0) as a:
        a.decode_chunk(offs[0])   # the archive's device mirror, before the threads start

        def worker(t):
            try:
                out = np.empty(CHUNK, np.uint8)
                for r in range(3):
                    for j in range(len(offs)):
                        i = (j + t + r) % len(offs)
                        out.fill(0xEE)
                        gpu.L.mc_archive_decode_chunk(a.a, offs[i], out.ctypes.data, 0)
                        if sha(out) != g["decoded_sha"][i]:
                            errors.append((t, r, g["names"][i]))
            except Exception as e:   # surfaced below
                errors.append((t, repr(e)))

        threads = [threading.Thread(target=worker, args=(t,)) for t in range(4)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
    assert not errors, errors[:5]


def test_archive_decode_paths(gpu, golden_chunks, tmp_path):
    """decode_chunk, per-block decode_block, read_region(s) on a GPU-built archive."""
    g = golden_chunks
    path = str(tmp_path / "d.mca")
    _, offs = _append_sequence(gpu, path)
    with gpu.open(path, 1024, 1024, 1024, 6.0) as a:
        for i, co in enumerate(offs):
            assert sha(a.decode_chunk(co)) == g["decoded_sha"][i], g["names"][i]
        co = offs[0]
        whole = a.decode_chunk(co).reshape(256, 256, 256)
        for bz, by, bx in [(0, 0, 0), (8, 8, 8), (15, 15, 15), (3, 12, 7), (12, 3, 9)]:
            blk = a.decode_block(co, bz, by, bx).reshape(16, 16, 16)
            assert np.array_equal(blk, whole[bz * 16:bz * 16 + 16, by * 16:by * 16 + 16, bx * 16:bx * 16 + 16])
        # region == crop of the decoded chunk (reference v6 test, section 5)
        reg = a.read_region(0, 10, 20, 30, 64, 64, 64).reshape(64, 64, 64)
        assert np.array_equal(reg, whole[10:74, 20:84, 30:94])
        # strided region output leaves the gaps untouched
        out = np.full(70 * 80 * 40, 0xAB, np.uint8)
        a.read_region(0, 100, 5, 250, 40, 30, 20, out=out, sz=80 * 70, sy=70)
        o = out.reshape(40, 80, 70)
        w1 = a.decode_chunk(a.chunk_offset(0, 0, 0, 1)).reshape(256, 256, 256)
        want = np.concatenate([whole[100:140, 5:35, 250:256], w1[100:140, 5:35, 0:14]], axis=2)
        assert np.array_equal(o[:, :30, :20], want)
        assert np.all(o[:, 30:, :] == 0xAB) and np.all(o[:, :30, 20:] == 0xAB)
        # batch == per-region, boxes crossing into absent chunks and past the volume
        boxes = [(0, 0, 0), (10, 20, 30), (60, 100, 3), (64, 64, 300), (-8, 250, 1000)]
        batch = a.read_regions(0, boxes, 64, 64, 64).reshape(len(boxes), 64, 64, 64)
        for i, (z0, y0, x0) in enumerate(boxes):
            single = a.read_region(0, z0, y0, x0, 64, 64, 64).reshape(64, 64, 64)
            assert np.array_equal(batch[i], single), boxes[i]
        # absent chunk and the air sentinel decode to zeros
        assert not a.decode_chunk(0).any()
        assert not a.decode_chunk(1).any()


def test_against_reference_build(gpu, ref, golden_chunks, tmp_path):
    """Same calls on the reference build and the GPU library: same blocks."""
    path = str(tmp_path / "r.mca")
    _append_sequence(ref, path)
    with ref.open(path, 1024, 1024, 1024, 6.0) as ra:
        co = ra.chunk_offset(0, 0, 0, 1)
        want = ra.decode_chunk(co)
        wreg = ra.read_regions(0, [(5, 200, 200), (130, 7, 255)], 48, 48, 48)
    with gpu.open(path, 1024, 1024, 1024, 6.0) as ga:   # the GPU library reads the reference's file
        assert np.array_equal(ga.decode_chunk(co), want)
        assert np.array_equal(ga.read_regions(0, [(5, 200, 200), (130, 7, 255)], 48, 48, 48), wreg)


def test_synthetic_chunk_q6(gpu, oracle, tmp_path):
    """One 256^3 chunk of the benchmark generator at q=6 (40% air): GPU
    append_par blob == oracle blob; every block decoded per call == oracle."""
    import torch
    import volumes
    vox = volumes.chunk(0, 0.4, device="cuda").cpu().numpy().reshape(-1)
    want_blob = oracle.encode_chunk(vox, 6.0, 0)
    with gpu.open(str(tmp_path / "s.mca"), 256, 256, 256, 6.0) as a:
        assert a.append_par(0, 0, 0, 0, vox, 6.0) == 0
        co = a.chunk_offset(0, 0, 0, 0)
        got_blob = bytes(np.fromfile(str(tmp_path / "s.mca"), np.uint8)[co:co + len(want_blob)])
        assert got_blob == want_blob
        want = oracle.decode_chunk(want_blob).reshape(256, 256, 256)
        got = a.decode_chunk(co).reshape(256, 256, 256)
        assert np.array_equal(got, want)
        for bi in range(0, 4096, 97):
            bz, by, bx = bi >> 8, (bi >> 4) & 15, bi & 15
            blk = a.decode_block(co, bz, by, bx).reshape(16, 16, 16)
            assert np.array_equal(blk, want[bz * 16:bz * 16 + 16, by * 16:by * 16 + 16, bx * 16:bx * 16 + 16])
        # device-output paths: decode_chunks_dev and a graph-captured plan
        d_out = torch.empty(2 * CHUNK, dtype=torch.uint8, device="cuda")
        assert a.decode_chunks_dev([co, 0], d_out.data_ptr()) == 0
        assert np.array_equal(d_out[:CHUNK].cpu().numpy(), want.reshape(-1))
        assert not d_out[CHUNK:].any().item()
        d2 = torch.zeros(CHUNK, dtype=torch.uint8, device="cuda")
        plan = a.plan_chunks([co], d2.data_ptr())
        plan.launch()
        torch.cuda.synchronize()
        assert np.array_equal(d2.cpu().numpy(), want.reshape(-1))
        launches, blocks, pbytes = plan.info()
        assert blocks == 4096 and launches >= 2
        plan.free()


def test_plan_stage_layouts(gpu, oracle, tmp_path):
    """Every stage layout of a decode plan -- two kernels in sequence, the long
    blocks on a second stream, one fused persistent kernel -- gives the
    oracle's voxels, on a batch with absent and all-air chunks, an odd number
    of blocks per sub-batch pair boundary and chunks of two qualities."""
    import torch
    import volumes
    with gpu.open(str(tmp_path / "f.mca"), 1024, 512, 256, 6.0) as a:
        coords = [(0, 0, 0), (0, 0, 1), (0, 1, 2), (0, 1, 3)]
        vox = [volumes.region(21 + i, (0, 256 * (c[1]), 256 * c[2]), (256, 256, 256), 0.4, device="cuda")
               for i, c in enumerate(coords)]
        vox[2].zero_()   # an all-air chunk
        for c, v, q in zip(coords, vox, (6.0, 6.0, 6.0, 3.0)):
            assert a.append_par(0, *c, v.cpu().numpy(), q) == 0
        offs = [a.chunk_offset(0, *c) for c in coords] + [a.chunk_offset(0, 0, 0, 3)]   # the last one absent
        data = np.fromfile(str(tmp_path / "f.mca"), np.uint8).tobytes()
        want = np.concatenate([oracle.decode_chunk(data[o:o + shapes.blob_len(data, o)]) if o > 1
                               else np.zeros(CHUNK, np.uint8) for o in offs])
        d_out = torch.empty(len(offs) * CHUNK, dtype=torch.uint8, device="cuda")
        plan = a.plan_chunks(offs, d_out.data_ptr())
        try:
            for stages in plan.STAGES:
                for ent, rec in ((5, 4), (3, 2)):
                    assert plan.set_config(ent, rec, stages) == 0
                    assert plan.config()["stages"] == stages
                    d_out.fill_(0xEE)
                    for _ in range(2):   # the work area is reset by every replay
                        plan.launch()
                    torch.cuda.synchronize()
                    assert np.array_equal(d_out.cpu().numpy(), want), (stages, ent, rec)
        finally:
            plan.free()


def test_mixed_quality_batch(gpu, oracle, tmp_path):
    """Chunks of different q in one batched append and one batched decode."""
    import torch
    import volumes
    qs = [1.0, 3.0, 6.0, 12.0]
    vox = [volumes.region(7 + i, (0, 0, 256 * i), (256, 256, 256), 0.3, device="cuda").cpu().numpy() for i in range(4)]
    with gpu.open(str(tmp_path / "m.mca"), 1024, 256, 256, 6.0) as a:
        for i, q in enumerate(qs):
            assert a.append_par(0, 0, 0, i, vox[i], q) == 0
        offs = [a.chunk_offset(0, 0, 0, i) for i in range(4)]
        d_out = torch.empty(4 * CHUNK, dtype=torch.uint8, device="cuda")
        assert a.decode_chunks_dev(offs, d_out.data_ptr()) == 0
        got = d_out.cpu().numpy()
        data = np.fromfile(str(tmp_path / "m.mca"), np.uint8).tobytes()
    for i, q in enumerate(qs):
        blob = data[offs[i]:offs[i] + shapes.blob_len(data, offs[i])]
        assert blob == oracle.encode_chunk(vox[i], q, 0), q
        assert np.array_equal(got[i * CHUNK:(i + 1) * CHUNK], oracle.decode_chunk(blob)), q


def test_preset_ladder_tau_bound(gpu, tmp_path):
    """Preset ladder through append_chunk_ctx: |err| <= tau on every voxel."""
    import volumes
    vox = volumes.region(3, (0, 0, 0), (256, 256, 256), 0.3, device="cuda").cpu().numpy()
    with gpu.open(str(tmp_path / "t.mca"), 256, 256, 256 * 8, 6.0) as a:
        for lvl, (q, tau) in enumerate(PRESETS):
            assert a.append_ctx(0, lvl, 0, 0, vox, 8.0, preset=lvl) == 0
            dec = a.decode_chunk(a.chunk_offset(0, lvl, 0, 0)).reshape(vox.shape)
            err = np.abs(dec.astype(int) - vox.astype(int))
            assert err.max() <= tau, (lvl, err.max())


def test_fused_layout_gives_up_waiting(gpu, oracle, tmp_path):
    """The fused layout's bounded wait: with a wait limit of zero polls every
    CTA that meets an unfilled completion-list position hands it to
    k_fused_tail at once and leaves, so the tail kernel reconstructs most
    pairs; the voxels are still the oracle's. Nothing here waits forever or
    faults: the wait simply ends."""
    import torch
    import volumes
    with gpu.open(str(tmp_path / "w.mca"), 512, 256, 256, 6.0) as a:
        for c in range(2):
            v = volumes.region(41 + c, (0, 0, 256 * c), (256, 256, 256), 0.45, device="cuda").cpu().numpy()
            assert a.append_par(0, 0, 0, c, v, 6.0) == 0
        offs = [a.chunk_offset(0, 0, 0, c) for c in range(2)]
        data = np.fromfile(str(tmp_path / "w.mca"), np.uint8).tobytes()
        want = np.concatenate([oracle.decode_chunk(data[o:o + shapes.blob_len(data, o)]) for o in offs])
        d_out = torch.empty(2 * CHUNK, dtype=torch.uint8, device="cuda")
        plan = a.plan_chunks(offs, d_out.data_ptr())
        try:
            if plan.set_config(5, 5, "fused") != 0:
                pytest.skip("the fused kernel cannot launch on this device")
            for polls in (0, 1, 1 << 15):
                assert plan.set_fused_wait(polls) == 0
                d_out.fill_(0xEE)
                for _ in range(2):
                    plan.launch()
                torch.cuda.synchronize()
                assert np.array_equal(d_out.cpu().numpy(), want), polls
        finally:
            plan.free()


def test_plan_entropy_shapes(gpu, oracle, tmp_path):
    """Every entropy launch shape the autotuner may pick -- 2, 4 or 8 warps per
    CTA, several CTAs per SM, queue claims of 1, 2 or 4 entries, the longest
    blocks on single-thread warps or not -- gives the oracle's voxels, at three
    qualities in one batch."""
    import torch
    import volumes
    with gpu.open(str(tmp_path / "e.mca"), 768, 256, 256, 6.0) as a:
        for c, q in enumerate((6.0, 1.0, 12.0)):
            v = volumes.region(61 + c, (0, 0, 256 * c), (256, 256, 256), 0.35, device="cuda").cpu().numpy()
            assert a.append_par(0, 0, 0, c, v, q) == 0
        offs = [a.chunk_offset(0, 0, 0, c) for c in range(3)]
        data = np.fromfile(str(tmp_path / "e.mca"), np.uint8).tobytes()
        want = np.concatenate([oracle.decode_chunk(data[o:o + shapes.blob_len(data, o)]) for o in offs])
        d_out = torch.empty(3 * CHUNK, dtype=torch.uint8, device="cuda")
        plan = a.plan_chunks(offs, d_out.data_ptr())
        try:
            t = plan.tuning()
            assert t["entropy_warps_per_cta"] in (2, 4, 8) and t["entropy_claim"] in (1, 2, 4)
            # solo share: 1/16 of the blocks on single-thread warps; 2 asks for
            # more than half of the warps and is clamped to that; 1 is the
            # single-thread kernel
            for warps, ctas, claim, solo, stages in (
                    (2, 12, 1, 0, "sequential"), (4, 5, 2, 16, "sequential"), (8, 3, 4, 0, "sequential"),
                    (4, 1, 1, 2, "sequential"), (2, 3, 64, 1, "sequential"), (4, 5, 1, 64, "sequential"),
                    (4, 5, 1, 1, "long_blocks_on_second_stream"), (4, 5, 1, 8, "fused"), (4, 5, 1, 1, "fused")):
                assert plan.set_tuning(warps, ctas, claim, 4, stages, solo) == 0
                assert plan.tuning()["entropy_warps_per_cta"] == warps
                assert plan.tuning()["entropy_solo_share"] == solo
                d_out.fill_(0xEE)
                plan.launch()
                torch.cuda.synchronize()
                assert np.array_equal(d_out.cpu().numpy(), want), (warps, ctas, claim, solo, stages)
            with pytest.raises(RuntimeError, match="bad arguments"):   # 3 warps per CTA: refused
                plan.set_tuning(3, 4, 1, 4, "sequential")
        finally:
            plan.free()


def test_host_region_batch_through_bounce_buffers(gpu, tmp_path):
    """A host-output region batch larger than one pinned bounce piece (crops
    of 3.1 MB, a stride with a gap, about 22 MB in all, so crops straddle the
    8 MiB pieces) equals the device-output batch crop for crop, twice in a
    row, and leaves the gaps between crops as they were."""
    import ctypes as C
    import torch
    from mcb200 import McBox
    with gpu.open(str(tmp_path / "hb.mca"), 1024, 1024, 1024, 6.0) as a:
        for st in shapes.archive_sequence()[:2]:
            assert a.append_par(0, *st["at"], shapes.chunk_source(st["src"]), st["q"]) == 0
        boxes = [(0, 0, 0), (10, 20, 30), (60, 100, 200), (64, 64, 300), (-8, 250, 1000), (200, 200, 450),
                 (100, 0, 0)]
        dz, dy, dx = 96, 160, 200
        crop = dz * dy * dx
        stride = crop + 4099
        want = torch.zeros(stride * len(boxes), dtype=torch.uint8, device="cuda")
        assert a.read_regions_dev(0, boxes, dz, dy, dx, want.data_ptr(), stride) == 0
        w = want.cpu().numpy()
        arr = (McBox * len(boxes))(*[McBox(*b) for b in boxes])
        host = np.full(stride * (len(boxes) - 1) + crop, 0xA5, np.uint8)
        for _ in range(2):
            a.L.mc_archive_read_regions(a.a, 0, C.cast(arr, C.c_void_p), len(boxes), dz, dy, dx,
                                        host.ctypes.data, stride, 0)
            for i in range(len(boxes)):
                assert np.array_equal(host[i * stride:i * stride + crop], w[i * stride:i * stride + crop]), boxes[i]
                if i + 1 < len(boxes):
                    assert np.all(host[i * stride + crop:(i + 1) * stride] == 0xA5)


def test_region_plan(gpu, tmp_path):
    """A graph-captured plan of a region batch (boxes across chunk borders,
    into absent chunks and past the volume, strided output) gives what
    mc_b200_read_regions_dev and the host read_regions give, replay after
    replay, and leaves the gaps between crops untouched."""
    import torch
    with gpu.open(str(tmp_path / "rp.mca"), 1024, 1024, 1024, 6.0) as a:
        for st in shapes.archive_sequence()[:2]:
            assert a.append_par(0, *st["at"], shapes.chunk_source(st["src"]), st["q"]) == 0
        boxes = [(0, 0, 0), (10, 20, 30), (60, 100, 200), (64, 64, 300), (-8, 250, 1000), (200, 200, 450)]
        dz, dy, dx = 48, 64, 80
        crop = dz * dy * dx
        stride = crop + 1000
        want = torch.full((stride * len(boxes),), 0x5A, dtype=torch.uint8, device="cuda")
        assert a.read_regions_dev(0, boxes, dz, dy, dx, want.data_ptr(), stride) == 0
        got = torch.full_like(want, 0x5A)
        plan = a.plan_regions(0, boxes, dz, dy, dx, got.data_ptr(), stride)
        try:
            for _ in range(3):
                plan.launch()
            torch.cuda.synchronize()
        finally:
            plan.free()
        assert torch.equal(got, want)
        g = got.cpu().numpy()
        for i in range(len(boxes)):
            assert np.all(g[i * stride + crop:(i + 1) * stride] == 0x5A)
        host = a.read_regions(0, boxes, dz, dy, dx, batch_stride=stride)
        for i in range(len(boxes)):
            assert np.array_equal(g[i * stride:i * stride + crop], host[i * stride:i * stride + crop]), boxes[i]
