"""ctypes binding of the matter-compressor C ABI.

The same class binds the B200 library (libmc_b200.so beside this file) and,
for the drop-in part of the ABI, any library exporting the reference's
symbols, so one call sequence can be replayed against both. Pass
``b200=False`` for a library without the mc_b200_* additions.

The B200 library has no CPU path: `McLib.product()` raises when the library
is missing or when no sm_100 device is usable.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmc_b200.so")
CHUNK = 256 * 256 * 256


class McBuf(C.Structure):
    _fields_ = [("p", C.c_void_p), ("len", C.c_size_t), ("cap", C.c_size_t)]


class McBox(C.Structure):
    _fields_ = [("z0", C.c_long), ("y0", C.c_long), ("x0", C.c_long)]


_libc = C.CDLL(None)
_libc.free.argtypes = [C.c_void_p]


class McRequest(C.Structure):
    """mc_b200_request (include/matter_compressor_b200.h)."""
    _fields_ = [("kind", C.c_int), ("lod", C.c_int), ("z", C.c_long), ("y", C.c_long), ("x", C.c_long),
                ("dz", C.c_long), ("dy", C.c_long), ("dx", C.c_long), ("out", C.c_void_p),
                ("sz", C.c_size_t), ("sy", C.c_size_t)]


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


class McLib:
    """Binding of one library; methods mirror the C entry points."""

    def __init__(self, path, b200=True):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (run __graft_entry__.build())")
        self.path = path
        self.L = L = C.CDLL(path)
        self.b200 = b200
        vp, u8p, i, f, u32, u64, sz, lg = (C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_uint32,
                                            C.c_uint64, C.c_size_t, C.c_long)
        sig = {
            "mc_codec_init": (None, []),
            "mc_codec_ctx_new": (vp, []),
            "mc_codec_ctx_free": (None, [vp]),
            "mc_codec_ctx_set_quality": (None, [vp, f]),
            "mc_codec_ctx_get_quality": (f, [vp]),
            "mc_codec_ctx_set_max_error": (None, [vp, i]),
            "mc_codec_ctx_get_max_error": (i, [vp]),
            "mc_apply_preset": (f, [vp, i]),
            "mc_preset_quality": (f, [i]),
            "mc_preset_tau": (i, [i]),
            "mc_preset_name": (C.c_char_p, [i]),
            "mc_codec_set_priors": (None, [vp, vp]),
            "mc_enc_block": (i, [vp, u8p, C.POINTER(McBuf), C.POINTER(u32)]),
            "mc_dec_block": (None, [vp, u8p, u32, u8p]),
            "mc_enc_fracmap": (u32, [u8p, u8p, sz]),
            "mc_dec_fracmap": (None, [u8p, u32, u8p]),
            "mc_xxh64": (u64, [vp, sz, u64]),
            "mc_archive_open": (vp, [C.c_char_p, i, f]),
            "mc_archive_open_dims": (vp, [C.c_char_p, i, i, i, f]),
            "mc_archive_close": (None, [vp]),
            "mc_archive_chunk_offset": (u64, [vp, i, i, i, i]),
            "mc_archive_chunk_coverage": (i, [vp, i, i, i, i]),
            "mc_archive_data_len": (u64, [vp]),
            "mc_archive_set_metadata": (i, [vp, vp, sz]),
            "mc_archive_decode_block": (None, [vp, u64, i, i, i, u8p]),
            "mc_archive_decode_chunk": (None, [vp, u64, u8p, i]),
            "mc_archive_read_region": (None, [vp, i, lg, lg, lg, lg, lg, lg, u8p, sz, sz, i]),
            "mc_archive_read_regions": (None, [vp, i, vp, i, lg, lg, lg, u8p, sz, i]),
            "mc_archive_append_chunk_par": (i, [vp, i, i, i, i, u8p, f, i]),
            "mc_archive_append_chunk_ctx": (i, [vp, vp, i, i, i, i, u8p]),
            "mc_archive_append_chunk_raw": (i, [vp, i, i, i, i, u8p]),
            "mc_archive_append_chunk_raw_q": (i, [vp, i, i, i, i, u8p, f]),
            "mc_archive_append_chunk_compressed": (i, [vp, i, i, i, i, u8p, sz]),
            "mc_archive_reserve_index": (i, [vp, i, i, i, i]),
            "mc_archive_block_present": (i, [vp, i, i, i, i]),
            "mc_archive_block_fraction": (f, [vp, i, i, i, i]),
            "mc_archive_sample_boxes": (i, [vp, i, u64, i, lg, lg, lg, f, vp]),
            "mc_archive_set_priors": (i, [vp, vp, vp]),
            "mc_archive_block_blob": (i, [vp, u64, i, i, i, C.POINTER(C.c_void_p), C.POINTER(u32)]),
            "mc_chunk_compute_hash": (u64, [u8p, u64]),
            "mc_verify_archive": (lg, [u8p, sz, i]),
        }
        if b200:
            sig.update({
                "mc_b200_init": (i, []),
                "mc_b200_device": (i, []),
                "mc_b200_last_error": (C.c_char_p, []),
                "mc_b200_clear_error": (None, []),
                "mc_b200_last_bad_blocks": (u32, []),
                "mc_b200_set_entropy_solo": (i, [i]),
                "mc_b200_decode_chunk_blobs": (i, [vp, vp, i, u8p, sz]),
                "mc_b200_archive_sync": (i, [vp, C.POINTER(C.c_void_p), C.POINTER(u64)]),
                "mc_b200_decode_chunks_dev": (i, [vp, vp, i, vp, sz, vp]),
                "mc_b200_read_regions_dev": (i, [vp, i, vp, i, lg, lg, lg, vp, sz, vp]),
                "mc_b200_plan_decode_chunks": (vp, [vp, vp, i, vp, sz]),
                "mc_b200_plan_launch": (i, [vp, vp]),
                "mc_b200_plan_launch_stage": (i, [vp, i, vp]),
                "mc_b200_plan_info": (None, [vp, C.POINTER(i), C.POINTER(lg), C.POINTER(u64)]),
                "mc_b200_plan_free": (None, [vp]),
                "mc_b200_plan_config": (None, [vp, vp]),
                "mc_b200_plan_set_config": (i, [vp, vp]),
                "mc_b200_plan_set_fused_wait": (i, [vp, u32]),
                "mc_b200_plan_tuning": (None, [vp, vp]),
                "mc_b200_plan_set_tuning": (i, [vp, vp]),
                "mc_b200_plan_read_regions": (vp, [vp, i, vp, i, lg, lg, lg, vp, sz]),
                "mc_b200_deblock_dev": (i, [vp, i, sz, i, i, i, f, vp]),
                "mc_b200_decimate_dev": (i, [vp, i, i, i, vp, vp]),
                "mc_b200_verify_archive_dev": (lg, [vp, vp, sz, i]),
                "mc_b200_sample_boxes": (i, [vp, i, u64, i, lg, lg, lg, f, vp]),
                "mc_open": (vp, [vp, sz]),
                "mc_open_streaming": (vp, [vp, vp, u64]),
                "mc_close": (None, [vp]),
                "mc_reader_set_quality": (None, [vp, f]),
                "mc_reader_set_partial_fetch": (None, [vp, i]),
                "mc_chunk_offset": (u64, [vp, i, i, i, i]),
                "mc_chunk_offset_chk": (u64, [vp, i, i, i, i, C.POINTER(i)]),
                "mc_decode_block": (None, [vp, u64, i, i, i, vp]),
                "mc_reader_chunk_blob_len": (u64, [vp, u64]),
                "mc_reader_read_blob": (i, [vp, u64, sz, vp]),
                "mc_reader_dims": (None, [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i)]),
                "mc_reader_quality": (f, [vp]),
                "mc_reader_nlods": (i, [vp]),
                "mc_b200_reader_decode_blocks": (i, [vp, u64, vp, i, vp, vp]),
                "mc_b200_append_pyramid": (i, [vp, vp, i, i, i, f, C.POINTER(i)]),
                "mc_deblock": (None, [vp, i, i, i, f]),
                "mc_b200_append_chunks": (i, [vp, vp, i, vp, i, vp, i, f]),
                "mc_b200_decode_blocks_noalloc": (i, [vp, vp, i, f, vp, vp]),
                "mc_b200_server_open": (vp, [vp, sz, sz, i]),
                "mc_b200_server_submit": (lg, [vp, C.POINTER(McRequest)]),
                "mc_b200_server_poll": (i, [vp, lg]),
                "mc_b200_server_wait": (i, [vp, lg]),
                "mc_b200_server_ticket_times": (i, [vp, lg, C.POINTER(u64), C.POINTER(u64)]),
                "mc_b200_server_replay": (i, [vp, C.POINTER(McRequest), vp, i, vp]),
                "mc_b200_server_stats": (None, [vp, vp]),
                "mc_b200_server_close": (None, [vp]),
            })
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args

    # ------------------------------------------------------------ construction
    @classmethod
    def product(cls):
        """The B200 library, checked to have a usable device."""
        lib = cls(LIB_PATH, b200=True)
        if lib.L.mc_b200_init() != 0:
            raise RuntimeError("matter-compressor-b200: " + (lib.last_error() or "no usable GPU"))
        return lib

    def last_error(self):
        e = self.L.mc_b200_last_error() if self.b200 else None
        return e.decode() if e else None

    def check(self):
        if self.b200:
            e = self.last_error()
            if e:
                self.L.mc_b200_clear_error()
                raise RuntimeError("matter-compressor-b200: " + e)

    # ------------------------------------------------------------ codec
    def ctx(self, q=8.0, tau=0):
        c = self.L.mc_codec_ctx_new()
        self.L.mc_codec_ctx_set_quality(c, q)
        self.L.mc_codec_ctx_set_max_error(c, tau)
        return c

    def enc_block(self, vox, q, tau=0):
        vox = np.ascontiguousarray(vox, dtype=np.uint8).reshape(-1)
        c = self.ctx(q, tau)
        buf = McBuf()
        n = C.c_uint32(0)
        coded = self.L.mc_enc_block(c, _ptr(vox), C.byref(buf), C.byref(n))
        out = C.string_at(buf.p, n.value) if coded else b""
        if buf.p:
            _libc.free(buf.p)
        self.L.mc_codec_ctx_free(c)
        self.check()
        return out

    def dec_block(self, payload, q):
        c = self.ctx(q)
        dst = np.zeros(4096, np.uint8)
        src = np.frombuffer(payload, np.uint8) if payload else np.zeros(1, np.uint8)
        src = np.ascontiguousarray(src)
        self.L.mc_dec_block(c, _ptr(src), len(payload), _ptr(dst))
        self.L.mc_codec_ctx_free(c)
        self.check()
        return dst

    def deblock(self, vol, quality):
        """mc_deblock in place on a dense (nz, ny, nx) u8 host volume; returns it."""
        v = np.ascontiguousarray(vol, np.uint8)
        nz, ny, nx = v.shape
        self.L.mc_deblock(_ptr(v), nz, ny, nx, quality)
        self.check()
        return v

    def deblock_dev(self, d_vol, count, vol_stride, nz, ny, nx, quality, stream=None):
        """Deblock `count` dense device volumes in place (mc_b200_deblock_dev)."""
        rc = self.L.mc_b200_deblock_dev(C.c_void_p(d_vol), count, vol_stride, nz, ny, nx, quality,
                                        C.c_void_p(stream) if stream else None)
        self.check()
        return rc

    def decimate_dev(self, d_src, nz, ny, nx, d_dst, stream=None):
        """2x LOD decimation of a dense device volume (mc_b200_decimate_dev)."""
        rc = self.L.mc_b200_decimate_dev(C.c_void_p(d_src), nz, ny, nx, C.c_void_p(d_dst),
                                         C.c_void_p(stream) if stream else None)
        self.check()
        return rc

    def set_priors(self, plo, phi):
        if plo is None:
            self.L.mc_codec_set_priors(None, None)
        else:
            plo = np.ascontiguousarray(plo, np.uint16)
            phi = np.ascontiguousarray(phi, np.uint16)
            self.L.mc_codec_set_priors(_ptr(plo), _ptr(phi))

    # ------------------------------------------------------------ archive
    def open(self, path, nx, ny=None, nz=None, q=6.0):
        a = self.L.mc_archive_open_dims(str(path).encode(), nx, ny or nx, nz or nx, q)
        if not a:
            raise RuntimeError(f"mc_archive_open_dims({path}) failed")
        return Archive(self, a)


class Archive:
    """One open archive handle of a bound library."""

    def __init__(self, lib, handle):
        self.lib, self.a, self.L = lib, handle, lib.L

    def close(self):
        if self.a:
            self.L.mc_archive_close(self.a)
            self.a = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def chunk_offset(self, lod, cz, cy, cx):
        return self.L.mc_archive_chunk_offset(self.a, lod, cz, cy, cx)

    def append_par(self, lod, cz, cy, cx, vox, q, nthreads=0):
        vox = np.ascontiguousarray(vox, np.uint8)
        assert vox.size == CHUNK
        rc = self.L.mc_archive_append_chunk_par(self.a, lod, cz, cy, cx, _ptr(vox), q, nthreads)
        self.lib.check()
        return rc

    def append_ctx(self, lod, cz, cy, cx, vox, q, tau=0, preset=None):
        vox = np.ascontiguousarray(vox, np.uint8)
        c = self.lib.ctx(q, tau)
        if preset is not None:
            self.L.mc_apply_preset(c, preset)
        rc = self.L.mc_archive_append_chunk_ctx(self.a, c, lod, cz, cy, cx, _ptr(vox))
        self.L.mc_codec_ctx_free(c)
        self.lib.check()
        return rc

    def decode_block(self, co, bz, by, bx):
        dst = np.zeros(4096, np.uint8)
        self.L.mc_archive_decode_block(self.a, co, bz, by, bx, _ptr(dst))
        self.lib.check()
        return dst

    def decode_chunk(self, co, out=None, nthreads=0):
        if out is None:
            out = np.empty(CHUNK, np.uint8)
        self.L.mc_archive_decode_chunk(self.a, co, _ptr(out), nthreads)
        self.lib.check()
        return out

    def read_region(self, lod, z0, y0, x0, dz, dy, dx, out=None, sz=None, sy=None, nthreads=0):
        sy = dx if sy is None else sy
        sz = dy * sy if sz is None else sz
        if out is None:
            out = np.zeros(sz * dz, np.uint8)
        self.L.mc_archive_read_region(self.a, lod, z0, y0, x0, dz, dy, dx, _ptr(out), sz, sy, nthreads)
        self.lib.check()
        return out

    def read_regions(self, lod, boxes, dz, dy, dx, batch_stride=None, nthreads=0):
        n = len(boxes)
        arr = (McBox * n)(*[McBox(*b) for b in boxes])
        crop = dz * dy * dx
        stride = crop if batch_stride is None else batch_stride
        out = np.zeros(stride * (n - 1) + crop, np.uint8)
        self.L.mc_archive_read_regions(self.a, lod, C.cast(arr, C.c_void_p), n, dz, dy, dx, _ptr(out), stride,
                                       nthreads)
        self.lib.check()
        return out

    def sample_boxes(self, lod, seed, count, dz, dy, dx, min_frac):
        arr = (McBox * count)()
        got = self.L.mc_archive_sample_boxes(self.a, lod, seed, count, dz, dy, dx, min_frac, C.cast(arr, C.c_void_p))
        return [(b.z0, b.y0, b.x0) for b in arr[:got]]

    def sample_boxes_dev(self, lod, seed, count, dz, dy, dx, min_frac):
        """mc_b200_sample_boxes: the same boxes as sample_boxes, scored on the device."""
        arr = (McBox * count)()
        got = self.L.mc_b200_sample_boxes(self.a, lod, seed, count, dz, dy, dx, min_frac, C.cast(arr, C.c_void_p))
        self.lib.check()
        return [(b.z0, b.y0, b.x0) for b in arr[:got]]

    def block_blob(self, co, bz, by, bx):
        p = C.c_void_p()
        n = C.c_uint32()
        if not self.L.mc_archive_block_blob(self.a, co, bz, by, bx, C.byref(p), C.byref(n)):
            return b""
        return C.string_at(p, n.value)

    # ---- B200 additions ----
    def append_chunks(self, lod, coords, vox_list, q, ctx_q=None, ctx_tau=0, on_device=False):
        n = len(coords)
        cc = np.ascontiguousarray(np.asarray(coords, np.int32).reshape(-1))
        if on_device:
            ptrs = (C.c_void_p * n)(*[v for v in vox_list])
        else:
            keep = [np.ascontiguousarray(v, np.uint8) for v in vox_list]
            ptrs = (C.c_void_p * n)(*[k.ctypes.data for k in keep])
        c = self.lib.ctx(ctx_q, ctx_tau) if ctx_q is not None else None
        rc = self.L.mc_b200_append_chunks(self.a, c, lod, _ptr(cc), n, C.cast(ptrs, C.c_void_p), int(on_device), q)
        if c:
            self.L.mc_codec_ctx_free(c)
        self.lib.check()
        return rc

    def append_pyramid(self, d_vol, nz, ny, nx, q):
        """mc_b200_append_pyramid: every LOD of a dense device volume; returns (rc, levels)."""
        n = C.c_int()
        rc = self.L.mc_b200_append_pyramid(self.a, C.c_void_p(d_vol), nz, ny, nx, q, C.byref(n))
        self.lib.check()
        return rc, n.value

    def sync_device(self):
        base = C.c_void_p()
        n = C.c_uint64()
        rc = self.L.mc_b200_archive_sync(self.a, C.byref(base), C.byref(n))
        self.lib.check()
        return rc, base.value, n.value

    def decode_chunks_dev(self, offs, d_out, stride=CHUNK, stream=None):
        o = np.ascontiguousarray(np.asarray(offs, np.uint64))
        rc = self.L.mc_b200_decode_chunks_dev(self.a, _ptr(o), len(o), C.c_void_p(d_out), stride,
                                              C.c_void_p(stream) if stream else None)
        self.lib.check()
        return rc

    def read_regions_dev(self, lod, boxes, dz, dy, dx, d_out, batch_stride=None, stream=None):
        n = len(boxes)
        arr = (McBox * n)(*[McBox(*b) for b in boxes])
        stride = dz * dy * dx if batch_stride is None else batch_stride
        rc = self.L.mc_b200_read_regions_dev(self.a, lod, C.cast(arr, C.c_void_p), n, dz, dy, dx,
                                             C.c_void_p(d_out), stride, C.c_void_p(stream) if stream else None)
        self.lib.check()
        return rc

    def plan_chunks(self, offs, d_out, stride=CHUNK):
        o = np.ascontiguousarray(np.asarray(offs, np.uint64))
        p = self.L.mc_b200_plan_decode_chunks(self.a, _ptr(o), len(o), C.c_void_p(d_out), stride)
        self.lib.check()
        if not p:
            raise RuntimeError("plan build failed")
        return Plan(self.lib, p)

    def plan_regions(self, lod, boxes, dz, dy, dx, d_out, batch_stride=None):
        """A graph-captured decode plan of a read_regions batch into device memory."""
        n = len(boxes)
        arr = (McBox * n)(*[McBox(*b) for b in boxes])
        stride = dz * dy * dx if batch_stride is None else batch_stride
        p = self.L.mc_b200_plan_read_regions(self.a, lod, C.cast(arr, C.c_void_p), n, dz, dy, dx, C.c_void_p(d_out),
                                             stride)
        self.lib.check()
        if not p:
            raise RuntimeError("region plan build failed")
        return Plan(self.lib, p)


class Plan:
    def __init__(self, lib, handle):
        self.lib, self.p = lib, handle

    def launch(self, stream=None):
        rc = self.lib.L.mc_b200_plan_launch(self.p, C.c_void_p(stream) if stream else None)
        self.lib.check()
        return rc

    def launch_stage(self, stage, stream=None):
        rc = self.lib.L.mc_b200_plan_launch_stage(self.p, stage, C.c_void_p(stream) if stream else None)
        self.lib.check()
        return rc

    def info(self):
        n, b, pb = C.c_int(), C.c_long(), C.c_uint64()
        self.lib.L.mc_b200_plan_info(self.p, C.byref(n), C.byref(b), C.byref(pb))
        return n.value, b.value, pb.value

    def config(self):
        out = np.zeros(3, np.int32)
        self.lib.L.mc_b200_plan_config(self.p, _ptr(out))
        return {"entropy_ctas_per_sm": int(out[0]), "reconstruct_ctas_per_sm": int(out[1]),
                "stages": ("sequential", "long_blocks_on_second_stream", "fused")[int(out[2])]}

    STAGES = ("sequential", "long_blocks_on_second_stream", "fused")

    def tuning(self):
        """The autotuner's full choice (mc_b200_plan_tuning)."""
        out = np.zeros(6, np.int32)
        self.lib.L.mc_b200_plan_tuning(self.p, _ptr(out))
        return {"entropy_warps_per_cta": int(out[0]), "entropy_ctas_per_sm": int(out[1]),
                "entropy_claim": int(out[2]), "reconstruct_ctas_per_sm": int(out[3]),
                "stages": self.STAGES[int(out[4])], "entropy_solo_share": int(out[5])}

    def set_tuning(self, warps, ctas_per_sm, claim, reconstruct_ctas_per_sm, stages, solo_share=0):
        """solo_share: the longest coded/solo_share blocks decoded one per warp by one thread (0: none)."""
        cfg = np.array([warps, ctas_per_sm, claim, reconstruct_ctas_per_sm, self.STAGES.index(stages), solo_share],
                       np.int32)
        rc = self.lib.L.mc_b200_plan_set_tuning(self.p, _ptr(cfg))
        self.lib.check()
        return rc

    def set_config(self, entropy_ctas_per_sm, reconstruct_ctas_per_sm, stages):
        """Override the autotuned launch shape and recapture the plan."""
        cfg = np.array([entropy_ctas_per_sm, reconstruct_ctas_per_sm, self.STAGES.index(stages)], np.int32)
        rc = self.lib.L.mc_b200_plan_set_config(self.p, _ptr(cfg))
        self.lib.check()
        return rc

    def set_fused_wait(self, polls):
        """Polls before a fused-layout CTA hands an unfilled list position to the tail kernel."""
        rc = self.lib.L.mc_b200_plan_set_fused_wait(self.p, polls)
        self.lib.check()
        return rc

    def free(self):
        if self.p:
            self.lib.L.mc_b200_plan_free(self.p)
            self.p = None


REQ_BLOCK, REQ_REGION, REQ_CHUNK = 0, 1, 2


class Server:
    """mc_b200_server: continuous batching of block / region / chunk reads
    behind an HBM decoded-block cache."""

    STATS = ("requests", "batches", "blocks", "hits", "misses", "zero_blocks", "evictions", "bytes")

    def __init__(self, archive, cache_bytes, batch_bytes=0, on_device=True):
        self.lib = archive.lib
        self.s = self.lib.L.mc_b200_server_open(archive.a, cache_bytes, batch_bytes, 1 if on_device else 0)
        if not self.s:
            self.lib.check()
            raise RuntimeError("mc_b200_server_open failed")

    @staticmethod
    def request(kind, lod, z, y, x, out, dz=0, dy=0, dx=0, sz=0, sy=0):
        return McRequest(kind, lod, z, y, x, dz, dy, dx, out, sz, sy)

    def submit(self, req):
        return self.lib.L.mc_b200_server_submit(self.s, C.byref(req))

    def wait(self, ticket):
        return self.lib.L.mc_b200_server_wait(self.s, ticket)

    def poll(self, ticket):
        return self.lib.L.mc_b200_server_poll(self.s, ticket)

    def times(self, ticket):
        a, b = C.c_uint64(), C.c_uint64()
        st = self.lib.L.mc_b200_server_ticket_times(self.s, ticket, C.byref(a), C.byref(b))
        return st, a.value, b.value

    def replay(self, reqs, arrival_ns):
        n = len(reqs)
        arr = (McRequest * n)(*reqs)
        t = np.ascontiguousarray(arrival_ns, np.uint64)
        lat = np.zeros(n, np.uint64)
        rc = self.lib.L.mc_b200_server_replay(self.s, arr, _ptr(t), n, _ptr(lat))
        return rc, lat

    def stats(self):
        out = np.zeros(8, np.uint64)
        self.lib.L.mc_b200_server_stats(self.s, _ptr(out))
        return dict(zip(self.STATS, (int(v) for v in out)))

    def close(self):
        if self.s:
            self.lib.L.mc_b200_server_close(self.s)
            self.s = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def decode_chunk_blobs(lib, blobs, out=None):
    """mc_b200_decode_chunk_blobs over a list of bytes/ndarray blobs (host in, host out)."""
    n = len(blobs)
    arrs = [np.frombuffer(b, np.uint8) if isinstance(b, (bytes, bytearray)) else b for b in blobs]
    ptrs = (C.c_void_p * n)(*[a.ctypes.data for a in arrs])
    lens = np.asarray([a.size for a in arrs], np.uint64)
    if out is None:
        out = np.empty(n * CHUNK, np.uint8)
    rc = lib.L.mc_b200_decode_chunk_blobs(C.cast(ptrs, C.c_void_p), _ptr(lens), n, _ptr(out), CHUNK)
    lib.check()
    if rc:
        raise RuntimeError("mc_b200_decode_chunk_blobs failed")
    return out


READ_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p)
_READER_SIGS = {
    "mc_open": (C.c_void_p, [C.c_void_p, C.c_size_t]),
    "mc_open_streaming": (C.c_void_p, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "mc_close": (None, [C.c_void_p]),
    "mc_reader_set_quality": (None, [C.c_void_p, C.c_float]),
    "mc_reader_set_partial_fetch": (None, [C.c_void_p, C.c_int]),
    "mc_chunk_offset": (C.c_uint64, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]),
    "mc_chunk_offset_chk": (C.c_uint64, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "mc_decode_block": (None, [C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "mc_reader_chunk_blob_len": (C.c_uint64, [C.c_void_p, C.c_uint64]),
    "mc_reader_read_blob": (C.c_int, [C.c_void_p, C.c_uint64, C.c_size_t, C.c_void_p]),
    "mc_reader_dims": (None, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "mc_reader_quality": (C.c_float, [C.c_void_p]),
    "mc_reader_nlods": (C.c_int, [C.c_void_p]),
}


class Reader:
    """A read-only reader (mc_open / mc_open_streaming) of either library:
    over archive bytes in memory, or over a file through a byte-range
    callback that counts the bytes and calls it serves."""

    def __init__(self, lib, data=None, path=None, partial=False):
        L = self.L = lib.L
        self.lib = lib
        for name, (res, args) in _READER_SIGS.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        self.bytes = self.calls = 0
        if data is not None:
            self.data = np.ascontiguousarray(np.frombuffer(data, np.uint8))
            self.r = L.mc_open(self.data.ctypes.data, self.data.size)
        else:
            self.f = open(path, "rb")
            size = os.path.getsize(path)

            def read(ud, off, n, dst):
                if off + n > size:
                    return -1
                self.f.seek(off)
                b = self.f.read(n)
                C.memmove(dst, b, n)
                self.bytes += n
                self.calls += 1
                return 0
            self._cb = READ_FN(read)
            self.r = L.mc_open_streaming(C.cast(self._cb, C.c_void_p), None, size)
            if partial:
                L.mc_reader_set_partial_fetch(self.r, 1)
        if not self.r:
            raise RuntimeError("reader open failed")

    def close(self):
        if self.r:
            self.L.mc_close(self.r)
            self.r = None
        if hasattr(self, "f"):
            self.f.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def chunk_offset(self, lod, cz, cy, cx):
        return self.L.mc_chunk_offset(self.r, lod, cz, cy, cx)

    def chunk_offset_chk(self, lod, cz, cy, cx):
        err = C.c_int()
        co = self.L.mc_chunk_offset_chk(self.r, lod, cz, cy, cx, C.byref(err))
        return co, err.value

    def decode_block(self, co, bz, by, bx):
        out = np.zeros(4096, np.uint8)
        self.L.mc_decode_block(self.r, co, bz, by, bx, out.ctypes.data)
        return out

    def blob(self, co):
        n = self.L.mc_reader_chunk_blob_len(self.r, co)
        out = np.zeros(n, np.uint8)
        if n and self.L.mc_reader_read_blob(self.r, co, n, out.ctypes.data) != 0:
            return None
        return out.tobytes()

    def info(self):
        x, y, z = C.c_int(), C.c_int(), C.c_int()
        self.L.mc_reader_dims(self.r, C.byref(x), C.byref(y), C.byref(z))
        return (x.value, y.value, z.value), self.L.mc_reader_quality(self.r), self.L.mc_reader_nlods(self.r)

    def decode_blocks_dev(self, co, coords, d_out, stream=None):
        """mc_b200_reader_decode_blocks (this library only)."""
        cc = np.ascontiguousarray(np.asarray(coords, np.int32).reshape(-1))
        rc = self.L.mc_b200_reader_decode_blocks(self.r, co, cc.ctypes.data, len(coords), C.c_void_p(d_out),
                                                 C.c_void_p(stream) if stream else None)
        self.lib.check()
        return rc
