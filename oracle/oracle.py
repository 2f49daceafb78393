"""ctypes binding of the oracle (TEST INFRASTRUCTURE ONLY).

Two checkers live under oracle/:
  * liboracle.so        -- our C restatement of the reference codec (mc_oracle.c)
  * _ref/libmcref.so    -- the reference's own sources, strict IEEE build, when
                           built here (oracle/Makefile); absent on machines
                           without the reference checkout unless shipped.
Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use them.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libmcref.so")
REF_FAST_LIB = os.path.join(HERE, "_ref", "libmcref_fast.so")


def _p(a):
    return C.c_void_p(a.ctypes.data)


class Oracle:
    def __init__(self, path=ORACLE_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run make -C oracle")
        L = self.L = C.CDLL(path)
        vp, f, i, u32, u64, sz = C.c_void_p, C.c_float, C.c_int, C.c_uint32, C.c_uint64, C.c_size_t
        for name, res, args in [
            ("or_set_priors", None, [vp, vp]),
            ("or_priors_for_q", None, [f, vp]),
            ("or_sanitize_q", f, [f]),
            ("or_step_table", None, [f, vp, vp]),
            ("or_scan_table", None, [vp]),
            ("or_enc_block", u32, [vp, f, i, vp, u32]),
            ("or_dec_block", None, [vp, u32, f, vp]),
            ("or_dec_block_levels", None, [vp, u32, f, vp, vp]),
            ("or_enc_fracmap", u32, [vp, vp, u32]),
            ("or_dec_fracmap", None, [vp, u32, vp]),
            ("or_frac_nibble", C.c_uint8, [vp]),
            ("or_xxh64", u64, [vp, sz, u64]),
            ("or_blob_hash", u64, [vp, u64]),
            ("or_encode_chunk", sz, [vp, f, f, i, vp, sz]),
            ("or_decode_chunk", None, [vp, u64, vp]),
            ("or_decode_chunk_block", None, [vp, u64, i, i, i, vp]),
            ("or_deblock", None, [vp, i, i, i, f]),
            ("or_decimate", None, [vp, i, i, i, vp]),
        ]:
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args

    def enc_block(self, vox, q, tau=0):
        vox = np.ascontiguousarray(vox, np.uint8).reshape(-1)
        out = np.zeros(17408, np.uint8)
        n = self.L.or_enc_block(_p(vox), q, tau, _p(out), out.size)
        return out[:n].tobytes()

    def dec_block(self, payload, q):
        dst = np.zeros(4096, np.uint8)
        src = np.ascontiguousarray(np.frombuffer(payload, np.uint8)) if payload else np.zeros(1, np.uint8)
        self.L.or_dec_block(_p(src), len(payload), q, _p(dst))
        return dst

    def dec_levels(self, payload, q):
        lv = np.zeros(4096, np.int16)
        info = np.zeros(8, np.int32)
        src = np.ascontiguousarray(np.frombuffer(payload, np.uint8)) if payload else np.zeros(1, np.uint8)
        self.L.or_dec_block_levels(_p(src), len(payload), q, _p(lv), _p(info))
        return lv, info

    def enc_fracmap(self, frac):
        frac = np.ascontiguousarray(frac, np.uint8)
        out = np.zeros(2112, np.uint8)
        n = self.L.or_enc_fracmap(_p(frac), _p(out), out.size)
        return out[:n].tobytes()

    def dec_fracmap(self, data):
        frac = np.zeros(4096, np.uint8)
        src = np.ascontiguousarray(np.frombuffer(data, np.uint8))
        self.L.or_dec_fracmap(_p(src), len(data), _p(frac))
        return frac

    def xxh64(self, data, seed):
        a = np.ascontiguousarray(np.frombuffer(data, np.uint8)) if len(data) else np.zeros(1, np.uint8)
        return self.L.or_xxh64(_p(a), len(data), seed)

    def blob_hash(self, blob):
        a = np.ascontiguousarray(np.frombuffer(blob, np.uint8))
        return self.L.or_blob_hash(_p(a), len(blob))

    def encode_chunk(self, vox, q, tau=0, header_q=None):
        vox = np.ascontiguousarray(vox, np.uint8).reshape(-1)
        cap = 64 << 20
        out = np.zeros(cap, np.uint8)
        n = self.L.or_encode_chunk(_p(vox), q if header_q is None else header_q, q, tau, _p(out), cap)
        return out[:n].tobytes()

    def decode_chunk(self, blob):
        out = np.zeros(256 ** 3, np.uint8)
        a = np.ascontiguousarray(np.frombuffer(blob, np.uint8))
        self.L.or_decode_chunk(_p(a), len(blob), _p(out))
        return out

    def deblock(self, vol, quality):
        """In-place deblock of a dense (nz, ny, nx) u8 volume; returns it."""
        v = np.ascontiguousarray(vol, np.uint8)
        nz, ny, nx = v.shape
        self.L.or_deblock(_p(v), nz, ny, nx, quality)
        return v

    def decimate(self, vol):
        """2x LOD decimation of a dense (DZ, DY, DX) u8 volume."""
        v = np.ascontiguousarray(vol, np.uint8)
        dz, dy, dx = v.shape
        out = np.zeros(((dz + 1) // 2, (dy + 1) // 2, (dx + 1) // 2), np.uint8)
        self.L.or_decimate(_p(v), dz, dy, dx, _p(out))
        return out

    def priors_for_q(self, q):
        out = np.zeros(256, np.uint16)
        self.L.or_priors_for_q(q, _p(out))
        return out

    def set_priors(self, plo, phi):
        if plo is None:
            self.L.or_set_priors(None, None)
        else:
            self._keep = (np.ascontiguousarray(plo, np.uint16), np.ascontiguousarray(phi, np.uint16))
            self.L.or_set_priors(_p(self._keep[0]), _p(self._keep[1]))
