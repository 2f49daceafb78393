"""mc_b200_decode_blocks_noalloc: the allocation-free block decode, through
the C ABI, against the library's regular entry points (mc_b200_decode_chunk_blobs,
mc_dec_block) and the reference's golden digests.

This file sorts last so that it runs both in a fresh process (alone: the
first GPU call of the library is the no-alloc one, whose first call sets up
its tables itself) and after every other GPU test (runtime already up). The
cold first call is also checked in a child process of its own, where nothing
else has touched the library before it.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ctx_q, sha

MAX_BLOCKS = 4096
MAX_ENTRIES = 4 << 20


def entry_cap(n):
    return min(12288, 8 * n + 64)


def blob_blocks(blob):
    """Header q and {block index: payload bytes} of one chunk blob
    ([f32 q][u64 hash][u16 fmaplen][fmap][512 B bitmap][u16 lens][payloads])."""
    blob = bytes(blob)
    q = float(np.frombuffer(blob, np.float32, 1, 0)[0])
    fml = int.from_bytes(blob[12:14], "little")
    bm = np.frombuffer(blob, np.uint8, 512, 14 + fml)
    present = [i for i in range(4096) if (bm[i >> 3] >> (i & 7)) & 1]
    lens = np.frombuffer(blob, np.uint16, len(present), 14 + fml + 512).astype(np.int64)
    pos = 14 + fml + 512 + 2 * len(present)
    out = {}
    for i, n in zip(present, lens):
        out[i] = blob[pos:pos + n]
        pos += n
    return q, out


def batches(items, nbytes, max_blocks=MAX_BLOCKS):
    """Split a list of blocks (payload sizes nbytes(item)) into calls within
    the entry point's limits."""
    cur, ent = [], 0
    for p in items:
        e = entry_cap(nbytes(p))
        if cur and (len(cur) == max_blocks or ent + e > MAX_ENTRIES):
            yield cur
            cur, ent = [], 0
        cur.append(p)
        ent += e
    if cur:
        yield cur


class NoAlloc:
    """Device buffers for one call (allocated by the test, not the library)."""

    def __init__(self, lib, payloads, stream):
        import torch
        offs = np.zeros(len(payloads) + 1, np.uint64)
        offs[1:] = np.cumsum([len(p) for p in payloads])
        host = np.zeros(int(offs[-1]) + 16, np.uint8)   # 16 readable bytes past the last payload
        for p, o in zip(payloads, offs[:-1]):
            host[int(o):int(o) + len(p)] = np.frombuffer(p, np.uint8)
        self.d_pay = torch.from_numpy(host).to("cuda")
        self.d_out = torch.full((len(payloads) * 4096,), 0xCD, dtype=torch.uint8, device="cuda")
        self.offs = offs
        self.lib, self.stream = lib, stream

    def launch(self, q):
        return self.lib.L.mc_b200_decode_blocks_noalloc(
            self.d_pay.data_ptr(), self.offs.ctypes.data, len(self.offs) - 1, q, self.d_out.data_ptr(),
            self.stream.cuda_stream)

    def result(self):
        return self.d_out.cpu().numpy().reshape(-1, 4096)


@pytest.fixture(scope="module")
def raw_lib():
    """The library without mc_b200_init: the no-alloc entry point needs none."""
    from mcb200 import LIB_PATH as path, McLib
    return McLib(path)


@pytest.mark.gpu
def test_chunk_blocks_two_calls(raw_lib, golden_chunks):
    """Every present block of the golden chunks, decoded by two back-to-back
    calls on one stream, == the blocks of mc_b200_decode_chunk_blobs."""
    import torch
    from mcb200 import McLib, decode_chunk_blobs
    g = golden_chunks
    blobs = [g["blobs"][g["offs"][i]:g["offs"][i + 1]] for i in range(len(g["offs"]) - 1)]
    # every present block, calls launched back to back on one stream (in a
    # fresh process the first of them is the library's first GPU call)
    stream = torch.cuda.Stream()
    calls = []
    for ci, b in enumerate(blobs):
        if not b.size:
            continue
        q, blocks = blob_blocks(b)
        idx = sorted(blocks)
        for part in batches(idx, lambda i: len(blocks[i]), 1500):
            na = NoAlloc(raw_lib, [blocks[i] for i in part], stream)
            assert na.launch(q) == 0
            calls.append((ci, part, na))
    assert len(calls) >= 2
    stream.synchronize()
    got = [(ci, part, na.result()) for ci, part, na in calls]
    want = decode_chunk_blobs(McLib.product(), blobs).reshape(len(blobs), 256, 256, 256)
    for ci, idx, res in got:
        for k, bi in enumerate(idx):
            bz, by, bx = bi >> 8, (bi >> 4) & 15, bi & 15
            w = want[ci, bz * 16:bz * 16 + 16, by * 16:by * 16 + 16, bx * 16:bx * 16 + 16].reshape(-1)
            assert np.array_equal(res[k], w), (str(g["names"][ci]), bi)


@pytest.mark.gpu
def test_golden_blocks(raw_lib, golden_blocks):
    """The reference's block vectors, one call per quality (the raw quality,
    sanitised inside), == the golden digests and mc_dec_block."""
    import torch
    from mcb200 import McLib
    g = golden_blocks
    stream = torch.cuda.Stream()
    groups = {}
    for i in range(len(g["q"])):
        p = g["payload"][g["offs"][i]:g["offs"][i + 1]].tobytes()
        if p:
            groups.setdefault(float(g["q"][i]), []).append((i, p))
    runs = []
    for q, cases in groups.items():
        for part in batches(cases, lambda c: len(c[1])):
            na = NoAlloc(raw_lib, [p for _, p in part], stream)
            assert na.launch(q) == 0
            runs.append((q, part, na))
    stream.synchronize()
    lib = McLib.product()
    for q, cases, na in runs:
        res = na.result()
        for k, (i, p) in enumerate(cases):
            assert sha(res[k]) == g["decoded_sha"][i], f"case {i} q={q}"
            assert np.array_equal(res[k], lib.dec_block(p, ctx_q(q))), f"case {i} q={q}"


@pytest.mark.gpu
def test_corrupt_streams(raw_lib, golden_corrupt):
    """Arbitrary and damaged byte strings in calls of 16 (their overflow stays
    within the fixed spill area) == the reference's digests and mc_dec_block."""
    import torch
    from mcb200 import McLib
    g = golden_corrupt
    stream = torch.cuda.Stream()
    cases = [(i, g["payload"][g["offs"][i]:g["offs"][i + 1]].tobytes(), float(g["q"][i])) for i in range(len(g["q"]))]
    runs = []
    for q in sorted({c[2] for c in cases}):
        sel = [c for c in cases if c[2] == q]
        for j in range(0, len(sel), 16):
            part = sel[j:j + 16]
            na = NoAlloc(raw_lib, [p for _, p, _ in part], stream)
            assert na.launch(q) == 0
            runs.append((part, na))
    stream.synchronize()
    lib = McLib.product()
    for part, na in runs:
        res = na.result()
        for k, (i, p, q) in enumerate(part):
            assert sha(res[k]) == g["decoded_sha"][i], f"stream {i}"
            assert np.array_equal(res[k], lib.dec_block(p, q)), f"stream {i}"


def test_limits_rejected():
    """Requests beyond the fixed scratch are refused before any GPU work
    (runs without a GPU: nothing is launched)."""
    from mcb200 import LIB_PATH as path, McLib
    L = McLib(path).L
    fake = 0x10000   # never dereferenced: every case fails its host-side check
    offs = np.zeros(MAX_BLOCKS + 2, np.uint64)
    assert L.mc_b200_decode_blocks_noalloc(fake, offs.ctypes.data, 0, 6.0, fake, None) == 0
    assert L.mc_b200_decode_blocks_noalloc(fake, offs.ctypes.data, MAX_BLOCKS + 1, 6.0, fake, None) == -2
    big = np.arange(401, dtype=np.uint64) * 2000   # 400 blocks x 12288 entries > 4M
    assert L.mc_b200_decode_blocks_noalloc(fake, big.ctypes.data, 400, 6.0, fake, None) == -3
    assert L.mc_b200_decode_blocks_noalloc(fake + 1, big.ctypes.data, 4, 6.0, fake, None) == -1
    bad = np.array([0, 10, 5], np.uint64)
    assert L.mc_b200_decode_blocks_noalloc(fake, bad.ctypes.data, 2, 6.0, fake, None) == -1
    assert L.mc_b200_decode_blocks_noalloc(None, offs.ctypes.data, 1, 6.0, fake, None) == -1


@pytest.mark.gpu
def test_empty_payloads_decode_to_zeros(raw_lib, golden_blocks):
    """Empty payloads (absent blocks) between real ones decode to zeros, as
    mc_dec_block does with plen = 0 (src/mc_codec.c:739-759), and leave their
    neighbours intact; two calls in a row."""
    import torch
    from mcb200 import McLib
    g = golden_blocks
    real = [(i, g["payload"][g["offs"][i]:g["offs"][i + 1]].tobytes()) for i in range(len(g["q"]))
            if float(g["q"][i]) == 6.0 and g["offs"][i + 1] > g["offs"][i]][:24]
    pays = []
    for k, (i, p) in enumerate(real):
        pays.append(b"")
        pays.append(p)
        if k % 3 == 0:
            pays.append(b"")
    lib = McLib.product()
    assert not lib.dec_block(b"", 6.0).any()
    stream = torch.cuda.Stream()
    runs = []
    for _ in range(2):
        na = NoAlloc(raw_lib, pays, stream)
        assert na.launch(6.0) == 0
        runs.append(na)
    stream.synchronize()
    for na in runs:
        res = na.result()
        for k, p in enumerate(pays):
            want = lib.dec_block(p, 6.0) if p else np.zeros(4096, np.uint8)
            assert np.array_equal(res[k], want), k


def test_empty_payload_reference(ref):
    """The reference's own mc_dec_block on an empty payload: zeros (the
    behaviour the no-alloc call's empty payloads reproduce)."""
    assert not ref.dec_block(b"", 6.0).any()
    assert not ref.dec_block(b"", 1.0).any()


_COLD = r"""
import sys, hashlib
import numpy as np
import torch
sys.path[:0] = [{pkg!r}, {golden!r}]
from mcb200 import LIB_PATH, McLib
g = np.load({blocks!r})
lib = McLib(LIB_PATH)            # no mc_b200_init: the no-alloc call comes first
pays, want = [], []
for i in range(len(g["q"])):
    if float(g["q"][i]) == 6.0 and g["offs"][i + 1] > g["offs"][i]:
        pays.append(g["payload"][g["offs"][i]:g["offs"][i + 1]].tobytes())
        want.append(str(g["decoded_sha"][i]))
offs = np.zeros(len(pays) + 1, np.uint64)
offs[1:] = np.cumsum([len(p) for p in pays])
host = np.zeros(int(offs[-1]) + 16, np.uint8)
for p, o in zip(pays, offs[:-1]):
    host[int(o):int(o) + len(p)] = np.frombuffer(p, np.uint8)
d_pay = torch.from_numpy(host).cuda()
for call in range(2):
    d_out = torch.full((len(pays) * 4096,), 0xCD, dtype=torch.uint8, device="cuda")
    rc = lib.L.mc_b200_decode_blocks_noalloc(d_pay.data_ptr(), offs.ctypes.data, len(pays), 6.0, d_out.data_ptr(), None)
    assert rc == 0, rc
    torch.cuda.synchronize()
    res = d_out.cpu().numpy().reshape(-1, 4096)
    for k in range(len(pays)):
        assert hashlib.sha256(res[k].tobytes()).hexdigest() == want[k], (call, k)
print("cold no-alloc OK", len(pays))
"""


@pytest.mark.gpu
def test_cold_first_call_in_fresh_process(golden_blocks):
    """In a child process whose first library call is the no-alloc one (its
    one-time set-up: the scratch's address and the tables), two calls give
    the reference's golden digests."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = _COLD.format(pkg=os.path.join(root, "matter-compressor_b200"), golden=os.path.join(root, "tests", "golden"),
                        blocks=os.path.join(root, "tests", "golden", "blocks.npz"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "cold no-alloc OK" in r.stdout
