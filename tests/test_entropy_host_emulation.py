"""The entropy stage's device code, compiled for the host and run one lane at
a time, against the oracle's block decoder.

The lane state machine of k_entropy (lane_begin, fast_step, fast_event,
slow_work, lane_finish and the warp loop run_lanes in csrc/mcb_decode.cu) and
the single-block loop of k_decode_one are lifted out of the CUDA source, their
few device intrinsics replaced by host equivalents (a warp vote over one lane
is that lane's own predicate), and built with g++. Each stream is decoded
twice -- by run_lanes with one lane and by the single-block loop -- and both
must give the oracle's levels, dc, flags and coefficient count
(oracle/mc_oracle.c or_dec_block_levels, which follows src/mc_codec.c:739-757,
353-375). Inputs: the golden block payloads, the corrupt-stream corpus and
random streams, so the state machine is covered without a GPU; the GPU tests
run the same code on the device.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "matter-compressor_b200", "csrc")
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")

_PRELUDE = r'''#include <stdint.h>
#include <string.h>
#include <algorithm>
#include "mcb_format.h"
#include "mcb_kernels.h"
using std::min;
template <class T> static T LDG(const T *p) { return *p; }
static uint32_t ATOMIC_ADD(uint32_t *p, uint32_t v) { uint32_t o = *p; *p += v; return o; }
static bool ANY_SYNC(unsigned, bool p) { return p; }   // a one-lane warp
static bool ALL_SYNC(unsigned, bool p) { return p; }
// __byte_perm: byte n of the result is byte (s >> 4n) & 7 of y:x
static uint32_t BYTE_PERM(uint32_t x, uint32_t y, uint32_t s) {
    const uint64_t v = ((uint64_t)y << 32) | x;
    uint32_t r = 0;
    for (int n = 0; n < 4; ++n) r |= (uint32_t)((v >> (8 * ((s >> (4 * n)) & 7))) & 0xFF) << (8 * n);
    return r;
}
namespace mcb {
'''


_DRIVER = r'''
#include <vector>
#include "mcb_tables.h"
using namespace mcb;
extern "C" int emu_block(const uint8_t *pay, uint32_t len, float q, int mode, int16_t *levels, int *info) {
    static uint16_t scan[kN3];
    static bool init = false;
    if (!init) { table_scan(scan); init = true; }
    uint16_t s_bend[9];
    for (int i = 1; i < kN3; ++i) {
        const uint32_t b = scan[i] >> 12;
        if ((uint32_t)(scan[i - 1] >> 12) != b) s_bend[b - 1] = (uint16_t)i;
    }
    s_bend[7] = kN3;
    s_bend[8] = 0xFFFF;
    static QTab qt;
    table_qtab(sanitize_q(q), &qt);
    // the payload at an odd address inside a larger buffer, as in an archive
    std::vector<uint8_t> buf(len + 64, 0xA5);
    const uint32_t shift = (len * 7 + 3) % 8;
    if (len) memcpy(buf.data() + shift, pay, len);
    DecItem it{};
    it.src = (uint64_t)(uintptr_t)(buf.data() + shift);
    it.len = len;
    uint64_t base = 0;
    const uint32_t cap = entry_cap(len);
    std::vector<uint32_t> entries(kEntryMax + 4);   // arena, then the overflow pool
    EntHdr hdr{};
    uint32_t status[4] = {0, 0, 0, 0};
    EntParams P{};
    P.items = &it; P.order = nullptr; P.n = 1; P.ncoded = 1; P.base = &base; P.arena = entries.data();
    P.hdr = &hdr; P.pool = entries.data() + cap; P.pool_cap = kEntryMax - cap; P.pool_used = status + 1;
    P.qtab = &qt; P.scan = scan; P.status = status;
    static uint32_t ctx[kCtxSlots * 32];
    LaneState L;
    if (mode == 0) {   // run_lanes, the k_entropy loop, with one lane and a queue of one block
        uint32_t counter = 0;
        P.counter = &counter;
        P.claim = 1;
        int done = 0;
        run_lanes(L, P, ctx, s_bend, 0, 1, [&](int) { done++; });
        if (done != 1) return -1;
    } else {           // k_decode_one's loop
        memset(&L, 0, sizeof L);
        lane_begin(L, P, ctx, s_bend, 0);
        solo_entropy(L, P, ctx, s_bend);
        lane_finish(L, P);
    }
    memset(levels, 0, 2 * kN3);
    for (uint32_t j = 0; j < hdr.nnz; ++j) {
        const uint32_t e = entries[j];   // arena and pool are contiguous here
        levels[scan[e & 0xFFF] & 0xFFF] = (int16_t)(e >> 16);
    }
    info[0] = hdr.dc; info[1] = hdr.flags; info[2] = hdr.nnz; info[3] = hdr.ncorr; info[4] = hdr.bad;
    return 0;
}
'''


def _cut(src, start, end):
    a = src.find(start)
    b = src.find(end, a)
    assert a >= 0 and b > a, f"marker not found in mcb_decode.cu: {start[:40]!r} / {end[:40]!r}"
    return src[a:b]


def _host_source():
    src = open(os.path.join(CSRC, "mcb_decode.cu")).read()
    # stage 1 up to k_entropy: the lane step functions, run_lanes and the
    # single-thread loop solo_entropy
    body = _cut(src, "// ---------------------------------------------------------------- stage 1",
                "template <int WARPS>\n__global__")
    for dev, host in (("__device__ __forceinline__", "static inline"), ("__ldg(", "LDG("),
                      ("atomicAdd(", "ATOMIC_ADD("), ("__byte_perm(", "BYTE_PERM("),
                      ("__popc(", "__builtin_popcount("), ("__any_sync(", "ANY_SYNC("),
                      ("__all_sync(", "ALL_SYNC(")):
        body = body.replace(dev, host)
    assert "asm" not in body and "__shared__" not in body, "device-only code left in the host build"
    return _PRELUDE + body + "\n}  // namespace mcb\n" + _DRIVER


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("emu")
    cpp = d / "emu.cpp"
    cpp.write_text(_host_source())
    so = d / "libemu.so"
    subprocess.run([gxx, "-std=c++17", "-O2", "-shared", "-fPIC", "-ffp-contract=off", "-I", CSRC, "-I", CUDA_INC,
                    "-o", str(so), str(cpp), os.path.join(CSRC, "mcb_tables.cpp")], check=True)
    lib = C.CDLL(str(so))
    lib.emu_block.argtypes = [C.c_void_p, C.c_uint32, C.c_float, C.c_int, C.c_void_p, C.c_void_p]
    lib.emu_block.restype = C.c_int
    return lib


def _run(lib, payload, q, mode):
    lv = np.zeros(4096, np.int16)
    info = np.zeros(8, np.int32)
    src = np.frombuffer(payload, np.uint8) if len(payload) else np.zeros(1, np.uint8)
    assert lib.emu_block(src.ctypes.data, len(payload), q, mode, lv.ctypes.data, info.ctypes.data) == 0
    return lv, info


def _check(lib, oracle, payload, q, what):
    olv, oinfo = oracle.dec_levels(payload, q)
    for mode in (0, 1):
        lv, info = _run(lib, payload, q, mode)
        assert np.array_equal(lv, olv), (what, mode, "levels")
        assert (info[0], info[1], info[2]) == (oinfo[0], oinfo[1], oinfo[6]), (what, mode, "dc/flags/nnz")
        if oinfo[7] == 0:
            assert info[4] == 0, (what, mode, "cut short")


def test_golden_blocks(emu, oracle, golden_blocks):
    g = golden_blocks
    for i in range(len(g["q"])):
        p = g["payload"][g["offs"][i]:g["offs"][i + 1]].tobytes()
        _check(emu, oracle, p, float(g["q"][i]), f"block {i}")


def test_corrupt_streams(emu, oracle, golden_corrupt):
    g = golden_corrupt
    for i in range(len(g["q"])):
        p = g["payload"][g["offs"][i]:g["offs"][i + 1]].tobytes()
        _check(emu, oracle, p, float(g["q"][i]), f"corrupt {i}")


def test_random_streams(emu, oracle):
    rng = np.random.default_rng(11)
    qs = [0.25, 1.0, 3.0, 6.0, 12.0, 40.0]
    for t in range(300):
        n = int(rng.integers(0, 600)) if t % 3 else int(rng.integers(600, 16000))
        p = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        _check(emu, oracle, p, qs[t % len(qs)], f"random {t}")


def test_biased_streams(emu, oracle):
    """Streams of biased random bits (runs of ones): long Exp-Golomb prefixes,
    suffixes decoded bit by bit, suffixes of more than 16 bits (the batched
    division path) and prefixes that reach the cap."""
    rng = np.random.default_rng(5)
    for t in range(1500):
        n = int(rng.integers(1, 3000))
        bias = float(rng.choice([0.5, 0.9, 0.97, 0.995]))
        p = np.packbits((rng.random(n * 8) < bias).astype(np.uint8)).tobytes()[:n]
        _check(emu, oracle, p, float(rng.choice([0.5, 1.0, 6.0, 40.0])), f"biased {t}")
