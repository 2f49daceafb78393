"""The C ABI: the shared library loads, exports exactly what include/ declares,
and reports -- rather than hides -- the absence of a usable GPU."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "matter_compressor_b200.h")
LIB = os.path.join(ROOT, "matter-compressor_b200", "libmc_b200.so")


def declared():
    return set(re.findall(r"\b(mc_[a-z0-9_]+)\s*\(", open(HEADER).read()))


def exported():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    return {l.split()[-1] for l in out.splitlines() if " T " in l}


def test_exports_match_header():
    d, e = declared(), exported()
    assert d - e == set(), f"declared but not exported: {sorted(d - e)}"
    assert {s for s in e if s.startswith("mc_")} - d == set()


def test_header_cites_reference_for_dropin():
    text = open(HEADER).read()
    part1 = text[text.index("part 1"):text.index("part 2")]
    for name in re.findall(r"\b(mc_[a-z0-9_]+)\s*\(", part1):
        line = next(l for l in part1.splitlines() if name + "(" in l)
        blk = part1[part1.index(line):part1.index(line) + 400]
        assert "/*" in blk, name


def test_binding_loads_every_symbol():
    from mcb200 import McLib
    lib = McLib(LIB)   # binds every entry point with its signature
    assert lib.L.mc_preset_tau(3) == 8
    assert lib.L.mc_preset_name(0) == b"archival"


def test_no_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from mcb200 import McLib
    lib = McLib(LIB)
    assert lib.L.mc_b200_init() == -1
    assert "device" in (lib.last_error() or "")
    with pytest.raises(RuntimeError):
        McLib.product()
    # the drop-in decode zeroes its output and records the error
    ctx = lib.ctx(6.0)
    dst = np.full(4096, 7, np.uint8)
    src = np.zeros(16, np.uint8)
    lib.L.mc_dec_block(ctx, src.ctypes.data, 16, dst.ctypes.data)
    assert not dst.any()
    assert lib.last_error()
