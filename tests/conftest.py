"""Shared fixtures. Tests marked `gpu` need an sm_100 device; everything else
runs on CPU (the oracle, the golden vectors, the host-side archive format and
the C ABI's exports)."""
import hashlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "matter-compressor_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    """The reference's own strict build, when it was compiled here."""
    from oracle import REF_LIB
    from mcb200 import McLib
    if not os.path.exists(REF_LIB):
        pytest.skip("reference build oracle/_ref/libmcref.so not present")
    lib = McLib(REF_LIB, b200=False)
    lib.L.mc_codec_init()
    return lib


@pytest.fixture(scope="session")
def gpu():
    """The B200 library with a usable device (GPU tests only)."""
    from mcb200 import McLib
    return McLib.product()


@pytest.fixture(scope="session")
def golden_blocks():
    return np.load(os.path.join(GOLDEN, "blocks.npz"))


@pytest.fixture(scope="session")
def golden_corrupt():
    return np.load(os.path.join(GOLDEN, "corrupt.npz"))


@pytest.fixture(scope="session")
def golden_meta():
    return np.load(os.path.join(GOLDEN, "meta.npz"))


@pytest.fixture(scope="session")
def golden_chunks():
    return np.load(os.path.join(GOLDEN, "chunks.npz"))


def ctx_q(q):
    """The quality a codec context ends up with (mc_codec_ctx_set_quality)."""
    return q if (q == q and 0 < q <= 1024) else 8.0
