"""Builds libmc_b200.so (sm_100a kernels + C ABI) in-tree with nvcc.

Usage: python build.py [--force]. Object files go to _build/ next to this
script; the shared library lands beside it so it ships with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmc_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Device arithmetic must round like the reference's strict IEEE build: no
# multiply-add contraction anywhere (-fmad=false, -ffp-contract=off on host),
# no flush-to-zero, IEEE division and square root.
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-ftz=false", "-prec-div=true", "-prec-sqrt=true",
          "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math,-Wall", "-I", CSRC]
SOURCES = ["mcb_decode.cu", "mcb_encode.cu", "mcb_tables.cpp", "mcb_runtime.cpp", "mcb_host_codec.cpp",
           "mcb_archive.cpp", "mcb_api.cpp", "mcb_noalloc.cu", "mcb_gather.cu", "mcb_server.cpp", "mcb_deblock.cu", "mcb_lod.cu", "mcb_sample.cu", "mcb_reader.cpp"]


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "matter_compressor_b200.h"))
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [NVCC] + ARCH + COMMON + ["-c", path, "-o", obj]
            if src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if verbose else []
            else:
                cmd += ["-x", "c++"]
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xlinker", "-Bsymbolic", "-lpthread", "-ldl", "-lrt"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
