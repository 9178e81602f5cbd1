"""Compile the CUDA sources into ``hulktracer_b200/libhulkcuda.so`` (sm_100a).

Usage: ``python -m hulktracer_b200.build`` (or ``python hulktracer_b200/build.py``).
Objects go to ``hulktracer_b200/_build``; a source is rebuilt when it, or any
header in ``csrc``/``include``, is newer than its object.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libhulkcuda.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: the traversal, shading and build arithmetic must round after
# every operation in source order to reproduce the reference bit for bit.
# -Xcompiler -ffp-contract=off does the same for host code (the AFF splines and
# matrices reproduce the reference's x86 arithmetic).
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-ffp-contract=off",
           "-Xptxas", "-warn-spills", "-I" + os.path.join(ROOT, "include")]
# files whose arithmetic has no parity constraint may contract (none: the
# network's tile code is shared by the builder and hk_mlp_forward, which must
# agree bit for bit)
FMAD_OK: set = set()


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return p


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [0])
    objs = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if not force and os.path.exists(o) and os.path.getmtime(o) >= max(os.path.getmtime(s), hdr_mtime):
            continue
        flags = list(NVFLAGS)
        if os.path.basename(s) in FMAD_OK:
            flags = [f for f in flags if f != "-fmad=false"]
        cmd = [nvcc()] + ARCH + flags + ["-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
