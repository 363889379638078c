"""Builds libibpm_b200.so in-tree for sm_100a (nvcc, no JIT cache).

Translation units: ibpm.cu (transforms, stencils, host runtime and C ABI);
coupling.cu, compiled with -fmad=false so the regularised-delta weights and the
E / E^T sums round exactly like the reference (no fused multiply-add);
noalloc.cu (the allocation-free Laplacian-inverse entry point);
warmstart.cu (the learned CG warm start's network); and tc_dst.cu (dense DST-I
passes on the tensor cores for the preconditioner's B assembly).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "lib", "obj")
OUT = os.path.join(HERE, "lib", "libibpm_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-diag-suppress", "550"]
UNITS = [("ibpm.cu", []), ("coupling.cu", ["-fmad=false"]), ("noalloc.cu", []), ("warmstart.cu", []), ("tc_dst.cu", [])]


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "ibpm_b200.h")]


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    if not force and os.path.exists(OUT):
        t = os.path.getmtime(OUT)
        if all(os.path.getmtime(p) <= t for p in _deps()):
            return OUT
    objs = []
    for src, extra in UNITS:
        obj = os.path.join(OBJ, src.replace(".cu", ".o"))
        cmd = [NVCC, *COMMON, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC, *ARCH, "-shared", "-o", OUT, *objs]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
