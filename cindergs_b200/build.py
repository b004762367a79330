"""Builds the sm_100a CUDA library ``cindergs_b200/_lib/libcindergs.so``.

Each translation unit is compiled by nvcc for ``sm_100a`` only. Stages 1 and
2 are compiled with ``-fmad=false`` so that every product and sum is rounded
separately, in the reference's operand order; Stage 3's binning rounds the
expressions its keys depend on explicitly (__fmul_rn / __fadd_rn). Their
integer outputs -- tile counts, offsets, keys -- are bit-exact against the
host restatement.
The library links the CUDA runtime statically and exports only the C ABI of
``include/cgs.h``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libcindergs.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
          "--expt-relaxed-constexpr", "-I", CSRC, "-I", INCLUDE]
# (source, extra flags)
UNITS = [
    ("stage1_deform.cu", ["-fmad=false"]),
    ("stage1_mvc.cu", ["-fmad=false"]),
    ("stage2_project.cu", ["-fmad=false"]),
    ("stage3_bin.cu", []),  # explicit __fmul_rn/__fadd_rn where the keys depend on rounding
    ("sh_rotate.cu", ["-fmad=false"]),
    ("springs.cu", ["-fmad=false"]),
    ("radix_sort.cu", []),
    ("stage4_composite.cu", []),
    ("mvc_field.cu", []),
    ("mvc_field_tc.cu", []),
    ("field.cu", []),
    ("pipeline.cu", []),
    ("noalloc.cu", []),
]
HEADERS = ["common.cuh", "detmath.h", "kernels.h", "field.h"]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _mtime(path: str) -> float:
    return os.path.getmtime(path) if os.path.exists(path) else -1.0


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    """Compiles changed units and relinks the library; returns its path."""
    os.makedirs(os.path.join(LIBDIR, "obj"), exist_ok=True)
    hdr_time = max(_mtime(os.path.join(CSRC, h)) for h in HEADERS)
    hdr_time = max(hdr_time, _mtime(os.path.join(INCLUDE, "cgs.h")))
    objs = []
    relink = force or not os.path.exists(LIB)
    nvcc = _nvcc()
    for src, extra in UNITS:
        sp = os.path.join(CSRC, src)
        op = os.path.join(LIBDIR, "obj", src.replace(".cu", ".o"))
        objs.append(op)
        if not force and _mtime(op) > max(_mtime(sp), hdr_time):
            continue
        cmd = [nvcc, *ARCH, *COMMON, *extra, "-c", sp, "-o", op]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        relink = True
    if relink or any(_mtime(o) > _mtime(LIB) for o in objs):
        cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
