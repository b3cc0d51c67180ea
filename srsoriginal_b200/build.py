"""Builds libsrs_b200.so in-tree with nvcc for sm_100a (B200).

    python -m srsoriginal_b200.build        # or __graft_entry__.build()

Translation units whose results must match the reference's IEEE-double arithmetic (the RK4 and the
plain FP64 sums, plus the host geometry) are compiled with -fmad=false: no multiply-add contraction.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsrs_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC]
# (source, exact IEEE double: -fmad=false)
SOURCES = [
    ("rk4.cu", True),
    ("rk4_shoot.cu", True),
    ("sums_fp64.cu", True),
    ("sums_mixed.cu", False),
    ("queue.cu", False),
    ("adjoint.cu", True),
    ("capi.cu", True),
    ("sim.cpp", True),
    ("field_files.cpp", True),
    ("peaks.cu", False),
]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src, exact, verbose=False):
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "srs_b200.h"))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    cmd = [nvcc(), "-x", "cu", "-c", path, "-o", obj] + ARCH + COMMON
    cmd += ["-fmad=false"] if exact else ["-fmad=true"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose=False, force=False):
    """Compiles every CUDA/C++ source for sm_100a and links libsrs_b200.so (CUDA runtime linked
    statically, so the library needs only the driver)."""
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s[0], s[1], verbose), SOURCES))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-cudart", "static", "-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
