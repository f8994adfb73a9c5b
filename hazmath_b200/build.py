"""Build the CUDA library hazmath_b200/libhazb200.so for sm_100a (in tree).

    python -m hazmath_b200.build [-v]

Every CUDA translation unit is compiled with
``-gencode arch=compute_100a,code=sm_100a -O3 -lineinfo``.  The parity
kernels need separately rounded products and sums (the reference's C loops
are built without FMA), so all files except the dense coarse factorisation
use ``-fmad=false``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhazb200.so")
ROOT = os.path.dirname(HERE)

SOURCES = [
    ("hzb_kernels.cu", False),
    ("hzb_sell.cu", False),
    ("hzb_setup.cu", False),
    ("hzb_dense.cu", True),
    ("hzb_solver.cu", False),
    ("hzb_batch.cu", False),
    ("hzb_gmres.cu", False),
    ("hzb_cycles.cu", False),
    ("hzb_minres.cu", False),
    ("hzb_sa.cu", False),
    ("hzb_bsr.cu", False),
    ("hzb_vmb.cu", False),
    ("hzb_hec.cu", False),
    ("hzb_assemble.cu", False),
    ("hzb_learn.cu", False),
    ("hzb_gnn.cu", True),
    ("hzb_api.cu", False),
]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _compile(src: str, fmad: bool, verbose: bool) -> str:
    out = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
           "-I", os.path.join(ROOT, "include"), f"-fmad={'true' if fmad else 'false'}",
           "-c", os.path.join(SRC, src), "-o", out]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr)
    return out


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(SRC, f) for f in os.listdir(SRC)]
    deps.append(os.path.join(ROOT, "include", "hazmath_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s[0], s[1], verbose), SOURCES))
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    v = "-v" in sys.argv
    print(build(verbose=v, force=True))
