"""Builds ``libb2simplec.so`` in-tree with nvcc for sm_100a (no JIT, no torch extension).

``python -m gputest_b200.csrc.build`` or ``build()``. Flags: ``-fmad=false`` keeps IEEE
multiply-then-add semantics, so per-cell sums can match the reference's NumPy results to the
bit; ``-lineinfo`` for profiling; the CUDA runtime is linked statically.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
INCLUDE = os.path.join(ROOT, "include")
SOURCES = ["b2s_setup.cu", "b2s_fv.cu", "b2s_krylov.cu", "b2s_amg.cu", "b2s_amg_setup.cu", "b2s_batch.cu", "b2s_adjoint.cu", "b2s_noalloc.cu", "b2s_sst.cu"]
HEADERS = ["b2s_common.cuh", "b2s_fv.cuh"]
LIB = os.path.join(HERE, "libb2simplec.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libb2simplec.so")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(HERE, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "b2simplec.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and not _stale():
        return LIB
    nvcc = _nvcc()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [nvcc, *ARCH, *FLAGS, *extra, "-I", INCLUDE, "-I", HERE, "-c", os.path.join(HERE, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        cp = subprocess.run(cmd, capture_output=True, text=True)
        if cp.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{cp.stdout}\n{cp.stderr}")
        if verbose and (cp.stdout or cp.stderr):
            print(cp.stdout, cp.stderr, flush=True)
        objs.append(obj)
    tmp = LIB + f".{os.getpid()}.tmp"
    cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs]
    cp = subprocess.run(cmd, capture_output=True, text=True)
    if cp.returncode != 0:
        raise RuntimeError(f"linking libb2simplec.so failed:\n{cp.stdout}\n{cp.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else ()))
