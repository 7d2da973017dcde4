"""In-tree build of the native libraries.

- ``libgraph_cuda.so`` / ``libgraph_cuda.a``: the sm_100a engine and its C ABI
  (``include/graph_cuda.h``), from ``csrc/engine.cu`` (and, once present,
  ``csrc/batch.cu``, ``csrc/adjoint.cu``).
- ``libgraph_synth.so``: the host-side synthetic graph generators.

The shared objects land next to this file so they travel with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]

CUDA_UNITS = ["engine.cu"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the sm_100a engine cannot be built")


def _cc() -> str:
    for cand in ("/usr/bin/gcc", shutil.which("gcc") or ""):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("gcc not found")


def _stale(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _deps():
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h", ".c")):
                out.append(os.path.join(d, f))
    return out


def build_cuda(force: bool = False, verbose: bool = False) -> str:
    so = os.path.join(HERE, "libgraph_cuda.so")
    a = os.path.join(HERE, "libgraph_cuda.a")
    units = [os.path.join(CSRC, u) for u in CUDA_UNITS if os.path.exists(os.path.join(CSRC, u))]
    if not force and not _stale(so, _deps()) and not _stale(a, _deps()):
        return so
    nvcc = _nvcc()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for u in units:
        o = os.path.join(objdir, os.path.basename(u) + ".o")
        cmd = [nvcc, *NVCC_FLAGS, *ARCH, "-rdc=false", "-c", u, "-o", o]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        objs.append(o)
    subprocess.run([nvcc, *ARCH, "-shared", "-o", so, *objs], check=True)
    if os.path.exists(a):
        os.remove(a)
    subprocess.run(["ar", "rcs", a, *objs], check=True)
    return so


def build_synth(force: bool = False) -> str:
    so = os.path.join(HERE, "libgraph_synth.so")
    src = os.path.join(CSRC, "synth.c")
    if force or _stale(so, [src]):
        subprocess.run([_cc(), "-O2", "-fPIC", "-shared", "-std=c11", "-o", so, src, "-lm"], check=True)
    return so


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_synth(force)
    build_cuda(force, verbose)


if __name__ == "__main__":
    import sys

    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
