"""Builds libpu_dycore.so in-tree (porturb_b200/_lib/) with nvcc for sm_100a.

Each (stencil type, tracer count) instantiation of the dycore is its own
translation unit, compiled in parallel, then linked with the C entry points
into one shared library.  The CUDA runtime is linked statically so the
library only needs the driver at run time.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIB = os.path.join(LIBDIR, "libpu_dycore.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]
INSTANCES = [(r, n) for r in ("float", "double") for n in (1, 2, 3, 4)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources_mtime() -> float:
    m = 0.0
    for fn in os.listdir(CSRC):
        if fn.endswith((".cu", ".cuh", ".h")):
            m = max(m, os.path.getmtime(os.path.join(CSRC, fn)))
    for hdr in ("pu_dycore.h", "pu_physics.h"):
        m = max(m, os.path.getmtime(os.path.join(HERE, "..", "include", hdr)))
    return m


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s" % (" ".join(cmd), r.stdout[-6000:]))
    return r.stdout


def build(force: bool = False, verbose: bool = False, ptxas_report: bool = False) -> str:
    """Compile and link; returns the library path.  Skips the work when the
    library is newer than every source file."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _sources_mtime():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    tables = os.path.join(CSRC, "weno9_tables.cuh")
    if not os.path.exists(tables):
        with open(tables, "w") as f:
            subprocess.run([sys.executable, os.path.join(CSRC, "gen_weno9.py")], stdout=f, check=True)
    extra = ["-Xptxas", "-v"] if ptxas_report else []
    jobs = []
    for real, ntr in INSTANCES:
        tag = ("f32_%d" if real == "float" else "f64_%d") % ntr
        obj = os.path.join(OBJDIR, "impl_%s.o" % tag)
        cmd = [nvcc()] + NVFLAGS + extra + ["-DPU_REAL=%s" % real, "-DPU_NTR=%d" % ntr, "-DPU_TAG=%s" % tag,
                                            "-c", os.path.join(CSRC, "impl_inst.cu"), "-o", obj]
        jobs.append((obj, cmd))
    for src in ("pu_dycore", "pu_noalloc", "physics"):
        jobs.append((os.path.join(OBJDIR, src + ".o"),
                     [nvcc()] + NVFLAGS + extra + ["-c", os.path.join(CSRC, src + ".cu"), "-o",
                                                   os.path.join(OBJDIR, src + ".o")]))
    with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
        outs = list(ex.map(lambda j: _run(j[1]), jobs))
    if verbose:
        for o in outs:
            sys.stdout.write(o)
    tmp = LIB + ".tmp"
    _run([nvcc()] + ARCH + ["-shared", "-o", tmp] + [j[0] for j in jobs])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_report="--ptxas" in sys.argv)
    print(LIB)
