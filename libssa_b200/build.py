"""Builds the libssa B200 shared libraries in-tree (libssa_b200/_lib/).

    python -m libssa_b200.build        # or: python libssa_b200/build.py

* ``libssa.so``      -- the drop-in library: libssa.h + libssa_b200.h, host C++
  and the sm_100a CUDA kernels (``-gencode arch=compute_100a,code=sm_100a``),
  CUDA runtime linked statically.  Its ssa_db_* imports are resolved from the
  database plugin loaded before it.
* ``libsdb_b200.so`` -- the database plugin implementing libssa_extern_db.h.

Compilation is incremental on file modification times; objects live in
``libssa_b200/_lib/obj``.
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
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(HERE, "_lib")
OBJ = os.path.join(OUT, "obj")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-Wall", "-I" + INCLUDE, "-I" + CSRC]

CU_SOURCES = ["engine.cu", "emul_kernel.cu", "traceback_kernels.cu", "diag_kernels.cu", "sw_fast_kernel.cu",
              "noalloc.cu", "sw_qpair_kernel.cu", "pair_kernel.cu"]
CPP_SOURCES = ["api.cpp", "replay.cpp", "tuning.cpp"]
HEADERS = ["device_common.cuh", "wavefront.cuh", "stripe_pipeline.cuh", "ssa_internal.h", "builtin_matrices.inc"]

LIB = os.path.join(OUT, "libssa.so")
PLUGIN = os.path.join(OUT, "libsdb_b200.so")


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def cuda_include() -> str:
    return os.path.join(os.path.dirname(os.path.dirname(nvcc())), "include")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"compile failed: {cmd[-1]}")


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, h) for h in os.listdir(INCLUDE)]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            jobs.append([nvcc(), *ARCH, *NVCC_FLAGS, "-c", s, "-o", o])
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            jobs.append(["g++", *CXX_FLAGS, "-I" + cuda_include(), "-c", s, "-o", o])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            list(ex.map(_run, jobs))
    if _stale(LIB, objs):
        _run([nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-cudart", "static", "-o", LIB, *objs,
              "-Xlinker", "--no-undefined", "-Xlinker", "--unresolved-symbols=ignore-in-object-files",
              "-lpthread", "-ldl", "-lrt"])
    plugin_src = os.path.join(CSRC, "sdb_plugin.c")
    if _stale(PLUGIN, [plugin_src, os.path.join(INCLUDE, "libssa_extern_db.h")]):
        _run(["gcc", "-O2", "-std=c99", "-fPIC", "-shared", "-I" + INCLUDE, "-o", PLUGIN, plugin_src])
    if verbose:
        print("built", LIB, PLUGIN)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
