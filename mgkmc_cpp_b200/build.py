"""Build recipe of the native library (libmgkmc_b200.so) and the CLI.

nvcc cross-compiles every CUDA source for sm_100a (no GPU needed).  Host code
is compiled with -ffp-contract=off so the host-side random draws and the
reference-order arithmetic (libstdc++ distributions, the Gillespie clock) round
exactly as the reference's own build does.  Objects go to mgkmc_cpp_b200/_build,
the library and the CLI binary next to this file (in-tree, so they travel with
the repository snapshot).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmgkmc_b200.so")
CLI = os.path.join(HERE, "mgkmc_b200")

SOURCES = ["ls.cu", "kmc_kernels.cu", "engine.cu", "batch.cu", "elastic.cu", "fieldgen.cu", "capi.cu", "vtu.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_FLAGS = "-fPIC,-O2,-ffp-contract=off,-fvisibility=hidden"


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _newer(src_paths, out) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(p) > t for p in src_paths)


def _deps(src):
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hdrs.append(os.path.join(HERE, "..", "include", "mgkmc_b200.h"))
    return [os.path.join(CSRC, src)] + hdrs


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, src + ".o")
    if not _newer(_deps(src), obj):
        return obj
    cmd = [nvcc(), *ARCH, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", HOST_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    if src.endswith(".cpp"):
        cmd.insert(1, "-x")
        cmd.insert(2, "cu")
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s" % (src, r.stderr[-6000:]))
    return obj


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if _newer(objs, LIB):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", HOST_FLAGS, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s" % r.stderr[-6000:])
    cli_src = os.path.join(CSRC, "main.cpp")
    if os.path.exists(cli_src) and _newer([cli_src, LIB] + _deps("main.cpp")[1:], CLI):
        cmd = [nvcc(), *ARCH, "-O2", "-std=c++17", "-x", "cu", cli_src, "-o", CLI, "-Xcompiler", "-O2,-ffp-contract=off",
               "-L" + HERE, "-lmgkmc_b200", "-Xlinker", "-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("CLI build failed:\n%s" % r.stderr[-6000:])
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print("built", LIB)
