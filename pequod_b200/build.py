"""Build the pequod_b200 shared library for sm_100a with nvcc.

The library is built in-tree (pequod_b200/_lib/libpequod_b200.so) so that it
ships with the source tree.  Host code is compiled without floating-point
contraction so that the set-up tables (pivots, correction function) follow the
reference's operation order; device code uses nvcc's default FMA contraction.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
SRC = os.path.join(PKG, "csrc")
OUT_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(OUT_DIR, "libpequod_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(SRC, "*.cu")) + glob.glob(os.path.join(SRC, "*.cpp")))


def headers():
    return sorted(glob.glob(os.path.join(SRC, "*.h")) + glob.glob(os.path.join(SRC, "*.cuh")) +
                  glob.glob(os.path.join(ROOT, "include", "*.h")))


OBJ_DIR = os.path.join(PKG, "_build")


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in sources() + headers() + [__file__])


def _flags():
    return [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
            "-Xptxas", "-warn-spills", "-I", os.path.join(ROOT, "include"), "-I", SRC]


def _compile(src, verbose):
    obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
    newest = max(os.path.getmtime(f) for f in [src, __file__] + headers())
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj
    cmd = [nvcc(), *_flags(), "-c", "-o", obj + ".tmp", src]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(obj + ".tmp", obj)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source to an object in parallel (only those older than
    their inputs), then link the shared library."""
    from concurrent.futures import ThreadPoolExecutor

    if not force and up_to_date():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    if force:
        for f in glob.glob(os.path.join(OBJ_DIR, "*.o")):
            os.remove(f)
    with ThreadPoolExecutor(max_workers=max(1, min(len(sources()), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(lambda src: _compile(src, verbose), sources()))
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "--shared", "-Xcompiler", "-fPIC", "-o", tmp, *objs, "-lcuda"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
