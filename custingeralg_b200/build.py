"""Build the native libraries in-tree (no JIT cache, so the .so files travel with the repo).

  custingeralg_b200/libcustinger_tc.so  CUDA kernels + C ABI + cuStinger-compatible C++ layer,
                                         nvcc -gencode arch=compute_100a,code=sm_100a
  custingeralg_b200/libtcgen.so          seeded graph generators, graph file readers and the binary
                                         CSR cache (host C++/OpenMP)

Usage: python -m custingeralg_b200.build [--force] [--verbose] [--define NAME=VALUE ...]

--define passes a preprocessor definition to every CUDA source: the kernels' tuning constants
(TC_HUB_UNIT, TC_HUB_ITEM_LOG2, TC_HUB_THREADS, TC_DELTA_MIN_BLOCKS) take their defaults unless
given, which is how their alternatives were measured. Use it with --force, and rebuild with
--force and no --define to return to the defaults.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-Wall", "-I", INCLUDE, "-I", CSRC]

LIB_TC = os.path.join(HERE, "libcustinger_tc.so")
LIB_GEN = os.path.join(HERE, "libtcgen.so")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)
    return r


def build_tc(force=False, verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "**", "*.h*"),
                                                                          recursive=True))
    objs = []
    jobs = []
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _newer(obj, [src] + headers):
            jobs.append([NVCC] + ARCH + NVCC_FLAGS + list(extra) + ["-c", src, "-o", obj])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            list(ex.map(lambda c: _run(c, verbose), jobs))
    if force or jobs or _newer(LIB_TC, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB_TC] + objs + ["-lcudart"], verbose)
    return LIB_TC


def build_gen(force=False, verbose=False):
    srcs = [os.path.join(CSRC, "tcgen.cpp"), os.path.join(CSRC, "tcgen_io.cpp")]
    hdrs = [os.path.join(INCLUDE, "tc_gen.h"), os.path.join(INCLUDE, "cuStingerDefs.hpp")]
    if force or _newer(LIB_GEN, srcs + hdrs):
        _run(["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-Wall"] + srcs + ["-o", LIB_GEN], verbose)
    return LIB_GEN


def build_all(force=False, verbose=False, defines=()):
    build_gen(force, verbose)
    build_tc(force, verbose, extra=[f"-D{d}" for d in defines])


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--define", action="append", default=[], metavar="NAME=VALUE",
                    help="preprocessor definition for the CUDA sources (a tuning constant)")
    a = ap.parse_args()
    build_all(a.force, a.verbose, a.define)
    print("built", LIB_TC, LIB_GEN)
