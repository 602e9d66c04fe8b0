"""Build recipe of the engine: nvcc for sm_100a -> libmgagcd.so and MG_GCD.

Usage: python mg-alphagcd_b200/build.py [--force] [--jobs N]
Objects go to mg-alphagcd_b200/_build/ (git-ignored); the shared library and
the CLI binary are written next to this file.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
            "-ccbin", "/usr/bin/g++", "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]
SOURCES = ["primitives.cu", "bins.cu", "local_move.cu", "local_move_batch.cu", "coarsen.cu", "graph.cu",
           "louvain.cu", "batch.cu", "serve.cu", "capi.cu",
           "mtx.cpp", "noalloc.cu"]
LIB = os.path.join(HERE, "libmgagcd.so")
CLI = os.path.join(HERE, "MG_GCD")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
        os.path.join(ROOT, "include", "mgagcd.h")]


def _compile(src: str, force: bool) -> str:
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    if force or _newer(obj, [path] + _headers()):
        lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
        cmd = [NVCC] + ARCH + CXXFLAGS + lang + ["-c", path, "-o", obj]
        subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), SOURCES))
    if force or _newer(LIB, objs):
        subprocess.run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"], check=True)
    main = os.path.join(CSRC, "main.cpp")
    if force or _newer(CLI, [main, LIB, os.path.join(ROOT, "include", "mgagcd.h")]):
        subprocess.run(["/usr/bin/g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), main,
                        "-o", CLI, "-L", HERE, "-lmgagcd", "-Wl,-rpath,$ORIGIN"], check=True)
    if verbose:
        print(f"built {LIB} and {CLI}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=8)
    a = ap.parse_args()
    try:
        build(a.force, a.jobs, verbose=True)
    except subprocess.CalledProcessError as e:
        sys.exit(e.returncode)
