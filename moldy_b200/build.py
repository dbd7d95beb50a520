"""Builds libmoldy_gpu.so in-tree with nvcc for sm_100a.

Each source is compiled to its own object (in parallel, one nvcc per file)
under moldy_b200/_build/, then linked into the shared library."""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmoldy_gpu.so")
SOURCES = ["api.cu", "cells.cu", "nlist.cu", "eam.cu", "pairs.cu", "noalloc.cu", "adjoint.cu", "batch.cu", "rdf.cu", "tables.cpp"]
HEADERS = ["common.cuh", "engine.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off",
    "-Xptxas", "-warn-spills",
]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "moldy_gpu.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def _nvcc() -> list:
    cmd = [os.environ.get("NVCC", "nvcc")]
    # nvcc's host compiler: the system g++ (a CC/CXX from the environment may
    # point at a wrapper without the full runtime)
    if os.path.exists("/usr/bin/g++"):
        cmd += ["-ccbin", "/usr/bin/g++"]
    return cmd


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    objs = [os.path.join(OBJ, os.path.splitext(f)[0] + ".o") for f in SOURCES]
    jobs = [_nvcc() + NVCC_FLAGS + ["-c", os.path.join(CSRC, f), "-o", o] for f, o in zip(SOURCES, objs)]
    if verbose:
        for j in jobs:
            print(" ".join(j), file=sys.stderr)

    def run(cmd):
        return subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as pool:
        results = list(pool.map(run, jobs))
    for r in results:
        if r.stderr:
            print(r.stderr, end="", file=sys.stderr)
    bad = [j for j, r in zip(jobs, results) if r.returncode != 0]
    if bad:
        raise subprocess.CalledProcessError(1, bad[0])
    link = _nvcc() + ["-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs, "-lcudart"]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
