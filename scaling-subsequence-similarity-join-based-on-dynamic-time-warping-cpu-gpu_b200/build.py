"""Builds libdtwj.so (CUDA, sm_100a) and the `dtwj` CLI in-tree.

    python build.py            # incremental
    python build.py --clean    # from scratch

Outputs: lib/libdtwj.so, bin/dtwj (objects in _build/).  nvcc cross-compiles
sm_100a without a GPU, so this runs on any machine with the CUDA toolkit.
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
LIB = os.path.join(HERE, "lib")
BIN = os.path.join(HERE, "bin")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE]
CU_SOURCES = ["prep.cu", "mp.cu", "lb.cu", "runs.cu", "paa.cu", "pairs.cu", "petitjean.cu", "join.cu", "noalloc.cu", "mlp.cu",
              "features.cu", "load.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(src_list, dst) -> bool:
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(s) > t for s in src_list)


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
        os.path.join(INCLUDE, "dtwj.h")
    ]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def build(verbose: bool = False) -> str:
    nvcc = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    heads = _headers()
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if _newer([s] + heads, o):
            jobs.append([nvcc] + ARCH + NVCC_FLAGS + ["-c", s, "-o", o])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            for r in ex.map(_run, jobs):
                if verbose:
                    sys.stderr.write(r.stderr)
    so = os.path.join(LIB, "libdtwj.so")
    if _newer(objs, so):
        _run([nvcc] + ARCH + ["-shared", "-cudart=static", "-o", so] + objs)
    cli = os.path.join(BIN, "dtwj")
    cli_src = os.path.join(CSRC, "cli.cpp")
    if _newer([cli_src, so, os.path.join(INCLUDE, "dtwj.h")], cli):
        cxx = shutil.which("g++") or "g++"
        _run([cxx, "-O2", "-std=c++17", "-I" + INCLUDE, cli_src, "-o", cli, "-L" + LIB,
              "-ldtwj", "-Wl,-rpath,$ORIGIN/../lib"])
    return so


if __name__ == "__main__":
    if "--clean" in sys.argv:
        for d in (BUILD, LIB, BIN):
            shutil.rmtree(d, ignore_errors=True)
    print(build(verbose="-v" in sys.argv))
