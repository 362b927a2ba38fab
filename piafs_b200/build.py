"""Build the native library and CLI of the GPU path (nvcc, sm_100a).

Produces, in-tree:
  piafs_b200/libpiafs_gpu.so   the C-ABI library (include/piafs_gpu.h)
  piafs_b200/bin/piafs-gpu     command-line drop-in for the reference binary
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpiafs_gpu.so")
CLI = os.path.join(HERE, "bin", "piafs-gpu")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
SOURCES = ["kernels.cu", "crweno.cu", "crweno_line.cu", "crweno_char.cu", "api.cu", "deck.cpp", "noalloc.cu", "batch.cu", "batch_stage_fp64.cu",
           "batch_stage_mixed.cu"]


def _nvcc():
    for c in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if os.path.sep not in c or os.path.exists(c):
            return c
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "piafs_gpu.h"))
    nvcc = _nvcc()
    jobs = []
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            lang = [] if src.endswith(".cu") else ["-x", "cu"] if False else []
            jobs.append([nvcc] + ARCH + FLAGS + lang + ["-c", s, "-o", o])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose:
            sys.stdout.write(r.stdout + r.stderr)

    with ThreadPoolExecutor(max_workers=len(jobs) or 1) as ex:
        list(ex.map(run, jobs))
    if force or _stale(LIB, objs):
        run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    main = os.path.join(CSRC, "main_cli.cpp")
    if force or _stale(CLI, [main, LIB]):
        run([nvcc] + ARCH + ["-O2", "-std=c++17", "-o", CLI, main, "-L" + HERE, "-lpiafs_gpu",
                             "-Xlinker", "-rpath,$ORIGIN/.."])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
