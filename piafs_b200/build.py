"""Build the native library and CLI of the GPU path (nvcc, sm_100a).

Produces, in-tree:
  piafs_b200/libpiafs_gpu.so   the C-ABI library (include/piafs_gpu.h)
  piafs_b200/bin/piafs-gpu     command-line drop-in for the reference binary
  piafs_b200/libpiafs_hypar.so the entry points on the reference's own
                               simulation objects (include/piafs_hypar.h);
                               built when the reference's include/ is found
                               (PIAFS_REF names its source tree), because it
                               takes the layout of HyPar and the other
                               structures from those headers
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
HYPAR_LIB = os.path.join(HERE, "libpiafs_hypar.so")
CUDA_INC = "/usr/local/cuda/include"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
SOURCES = ["kernels.cu", "crweno.cu", "crweno_line.cu", "crweno_char.cu", "api.cu", "deck.cpp", "noalloc.cu", "batch.cu", "batch_stage_fp64.cu",
           "batch_stage_mixed.cu", "slab.cu"]


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
    build_hypar(force, verbose)
    return LIB


def reference_include():
    """The reference's include/ directory, if its source tree is named by
    PIAFS_REF and present."""
    ref = os.environ.get("PIAFS_REF")
    if ref and os.path.exists(os.path.join(ref, "include", "hypar.h")):
        return os.path.join(ref, "include")
    return None


def build_hypar(force: bool = False, verbose: bool = False):
    """libpiafs_hypar.so from csrc/hypar_attach.cpp, compiled with the
    reference's headers in their single-rank (-Dserial) layout."""
    inc = reference_include()
    src = os.path.join(CSRC, "hypar_attach.cpp")
    # it links libpiafs_gpu.so dynamically: only the structures it shares
    # with the library (these headers) make it stale
    deps = [src, os.path.join(HERE, "..", "include", "piafs_hypar.h"), os.path.join(HERE, "..", "include", "piafs_gpu.h"),
            os.path.join(CSRC, "deck.h"), os.path.join(CSRC, "common.cuh"), os.path.join(CSRC, "kernels.h")]
    if inc is None:
        # without the reference's headers it cannot be rebuilt; one built
        # against older library structures must not be loaded
        if os.path.exists(HYPAR_LIB) and _stale(HYPAR_LIB, deps):
            sys.stderr.write("removing " + HYPAR_LIB + ": older than the library and no PIAFS_REF to rebuild it\n")
            os.remove(HYPAR_LIB)
        return None
    if not (force or _stale(HYPAR_LIB, deps)):
        return HYPAR_LIB
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Dserial", "-I" + inc, "-I" + CUDA_INC, src,
           "-o", HYPAR_LIB, "-L" + HERE, "-lpiafs_gpu", "-L/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if verbose:
        sys.stdout.write(r.stdout + r.stderr)
    return HYPAR_LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
