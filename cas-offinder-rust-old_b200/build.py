"""Builds libcof.so (the CUDA engine + C ABI) and the cof-offinder CLI in-tree.

Kernels are compiled for sm_100a only (B200).  Objects go to _build/ beside
this file; the shared library and CLI are written next to this file so they
travel with the source tree.  Rebuilds only what is older than its sources.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcof.so")
CLI = os.path.join(HERE, "cof-offinder")
PEAK_LIB = os.path.join(HERE, "libcof_peak.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
          "-I" + os.path.join(ROOT, "include")]
HEADERS = [os.path.join(CSRC, "cof_engine.h"), os.path.join(CSRC, "engine_dev.cuh"),
           os.path.join(CSRC, "textout.h"),
           os.path.join(ROOT, "include", "cof.h")]

SOURCES = ["engine.cu", "bulge.cu", "raw.cu", "loader.cpp", "cabi.cpp", "server.cpp", "noalloc.cu",
           "textout.cpp",
           "hostpool.cpp", "twobit.cu", "fasta_dev.cu"]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if _stale(obj, [path] + HEADERS):
            cmd = [NVCC] + ARCH + COMMON + ["-c", path, "-o", obj]
            if ptxas_info and src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            _run(cmd, verbose)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"], verbose)
    peak_src = os.path.join(CSRC, "intpeak.cu")
    if _stale(PEAK_LIB, [peak_src]):
        _run([NVCC] + ARCH + COMMON + ["-shared", peak_src, "-o", PEAK_LIB], verbose)
    cli_src = os.path.join(CSRC, "cli.cpp")
    if _stale(CLI, [cli_src, LIB] + HEADERS):
        _run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), cli_src,
              "-o", CLI, "-L" + HERE, "-lcof", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
