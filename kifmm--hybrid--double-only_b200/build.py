"""Build recipe for libkifmm_b200.so and the fmmd--b200 driver (sm_100a).

Run as ``python kifmm--hybrid--double-only_b200/build.py`` or through
``__graft_entry__.build()``.  nvcc cross-compiles for sm_100a without a GPU.
Host C++ is compiled with -ffp-contract=off so the tree centres and operator
matrices round exactly like the reference's gcc -O3 -msse3 build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libkifmm_b200.so")
CLI = os.path.join(HERE, "fmmd--b200")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["plan.cu", "peaks.cu", "noalloc.cu", "tree.cc", "tree_gpu.cu", "operators.cc", "mlp.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
          "-Xcompiler", "-fPIC,-ffp-contract=off,-fopenmp"]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    deps = [os.path.join(CSRC, s) for s in os.listdir(CSRC)] + [
        os.path.join(ROOT, "include", "kifmm_b200.h"), __file__]
    if force or _stale(LIB, deps):
        objs = []
        for s in SOURCES:
            src = os.path.join(CSRC, s)
            obj = os.path.join(CSRC, s + ".o")
            _run([NVCC] + ARCH + COMMON + ["-c", src, "-o", obj], verbose)
            objs.append(obj)
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fopenmp",
                                                               "-lgomp"], verbose)
        for o in objs:
            os.remove(o)
    cli_src = os.path.join(CSRC, "fmmd_b200.cc")
    if os.path.exists(cli_src) and (force or _stale(CLI, [cli_src, LIB])):
        _run([NVCC] + ARCH + ["-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-Xcompiler",
              "-ffp-contract=off", cli_src, "-o", CLI, "-L", HERE, "-l:libkifmm_b200.so",
              "-Xlinker", "-rpath,$ORIGIN", "-lm"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
