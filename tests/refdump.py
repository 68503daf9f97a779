"""Reader for the binary dumps written by oracle/ref_harness.cc and helpers
to run the reference build (oracle/_ref) from tests.

Record layout: name (32 bytes, NUL padded), dtype (int32: 0 float64,
1 int32), count (int64), payload.
"""
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def read_dump(path):
    out = {}
    with open(path, "rb") as f:
        while True:
            head = f.read(32)
            if len(head) < 32:
                break
            name = head.split(b"\0", 1)[0].decode()
            dtype = np.frombuffer(f.read(4), np.int32)[0]
            count = int(np.frombuffer(f.read(8), np.int64)[0])
            dt = np.float64 if dtype == 0 else np.int32
            out[name] = np.frombuffer(f.read(count * np.dtype(dt).itemsize), dt).copy()
    return out


def harness(variant="omp"):
    return os.path.join(REF_DIR, f"ref_harness--{variant}")


def have_reference_build(variant="omp"):
    return os.path.exists(harness(variant))


def reference_env(**kw):
    """Environment for reference runs: large allocations from fresh zeroed
    pages, because compute_fft_src (fmm/omp.cc:396-397) never zeroes its
    regular-grid buffer."""
    env = dict(os.environ, GLIBC_TUNABLES="glibc.malloc.mmap_threshold=4096")
    env.update(kw)
    return env


def run_reference(n, dist, ppb, np_, out_path, coincide=0, nv=100, variant="omp",
                  tree_only=False, threads=None, reverse_sums=False):
    """reverse_sums: the oracle build's FFTW and MKL stand-ins sum in reverse
    order (KFMM_SHIM_SUM_ORDER=1), a legal reordering those libraries do not
    rule out; the distance between the two runs is the reference's own FP64
    rounding floor."""
    env = reference_env(NP=str(np_), C=str(coincide), NV=str(nv))
    env["KFMM_SHIM_SUM_ORDER"] = "1" if reverse_sums else "0"
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    cmd = [harness(variant), str(n), dist, str(ppb), out_path] + (["tree"] if tree_only else [])
    subprocess.run(cmd, env=env, check=True, stdout=subprocess.DEVNULL,
                   stderr=subprocess.DEVNULL)
    return read_dump(out_path)
