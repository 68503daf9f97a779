"""The drop-in binaries against the reference driver.

fmmd--b200-dropin is the reference's own driver, tree and operator code
(oracle/_ref, built from the reference sources) with this library in place of
the GPU evaluator; fmmd--b200 is this repository's stand-alone driver with the
same CLI and output lines.  Both must report the same "Relative error" (the
reference's direct-sum check, fmm/driver.cc:142-206) as fmmd--omp for the same
command line.

The reference driver's check accumulates into an array it never zeroes
(chkPot, fmm/driver.cc:157).  The reference binaries here run with
glibc.malloc.mmap_threshold=4096 and NV >= 512, so that array (8 NV bytes)
comes from fresh zeroed pages in every binary.
"""
import os
import re
import subprocess

import pytest

from refdump import REF_DIR, reference_env

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "kifmm--hybrid--double-only_b200", "fmmd--b200")
DROPIN = os.path.join(REF_DIR, "fmmd--b200-dropin")
REF_OMP = os.path.join(REF_DIR, "fmmd--omp")


def run(exe, args, **env):
    r = subprocess.run([exe] + [str(a) for a in args], env=reference_env(**env),
                       capture_output=True, text=True, timeout=600)
    return r


def rel_error(r):
    m = re.search(r"Relative error:\s*([0-9.eE+-]+)", r.stderr)
    assert m, r.stderr[-500:]
    return float(m.group(1))


def test_cli_usage_and_errors():
    r = subprocess.run([CLI], capture_output=True, text=True)
    assert r.returncode != 0 and "usage" in r.stderr
    r = subprocess.run([CLI, "100", "noSuchDistribution", "8"], capture_output=True, text=True)
    assert r.returncode != 0 and "unknown distribution" in r.stderr


CASES = [("uniform", 65536, 128, 4, 0), ("ellipseUniformAngles", 20000, 32, 3, 0),
         ("uniform", 30000, 64, 6, 1)]


@pytest.mark.gpu
@pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(REF_OMP)),
                    reason="oracle/_ref drop-in not built")
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1]}-{c[2]}-np{c[3]}-C{c[4]}")
def test_dropin_matches_reference_driver(case):
    dist, n, ppb, np_, c = case
    env = {"NP": str(np_), "NV": "600", "C": str(c)}
    ref = run(REF_OMP, [n, dist, ppb], **env)
    assert ref.returncode == 0, ref.stderr[-500:]
    e_ref = rel_error(ref)
    drop = run(DROPIN, [n, dist, ppb], **env)
    assert drop.returncode == 0, drop.stderr[-500:]
    assert "== Timing for FMM3d ==" in drop.stderr and "Code: b200-fp64" in drop.stdout
    e_drop = rel_error(drop)
    cli = run(CLI, [n, dist, ppb], **env)
    assert cli.returncode == 0, cli.stderr[-500:]
    e_cli = rel_error(cli)
    mixed = run(DROPIN, [n, dist, ppb], KFMM_MIXED="1", **env)
    assert mixed.returncode == 0, mixed.stderr[-500:]
    e_mixed = rel_error(mixed)
    print(f"{case}: reference {e_ref:.6e} drop-in {e_drop:.6e} fmmd--b200 {e_cli:.6e} "
          f"drop-in mixed {e_mixed:.6e}")
    # |e_a - e_b| <= max per-target relative deviation of the potentials
    # (triangle inequality), which is the FP64 rounding floor for the same
    # operators (~0.1^-(np+1) * 1e-17, see test_gpu_parity); plus the 7
    # significant digits the driver prints
    floor = 1e-17 * 10.0 ** (np_ + 1) * 20
    assert abs(e_drop - e_ref) <= 1e-6 * e_ref + floor
    # own pseudo-inverses: differences at the SVD's rounding level
    assert abs(e_cli - e_ref) <= 1e-6 * e_ref + 5 * floor
    assert e_mixed <= 2.0 * e_ref
