"""Generates the golden fixtures in this folder from the reference build.

Runs oracle/_ref/ref_harness--omp (the reference fmm/omp.cc evaluator compiled
from its own sources, see oracle/Makefile) on small cases and stores, per case,
the tree and lists, the leaf-order permutations, the operator matrices (NP 3
and 4 only; NP 6 keeps checksums), the per-node expansions on a subset of
nodes, the potentials, and the reference's own direct-sum check.  Points are
not stored: they are regenerated from the reference generator (srand48(26)).

  python tests/golden/make_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from refdump import run_reference  # noqa: E402

CASES = [
    # name, distribution, N, pts/box, NP, coincide
    ("uniform_n8192_ppb64_np4", "uniform", 8192, 64, 4, 0),
    ("ellipse_n6000_ppb24_np3", "ellipseUniformAngles", 6000, 24, 3, 0),
    ("uniform_n6000_ppb32_np6", "uniform", 6000, 32, 6, 0),
    ("ellipsoid_n8000_ppb40_np4", "ellipsoidSurface", 8000, 40, 4, 0),
    ("uniform_n4096_ppb128_np4_C1", "uniform", 4096, 128, 4, 1),
]
TREE = ("parent", "child", "depth", "tag", "path", "src_beg", "src_num", "trg_beg", "trg_num",
        "src_perm", "trg_perm", "node_level", "u_ptr", "u_idx", "v_ptr", "v_idx", "w_ptr",
        "w_idx", "x_ptr", "x_idx")


def main():
    for name, dist, n, ppb, np_, c in CASES:
        with tempfile.TemporaryDirectory() as td:
            R = run_reference(n, dist, ppb, np_, os.path.join(td, "r.bin"), c, nv=200)
        out = {k: R[k].astype(np.int32) for k in TREE}
        out["meta"] = np.array([n, ppb, np_, c], np.int32)
        out["dist"] = np.array(dist)
        out["pot"] = R["pot"]
        out["check_ids"] = R["check_ids"]
        out["check_direct"] = R["check_direct"]
        P = int(R["sizes"][0])
        nn = len(R["parent"])
        sel = np.arange(0, nn, max(1, nn // 64))
        out["sel_nodes"] = sel.astype(np.int32)
        for k in ("src_upw_equ_den", "trg_dwn_chk_val", "trg_dwn_equ_den"):
            out[k + "_sel"] = R[k].reshape(nn, P)[sel]
        if np_ <= 4:
            out["uc2ue"] = R["uc2ue"]
            out["dc2de"] = R["dc2de"]
            out["ue2uc_0"] = R["ue2uc_0"]
            out["de2dc_7"] = R["de2dc_7"]
        out["ue2dc_checksum"] = np.array([np.sum(R["ue2dc"]), np.sum(np.abs(R["ue2dc"]))])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "nodes", nn, "W", len(R["w_idx"]), "X", len(R["x_idx"]))


if __name__ == "__main__":
    main()
