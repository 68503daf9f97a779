"""Numerical design checks on the CPU (no GPU): why the level products stay
FP64 in the mixed form.

The check-to-equivalent operators are pseudo-inverses with condition bound
0.1^-(np+1) (1e7 at NP=6); their products cancel heavily.  Carrying the
operator products (S2M/M2M/L2L matrix-vector products) in FP32, or as
split-TF32 three-pass products with FP32 accumulation, wrecks the potentials,
while the FMM's own FP64 error is ~2e-7 at NP=6.  The mixed form therefore
keeps those products in FP64 (DMMA) and uses FP32 only where it measures
harmless: the P2P sums and the V-list Hadamard products.
"""
import numpy as np
import pytest


@pytest.mark.parametrize("np_,n,ppb", [(6, 30000, 128), (4, 20000, 64)])
def test_reduced_precision_level_products_are_not_viable(K, oracle_mod, np_, n, ppb):
    pts = K.generate_points(n, "uniform", 0, 26, 300)
    t = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
    tree = {k: t.array(k) for k in oracle_mod.TREE_FIELDS}
    ops = K.operators(np_)
    ref = oracle_mod.evaluate(tree, np_, ops, pts)
    ids = pts["check_ids"]
    d = oracle_mod.direct(pts["tx"][ids], pts["ty"][ids], pts["tz"][ids], pts["sx"], pts["sy"],
                          pts["sz"], pts["den"])
    e_fp64 = np.linalg.norm(ref[ids] - d) / np.linalg.norm(d)
    for mode in (1, 2):
        pot = oracle_mod.evaluate_reduced_products(tree, np_, ops, pts, mode)
        e = np.linalg.norm(pot[ids] - d) / np.linalg.norm(d)
        print(f"np={np_} mode {mode}: rel-L2 vs direct {e:.2e} (FP64 products {e_fp64:.2e})")
        assert e > 2.0 * e_fp64  # fails the mixed form's accuracy bar
