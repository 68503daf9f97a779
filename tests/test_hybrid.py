"""Hybrid CPU+GPU evaluation (kfmm_tuning.cpu_share_ppm): the host's cores sum
the U lists of the cheapest target leaves in FP64 while the GPU runs the rest
of the solve, as the reference's run--hybrid2 schedule does with the whole U
list (fmm/run--hybrid2.cu:25-47).  The potentials must not depend on who sums
what: the plain form's hybrid result equals the all-GPU result to FP64
reordering, and stays within the parity bar against the oracle."""
import numpy as np
import pytest


def _plan(K, pts, ppb, np_, prec, share):
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
    return tree, K.Plan(tree, np_, prec, tuning={"cpu_share_ppm": share} if share else None)


def test_share_out_of_range_is_refused(K):
    pts = K.generate_points(3000, "uniform", 0, 1)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 32)
    for bad in (-1, 1000001):
        with pytest.raises(K.KfmmError, match="tuning value out of range"):
            K.Plan(tree, 4, K.PLAIN_FP64, tuning={"cpu_share_ppm": bad})


@pytest.mark.gpu
@pytest.mark.parametrize("share", [20000, 250000, 1000000])
def test_plain_hybrid_equals_gpu(K, oracle_mod, cuda_ok, share):
    pts = K.generate_points(30000, "uniform", 0, 26)
    tree, gpu = _plan(K, pts, 64, 4, K.PLAIN_FP64, 0)
    want = gpu.evaluate(pts)
    full = gpu.stats()["u_pairs"]
    hyb = K.Plan(tree, 4, K.PLAIN_FP64, tuning={"cpu_share_ppm": share})
    st = hyb.stats()
    got = hyb.evaluate(pts)
    d = float(np.max(np.abs(got - want) / np.abs(want)))
    tarrs = {k: tree.array(k) for k in oracle_mod.TREE_FIELDS}
    ref = oracle_mod.evaluate(tarrs, 4, K.operators(4), pts)
    e = float(np.max(np.abs(got - ref) / np.abs(ref)))
    print(f"share {share} ppm: host pairs {st['host_pairs']:.4g} of {full:.4g}; hybrid vs GPU "
          f"{d:.2e}; hybrid vs oracle {e:.2e}")
    assert st["host_pairs"] > 0
    assert st["host_pairs"] <= share * 1e-6 * full * (1.0 + 1e-12) or share == 1000000
    assert st["u_pairs"] < full
    assert d <= 1e-13
    assert e <= 1e-12


@pytest.mark.gpu
def test_mixed_hybrid_whole_u_list(K, oracle_mod, cuda_ok):
    """The reference's schedule: the whole U list on the host (FP64), the
    rest in the mixed form on the GPU; error against the exact direct sum
    within 2x the plain path's."""
    pts = K.generate_points(40000, "uniform", 0, 26, 300)
    tree, mixed = _plan(K, pts, 64, 6, K.MIXED, 0)
    m = mixed.evaluate(pts)
    hyb = K.Plan(tree, 6, K.MIXED, tuning={"cpu_share_ppm": 1000000})
    h = hyb.evaluate(pts)
    plain = K.Plan(tree, 6, K.PLAIN_FP64).evaluate(pts)
    ids = pts["check_ids"]
    d = oracle_mod.direct(pts["tx"][ids], pts["ty"][ids], pts["tz"][ids], pts["sx"], pts["sy"],
                          pts["sz"], pts["den"])
    e_plain = np.linalg.norm(plain[ids] - d) / np.linalg.norm(d)
    e_h = np.linalg.norm(h[ids] - d) / np.linalg.norm(d)
    vs = np.linalg.norm(h - m) / np.linalg.norm(m)
    print(f"whole U list on the host: rel-L2 vs direct {e_h:.3e} (plain {e_plain:.3e}); "
          f"vs all-GPU mixed {vs:.2e}")
    assert vs <= 1e-6
    assert e_h <= 2.0 * e_plain


@pytest.mark.gpu
def test_hybrid_plan_refuses_device_only_calls(K, cuda_ok):
    pts = K.generate_points(20000, "uniform", 0, 3)
    tree, hyb = _plan(K, pts, 64, 4, K.MIXED, 100000)
    hyb.set_points(pts)
    with pytest.raises(K.KfmmError, match="use kfmm_evaluate"):
        hyb.run()
    with pytest.raises(K.KfmmError, match="use kfmm_evaluate"):
        K.Batch([hyb], 1)
    assert np.all(np.isfinite(hyb.evaluate(pts)))
