"""The autotuner (leaf size, then the kernels' launch choices by coordinate
descent) on a small surface cloud, and the table it ships for the batched
workload."""
import json
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TABLE = os.path.join(ROOT, "kifmm--hybrid--double-only_b200", "tuning_data",
                     "b200_batched_configs.json")


@pytest.mark.skipif(not os.path.exists(TABLE), reason="no tuning table")
def test_shipped_table_covers_the_batched_workload(K):
    from kifmm_b200 import autotune, batched
    with open(TABLE) as f:
        picks = json.load(f)
    fields = {n for n, _ in autotune.KNOBS}
    for prec in (K.MIXED, K.PLAIN_FP64):
        for sp in batched.specs(256):
            e = picks[autotune.ConfigTable.key(sp["distribution"], sp["n"], sp["np"], prec)]
            assert e["ppb"] in (32, 64, 128, 256)
            assert set(e["tuning"]) <= fields
            if prec != K.MIXED:
                assert not set(e["tuning"]) & set(autotune.MIXED_ONLY)


@pytest.mark.gpu
def test_tune_keeps_the_fastest_measured_config(K, cuda_ok):
    from kifmm_b200 import autotune
    pts = K.generate_points(60000, "ellipsoidSurface", 0, 3)
    knobs = (("job_rows", (0, 4)), ("nf_blocks", (0, 5, 6)), ("splitk_max", (0, 1)))
    r = autotune.tune(K, pts, 4, K.MIXED, candidates=(32, 64, 128), knobs=knobs)
    assert r["ppb"] in (32, 64, 128)
    measured = list(r["sweep"]["leaf"].values())
    for d in r["sweep"]["knobs"].values():
        measured += list(d.values())
    assert r["ms"] <= min(measured) * (1 + autotune.KEEP_GAIN) + 1e-9
    # launch choices other than the split-K factor do not change the
    # arithmetic: the tuned plan gives the automatic plan's potentials
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], r["ppb"])
    tun = {k: v for k, v in r["tuning"].items() if k != "splitk_max"}
    a = K.Plan(tree, 4, K.MIXED).evaluate(pts)
    b = K.Plan(tree, 4, K.MIXED, tuning=tun).evaluate(pts)
    assert np.array_equal(a, b)
    print(f"tuned: ppb {r['ppb']} {r['tuning']} {r['ms']:.3f} ms; sweep {r['sweep']}")


def test_plan_rejects_bad_tuning(K):
    pts = K.generate_points(2000, "uniform", 0, 1)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 32)
    for bad in ({"nf_blocks": 3}, {"job_rows": 7}, {"had_windows": 9}, {"splitk_max": -1}):
        with pytest.raises(K.KfmmError, match="tuning value out of range"):
            K.Plan(tree, 4, K.MIXED, tuning=bad)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_set_tuning_in_place(K, cuda_ok, precision):
    """Re-chunked near-field jobs, other resident-block counts and Hadamard
    shapes give the same potentials bit for bit; a different split-K factor
    reorders the level products' sums only: FP64 rounding, amplified by the
    pseudo-inverses' condition number, which the mixed form's FP32 rounding
    of spectra and sources then shows at its own level (~1e-7)."""
    prec = K.PLAIN_FP64 if precision == "plain" else K.MIXED
    pts = K.generate_points(50000, "uniform", 0, 9)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 64)
    want = K.Plan(tree, 6, prec).evaluate(pts)
    plan = K.Plan(tree, 6, prec)
    for cfg in ({"job_rows": 3}, {"job_rows": 1, "nf_blocks": 5, "had_windows": 2}, None):
        plan.set_tuning(cfg)
        assert np.array_equal(plan.evaluate(pts), want), cfg
    plan.set_tuning({"splitk_max": 1})
    got = plan.evaluate(pts)
    tol = 1e-9 if precision == "plain" else 1e-6
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < tol
