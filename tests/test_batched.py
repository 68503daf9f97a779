"""Batched solves under one CUDA graph (kfmm_batch_*), with leaf sizes and
launch choices from the autotuner: a smaller instance of the batched
workload (solves of uneven size, uniform cube and ellipsoid surface, NP 3 and
4, mixed form).

* every solve's potentials from the graph replay equal, bit for bit, those of
  the same plan run on its own (the kernels are deterministic), on two
  launches in a row;
* every solve's relative L2 error against an exact direct sum on sampled
  targets is at most 2x the plain FP64 form's error for the same tree.
"""
import numpy as np
import pytest


@pytest.mark.gpu
def test_batched_graph_matches_single_runs(K, oracle_mod, cuda_ok, tmp_path):
    from kifmm_b200 import autotune, batched
    table = autotune.ConfigTable(str(tmp_path / "configs.json"),
                                 knobs=(("job_rows", (0, 4)), ("nf_blocks", (0, 5))),
                                 candidates=(16, 32, 64))
    sp = batched.specs(12, nmin=4096, nmax=40000, seed=7)
    B = batched.BatchedSolves(K, sp, K.MIXED, table=table, nstreams=4, num_check=60)
    single = []
    for s in B.solves:
        s["plan"].run()
        single.append(s["plan"].potentials())
    for rep in range(2):
        B.launch()
        got = B.potentials()
        for i, (a, b) in enumerate(zip(got, single)):
            assert np.array_equal(a, b), f"solve {i} launch {rep}"
    for s, pot in zip(B.solves, single):
        pts = s["pts"]
        plain = K.Plan(s["tree"], s["np"], K.PLAIN_FP64).evaluate(pts)
        ids = pts["check_ids"]
        d = oracle_mod.direct(pts["tx"][ids], pts["ty"][ids], pts["tz"][ids], pts["sx"], pts["sy"],
                              pts["sz"], pts["den"])
        e_mixed = np.linalg.norm(pot[ids] - d) / np.linalg.norm(d)
        e_plain = np.linalg.norm(plain[ids] - d) / np.linalg.norm(d)
        print(f"{s['distribution']} n={s['n']} np={s['np']} ppb={s['ppb']}: mixed {e_mixed:.3e} "
              f"plain {e_plain:.3e}")
        assert e_mixed <= 2.0 * e_plain
    assert (tmp_path / "configs.json").exists()
    assert any(s["tuning"] is not None for s in B.solves)
    B.close()


def test_batch_rejects_bad_arguments(K):
    import ctypes
    h = ctypes.c_void_p()
    arr = (ctypes.c_void_p * 1)(None)
    assert K.lib().kfmm_batch_create(arr, 1, 1, ctypes.byref(h)) != 0
    assert K.lib().kfmm_batch_create(arr, 0, 1, ctypes.byref(h)) != 0
    assert K.lib().kfmm_batch_launch(None, None) != 0


def test_specs_follow_the_batched_workload():
    from kifmm_b200 import batched
    sp = batched.specs(256)
    ns = np.array([s["n"] for s in sp])
    assert ns.min() >= 4096 and ns.max() <= 262144
    assert sum(s["distribution"] == "uniform" for s in sp) == 128
    assert {s["np"] for s in sp} == {3, 4}
