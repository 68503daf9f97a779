"""kfmm_evaluate_async: back-to-back solves on one plan with different inputs.

Each call's host->device copies run while the previous call's solve is still
on the GPU, through the plan's single set of staging and device buffers; the
events between the plan's streams must keep every call's inputs and outputs
apart.  Three calls with different densities, queued without waiting, must
give exactly the potentials of three synchronous kfmm_evaluate calls (same
kernels, same order of operations: bit for bit).
"""
import ctypes

import numpy as np
import pytest


def _cargs(d, out):
    fp = ctypes.POINTER(ctypes.c_double)
    return [ctypes.cast(d[k].data_ptr(), fp) for k in ("sx", "sy", "sz", "den", "tx", "ty",
                                                       "tz")] + [ctypes.cast(out.data_ptr(), fp)]


def test_async_entry_points_reject_null(K):
    assert K.lib().kfmm_evaluate_join(None, None) == 1
    assert K.lib().kfmm_evaluate_wait(None, None) == 1
    assert K.lib().kfmm_evaluate_async(None, *([None] * 8), None) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_async_back_to_back_matches_sync(K, cuda_ok, precision):
    import torch
    prec = K.PLAIN_FP64 if precision == "plain" else K.MIXED
    n = 60000
    base = K.generate_points(n, "uniform", 0, 26)
    tree = K.Tree(base["sx"], base["sy"], base["sz"], base["tx"], base["ty"], base["tz"], 64)
    plan = K.Plan(tree, 4, prec)
    rng = np.random.default_rng(1)
    inputs = []
    for c in range(3):  # same points (the plan's tree), different densities
        d = dict(base)
        d["den"] = base["den"] * (c + 1) + rng.uniform(-1, 1, n)
        inputs.append(d)
    want = [plan.evaluate(d) for d in inputs]
    pinned = [{k: torch.from_numpy(np.ascontiguousarray(d[k])).pin_memory()
               for k in ("sx", "sy", "sz", "den", "tx", "ty", "tz")} for d in inputs]
    outs = [torch.full((n,), np.nan, dtype=torch.float64).pin_memory() for _ in inputs]
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # twice, so the second round also follows queued work
        for d, o in zip(pinned, outs):
            K.check(K.lib().kfmm_evaluate_async(plan.handle, *_cargs(d, o), stream),
                    "evaluate_async")
        K.check(K.lib().kfmm_evaluate_wait(plan.handle, stream), "evaluate_wait")
        for w, o in zip(want, outs):
            assert np.array_equal(o.numpy(), w)
        for o in outs:
            o.fill_(np.nan)
