"""Error reporting of the kernels' bounded waits, driven without a fault.

The mixed V list copies each frequency block's translation spectra into
shared memory with a bulk copy and waits on an mbarrier for a bounded number
of tries; when the tries run out the kernel sets the plan's error flag and
returns (after letting the copy land).  kfmm_set_wait_limit(plan, 0) makes
that wait give up at once, so the error path runs on every launch: the solve
must then report KFMM_ERR_CUDA through every call that hands back potentials,
and the next solve with the default limit must succeed with the same
potentials as an untouched plan (the flag is cleared at the start of each
solve).  The reference has no such path: it exits on any CUDA error
(fmm/cuda.cu:19-30).
"""
import numpy as np
import pytest


def _setup(K, n=20000, ppb=32, np_=4):
    pts = K.generate_points(n, "uniform", 0, 26)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
    return pts, tree


def test_set_wait_limit_rejects_null_plan(K):
    assert K.lib().kfmm_set_wait_limit(None, 0) == 1
    assert K.lib().kfmm_batch_wait(None, None) == 1


@pytest.mark.gpu
def test_wait_timeout_reported_then_cleared(K, cuda_ok):
    import torch
    pts, tree = _setup(K)
    want = K.Plan(tree, 4, K.MIXED).evaluate(pts)
    plan = K.Plan(tree, 4, K.MIXED)
    plan.set_wait_limit(0)
    with pytest.raises(K.KfmmError, match="bounded wait"):
        plan.evaluate(pts)
    plan.run()
    with pytest.raises(K.KfmmError, match="bounded wait"):
        plan.potentials()
    out = torch.empty(len(want), dtype=torch.float64, device="cuda:0")
    rc = K.lib().kfmm_get_potentials_device(plan.handle, out.data_ptr(), None)
    assert rc == 2 and b"bounded wait" in K.lib().kfmm_last_error()
    plan.set_wait_limit(-1)
    got = plan.evaluate(pts)
    assert np.array_equal(got, want)
    assert K.lib().kfmm_get_potentials_device(plan.handle, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), want)


@pytest.mark.gpu
def test_batch_wait_reports_timeout(K, cuda_ok):
    pts, tree = _setup(K, n=15000)
    plans = [K.Plan(tree, 4, K.MIXED) for _ in range(2)]
    for p in plans:
        p.set_points(pts)
    want = K.Plan(tree, 4, K.MIXED).evaluate(pts)
    plans[1].set_wait_limit(0)
    batch = K.Batch(plans, nstreams=2)  # the limit is captured with the launch
    batch.launch()
    with pytest.raises(K.KfmmError, match="solve 1"):
        batch.wait()
    batch.close()
    plans[1].set_wait_limit(-1)
    batch = K.Batch(plans, nstreams=2)
    batch.launch()
    batch.wait()
    for p in plans:
        assert np.array_equal(p.potentials(), want)
    batch.close()
