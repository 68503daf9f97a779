"""The allocation-free S2M entry point (kfmm_s2m_noalloc).

Some callers cannot allocate device memory when they call the solver: a host
framework that owns all device memory through its own pool, or a solver step
run while such a framework holds the memory budget.  For them
kfmm_s2m_noalloc turns source points into upward equivalent densities with
caller-provided buffers and a fixed scratch array inside the library.  This
test calls it through the C ABI twice in a row and checks both results
against the equivalent densities the regular plan computes for the same
leaves (kfmm_up_calc via kfmm_run), within the per-node tolerance the parity
tests use.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("np_,n,ppb", [(4, 30000, 64), (6, 40000, 96)])
def test_s2m_noalloc_matches_plan(K, cuda_ok, np_, n, ppb):
    import torch
    dev = torch.device("cuda:0")
    pts = K.generate_points(n, "uniform", 0, 26)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
    plan = K.Plan(tree, np_, K.PLAIN_FP64)
    plan.evaluate(pts)
    P, Q, _ = K.sizes(np_)
    nn = tree.desc.num_nodes
    ref = plan.read(0, nn * P).reshape(nn, P)

    child, tag, depth = tree.array("child"), tree.array("tag"), tree.array("depth")
    path = tree.array("path").reshape(-1, 3)
    leaves = np.where((child == -1) & (tag & 1))[0]
    assert len(leaves) * Q <= 1 << 20
    perm = tree.array("src_perm")
    src4 = np.stack([pts["sx"][perm], pts["sy"][perm], pts["sz"][perm], pts["den"][perm]], 1)
    beg = tree.array("src_beg")[leaves].astype(np.int32)
    num = tree.array("src_num")[leaves].astype(np.int32)
    scale = 1.0 / (1 << depth[leaves]).astype(np.float64)
    ctr = np.concatenate([-1.0 + (2.0 * 1.0) * (path[leaves] + 0.5) * scale[:, None],
                          scale[:, None]], 1)
    uc2ue = K.operators(np_)["uc2ue"]
    d_src = torch.tensor(src4.ravel(), device=dev)
    d_beg = torch.tensor(beg, device=dev)
    d_num = torch.tensor(num, device=dev)
    d_ctr = torch.tensor(ctr.ravel(), device=dev)
    d_op = torch.tensor(uc2ue, device=dev)
    tol = 50 * 2.2e-16 * 10.0 ** (np_ + 1)  # the parity tests' per-node tolerance
    outs = []
    for call in range(2):
        d_out = torch.full((len(leaves) * P,), np.nan, dtype=torch.float64, device=dev)
        K.check(K.lib().kfmm_s2m_noalloc(np_, len(leaves), d_src.data_ptr(), d_beg.data_ptr(),
                                         d_num.data_ptr(), d_ctr.data_ptr(), d_op.data_ptr(),
                                         d_out.data_ptr(), None), "s2m_noalloc")
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().reshape(len(leaves), P)
        want = ref[leaves]
        err = np.max(np.abs(got - want).max(axis=1) / np.abs(want).max(axis=1))
        print(f"np={np_} call {call}: {len(leaves)} leaves, max per-leaf rel diff {err:.2e}")
        assert np.all(np.isfinite(got)) and err <= tol
        outs.append(got)
    assert np.array_equal(outs[0], outs[1])


def test_s2m_noalloc_rejects_oversized_batch(K):
    rc = K.lib().kfmm_s2m_noalloc(6, 4000, 1, 1, 1, 1, 1, 1, None)  # 4000 * 296 > 2^20
    assert rc == 1 and b"exceeds the fixed scratch" in K.lib().kfmm_last_error()
