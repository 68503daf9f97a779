"""The benchmark configurations at their full sizes (GPU).

At these sizes the oracle takes too long, so the checks are the reference's
own size-independent one, the relative L2 error against an exact FP64 direct
sum on 1000 sampled targets (fmm/driver.cc:142-206; the direct sum runs on
the GPU through kfmm_direct_evaluation, which test_gpu_parity pins to the
oracle), and the agreement of the two precision forms:

  1,048,576 uniform points, NP=6, 512 per leaf: plain FP64 and mixed; the
      mixed form's error <= 2x the plain form's, both at the NP=6 truncation
      level (< 1e-6);
  4,194,304 points on the ellipsoid surface, NP=4, 256 per leaf (deep
      adaptive tree, W and X lists in use): the same two checks at NP=4.
"""
import numpy as np
import pytest

CONFIGS = [
    # (distribution, N, pts/box, NP, bound on the plain error)
    ("uniform", 1048576, 512, 6, 1e-6),
    ("ellipsoidSurface", 4194304, 256, 4, 1e-3),
]


def _direct(K, pts, ids):
    import torch
    dev = torch.device("cuda:0")
    src = [torch.tensor(pts[k], device=dev) for k in ("sx", "sy", "sz", "den")]
    trg = [torch.tensor(pts[k][ids], device=dev) for k in ("tx", "ty", "tz")]
    out = torch.zeros(len(ids), dtype=torch.float64, device=dev)
    K.check(K.lib().kfmm_direct_evaluation(len(ids), *[x.data_ptr() for x in trg], out.data_ptr(),
                                           len(pts["sx"]), *[x.data_ptr() for x in src], None),
            "direct")
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: f"{c[0]}-{c[1]}-ppb{c[2]}-np{c[3]}")
def test_config_full_size(K, cuda_ok, cfg):
    dist, n, ppb, np_, bound = cfg
    pts = K.generate_points(n, dist, 0, 26, 1000)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
    pot = {}
    for name, prec in (("plain", K.PLAIN_FP64), ("mixed", K.MIXED)):
        plan = K.Plan(tree, np_, prec)
        pot[name] = plan.evaluate(pts)
        plan.close()
    ids = pts["check_ids"]
    d = _direct(K, pts, ids)
    err = {k: float(np.linalg.norm(v[ids] - d) / np.linalg.norm(d)) for k, v in pot.items()}
    vs = float(np.linalg.norm(pot["mixed"] - pot["plain"]) / np.linalg.norm(pot["plain"]))
    st = tree.desc
    print(f"{dist} n={n} ppb={ppb} np={np_}: nodes {st.num_nodes}, rel-L2 vs direct plain "
          f"{err['plain']:.3e} mixed {err['mixed']:.3e}; mixed vs plain {vs:.3e}")
    assert np.all(np.isfinite(pot["mixed"])) and np.all(np.isfinite(pot["plain"]))
    assert err["plain"] < bound
    assert err["mixed"] <= 2.0 * err["plain"]
    tree.close()
