"""GPU parity: the sm_100a path through the C ABI against the oracle (the
restated fmm/omp.cc evaluator, itself pinned bit-exactly to the reference
build) on the same tree, points and operators, phase by phase and end to end,
and against the reference CPU build itself where oracle/_ref is present.

Tolerances (plain FP64 path):
  potentials  : max over targets of |phi_gpu - phi_ref| / |phi_ref| (for the
                signed-density ellipsoid, / max|phi_ref|: per-target relative
                error is not defined where the potential crosses zero)
                <= max(1e-12, 2 * floor).  Against the reference build, floor
                is the same measure between two runs of the reference itself
                whose only difference is the summation order inside the
                third-party routines it calls (FFTW's transforms, MKL's
                matrix-vector products; KFMM_SHIM_SUM_ORDER), which those
                libraries leave open.  Against the oracle, floor is the oracle
                vs itself with every sum reversed.  Either floor is the
                algorithm's own FP64 rounding level: the check-to-equivalent
                pseudo-inverses amplify any reordering by up to their condition
                number 0.1^-(np+1); it is below 1e-12 for NP <= 4 and ~5e-11
                to 7e-11 at NP = 6.
  per-node expansions: max|d| <= 50 eps kappa * max|ref| per node, kappa =
                0.1^-(np+1) the pseudo-inverse's condition bound: a rounding
                difference in a check potential reaches the equivalent density
                amplified by up to kappa, and is filtered out again on the way
                to the potentials.
"""
import os
import tempfile

import numpy as np
import pytest

from refdump import have_reference_build, run_reference

CASES = [
    # (distribution, N, pts/box, NP, coincide)
    ("uniform", 20000, 64, 4, 0),
    ("ellipseUniformAngles", 20000, 32, 3, 0),
    ("uniform", 30000, 128, 6, 0),
    ("ellipsoidSurface", 30000, 48, 4, 0),
    ("uniform", 12000, 40, 5, 1),
    ("ellipseUniformAngles", 6000, 16, 8, 0),
    ("uniform", 65536, 128, 4, 1),  # the CPU-runnable benchmark configuration (fmmd--omp)
    ("uniform", 8000, 24, 7, 0),
]
# the metric's NP and leaf size (512 per box) at a size the reference runs in
# seconds: depth 3-4 adaptive tree, V lists at depths 2-4, W and X lists
REF_CASES = CASES + [("uniform", 262144, 512, 6, 0)]


def _ids(c):
    return f"{c[0]}-{c[1]}-ppb{c[2]}-np{c[3]}-C{c[4]}"


def _pot_err(pot, ref, signed):
    d = np.abs(pot - ref)
    if signed:
        return float(d.max() / np.abs(ref).max())
    return float((d / np.abs(ref)).max())


def _node_err(a, b, P, nodes):
    a = a.reshape(-1, P)[nodes]
    b = b.reshape(-1, P)[nodes]
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return float((np.abs(a - b).max(axis=1) / scale).max()) if len(nodes) else 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_plain_fp64_vs_oracle(K, oracle_mod, cuda_ok, case):
    dist, n, ppb, np_, coincide = case
    pts = K.generate_points(n, dist, coincide, 26)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
    plan = K.Plan(tree, np_, K.PLAIN_FP64)
    pot = plan.evaluate(pts)
    ops = K.operators(np_)
    tarrs = {k: tree.array(k) for k in oracle_mod.TREE_FIELDS}
    ref, (ud, dc, dd) = oracle_mod.evaluate(tarrs, np_, ops, pts, want_phases=True)
    P, _, _ = K.sizes(np_)
    nn = tree.desc.num_nodes
    tag = tarrs["tag"]
    # equivalent densities above depth 2 are never read and not computed
    src_nodes = np.where((tag & 1) & (tarrs["depth"] >= 2))[0]
    trg_nodes = np.where(tag & 2)[0]
    e_ud = _node_err(plan.read(0, nn * P), ud, P, src_nodes)
    e_dc = _node_err(plan.read(1, nn * P), dc, P, trg_nodes)
    e_dd = _node_err(plan.read(2, nn * P), dd, P, trg_nodes)
    e_pot = _pot_err(pot, ref, dist == "ellipsoidSurface")
    floor = _pot_err(oracle_mod.evaluate_reordered(tarrs, np_, ops, pts), ref,
                     dist == "ellipsoidSurface")
    print(f"{_ids(case)}: uden {e_ud:.2e} dchk {e_dc:.2e} dden {e_dd:.2e} pot {e_pot:.2e} "
          f"(floor {floor:.2e})")
    tol_exp = 50 * 2.2e-16 * 10.0 ** (np_ + 1)
    assert e_ud <= tol_exp and e_dc <= tol_exp and e_dd <= tol_exp
    assert e_pot <= max(1e-12, 2 * floor)


@pytest.mark.gpu
@pytest.mark.skipif(not have_reference_build(), reason="oracle/_ref not built")
@pytest.mark.parametrize("case", REF_CASES, ids=_ids)
def test_plain_fp64_vs_reference_build(K, oracle_mod, cuda_ok, case):
    """End to end against fmmd--omp itself, run here from oracle/_ref.  With
    the reference's own operator matrices handed to the plan (as the drop-in
    preproc does) the potentials agree to 1e-12 per target (NP <= 4), or to
    twice the reference's own reordering floor (NP >= 5); with this library's
    own pseudo-inverses (one-sided Jacobi instead of LAPACK DGESVD) they agree
    to the SVD's rounding times kappa."""
    dist, n, ppb, np_, coincide = case
    with tempfile.TemporaryDirectory() as td:
        R = run_reference(n, dist, ppb, np_, os.path.join(td, "r.bin"), coincide, nv=200)
        R2 = run_reference(n, dist, ppb, np_, os.path.join(td, "r2.bin"), coincide, nv=200,
                           reverse_sums=True)
    pts = {k: R[k] for k in ("sx", "sy", "sz", "den", "tx", "ty", "tz")}
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
    for k in ("child", "tag", "src_perm", "trg_perm", "u_idx", "v_idx", "w_idx", "x_idx"):
        assert np.array_equal(tree.array(k), R[k]), k
    signed = dist == "ellipsoidSurface"
    plan = K.Plan(tree, np_, K.PLAIN_FP64, operators=oracle_mod.ops_from_dump(R))
    pot = plan.evaluate(pts)
    e_same_ops = _pot_err(pot, R["pot"], signed)
    plan.close()
    plan = K.Plan(tree, np_, K.PLAIN_FP64)
    pot_own = plan.evaluate(pts)
    e_own_ops = _pot_err(pot_own, R["pot"], signed)
    floor = _pot_err(R2["pot"], R["pot"], signed)  # the reference's own floor
    print(f"{_ids(case)}: vs reference build: {e_same_ops:.2e} (reference operators), "
          f"{e_own_ops:.2e} (own operators), reference reordering floor {floor:.2e}")
    assert e_same_ops <= max(1e-12, 2 * floor)
    assert e_own_ops <= max(1e-12, 5 * floor)
    # the reference's own check, rel-L2 against the exact direct sum: no worse
    # than the reference's by more than the largest per-target deviation
    # (triangle inequality)
    ids = R["check_ids"]
    err = np.linalg.norm(pot[ids] - R["check_direct"]) / np.linalg.norm(pot[ids])
    ref_err = np.linalg.norm(R["pot"][ids] - R["check_direct"]) / np.linalg.norm(R["pot"][ids])
    assert err <= ref_err + 1.01 * e_same_ops + 1e-15


@pytest.mark.gpu
def test_direct_evaluation_entry(K, oracle_mod, cuda_ok):
    import torch
    rng = np.random.default_rng(3)
    nt, ns = 777, 1500
    t = rng.uniform(-1, 1, (3, nt))
    s = rng.uniform(-1, 1, (4, ns))
    s[:3, :5] = t[:, :5]  # coincident pairs are skipped
    s[3] = np.abs(s[3])
    dev = torch.device("cuda:0")
    T = [torch.tensor(v, device=dev) for v in t]
    Sd = [torch.tensor(v, device=dev) for v in s]
    pot = torch.full((nt,), 0.5, dtype=torch.float64, device=dev)
    K.check(K.lib().kfmm_direct_evaluation(nt, *[x.data_ptr() for x in T], pot.data_ptr(), ns,
                                           *[x.data_ptr() for x in Sd], None), "direct")
    torch.cuda.synchronize()
    ref = oracle_mod.direct(*t, *s) + 0.5
    assert np.max(np.abs(pot.cpu().numpy() - ref) / np.abs(ref)) <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_leaf_order_potentials(K, cuda_ok, precision):
    """kfmm_read_array(3) gives the potentials in leaf order, pot_leaf[i] =
    pot[trg_perm[i]], in both forms (the mixed near field stores original
    order itself; the leaf-order view is gathered on demand)."""
    prec = K.PLAIN_FP64 if precision == "plain" else K.MIXED
    pts = K.generate_points(12000, "ellipseUniformAngles", 0, 5)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 24)
    plan = K.Plan(tree, 4, prec)
    pot = plan.evaluate(pts)
    leaf = plan.read(3, len(pot))
    assert np.array_equal(leaf, pot[tree.array("trg_perm")])


@pytest.mark.gpu
def test_repeat_runs_identical(K, cuda_ok):
    """Same inputs, same plan: bitwise-identical results run to run."""
    pts = K.generate_points(15000, "ellipseUniformAngles", 0, 7)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 24)
    plan = K.Plan(tree, 4, K.PLAIN_FP64)
    a = plan.evaluate(pts)
    plan.run()
    b = plan.potentials()
    assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_adjacent_translation_spectra_ignored(K, cuda_ok, precision):
    """Offsets with |delta|_inf <= 1 are adjacent boxes, never V-list pairs
    (fmm/omp_sse_block.cc:581-593 visits V-list members only), and the window
    kernels skip them: a supplied translation table with garbage there gives
    the same potentials, bit for bit, as the plan's own table."""
    prec = K.PLAIN_FP64 if precision == "plain" else K.MIXED
    np_ = 4
    pts = K.generate_points(20000, "ellipsoidSurface", 0, 11)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 32)
    ops = K.operators(np_)
    F = K.sizes(np_)[2]
    bad = {k: v.copy() for k, v in ops.items()}
    t = bad["ue2dc"].reshape(343, 2 * F)
    rng = np.random.default_rng(5)
    for i3 in (-1, 0, 1):
        for i2 in (-1, 0, 1):
            for i1 in (-1, 0, 1):
                t[(i1 + 3) + 7 * (i2 + 3) + 49 * (i3 + 3)] = rng.normal(size=2 * F) * 1e3
    a = K.Plan(tree, np_, prec, operators=ops).evaluate(pts)
    b = K.Plan(tree, np_, prec, operators=bad).evaluate(pts)
    assert np.array_equal(a, b)


MIXED_CASES = [("uniform", 65536, 128, 6, 0), ("uniform", 60000, 64, 4, 1),
               ("ellipsoidSurface", 60000, 40, 4, 0), ("ellipseUniformAngles", 40000, 24, 5, 0),
               ("uniform", 40000, 32, 3, 0), ("uniform", 30000, 48, 7, 0),
               ("uniform", 20000, 48, 8, 0)]
# The mixed form's own rounding floor: FP32 pair terms, spectra and
# Hadamard products leave ~1e-7 of the potentials; where the plain path's
# error lies below that (NP >= 7) the mixed form's error is that floor.
MIXED_FLOOR = 3e-7


@pytest.mark.gpu
@pytest.mark.parametrize("case", MIXED_CASES, ids=_ids)
def test_mixed_precision_accuracy(K, oracle_mod, cuda_ok, case):
    """The mixed form (FP32 + compensated sums, FP64 final accumulation) is
    measured by the reference's own check, the relative L2 error against an
    exact FP64 direct sum on sampled targets: it must stay within 2x the
    plain FP64 path's error, or within the mixed form's own rounding floor
    (3e-7) where the plain error is smaller still (NP >= 7); its distance to
    the plain path is reported."""
    dist, n, ppb, np_, coincide = case
    pts = K.generate_points(n, dist, coincide, 26, 400)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
    plain = K.Plan(tree, np_, K.PLAIN_FP64).evaluate(pts)
    mixed = K.Plan(tree, np_, K.MIXED).evaluate(pts)
    ids = pts["check_ids"]
    d = oracle_mod.direct(pts["tx"][ids], pts["ty"][ids], pts["tz"][ids], pts["sx"], pts["sy"],
                          pts["sz"], pts["den"])
    e_plain = np.linalg.norm(plain[ids] - d) / np.linalg.norm(d)
    e_mixed = np.linalg.norm(mixed[ids] - d) / np.linalg.norm(d)
    vs_plain = np.linalg.norm(mixed - plain) / np.linalg.norm(plain)
    print(f"{_ids(case)}: rel-L2 vs direct: plain {e_plain:.3e} mixed {e_mixed:.3e}; "
          f"mixed vs plain {vs_plain:.3e}")
    assert np.all(np.isfinite(mixed))
    assert e_mixed <= max(2.0 * e_plain, MIXED_FLOOR)


@pytest.mark.gpu
def test_mixed_precision_deep_cluster(K, oracle_mod, cuda_ok):
    """A tight cluster inside a uniform background drives the leaves to depth
    ~17, where the mixed form's FP32 source offsets (relative to each leaf's
    centre, plus the exact offset between centres) matter most: its rel-L2
    error against the exact direct sum, on targets inside and outside the
    cluster, stays within 2x the plain path's."""
    rng = np.random.default_rng(17)

    def cloud():
        bg = rng.uniform(-1.0, 1.0, (30000, 3))
        cl = np.array([0.1, -0.2, 0.3]) + rng.normal(0.0, 2e-5, (20000, 3))
        return np.concatenate([bg, cl])

    s, t = cloud(), cloud()
    pts = {"sx": s[:, 0].copy(), "sy": s[:, 1].copy(), "sz": s[:, 2].copy(),
           "tx": t[:, 0].copy(), "ty": t[:, 1].copy(), "tz": t[:, 2].copy(),
           "den": rng.uniform(0.0, 1.0, len(s))}
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 32)
    depth = int(tree.array("depth").max())
    assert 14 <= depth <= 20, depth
    plain = K.Plan(tree, 4, K.PLAIN_FP64).evaluate(pts)
    mixed = K.Plan(tree, 4, K.MIXED).evaluate(pts)
    ids = np.concatenate([rng.choice(30000, 200, replace=False),
                          30000 + rng.choice(20000, 200, replace=False)])
    d = oracle_mod.direct(pts["tx"][ids], pts["ty"][ids], pts["tz"][ids], pts["sx"], pts["sy"],
                          pts["sz"], pts["den"])
    e_plain = np.linalg.norm(plain[ids] - d) / np.linalg.norm(d)
    e_mixed = np.linalg.norm(mixed[ids] - d) / np.linalg.norm(d)
    print(f"deep cluster (depth {depth}): rel-L2 vs direct: plain {e_plain:.3e} "
          f"mixed {e_mixed:.3e}")
    assert np.all(np.isfinite(mixed))
    assert e_mixed <= 2.0 * e_plain


@pytest.mark.gpu
@pytest.mark.parametrize("case", [("uniform", 65536, 128, 6, 0), ("ellipsoidSurface", 60000, 40, 4, 0),
                                  ("ellipseUniformAngles", 20000, 32, 3, 0)], ids=_ids)
def test_mixed_downward_check_vs_plain(K, cuda_ok, case):
    """The mixed form's V list (FP32 spectra and products, half-window sums in
    FP64) and S2L (FP32 P2P) against the plain path, on the downward check
    potentials they produce: per node max|d| / max|plain| <= 2e-5 (FP32
    rounding of the spectra and terms, ~6e-8 each, summed over up to 189
    V-list boxes)."""
    dist, n, ppb, np_, coincide = case
    pts = K.generate_points(n, dist, coincide, 26)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
    P, _, _ = K.sizes(np_)
    nn = tree.desc.num_nodes
    out = {}
    for prec in (K.PLAIN_FP64, K.MIXED):
        plan = K.Plan(tree, np_, prec)
        plan.evaluate(pts)
        out[prec] = plan.read(1, nn * P)
        plan.close()
    tag = tree.array("tag")
    nodes = np.where(((tag & 2) != 0) & (np.abs(out[K.PLAIN_FP64].reshape(-1, P)).max(axis=1) > 0))[0]
    e = _node_err(out[K.MIXED], out[K.PLAIN_FP64], P, nodes)
    print(f"{_ids(case)}: mixed vs plain downward check potentials {e:.2e} over {len(nodes)} nodes")
    assert len(nodes) > 0 and e <= 2e-5


TENSOR_CASES = [("uniform", 65536, 128, 6, 0, 2), ("uniform", 262144, 64, 4, 0, 2),
                ("uniform", 300000, 32, 3, 1, 2), ("uniform", 150000, 16, 5, 0, 2),
                ("uniform", 40000, 64, 8, 0, 2)]


@pytest.mark.gpu
@pytest.mark.parametrize("case", TENSOR_CASES, ids=lambda c: _ids(c) + f"-tc{c[5]}")
def test_tensor_core_hadamard(K, oracle_mod, cuda_ok, case):
    """The mixed form's Hadamard on the tcgen05 tensor cores (TF32 hi/lo
    split, three passes, FP32 accumulation in tensor memory) for the levels
    whose boxes are all present, against the same plan with the CUDA-core
    FP32 kernels everywhere (had_tensor 1): downward check potentials per
    node within 2e-5 of the plain FP64 path (the CUDA-core form's bar),
    potentials within 1e-6 (rel-L2) of the CUDA-core mixed form, and the
    reference's check (rel-L2 against the exact direct sum) within 2x the
    plain path's error (had_tensor 2: every complete level)."""
    dist, n, ppb, np_, coincide, mode = case
    pts = K.generate_points(n, dist, coincide, 26, 300)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
    P, _, _ = K.sizes(np_)
    nn = tree.desc.num_nodes
    res = {}
    for name, prec, tun in (("plain", K.PLAIN_FP64, None), ("cuda", K.MIXED, None),
                            ("tensor", K.MIXED, {"had_tensor": mode})):
        plan = K.Plan(tree, np_, prec, tuning=tun)
        pot = plan.evaluate(pts)
        res[name] = (pot, plan.read(1, nn * P), plan.stats()["tensor_levels"])
        plan.close()
    assert res["cuda"][2] == 0 and res["tensor"][2] >= 1, res["tensor"][2]
    tag = tree.array("tag")
    dplain = res["plain"][1]
    nodes = np.where(((tag & 2) != 0) & (np.abs(dplain.reshape(-1, P)).max(axis=1) > 0))[0]
    e_tc = _node_err(res["tensor"][1], dplain, P, nodes)
    e_cc = _node_err(res["cuda"][1], dplain, P, nodes)
    tc, cc, plain = res["tensor"][0], res["cuda"][0], res["plain"][0]
    vs_cuda = np.linalg.norm(tc - cc) / np.linalg.norm(cc)
    ids = pts["check_ids"]
    d = oracle_mod.direct(pts["tx"][ids], pts["ty"][ids], pts["tz"][ids], pts["sx"], pts["sy"],
                          pts["sz"], pts["den"])
    e_plain = np.linalg.norm(plain[ids] - d) / np.linalg.norm(d)
    e_tens = np.linalg.norm(tc[ids] - d) / np.linalg.norm(d)
    print(f"{_ids(case)} tc{mode}: {res['tensor'][2]} tensor levels; dchk vs plain: tensor "
          f"{e_tc:.2e}, CUDA cores {e_cc:.2e}; potentials tensor vs CUDA cores {vs_cuda:.2e}; "
          f"rel-L2 vs direct: plain {e_plain:.3e} tensor {e_tens:.3e}")
    assert np.all(np.isfinite(tc))
    assert e_tc <= 2e-5
    assert vs_cuda <= 1e-6
    assert e_tens <= max(2.0 * e_plain, MIXED_FLOOR)


@pytest.mark.gpu
def test_tensor_choice_fixed_at_creation(K, cuda_ok):
    """kfmm_plan_set_tuning leaves the tensor-core choice as created, and
    re-running after other changes gives the same potentials bit for bit."""
    pts = K.generate_points(262144, "uniform", 0, 5)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 64)
    assert K.Plan(tree, 4, K.MIXED).stats()["tensor_levels"] == 0  # automatic: CUDA cores
    plan = K.Plan(tree, 4, K.MIXED, tuning={"had_tensor": 2})
    levels = plan.stats()["tensor_levels"]
    assert levels == 3  # depths 2, 3 and 4 are complete
    want = plan.evaluate(pts)
    plan.set_tuning({"had_tensor": 1, "job_rows": 3})
    assert plan.stats()["tensor_levels"] == levels
    assert np.array_equal(plan.evaluate(pts), want)
    plan.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 9, 100, 700])
def test_tiny_inputs(K, oracle_mod, cuda_ok, n):
    """Trees of a single leaf up to two levels: both forms against the oracle
    and, for the plain form, the exact direct sum."""
    pts = K.generate_points(n, "uniform", 0, 26)
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 8)
    tarrs = {k: tree.array(k) for k in oracle_mod.TREE_FIELDS}
    ref = oracle_mod.evaluate(tarrs, 4, K.operators(4), pts)
    plain = K.Plan(tree, 4, K.PLAIN_FP64).evaluate(pts)
    mixed = K.Plan(tree, 4, K.MIXED).evaluate(pts)
    assert np.all(np.isfinite(plain)) and np.all(np.isfinite(mixed))
    assert np.max(np.abs(plain - ref) / np.abs(ref)) <= 1e-12
    assert np.max(np.abs(mixed - ref) / np.abs(ref)) <= 1e-5
    if tree.desc.num_nodes == 1:
        d = oracle_mod.direct(pts["tx"], pts["ty"], pts["tz"], pts["sx"], pts["sy"], pts["sz"],
                              pts["den"])
        assert np.max(np.abs(plain - d) / np.abs(d)) <= 1e-13
