"""kfmm_tree_build_device (point work on the GPU) against kfmm_tree_build
(the host restatement pinned to the reference's tree by test_tree_oracle):
every array of the description identical, on uniform, ellipse, ellipsoid and
coincident clouds, on points lying exactly on cell boundaries and the root
box faces, and at the benchmark's 4M-point sizes; a cloud that would need
more than 21 levels is refused with an error, not built."""
import time

import numpy as np
import pytest

FIELDS = ("parent", "child", "depth", "tag", "path", "src_beg", "src_num", "trg_beg", "trg_num",
          "src_perm", "trg_perm", "node_level", "u_ptr", "u_idx", "v_ptr", "v_idx", "w_ptr",
          "w_idx", "x_ptr", "x_idx")

CASES = [("uniform", 20000, 64, 0), ("ellipsoidSurface", 30000, 48, 0),
         ("ellipseUniformAngles", 20000, 32, 0), ("uniform", 12000, 40, 1),
         ("uniform", 4194304, 512, 0), ("ellipsoidSurface", 4194304, 256, 0)]


def _same(K, a, b):
    for f in FIELDS:
        x, y = a.array(f), b.array(f)
        assert np.array_equal(x, y), f


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1]}-ppb{c[2]}-C{c[3]}")
def test_device_tree_equals_host_tree(K, cuda_ok, case):
    dist, n, ppb, c = case
    pts = K.generate_points(n, dist, c, 26)
    args = [pts[k] for k in ("sx", "sy", "sz", "tx", "ty", "tz")]
    t0 = time.time()
    host = K.Tree(*args, ppb)
    t1 = time.time()
    K.Tree(*args, ppb, device=True).close()  # first call pays the CUDA start-up
    t2 = time.time()
    dev = K.Tree(*args, ppb, device=True)
    t3 = time.time()
    print(f"{dist} n={n} ppb={ppb}: nodes {host.desc.num_nodes}; host {t1 - t0:.3f} s, "
          f"device {t3 - t2:.3f} s")
    _same(K, host, dev)


@pytest.mark.gpu
def test_device_tree_boundary_points(K, cuda_ok):
    rng = np.random.default_rng(1)
    n = 5000
    x = rng.integers(-8, 8, n) / 8.0          # exactly on cell boundaries
    y = rng.uniform(-1, 1, n)
    z = np.where(rng.random(n) < 0.1, 1.0, rng.uniform(-1, 1, n))
    x[:10], x[10:20] = 1.0, -1.0             # root box faces
    y[20:30] = -0.5 - 2.0 ** -60              # rounds to a boundary when 1 is added
    y[30:40] = np.nextafter(0.0, -1.0)
    host = K.Tree(x, y, z, z, y, x, 16)
    dev = K.Tree(x, y, z, z, y, x, 16, device=True)
    _same(K, host, dev)


@pytest.mark.gpu
def test_device_tree_refuses_too_deep(K, cuda_ok):
    x = np.full(50, 0.25)
    with pytest.raises(K.KfmmError, match="21 levels"):
        K.Tree(x, x, x, x, x, x, 10, device=True)
