"""The C ABI library: it loads, exports every entry point include/kifmm_b200.h
declares, and rejects bad input with a status (no exit, no crash).  No GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "kifmm_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(kfmm_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("kfmm_plan_create", "kfmm_run", "kfmm_up_calc", "kfmm_vlist_calc",
                 "kfmm_ulist_calc", "kfmm_down_calc", "kfmm_copy_trg_val", "kfmm_tree_build",
                 "kfmm_evaluate", "kfmm_direct_evaluation", "kfmm_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(K):
    L = K.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_version_string(K):
    assert b"sm_100a" in K.lib().kfmm_version()


def test_sizes(K):
    assert K.sizes(6) == (152, 296, 1008)
    assert K.sizes(4) == (56, 152, 320)
    assert K.sizes(3) == (26, 98, 144)
    assert K.sizes(8) == (296, 488, 2304)
    P = ctypes.c_int()
    assert K.lib().kfmm_sizes(2, ctypes.byref(P), None, None) == 4  # UNSUPPORTED
    assert b"NP" in K.lib().kfmm_last_error()


def test_generate_unknown_distribution(K):
    with pytest.raises(K.KfmmError, match="unknown distribution"):
        K.generate_points(10, "gaussianBlob")


def test_tree_rejects_points_outside_root_box(K):
    pts = K.generate_points(100, "uniform")
    pts["sx"][3] = 1.5
    with pytest.raises(K.KfmmError, match="root box"):
        K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 8)
    pts["sx"][3] = np.nan
    with pytest.raises(K.KfmmError, match="root box"):
        K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 8)


def test_tree_refuses_empty_point_sets(K):
    """No sources, no targets or a leaf size below 1 is an argument error
    (status KFMM_ERR_INVALID), not a tree: the evaluation needs both sets."""
    pts = K.generate_points(50, "uniform")
    z = np.zeros(0)
    for args, ppb in (((z, z, z, z, z, z), 8), ((pts["sx"], pts["sy"], pts["sz"], z, z, z), 8),
                      ((z, z, z, pts["tx"], pts["ty"], pts["tz"]), 8),
                      ((pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"]), 0)):
        with pytest.raises(K.KfmmError, match="bad argument"):
            K.Tree(*args, ppb)


def test_plan_create_argument_errors(K):
    L = K.lib()
    h = ctypes.c_void_p()
    assert L.kfmm_plan_create(None, 6, 0, ctypes.byref(h)) == 1  # INVALID
    pts = K.generate_points(2000, "uniform")
    t = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 32)
    assert L.kfmm_plan_create(ctypes.byref(t.desc), 2, 0, ctypes.byref(h)) == 4
    assert L.kfmm_plan_create(ctypes.byref(t.desc), 6, 7, ctypes.byref(h)) == 1
    # corrupt a list entry: validation catches it before touching the device
    bad = K.TreeDesc.from_buffer_copy(t.desc)
    u = t.array("u_idx").astype(np.int32)
    u[0] = 10**7
    bad.u_idx = u.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    assert L.kfmm_plan_create(ctypes.byref(bad), 6, 0, ctypes.byref(h)) == 1
    assert b"out of range" in L.kfmm_last_error()
    # a repeated index in the leaf-order permutation (points reach leaf order
    # through its inverse)
    bad = K.TreeDesc.from_buffer_copy(t.desc)
    perm = t.array("src_perm").astype(np.int32)
    perm[1] = perm[0]
    bad.src_perm = perm.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    assert L.kfmm_plan_create(ctypes.byref(bad), 6, 0, ctypes.byref(h)) == 1
    assert b"not a permutation" in L.kfmm_last_error()


def test_plan_create_without_device_reports_status(K):
    """On a machine without a GPU a valid tree gets as far as the first device
    allocation and returns a status: no exit, no CPU fallback."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    pts = K.generate_points(3000, "uniform")
    t = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 32)
    h = ctypes.c_void_p()
    rc = K.lib().kfmm_plan_create(ctypes.byref(t.desc), 4, 0, ctypes.byref(h))
    assert rc in (2, 3) and not h.value


def test_null_plan_calls(K):
    L = K.lib()
    assert L.kfmm_run(None, None) == 1
    assert L.kfmm_plan_destroy(None) == 0
    assert L.kfmm_read_array(None, 0, None, 0) == 1


def test_tree_build_refuses_coincident_overflow(K):
    """More than pts_max coincident sources never separate: the reference's
    builder splits forever; this one stops at 30 levels with an error."""
    import numpy as np
    x = np.full(50, 0.25)
    with pytest.raises(K.KfmmError, match="coincident"):
        K.Tree(x, x, x, x, x, x, 10)
