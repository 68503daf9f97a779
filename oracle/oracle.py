"""TEST INFRASTRUCTURE — ctypes binding of the oracle (liboracle.so).

Used only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg,
always as the checker.  Build with ``make -C oracle restated``.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None
_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)

TREE_FIELDS = ("parent", "child", "depth", "tag", "path", "src_beg", "src_num", "trg_beg",
               "trg_num", "src_perm", "trg_perm", "node_level", "u_ptr", "u_idx", "v_ptr",
               "v_idx", "w_ptr", "w_idx", "x_ptr", "x_idx")


class OracleTree(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("num_nodes", "num_levels", "num_src", "num_trg")] + [
        (n, _i32p) for n in TREE_FIELDS]


class OracleOps(ctypes.Structure):
    _fields_ = [(n, _f64p) for n in ("uc2ue", "ue2uc", "dc2de", "de2dc", "ue2dc")]


def build():
    subprocess.check_call(["make", "-s", "-C", HERE, "restated"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.oracle_evaluate.argtypes = [ctypes.POINTER(OracleTree), ctypes.c_int,
                                      ctypes.POINTER(OracleOps)] + [_f64p] * 11
        L.oracle_evaluate.restype = ctypes.c_int
        L.oracle_direct.argtypes = [ctypes.c_int, _f64p, _f64p, _f64p, ctypes.c_int, _f64p,
                                    _f64p, _f64p, _f64p, _f64p]
        L.oracle_direct.restype = None
        L.oracle_set_order.argtypes = [ctypes.c_int]
        L.oracle_set_order.restype = None
        L.oracle_set_product_precision.argtypes = [ctypes.c_int]
        L.oracle_set_product_precision.restype = None
        _lib = L
    return _lib


def _p(a, t=_f64p):
    return a.ctypes.data_as(t)


def evaluate(tree, np_, ops, pts, want_phases=False):
    """tree: dict of int32 arrays (TREE_FIELDS + num_* entries); ops: dict with
    uc2ue, ue2uc (8 blocks concatenated), dc2de, de2dc, ue2dc; pts: dict of
    original-order float64 arrays.  Returns potentials (and per-node arrays)."""
    hold = {k: np.ascontiguousarray(tree[k], np.int32) for k in TREE_FIELDS}
    t = OracleTree(int(len(hold["parent"])), int(len(hold["node_level"]) - 1),
                   int(len(hold["src_perm"])), int(len(hold["trg_perm"])),
                   *[_p(hold[k], _i32p) for k in TREE_FIELDS])
    oh = {k: np.ascontiguousarray(ops[k], np.float64) for k in ("uc2ue", "ue2uc", "dc2de",
                                                               "de2dc", "ue2dc")}
    o = OracleOps(*[_p(oh[k]) for k in ("uc2ue", "ue2uc", "dc2de", "de2dc", "ue2dc")])
    P = int(round(len(oh["dc2de"]) ** 0.5))
    a = {k: np.ascontiguousarray(pts[k], np.float64) for k in ("sx", "sy", "sz", "den", "tx",
                                                                "ty", "tz")}
    pot = np.zeros(t.num_trg)
    nn = t.num_nodes
    ph = [np.zeros(nn * P) for _ in range(3)] if want_phases else None
    null = ctypes.cast(None, _f64p)
    rc = lib().oracle_evaluate(ctypes.byref(t), np_, ctypes.byref(o),
                               *[_p(a[k]) for k in ("sx", "sy", "sz", "den", "tx", "ty", "tz")],
                               _p(pot), *([_p(x) for x in ph] if ph else [null] * 3))
    if rc != 0:
        raise RuntimeError(f"oracle_evaluate failed: {rc}")
    return (pot, ph) if want_phases else pot


def evaluate_reordered(tree, np_, ops, pts):
    """The oracle with every direct sum and matrix-vector product summed in
    descending order: the spread to evaluate() is the FP64 rounding floor of
    the algorithm itself (the pseudo-inverses amplify it by up to their
    condition number)."""
    lib().oracle_set_order(1)
    try:
        return evaluate(tree, np_, ops, pts)
    finally:
        lib().oracle_set_order(0)


def evaluate_reduced_products(tree, np_, ops, pts, mode):
    """The oracle with its operator matrix-vector products in FP32 (mode 1)
    or split-TF32 three-pass with FP32 accumulation (mode 2)."""
    lib().oracle_set_product_precision(mode)
    try:
        return evaluate(tree, np_, ops, pts)
    finally:
        lib().oracle_set_product_precision(0)


def direct(tx, ty, tz, sx, sy, sz, den):
    """Exact FP64 direct sum at the given targets (fmm/driver.cc:142-206)."""
    t = [np.ascontiguousarray(v, np.float64) for v in (tx, ty, tz)]
    s = [np.ascontiguousarray(v, np.float64) for v in (sx, sy, sz, den)]
    out = np.zeros(len(t[0]))
    lib().oracle_direct(len(t[0]), *[_p(v) for v in t], len(s[0]), *[_p(v) for v in s], _p(out))
    return out


def ops_from_dump(R):
    """Operators in kfmm_operators layout from a reference dump."""
    return {"uc2ue": R["uc2ue"], "dc2de": R["dc2de"], "ue2dc": R["ue2dc"],
            "ue2uc": np.concatenate([R[f"ue2uc_{c}"] for c in range(8)]),
            "de2dc": np.concatenate([R[f"de2dc_{c}"] for c in range(8)])}
