"""ctypes binding of libkifmm_b200.so (include/kifmm_b200.h).

Python here is plumbing for tests and benchmarks: every computation runs in
the C++/CUDA library.  Loading fails loudly if the library has not been built;
there is no fallback path.

The directory name is not a Python identifier, so importers load this file by
path (see ``load_package`` in __graft_entry__.py) under the name
``kifmm_b200``.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkifmm_b200.so")
CLI_PATH = os.path.join(HERE, "fmmd--b200")

PLAIN_FP64 = 0
MIXED = 1

_lib = None

_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)
_f32p = ctypes.POINTER(ctypes.c_float)


class KfmmError(RuntimeError):
    pass


class TreeDesc(ctypes.Structure):
    _fields_ = [("num_nodes", ctypes.c_int), ("num_levels", ctypes.c_int),
                ("num_src", ctypes.c_int), ("num_trg", ctypes.c_int)] + [
        (n, _i32p) for n in ("parent", "child", "depth", "tag", "path", "src_beg", "src_num",
                             "trg_beg", "trg_num", "src_perm", "trg_perm", "node_level",
                             "u_ptr", "u_idx", "v_ptr", "v_idx", "w_ptr", "w_idx", "x_ptr",
                             "x_idx")]


class OperatorSet(ctypes.Structure):
    _fields_ = [(n, _f64p) for n in ("uc2ue", "ue2uc", "dc2de", "de2dc", "ue2dc")]


class Tuning(ctypes.Structure):
    """kfmm_tuning: launch choices, 0 = the plan's automatic choice."""
    _fields_ = [(n, ctypes.c_int) for n in ("nf_blocks", "job_rows", "had_windows",
                                             "splitk_max", "had_tensor", "cpu_share_ppm")]


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("u_pairs", "s2m_pairs", "s2l_pairs", "v_pairs",
                                                "hadamard_cmacs", "gemm_flops",
                                                "spectra_bytes")] + [
        (n, ctypes.c_int) for n in ("num_nodes", "P", "Q", "F", "launches", "tensor_levels")] + [
        ("host_pairs", ctypes.c_double)]


def lib():
    """Load libkifmm_b200.so once; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise KfmmError(f"{LIB_PATH} is not built; run kifmm--hybrid--double-only_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    sig = {
        "kfmm_generate_points": [i, ctypes.c_char_p, i, ctypes.c_long] + [_f64p] * 7 + [i, _i32p],
        "kfmm_tree_build": [i, _f64p, _f64p, _f64p, i, _f64p, _f64p, _f64p, i,
                            ctypes.POINTER(vp)],
        "kfmm_tree_describe": [vp, ctypes.POINTER(TreeDesc)],
        "kfmm_tree_build_device": [i, _f64p, _f64p, _f64p, i, _f64p, _f64p, _f64p, i, vp,
                                   ctypes.POINTER(vp)],
        "kfmm_sizes": [i, _i32p, _i32p, _i32p],
        "kfmm_operators": [i, _f64p, _f64p, _f64p, _f64p, _f64p],
        "kfmm_plan_create": [ctypes.POINTER(TreeDesc), i, i, ctypes.POINTER(vp)],
        "kfmm_plan_create_with_operators": [ctypes.POINTER(TreeDesc), i, i,
                                            ctypes.POINTER(OperatorSet), ctypes.POINTER(vp)],
        "kfmm_plan_create_tuned": [ctypes.POINTER(TreeDesc), i, i, ctypes.POINTER(OperatorSet),
                                   ctypes.POINTER(Tuning), ctypes.POINTER(vp)],
        "kfmm_plan_set_tuning": [vp, ctypes.POINTER(Tuning)],
        "kfmm_plan_destroy": [vp],
        "kfmm_set_sources": [vp, _f64p, _f64p, _f64p, _f64p, vp],
        "kfmm_set_targets": [vp, _f64p, _f64p, _f64p, vp],
        "kfmm_set_sources_device": [vp, vp, vp, vp, vp, vp],
        "kfmm_set_targets_device": [vp, vp, vp, vp, vp],
        "kfmm_run": [vp, vp],
        "kfmm_up_calc": [vp, vp],
        "kfmm_vlist_calc": [vp, vp],
        "kfmm_xlist_calc": [vp, vp],
        "kfmm_down_calc": [vp, vp],
        "kfmm_ulist_calc": [vp, vp],
        "kfmm_copy_trg_val": [vp, _f64p, vp],
        "kfmm_get_potentials_device": [vp, vp, vp],
        "kfmm_evaluate": [vp] + [_f64p] * 8 + [vp],
        "kfmm_evaluate_async": [vp] + [_f64p] * 8 + [vp],
        "kfmm_evaluate_join": [vp, vp],
        "kfmm_evaluate_wait": [vp, vp],
        "kfmm_direct_evaluation": [i, vp, vp, vp, vp, i, vp, vp, vp, vp, vp],
        "kfmm_read_array": [vp, i, _f64p, ctypes.c_size_t],
        "kfmm_plan_stats": [vp, ctypes.POINTER(Stats)],
        "kfmm_enable_timing": [vp, i],
        "kfmm_phase_times": [vp, ctypes.POINTER(ctypes.c_float)],
        "kfmm_kernel_times": [vp, ctypes.POINTER(ctypes.c_float)],
        "kfmm_measure_peak": [i, _f64p],
        "kfmm_s2m_noalloc": [i, i, vp, vp, vp, vp, vp, vp, vp],
        "kfmm_batch_create": [ctypes.POINTER(vp), i, i, ctypes.POINTER(vp)],
        "kfmm_batch_launch": [vp, vp],
        "kfmm_batch_wait": [vp, vp],
        "kfmm_set_wait_limit": [vp, ctypes.c_longlong],
        "kfmm_batch_destroy": [vp],
        "kfmm_mlp_param_count": [i, i, i, ctypes.POINTER(ctypes.c_longlong)],
        "kfmm_mlp_forward": [i, i, i, _f32p, i, _f32p, _f32p],
        "kfmm_mlp_gradients": [i, i, i, _f32p, i, _f32p, _f32p, _f32p, _f32p],
        "kfmm_mlp_train": [i, i, i, _f32p, i, _f32p, _f32p, i, ctypes.c_float, _f32p],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    L.kfmm_tree_destroy.argtypes = [vp]
    L.kfmm_tree_destroy.restype = None
    L.kfmm_last_error.restype = ctypes.c_char_p
    L.kfmm_version.restype = ctypes.c_char_p
    _lib = L
    return L


def check(status, what=""):
    if status != 0:
        msg = lib().kfmm_last_error().decode()
        raise KfmmError(f"{what}: status {status}: {msg}")


def _p(a, t=_f64p):
    return a.ctypes.data_as(t)


PEAK_KINDS = {"fp64_fma_tflops": 0, "fp32_fma_tflops": 1, "fp32_rsqrt_tops": 2,
              "fp64_rsqrt_tops": 3, "fp64_dmma_tflops": 4}


def measure_peaks():
    """Micro-benchmarked pipe throughputs of the current device."""
    out = {}
    for name, k in PEAK_KINDS.items():
        v = ctypes.c_double()
        check(lib().kfmm_measure_peak(k, ctypes.byref(v)), "measure_peak")
        out[name] = v.value
    return out


def sizes(np_):
    P, Q, F = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    check(lib().kfmm_sizes(np_, ctypes.byref(P), ctypes.byref(Q), ctypes.byref(F)), "sizes")
    return P.value, Q.value, F.value


def generate_points(n, distribution="uniform", coincide=0, seed=26, num_check=0):
    """Reference generators (drand48 stream): dict of float64 arrays."""
    out = {k: np.empty(n, np.float64) for k in ("sx", "sy", "sz", "den", "tx", "ty", "tz")}
    ids = np.empty(max(num_check, 1), np.int32)
    check(lib().kfmm_generate_points(n, distribution.encode(), coincide, seed,
                                     *[_p(out[k]) for k in ("sx", "sy", "sz", "den", "tx", "ty",
                                                            "tz")],
                                     num_check, _p(ids, _i32p)), "generate_points")
    out["check_ids"] = ids[:num_check]
    return out


def operators(np_):
    P, Q, F = sizes(np_)
    o = {"uc2ue": np.empty(P * Q), "ue2uc": np.empty(8 * Q * P), "dc2de": np.empty(P * P),
         "de2dc": np.empty(8 * P * P), "ue2dc": np.empty(343 * 2 * F)}
    check(lib().kfmm_operators(np_, *[_p(o[k]) for k in ("uc2ue", "ue2uc", "dc2de", "de2dc",
                                                         "ue2dc")]), "operators")
    return o


class Tree:
    """Octree + interaction lists built by the library (fmm/input.cc)."""

    def __init__(self, sx, sy, sz, tx, ty, tz, pts_max, device=False, stream=None):
        """device=True builds with the point work on the GPU
        (kfmm_tree_build_device); the result is the same tree."""
        self._arrays = [np.ascontiguousarray(a, np.float64) for a in (sx, sy, sz, tx, ty, tz)]
        sx, sy, sz, tx, ty, tz = self._arrays
        h = ctypes.c_void_p()
        if device:
            check(lib().kfmm_tree_build_device(len(sx), _p(sx), _p(sy), _p(sz), len(tx), _p(tx),
                                               _p(ty), _p(tz), pts_max, stream, ctypes.byref(h)),
                  "tree_build_device")
        else:
            check(lib().kfmm_tree_build(len(sx), _p(sx), _p(sy), _p(sz), len(tx), _p(tx), _p(ty),
                                        _p(tz), pts_max, ctypes.byref(h)), "tree_build")
        self.handle = h
        self.desc = TreeDesc()
        check(lib().kfmm_tree_describe(h, ctypes.byref(self.desc)), "tree_describe")

    def array(self, name):
        d = self.desc
        nn = d.num_nodes
        n = {"path": 3 * nn, "src_perm": d.num_src, "trg_perm": d.num_trg,
             "node_level": d.num_levels + 1}.get(name, nn)
        if name.endswith("_ptr"):
            n = nn + 1
        if name.endswith("_idx"):
            n = self.array(name[:-4] + "_ptr")[-1]
        ptr = getattr(d, name)
        return np.ctypeslib.as_array(ptr, shape=(int(n),)).copy() if n > 0 else np.zeros(0, np.int32)

    def close(self):
        if self.handle:
            lib().kfmm_tree_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """An evaluation plan on the current CUDA device."""

    def __init__(self, tree, np_, precision=PLAIN_FP64, operators=None, tuning=None):
        """operators: optional dict (uc2ue, ue2uc, dc2de, de2dc[, ue2dc]) in
        kfmm_operators layout, e.g. the reference's own matrices.  tuning:
        optional dict of kfmm_tuning fields (launch choices)."""
        self.tree = tree
        self.np = np_
        h = ctypes.c_void_p()
        ops = None
        if operators is not None:
            self._ops = {k: np.ascontiguousarray(operators[k], np.float64)
                         for k in ("uc2ue", "ue2uc", "dc2de", "de2dc", "ue2dc") if k in operators}
            null = ctypes.cast(None, _f64p)
            ops = ctypes.byref(OperatorSet(*[_p(self._ops[k]) if k in self._ops else null
                                             for k in ("uc2ue", "ue2uc", "dc2de", "de2dc",
                                                       "ue2dc")]))
        tune = ctypes.byref(Tuning(**{k: int(v) for k, v in tuning.items()})) if tuning else None
        check(lib().kfmm_plan_create_tuned(ctypes.byref(tree.desc), np_, precision, ops, tune,
                                           ctypes.byref(h)), "plan_create")
        self.handle = h
        self.nt = tree.desc.num_trg
        self.ns = tree.desc.num_src

    def set_points(self, pts, stream=None):
        a = {k: np.ascontiguousarray(pts[k], np.float64) for k in ("sx", "sy", "sz", "den", "tx",
                                                                    "ty", "tz")}
        self._hold = a
        check(lib().kfmm_set_targets(self.handle, _p(a["tx"]), _p(a["ty"]), _p(a["tz"]), stream),
              "set_targets")
        check(lib().kfmm_set_sources(self.handle, _p(a["sx"]), _p(a["sy"]), _p(a["sz"]),
                                     _p(a["den"]), stream), "set_sources")

    def run(self, stream=None):
        check(lib().kfmm_run(self.handle, stream), "run")

    def potentials(self, stream=None):
        out = np.empty(self.nt, np.float64)
        check(lib().kfmm_copy_trg_val(self.handle, _p(out), stream), "copy_trg_val")
        return out

    def evaluate(self, pts, stream=None):
        a = {k: np.ascontiguousarray(pts[k], np.float64) for k in ("sx", "sy", "sz", "den", "tx",
                                                                    "ty", "tz")}
        out = np.empty(self.nt, np.float64)
        check(lib().kfmm_evaluate(self.handle, *[_p(a[k]) for k in ("sx", "sy", "sz", "den",
                                                                     "tx", "ty", "tz")],
                                  _p(out), stream), "evaluate")
        return out

    def read(self, which, count):
        out = np.empty(count, np.float64)
        check(lib().kfmm_read_array(self.handle, which, _p(out), count), "read_array")
        return out

    def stats(self):
        s = Stats()
        check(lib().kfmm_plan_stats(self.handle, ctypes.byref(s)), "plan_stats")
        return {f: getattr(s, f) for f, _ in Stats._fields_}

    def set_tuning(self, tuning=None):
        """New launch choices (dict of kfmm_tuning fields; None: automatic)."""
        t = ctypes.byref(Tuning(**{k: int(v) for k, v in tuning.items()})) if tuning else None
        check(lib().kfmm_plan_set_tuning(self.handle, t), "plan_set_tuning")

    def set_wait_limit(self, tries):
        """Tries of the kernels' bounded waits; < 0 restores the default."""
        check(lib().kfmm_set_wait_limit(self.handle, tries), "set_wait_limit")

    def enable_timing(self, on=True):
        check(lib().kfmm_enable_timing(self.handle, 1 if on else 0), "enable_timing")

    def phase_times(self):
        ms = (ctypes.c_float * 6)()
        check(lib().kfmm_phase_times(self.handle, ms), "phase_times")
        return dict(zip(("up", "vlist", "xlist", "down", "ulist", "copy"), list(ms)))

    KERNEL_PHASES = ("s2m", "up_gemm", "fft_src", "hadamard", "ifft_trg", "s2l", "down_gemm",
                     "near_field", "copy")

    def kernel_times(self):
        """Per-kernel-group device times (ms) of the last timed run."""
        ms = (ctypes.c_float * 9)()
        check(lib().kfmm_kernel_times(self.handle, ms), "kernel_times")
        return dict(zip(self.KERNEL_PHASES, list(ms)))

    def close(self):
        if self.handle:
            lib().kfmm_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many plans replayed by one CUDA graph launch (kfmm_batch_create).  The
    plans must have their points set; they stay owned by the caller and must
    outlive the batch."""

    def __init__(self, plans, nstreams=16):
        self.plans = list(plans)
        arr = (ctypes.c_void_p * len(self.plans))(*[p.handle for p in self.plans])
        h = ctypes.c_void_p()
        check(lib().kfmm_batch_create(arr, len(self.plans), nstreams, ctypes.byref(h)),
              "batch_create")
        self.handle = h

    def launch(self, stream=None):
        check(lib().kfmm_batch_launch(self.handle, stream), "batch_launch")

    def wait(self, stream=None):
        """Wait for the last launch; raise if one of its solves gave up a
        bounded wait."""
        check(lib().kfmm_batch_wait(self.handle, stream), "batch_wait")

    def close(self):
        if self.handle:
            lib().kfmm_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MLP:
    """The cost-model network (kfmm_mlp_*): F inputs, H hidden, O outputs,
    FP32 parameters held on the host, every computation on the GPU."""

    def __init__(self, F, H, O, params=None, seed=0):
        self.F, self.H, self.O = F, H, O
        n = ctypes.c_longlong()
        check(lib().kfmm_mlp_param_count(F, H, O, ctypes.byref(n)), "mlp_param_count")
        self.n = n.value
        if params is None:
            rng = np.random.default_rng(seed)
            parts = []
            for fi, fo in ((F, H), (H, H), (H, O)):
                parts += [rng.normal(0, np.sqrt(2.0 / fi), fi * fo), np.zeros(fo)]
            params = np.concatenate(parts)
        self.params = np.ascontiguousarray(params, np.float32)
        assert self.params.size == self.n

    def forward(self, X):
        X = np.ascontiguousarray(X, np.float32)
        Y = np.empty((X.shape[0], self.O), np.float32)
        check(lib().kfmm_mlp_forward(self.F, self.H, self.O, _p(self.params, _f32p), X.shape[0],
                                     _p(X, _f32p), _p(Y, _f32p)), "mlp_forward")
        return Y

    def gradients(self, X, T):
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        g = np.empty(self.n, np.float32)
        loss = ctypes.c_float()
        check(lib().kfmm_mlp_gradients(self.F, self.H, self.O, _p(self.params, _f32p),
                                       X.shape[0], _p(X, _f32p), _p(T, _f32p), _p(g, _f32p),
                                       ctypes.byref(loss)), "mlp_gradients")
        return g, loss.value

    def train(self, X, T, steps, lr=1e-3):
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        losses = np.empty(steps, np.float32)
        check(lib().kfmm_mlp_train(self.F, self.H, self.O, _p(self.params, _f32p), X.shape[0],
                                   _p(X, _f32p), _p(T, _f32p), steps, lr, _p(losses, _f32p)),
              "mlp_train")
        return losses
