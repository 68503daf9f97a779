"""Learned cost model for the leaf size (points per box) and the near-field
kernel's launch choices.

A small network (kfmm_mlp_*: 3 layers, 64 hidden units, FP32, trained and
evaluated by this library's own CUDA kernels) maps tree statistics plus a
near-field configuration (job size in rows of 32 targets, resident blocks
per SM: CONFIGS) to the per-phase device times of one solve.  To pick for a
new cloud, the tree is built for every leaf-size candidate (on the GPU,
kfmm_tree_build_device: no plan, no solve), the network predicts the time of
every (leaf size, configuration) pair, and the fastest prediction wins.  When
the two best predictions are closer than `fallback_margin` (10%), those two
are measured and the faster one is taken: measurement stays the fallback,
and the exhaustive measured sweep the yardstick the model is scored
against.

Features of a (cloud, leaf size) tree: log point count, log leaf size, NP,
node counts per level (16 levels), histograms of the U, V, W and X list
lengths over target nodes (8 log2 bins each, as fractions), the log totals
of U-list point pairs and V, W, X box pairs, and the logs of the work the
kernels do as the plan counts it: near-field pairs (U + W + direct X + L2T),
the same padded to the warp's 32-target granularity, S2M and S2L pairs, the
box, leaf and V-list-box counts, the largest leaf's near-field work and the
work-weighted histogram of leaf work (8 bins, factors of 4); then the
configuration (rows per job / 6, 1 for 5 resident blocks).  Targets: log(ms)
of the phases up, vlist, xlist, down, ulist (kfmm_phase_times).

``harvest`` measures clouds with a pipeline: worker threads build the trees
(on the host), the features and the plans of the next (cloud, leaf size)
pairs while the main thread times the ready ones on the GPU, one at a time.

Clouds (``make_cloud``): the uniform cube, the ellipsoid surface, and
mixtures of 1 to 32 isotropic Gaussian clusters with sigma log-uniform in
[0.005, 0.1] (points outside the root box redrawn).
"""
import json
import math
import os

import numpy as np

PHASES = ("up", "vlist", "xlist", "down", "ulist")
LEAF_SIZES = (32, 64, 128, 256, 512, 1024)
# near-field launch choices the model ranks (kfmm_tuning fields)
CONFIGS = ({"job_rows": 6, "nf_blocks": 6}, {"job_rows": 4, "nf_blocks": 5})


def config_features(cfg):
    return [cfg["job_rows"] / 6.0, 1.0 if cfg["nf_blocks"] == 5 else 0.0]
NLEVELS = 16
NBINS = 8


def cluster_points(n, k, sigma, rng):
    centres = rng.uniform(-0.7, 0.7, (k, 3))
    out = np.empty((n, 3))
    filled = 0
    while filled < n:
        m = n - filled
        c = centres[rng.integers(0, k, m)]
        p = c + rng.normal(0.0, sigma, (m, 3))
        ok = np.all((p >= -1.0) & (p < 1.0), axis=1)
        p = p[ok]
        out[filled:filled + len(p)] = p
        filled += len(p)
    return out


def make_cloud(K, kind, n, seed):
    """Points dict (sx..tz, den) for kind 'uniform', 'ellipsoidSurface' or
    'clusters' (cluster count and width drawn from the seed)."""
    if kind in ("uniform", "ellipsoidSurface"):
        return K.generate_points(n, kind, 0, seed)
    rng = np.random.default_rng(seed)
    k = int(rng.integers(1, 33))
    sigma = float(np.exp(rng.uniform(np.log(0.005), np.log(0.1))))
    s = cluster_points(n, k, sigma, rng)
    t = cluster_points(n, k, sigma, np.random.default_rng(seed + 7919))
    return {"sx": s[:, 0].copy(), "sy": s[:, 1].copy(), "sz": s[:, 2].copy(),
            "tx": t[:, 0].copy(), "ty": t[:, 1].copy(), "tz": t[:, 2].copy(),
            "den": rng.uniform(0, 1, n), "clusters": k, "sigma": sigma}


def _hist(lengths):
    h = np.zeros(NBINS)
    if len(lengths):
        b = np.minimum(np.where(lengths > 0, np.floor(np.log2(np.maximum(lengths, 1))) + 1, 0),
                       NBINS - 1).astype(int)
        np.add.at(h, b, 1.0)
        h /= len(lengths)
    return h


def features(tree, np_, ppb, n, cfg=None):
    """Tree statistics of a (cloud, leaf size) followed by the near-field
    configuration's features (CONFIGS[0] when cfg is None)."""
    return np.concatenate([tree_features(tree, np_, ppb, n),
                           config_features(CONFIGS[0] if cfg is None else cfg)])


def tree_features(tree, np_, ppb, n):
    depth = tree.array("depth")
    tag = tree.array("tag")
    src_num = tree.array("src_num").astype(np.float64)
    trg_num = tree.array("trg_num").astype(np.float64)
    child = tree.array("child")
    levels = np.bincount(np.minimum(depth, NLEVELS - 1), minlength=NLEVELS)[:NLEVELS]
    f = [math.log(n), math.log(ppb), float(np_)]
    f += list(np.log1p(levels))
    trg_nodes = np.where(tag & 2)[0]
    totals = []
    for name in ("u", "v", "w", "x"):
        ptr = tree.array(name + "_ptr")
        idx = tree.array(name + "_idx")
        lens = (ptr[1:] - ptr[:-1])[trg_nodes]
        f += list(_hist(lens))
        if name == "u":
            # point pairs: targets of each leaf times the sources of its U list
            per = np.zeros(len(ptr) - 1)
            if len(idx):
                cs = np.concatenate([[0.0], np.cumsum(src_num[idx])])
                per = cs[ptr[1:]] - cs[ptr[:-1]]
            leaves = child == -1
            totals.append(float((trg_num * per)[leaves].sum()))
        else:
            totals.append(float(len(idx)))
    f += [math.log1p(t) for t in totals]
    # the work the kernels do, counted as the plan counts it: near-field
    # pairs (U + W + direct X + L2T) and the same padded to the warp's
    # 32-target granularity, S2M and S2L pairs, boxes, leaves, V-list boxes
    P = np_ ** 3 - (np_ - 2) ** 3
    Q = (np_ + 2) ** 3 - np_ ** 3
    nn = len(depth)
    leaves = child == -1

    def per_node(name, contrib):
        ptr = tree.array(name + "_ptr")
        idx = tree.array(name + "_idx")
        if not len(idx):
            return np.zeros(nn)
        cs = np.concatenate([[0.0], np.cumsum(contrib(idx))])
        return cs[ptr[1:]] - cs[ptr[:-1]]

    src_leaf = leaves & (src_num > 0)
    u = per_node("u", lambda i: src_num[i])
    w = per_node("w", lambda i: np.where(src_leaf[i] & (src_num[i] < P), src_num[i], P))
    x = per_node("x", lambda i: src_num[i])
    near = u + w + np.where(trg_num < P, x, 0.0) + np.where(depth >= 2, P, 0.0)
    tl = leaves & (trg_num > 0)
    nf = float((trg_num * near)[tl].sum())
    nf_pad = float((np.ceil(trg_num / 32.0) * 32.0 * near)[tl].sum())
    s2m = float(Q * src_num[src_leaf].sum())
    s2l = float((P * x)[(tag & 2).astype(bool) & ~(leaves & (trg_num < P))].sum())
    vptr = tree.array("v_ptr")
    f += [math.log1p(v) for v in (nf, nf_pad, s2m, s2l, nn, float(src_leaf.sum()),
                                  float(np.sum(vptr[1:] > vptr[:-1])))]
    # how the near-field work is spread over the leaves (the persistent
    # kernel's tail): largest leaf, and the work-weighted histogram of leaf
    # work in factors of 4
    lw = (np.ceil(trg_num / 32.0) * 32.0 * near)[tl]
    f.append(math.log1p(float(lw.max()) if len(lw) else 0.0))
    h = np.zeros(NBINS)
    if len(lw) and lw.sum() > 0:
        b = np.clip(np.floor(np.log(np.maximum(lw, 1.0) / 1e4) / np.log(4.0)) + 2, 0,
                    NBINS - 1).astype(int)
        np.add.at(h, b, lw / lw.sum())
    f += list(h)
    return np.array(f, np.float64)


def time_phases(K, plan, pts, reps=3, set_points=True, stream=None):
    """Per-phase device ms of one solve (minimum over reps after a warm-up),
    the copy phase counted into down.  `stream`: a non-blocking stream keeps
    other threads' synchronous copies (legacy stream) out of the timed
    region."""
    if set_points:
        plan.set_points(pts, stream)
    plan.run(stream)
    plan.enable_timing(True)
    best = None
    for _ in range(reps):
        plan.run(stream)
        ph = plan.phase_times()
        v = np.array([ph[p] for p in PHASES])
        v[PHASES.index("down")] += ph["copy"]
        best = v if best is None else np.minimum(best, v)
    plan.enable_timing(False)
    return best


def measure(K, pts, np_, ppb, precision, reps=2, device_tree=True, configs=CONFIGS):
    """The tree's features and, for each configuration, its per-phase ms:
    [(features, phase ms)] in the order of configs."""
    args = [pts[k] for k in ("sx", "sy", "sz", "tx", "ty", "tz")]
    tree = K.Tree(*args, ppb, device=device_tree)
    try:
        base = tree_features(tree, np_, ppb, len(pts["sx"]))
        out = []
        plan = K.Plan(tree, np_, precision, tuning=configs[0])
        try:
            for k, cfg in enumerate(configs):
                if k:
                    plan.set_tuning(cfg)
                out.append((np.concatenate([base, config_features(cfg)]),
                            time_phases(K, plan, pts, reps, set_points=(k == 0))))
        finally:
            plan.close()
        return out
    finally:
        tree.close()


def cloud_specs(count, nmin=65536, nmax=8388608, seed=5):
    rng = np.random.default_rng(seed)
    kinds = ("uniform", "ellipsoidSurface", "clusters")
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        out.append({"kind": kinds[i % 3], "n": n, "seed": seed * 1000 + i})
    return out


def plan_bytes(tree, np_, mixed=True):
    """Upper estimate of a plan's device memory: per node the FP64 expansions
    (3 x P), the leaf check potentials (Q) and two spectra (2 x (F padded to
    32) complex, FP32 in the mixed form), per point the coordinates in both
    orders, densities and potentials; 30% margin."""
    P = np_ ** 3 - (np_ - 2) ** 3
    Q = (np_ + 2) ** 3 - np_ ** 3
    F = (np_ + 1) * (2 * np_) ** 2
    fpad = (F + 31) // 32 * 32
    d = tree.desc
    per_node = 8.0 * (3 * P + Q) + 2 * (8.0 if mixed else 16.0) * fpad
    per_point = 8.0 * 16 + 16.0
    return 1.3 * (d.num_nodes * per_node + (d.num_src + d.num_trg) * per_point)


def harvest(K, specs, np_=6, precision=None, leaf_sizes=LEAF_SIZES, configs=CONFIGS,
            threads=8, device_bytes=100e9, log=None, checkpoint=None):
    """Measured dataset: one row per (cloud, leaf size, configuration).
    `threads` workers build host trees, features and plans ahead of the
    timing loop, which runs on its own non-blocking stream; at most
    `device_bytes` of plans (plan_bytes) are held at once.
    checkpoint(data): called with the rows so far every 100 clouds."""
    import queue
    import threading

    import torch
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    precision = K.MIXED if precision is None else precision
    ready = queue.Queue()
    held = [0.0]  # estimated device bytes of the plans built and not yet timed
    room = threading.Condition()

    def reserve(nbytes):
        with room:
            room.wait_for(lambda: held[0] == 0.0 or held[0] + nbytes <= device_bytes)
            held[0] += nbytes

    def release(nbytes):
        with room:
            held[0] -= nbytes
            room.notify_all()

    todo = list(enumerate(specs))
    todo_lock = threading.Lock()
    errors = []

    def worker():
        try:
            while True:
                with todo_lock:
                    if not todo:
                        return
                    ci, sp = todo.pop(0)
                pts = make_cloud(K, sp["kind"], sp["n"], sp["seed"])
                args = [pts[k] for k in ("sx", "sy", "sz", "tx", "ty", "tz")]
                for ppb in leaf_sizes:
                    if ppb * 8 > sp["n"]:
                        continue
                    tree = K.Tree(*args, ppb)
                    u = plan_bytes(tree, np_, precision == K.MIXED)
                    reserve(u)
                    base = tree_features(tree, np_, ppb, sp["n"])
                    plan = K.Plan(tree, np_, precision, tuning=configs[0])
                    ready.put((ci, ppb, pts, tree, base, plan, u))
                ready.put((ci, None, None, None, None, None, 0.0))
        except Exception as ex:  # reported by the timing loop
            errors.append(ex)
            ready.put(None)

    pool = [threading.Thread(target=worker, daemon=True) for _ in range(threads)]
    for t in pool:
        t.start()
    rows_f, rows_t, cloud, ppbs, cfgs = [], [], [], [], []
    done = 0

    def pack():
        return {"features": np.array(rows_f), "phase_ms": np.array(rows_t),
                "cloud": np.array(cloud), "ppb": np.array(ppbs), "config": np.array(cfgs),
                "n": np.array([specs[c]["n"] for c in cloud]),
                "kind": np.array([specs[c]["kind"] for c in cloud]),
                "seed": np.array([specs[c]["seed"] for c in cloud])}
    while done < len(specs):
        item = ready.get()
        if item is None:
            raise errors[0]
        ci, ppb, pts, tree, base, plan, u = item
        if ppb is None:
            done += 1
            if log:
                log(f"cloud {ci} {specs[ci]['kind']} n={specs[ci]['n']}: done ({done}/{len(specs)})")
            if checkpoint and done % 100 == 0:
                checkpoint(pack())
            continue
        for k, cfg in enumerate(configs):
            if k:
                plan.set_tuning(cfg)
            rows_f.append(np.concatenate([base, config_features(cfg)]))
            rows_t.append(time_phases(K, plan, pts, set_points=(k == 0), stream=sh))
            cloud.append(ci)
            ppbs.append(ppb)
            cfgs.append(k)
        plan.close()
        tree.close()
        release(u)
    for t in pool:
        t.join()
    return pack()


class CostModel:
    """Feature standardisation + the network; predicts per-phase log ms."""

    def __init__(self, K, mean=None, std=None, params=None, hidden=64, seed=0):
        self.K = K
        self.mean, self.std = mean, std
        self.hidden = hidden
        self.net = None
        if mean is not None:
            self.net = K.MLP(len(mean), hidden, len(PHASES), params=params, seed=seed)

    def _x(self, feats):
        return ((np.atleast_2d(feats) - self.mean) / self.std).astype(np.float32)

    def fit(self, feats, phase_ms, steps=4000, lr=2e-3, seed=0):
        self.mean = feats.mean(0)
        self.std = np.where(feats.std(0) > 1e-9, feats.std(0), 1.0)
        self.net = self.K.MLP(feats.shape[1], self.hidden, len(PHASES), seed=seed)
        T = np.log(np.maximum(phase_ms, 1e-3)).astype(np.float32)
        return self.net.train(self._x(feats), T, steps, lr)

    def predict_phase_ms(self, feats):
        return np.exp(self.net.forward(self._x(feats)))

    def predict_ms(self, feats):
        return self.predict_phase_ms(feats).sum(1)

    def save(self, path):
        np.savez(path, mean=self.mean, std=self.std, params=self.net.params,
                 hidden=self.hidden)

    @classmethod
    def load_default(cls, K):
        """The network trained on the committed B200 harvest (NP=6, mixed)."""
        return cls.load(K, os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                        "costmodel_data", "weights_b200_np6_mixed.npz"))

    @classmethod
    def load(cls, K, path):
        z = np.load(path)
        return cls(K, z["mean"], z["std"], z["params"], int(z["hidden"]))

    def pick(self, pts, np_=6, precision=None, leaf_sizes=LEAF_SIZES, configs=CONFIGS,
             fallback_margin=0.10):
        """((leaf size, configuration), {(leaf size, config index): predicted
        ms}, measured?) for a cloud."""
        K = self.K
        precision = K.MIXED if precision is None else precision
        n = len(pts["sx"])
        args = [pts[k] for k in ("sx", "sy", "sz", "tx", "ty", "tz")]
        cand = [b for b in leaf_sizes if b * 8 <= n] or [leaf_sizes[0]]
        keys, feats = [], []
        for ppb in cand:
            tree = K.Tree(*args, ppb, device=True)
            base = tree_features(tree, np_, ppb, n)
            tree.close()
            for k, cfg in enumerate(configs):
                keys.append((ppb, k))
                feats.append(np.concatenate([base, config_features(cfg)]))
        pred = dict(zip(keys, self.predict_ms(np.array(feats))))
        order = sorted(keys, key=pred.get)
        best = order[0]
        measured = len(order) > 1 and pred[order[1]] - pred[order[0]] < fallback_margin * pred[order[0]]
        if measured:
            from . import autotune
            ms = {key: autotune.time_leaf_size(K, pts, key[0], np_, precision,
                                               tuning=configs[key[1]]) for key in order[:2]}
            best = min(ms, key=ms.get)
        return (best[0], dict(configs[best[1]])), pred, measured


def evaluate_picks(model, data, clouds, default_ppb=512, fallback_margin=0.10):
    """For each cloud of the dataset, from the harvested measurements: the
    time of the model's pick over all measured (leaf size, configuration)
    rows, of the model with the measured fallback (the two best predictions
    measured when they are within fallback_margin), of the fixed default
    (leaf size 512 with the automatic configuration) and of the sweep's best.
    Ratios to the best."""
    out = []
    cfg_col = data["config"] if "config" in data else np.zeros(len(data["ppb"]), int)
    for c in clouds:
        m = data["cloud"] == c
        ppb = data["ppb"][m]
        cfg = cfg_col[m]
        total = data["phase_ms"][m].sum(1)
        pred = model.predict_ms(data["features"][m])
        best = total.min()
        order = np.argsort(pred)
        pick = order[0]
        fb = pick
        measured = len(order) > 1 and pred[order[1]] - pred[order[0]] < fallback_margin * pred[order[0]]
        if measured:
            fb = order[:2][np.argmin(total[order[:2]])]
        sel = (ppb == default_ppb) & (cfg == 0)
        dflt = total[sel][0] if np.any(sel) else total[-1]
        out.append({"cloud": int(c), "kind": str(data["kind"][m][0]), "n": int(data["n"][m][0]),
                    "pick_over_best": float(total[pick] / best),
                    "fallback_over_best": float(total[fb] / best), "measured": bool(measured),
                    "default_over_best": float(dflt / best),
                    "picked": (int(ppb[pick]), int(cfg[pick])),
                    "best": (int(ppb[np.argmin(total)]), int(cfg[np.argmin(total)]))})
    return out


def main(argv):
    """harvest <out.npz> <nclouds>  |  train <data.npz> <weights.npz> [steps]"""
    import __graft_entry__
    K = __graft_entry__.load_package()
    if argv[0] == "harvest":
        specs = cloud_specs(int(argv[2]))
        threads = int(argv[3]) if len(argv) > 3 else 8
        data = harvest(K, specs, threads=threads, log=lambda m: print(m, flush=True),
                       checkpoint=lambda d: np.savez_compressed(argv[1], **d))
        np.savez_compressed(argv[1], **data)
    elif argv[0] == "train":
        data = dict(np.load(argv[1]))
        train = data["cloud"] % 5 != 0  # every fifth cloud held out
        model = CostModel(K)
        losses = model.fit(data["features"][train], data["phase_ms"][train],
                           steps=int(argv[3]) if len(argv) > 3 else 4000)
        model.save(argv[2])
        held = sorted(set(data["cloud"][~train].tolist()))
        ev = evaluate_picks(model, data, held)
        print(json.dumps({"final_loss": float(losses[-1]), "held_out": ev}))


if __name__ == "__main__":
    import sys
    main(sys.argv[1:])
