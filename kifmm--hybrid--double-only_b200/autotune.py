"""Autotuner: a measured sweep over the leaf size and the kernels' launch
choices (kfmm_tuning).

The evaluator's cost splits between the near field (grows with the leaf
size) and the far field (grows with the number of boxes); the best leaf size
depends on the point distribution, the point count, NP and the precision
form.  At a given leaf size, the kernels' own shapes matter too: how many
targets one near-field job holds (leaf chunking, `job_rows`), how many
resident blocks per SM the mixed near-field kernel is compiled for
(`nf_blocks`, i.e. its register budget), how many sibling windows each warp
of a mixed Hadamard CTA takes (`had_windows`) and how far the level products
split their K dimension (`splitk_max`).

``tune`` measures, on the device (CUDA events, kfmm_kernel_times), first
every leaf-size candidate with the plan's automatic launch choices, then, at
the fastest leaf size, each launch choice in turn with the others held at
their best so far (coordinate descent); a change is kept only when it is
faster by more than 0.5%.  ``ConfigTable`` caches the result per
(distribution, log2 point-count bucket, NP, precision), tuned once per bucket
on a cloud of the bucket's geometric middle size, and can be persisted as
JSON.

The reference has no tuner: it takes the leaf size from its command line
(fmm/driver.cc:216) and fixes its thread-block sizes at compile time
(fmm/cuda.cu:35-105).
"""
import json
import math
import os

CANDIDATES = (16, 32, 64, 128, 256, 512, 1024)
# launch choices swept at the best leaf size, in this order; the first value
# of each is the plan's automatic choice.  nf_blocks and had_windows only act
# on mixed plans.
KNOBS = (("job_rows", (0, 3, 4, 5, 6)),
         ("nf_blocks", (0, 5, 6)),
         ("had_windows", (0, 2, 4, 6, 8)),
         ("splitk_max", (0, 1, 2, 4, 16)))
MIXED_ONLY = ("nf_blocks", "had_windows")
KEEP_GAIN = 0.005


def time_run(plan, reps=3):
    """Device milliseconds of one kfmm_run of a plan whose points are set
    (minimum over reps, after one warm-up run)."""
    plan.run()
    plan.enable_timing(True)
    best = math.inf
    for _ in range(reps):
        plan.run()
        best = min(best, sum(plan.kernel_times().values()))
    plan.enable_timing(False)
    return best


def time_plan(K, tree, pts, np_, precision, tuning=None, reps=3):
    """Device milliseconds of one kfmm_run of a plan over `tree` with the
    given launch choices; the plan is built and released here."""
    plan = K.Plan(tree, np_, precision, tuning=tuning or None)
    try:
        plan.set_points(pts)
        return time_run(plan, reps)
    finally:
        plan.close()


def time_leaf_size(K, pts, ppb, np_, precision, reps=3, tuning=None):
    """Device milliseconds of one kfmm_run with ppb points per leaf; the tree
    and plan are built and released here."""
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
    try:
        return time_plan(K, tree, pts, np_, precision, tuning, reps)
    finally:
        tree.close()


def best_leaf_size(K, pts, np_, precision, candidates=CANDIDATES, reps=3):
    """(fastest leaf size, {leaf size: ms}) over the candidates that give a
    tree of at least two levels."""
    n = len(pts["sx"])
    table = {}
    for ppb in candidates:
        if ppb * 8 > n:
            continue
        table[ppb] = time_leaf_size(K, pts, ppb, np_, precision, reps)
    if not table:
        table[candidates[0]] = time_leaf_size(K, pts, candidates[0], np_, precision, reps)
    return min(table, key=table.get), table


def tune(K, pts, np_, precision, candidates=CANDIDATES, knobs=KNOBS, reps=3):
    """Leaf size, then launch choices by coordinate descent.  Returns a dict:
    ppb, tuning (the kfmm_tuning fields that differ from automatic), ms, and
    the measured sweep (leaf: {ppb: ms}, knobs: {name: {value: ms}})."""
    ppb, leaf_ms = best_leaf_size(K, pts, np_, precision, candidates, reps)
    best, best_ms = {}, leaf_ms[ppb]
    sweep = {}
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
    plan = K.Plan(tree, np_, precision)  # one plan, its launch choices changed in place
    plan.set_points(pts)
    try:
        for name, values in knobs:
            if name in MIXED_ONLY and precision != K.MIXED:
                continue
            sweep[name] = {0: best_ms} if best.get(name, 0) == 0 else {}
            for v in values:
                if v == best.get(name, 0):
                    continue
                cfg = dict(best)
                if v:
                    cfg[name] = v
                else:
                    cfg.pop(name, None)
                plan.set_tuning(cfg)
                ms = time_run(plan, reps)
                sweep[name][v] = ms
                if ms < best_ms * (1.0 - KEEP_GAIN):
                    best, best_ms = cfg, ms
    finally:
        plan.close()
        tree.close()
    return {"ppb": ppb, "tuning": best, "ms": best_ms,
            "sweep": {"leaf": leaf_ms, "knobs": sweep}}


def bucket_of(n):
    return int(round(math.log2(max(n, 1))))


class ConfigTable:
    """Tuned (leaf size, launch choices) per (distribution, log2 N bucket,
    NP, precision), optionally persisted as JSON at `path`.  knobs=() tunes
    the leaf size only."""

    def __init__(self, path=None, knobs=KNOBS, candidates=None):
        self.path = path
        self.knobs = knobs
        self.candidates = candidates
        self.picks = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.picks = json.load(f)

    @staticmethod
    def key(distribution, n, np_, precision):
        return f"{distribution}/{bucket_of(n)}/{np_}/{precision}"

    def config(self, K, distribution, n, np_, precision, seed=1):
        """(leaf size, tuning dict): the cached pick, or tune on a cloud of
        2^bucket points of this distribution and cache it."""
        k = self.key(distribution, n, np_, precision)
        if k not in self.picks:
            m = 1 << bucket_of(n)
            pts = K.generate_points(m, distribution, 0, seed)
            cand = self.candidates or CANDIDATES
            r = tune(K, pts, np_, precision, cand, self.knobs)
            self.picks[k] = {"ppb": r["ppb"], "tuning": r["tuning"], "ms": r["ms"], "n": m,
                             "leaf_ms": {str(a): b for a, b in r["sweep"]["leaf"].items()}}
            if self.path:
                with open(self.path, "w") as f:
                    json.dump(self.picks, f, indent=1, sort_keys=True)
        e = self.picks[k]
        return e["ppb"], dict(e.get("tuning", {}))

    def leaf_size(self, K, distribution, n, np_, precision, seed=1):
        return self.config(K, distribution, n, np_, precision, seed)[0]


def main(argv):
    """batched <out.json>: tune every (distribution, size bucket, NP,
    precision) of the batched workload (batched.specs(256)) with the leaf
    candidates 32..256 and write the table.  Run through the package loader:
      python -c "import __graft_entry__ as g; g.load_package();
                 from kifmm_b200 import autotune; autotune.main(['batched', 'out.json'])"
    """
    import __graft_entry__
    from . import batched
    K = __graft_entry__.load_package()
    if argv[0] == "batched":
        table = ConfigTable(argv[1], candidates=(32, 64, 128, 256))
        for prec in (K.MIXED, K.PLAIN_FP64):
            for sp in batched.specs(256):
                table.config(K, sp["distribution"], sp["n"], sp["np"], prec)
        print(json.dumps(table.picks))
