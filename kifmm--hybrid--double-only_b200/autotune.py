"""Leaf-size autotuner: a measured sweep over points-per-box candidates.

The evaluator's cost splits between the near field (grows with the leaf
size) and the far field (grows with the number of boxes); the best leaf size
depends on the point distribution, the point count, NP and the precision
form.  ``best_leaf_size`` builds the tree and plan for every candidate on the
given cloud and times kfmm_run on the device (phase timers, CUDA events),
returning the fastest.  ``LeafSizeTable`` caches picks per (distribution,
log2 point-count bucket, NP, precision) so that a batch of many clouds is
tuned once per bucket on a representative cloud of the bucket's geometric
middle size.

The reference has no tuner: it takes the leaf size from its command line
(fmm/driver.cc:216).
"""
import json
import math
import os

CANDIDATES = (16, 32, 64, 128, 256, 512, 1024)


def time_leaf_size(K, pts, ppb, np_, precision, reps=3):
    """Device milliseconds of one kfmm_run (minimum over reps, after one
    warm-up run) with ppb points per leaf; the tree and plan are built and
    released here."""
    tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
    plan = K.Plan(tree, np_, precision)
    try:
        plan.set_points(pts)
        plan.run()
        plan.enable_timing(True)
        best = math.inf
        for _ in range(reps):
            plan.run()
            best = min(best, sum(plan.phase_times().values()))
        return best
    finally:
        plan.close()
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


def bucket_of(n):
    return int(round(math.log2(max(n, 1))))


class LeafSizeTable:
    """Leaf-size picks per (distribution, log2 N bucket, NP, precision),
    optionally persisted as JSON at `path`."""

    def __init__(self, path=None):
        self.path = path
        self.picks = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.picks = json.load(f)

    @staticmethod
    def key(distribution, n, np_, precision):
        return f"{distribution}/{bucket_of(n)}/{np_}/{precision}"

    def leaf_size(self, K, distribution, n, np_, precision, seed=1):
        """The cached pick, or tune on a cloud of 2^bucket points of this
        distribution and cache it."""
        k = self.key(distribution, n, np_, precision)
        if k not in self.picks:
            m = 1 << bucket_of(n)
            pts = K.generate_points(m, distribution, 0, seed)
            ppb, table = best_leaf_size(K, pts, np_, precision)
            self.picks[k] = {"ppb": ppb, "ms": {str(a): b for a, b in table.items()}, "n": m}
            if self.path:
                with open(self.path, "w") as f:
                    json.dump(self.picks, f, indent=1, sort_keys=True)
        return self.picks[k]["ppb"]
