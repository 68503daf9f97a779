"""Many independent solves of uneven size replayed by one CUDA graph.

``specs`` draws the solves of the batched workload: point counts
log-uniform in [nmin, nmax], half on the uniform cube and half on the
ellipsoid surface, NP from {3, 4}, seeds base + index.  ``BatchedSolves``
builds each solve's tree with the leaf size, and its plan with the launch
choices, that the autotuner picks for its (distribution, size bucket, NP,
precision), uploads the points and captures every kfmm_run into a single
graph (kfmm_batch_create); ``launch`` replays all solves, ``potentials``
waits for the launch and reads them back.
"""
import numpy as np

from . import autotune


def specs(count, nmin=4096, nmax=262144, seed=2024):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        dist = "uniform" if i % 2 == 0 else "ellipsoidSurface"
        np_ = int(rng.choice([3, 4]))
        out.append({"distribution": dist, "n": n, "np": np_, "seed": seed + i})
    return out


class BatchedSolves:
    def __init__(self, K, solves, precision, table=None, nstreams=16, num_check=0):
        self.K = K
        self.table = table if table is not None else autotune.ConfigTable()
        self.solves = []
        for sp in solves:
            pts = K.generate_points(sp["n"], sp["distribution"], 0, sp["seed"], num_check)
            ppb, tuning = self.table.config(K, sp["distribution"], sp["n"], sp["np"], precision)
            tree = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], ppb)
            plan = K.Plan(tree, sp["np"], precision, tuning=tuning)
            plan.set_points(pts)
            self.solves.append({**sp, "ppb": ppb, "tuning": tuning, "pts": pts, "tree": tree,
                                "plan": plan})
        self.batch = K.Batch([s["plan"] for s in self.solves], nstreams)

    @property
    def total_points(self):
        return sum(s["n"] for s in self.solves)

    def launch(self, stream=None):
        self.batch.launch(stream)

    def potentials(self, stream=None):
        self.batch.wait(stream)
        return [s["plan"].potentials() for s in self.solves]

    def close(self):
        self.batch.close()
        for s in self.solves:
            s["plan"].close()
            s["tree"].close()
