"""Benchmark: KIFMM 3-D Laplace solve throughput (Mpts/s) on B200.

Workload (one "step" = one full FMM evaluation of a fixed synthetic problem):
4,194,304 uniform points in [-1,1)^3 (the reference's "uniform" generator,
srand48(26)), densities in [0,1), NP=6, at most 512 points per leaf.  Tree,
lists and operators are built once (untimed, like the reference's preproc);
`value` times kfmm_run of the mixed form with inputs resident in HBM; `fp64`
the plain form the same way; `e2e` times kfmm_evaluate from pinned host
buffers (H2D of points and densities, the solve, D2H of the potentials).
The CPU reference (`cpu_baseline`, and `--impl reference`) is the
reference's own fmmd--omp_sse_block built from its sources, on the same
4,194,304-point configuration, all host threads.  Multi-GPU runs are replicas
(one independent solve per rank, weak scaling, no collective on the data
path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_POINTS = 4194304
NP = 6
PPB = 512
DIST = "uniform"
METRIC = "Mpts/s per FMM solve at 4M pts NP=6, mixed vs FP64 on B200, rel-L2 err vs FP64"
WORKLOAD = "KIFMM Laplace solve, 4194304 uniform points, NP=6, 512 pts/box"
FLOPS_PER_PAIR = 11.0    # reference convention, fmm/driver.cc:60
FLOPS_PER_CMAC = 8.0     # complex multiply-add, fmm/driver.cc:82 (4 * 2F per V pair)
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one near-field
# launch at this workload, from the latest ncu capture of each form on a B200
# of this pool (profiles/p2p_near_field_4m_np6.md); the algorithmic bytes
# (sources, targets, potentials and downward densities once each, FP64) are
# 348 MB.
NEAR_FIELD_DRAM_BYTES = {"mixed": 539.1e6, "fp64": 610.4e6}
# batched workload: independent solves, point counts log-uniform in
# [4096, 262144], half uniform cube / half ellipsoid surface, NP in {3, 4},
# leaf sizes and launch choices from the autotuner (its table for this
# workload, tuned on a B200, ships with the package; missing entries are
# tuned during the run), all solves in one CUDA graph
BATCH_SOLVES = 256
BATCH_LEAF_CANDIDATES = (32, 64, 128, 256)
BATCH_TABLE = os.path.join(ROOT, "kifmm--hybrid--double-only_b200", "tuning_data",
                           "b200_batched_configs.json")
# wall-clock budgets of the CPU reference runs (seconds): the warm-up and
# timed steps of `--impl reference` (one 4M-point solve takes ~8 s on 16
# host cores, so --steps 20 --warmup 5 fit), and the cpu_baseline leg of the
# GPU arm
REF_ARM_BUDGET_S = 330.0
CPU_BASELINE_BUDGET_S = 45.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_POINTS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-solves sub-measurement")
    ap.add_argument("--batch", type=int, default=BATCH_SOLVES)
    ap.add_argument("--no-sweep", action="store_true",
                    help="skip the leaf-size sweep of the metric's workload")
    ap.add_argument("--only", choices=["mixed", "fp64"], default=None,
                    help="profile one form only (no JSON line)")
    ap.add_argument("--had-tensor", action="store_true",
                    help="with --only mixed: the Hadamard on the tensor cores (kfmm_tuning.had_tensor 2)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(rank):
    """Each rank solves its own instance of the workload (replicas, weak
    scaling): same generator and sizes, seed 26 + rank."""
    return 26 + rank


def reduce_max(value, world, device):
    """Max over ranks of a per-rank time (the slowest replica sets the pace)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_mpts(n_per_rank, world, ms):
    """Whole-job throughput: all ranks' points over the slowest rank's time."""
    return n_per_rank * world / (ms * 1e3)


def sig(x, d=4):
    """Round floats for the JSON line (it must fit a log tail)."""
    if isinstance(x, float):
        return float(f"{x:.{d}g}")
    if isinstance(x, dict):
        return {k: sig(v, d) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [sig(v, d) for v in x]
    return x


def config_of(n):
    """The workload description shared by both arms (the reference arm runs
    the same points, NP and leaf size)."""
    return {"workload": WORKLOAD, "n_points": n, "np": NP, "pts_per_box": PPB,
            "distribution": DIST, "parallelism": "single",
            "l2": "inputs > L2 (points 268 MB, spectra 1.2 GB)"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def _run_ref_once(exe, n, env):
    t0 = time.time()
    r = subprocess.run([exe, str(n), DIST, str(PPB)], env=env, capture_output=True, text=True,
                       timeout=900)
    m = re.search(r"Total Execution Time:\s*([0-9.eE+-]+)", r.stderr)
    if r.returncode != 0 or not m:
        raise RuntimeError("fmmd--omp_sse_block failed: " + r.stderr[-300:])
    return float(m.group(1)), time.time() - t0


def run_reference_cpu(n, max_steps, warmup, budget_s):
    """The reference's own blocked-SSE CPU evaluator (fmmd--omp_sse_block,
    built from its sources into oracle/_ref) on the workload itself, all host
    threads pinned.  `warmup` untimed runs, then up to `max_steps` timed runs;
    runs stop early only when the next one would take the whole call past
    `budget_s` seconds of wall clock (at least one timed run).  Each run is
    one process: input generation and tree build are outside the reference's
    own 'Total Execution Time', which is what is timed."""
    import oracle  # noqa: F401  (checker package; only its build lives here)
    exe = os.path.join(ROOT, "oracle", "_ref", "fmmd--omp_sse_block")
    if not os.path.exists(exe):
        return None
    cores = os.cpu_count() or 1
    # the reference's own defaults NUMA=yes, BS=49, UPBS=1000 (fmm/util.c); threads
    # pinned one per core
    env = dict(os.environ, NP=str(NP), NV="1", OMP_NUM_THREADS=str(cores), OMP_PROC_BIND="true",
               OMP_PLACES="cores", GLIBC_TUNABLES="glibc.malloc.mmap_threshold=4096")
    t_start = time.time()
    walls = []
    done_warm = 0
    for _ in range(warmup):
        if walls and time.time() - t_start + max(walls) > budget_s:
            break
        walls.append(_run_ref_once(exe, n, env)[1])
        done_warm += 1
    times = []
    while len(times) < max(1, max_steps):
        if times and time.time() - t_start + max(walls) > budget_s:
            break
        t, wall = _run_ref_once(exe, n, env)
        times.append(t)
        walls.append(wall)
    t = statistics.median(times)
    # The reference computes its operators (SVD pseudo-inverses, translation
    # spectra) inside its timed Up/Down phases; this library does so at plan
    # creation, outside the timed solve.  A run of 32,768 points (same NP and
    # leaf size: every operator is built, the evaluation is a small share)
    # estimates that precompute, which is then taken off, so the comparison
    # times evaluation against evaluation.
    small = 32768
    pre, _ = _run_ref_once(exe, small, env)
    pre = min(pre, 0.5 * t)
    return {"value": n / (t - pre) / 1e6, "unit": "Mpts/s", "cores": cores, "kind": "reference",
            "cpu_model": cpu_model(),
            "runs": len(times), "warmup_runs": done_warm, "seconds": times, "precompute_s": pre,
            "value_with_precompute": n / t / 1e6,
            "sample": f"fmmd--omp_sse_block {n} {DIST} {PPB} NP={NP}, {cores} threads; median "
                      f"Total Execution Time of {len(times)} runs - precompute"}


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), or None."""
    try:
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    res = run_reference_cpu(N_POINTS, args.steps, args.warmup, REF_ARM_BUDGET_S)
    if res is None:
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/fmmd--omp_sse_block not built"}))
        return
    v = res["value"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mpts/s",
            "n_gpus": args.gpus, "steps": res["runs"], "warmup": res["warmup_runs"],
            "ms_per_step": 1e3 * statistics.median(res["seconds"]), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(N_POINTS),
            "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                 "precompute_s", "value_with_precompute",
                                                 "cpu_model")},
            "e2e": {"value": v, "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if res["runs"] < args.steps or res["warmup_runs"] < args.warmup:
        line["steps_note"] = (f"{res['warmup_runs']} warm-up and {res['runs']} timed runs of the "
                              f"{args.warmup} + {args.steps} requested fit the "
                              f"{REF_ARM_BUDGET_S:.0f} s budget of this arm")
    print(json.dumps(sig(line)))


SWEEP_LEAF_SIZES = (32, 64, 128, 256, 512)


def leaf_sweep(K, pts, sh, stream, steps, warmup, ids, direct):
    """The metric's workload in the mixed form at each candidate leaf size:
    device ms per kfmm_run (CUDA events on the launch stream, as `value`),
    and the reference's check (rel-L2 against the direct sum at the same
    sampled targets) at the fastest.  Trees are built on the device; each
    plan is released before the next is made."""
    import torch
    ms_by, best = {}, None
    args = [pts[k] for k in ("sx", "sy", "sz", "tx", "ty", "tz")]
    for ppb in SWEEP_LEAF_SIZES:
        tree = K.Tree(*args, ppb, device=True)
        plan = K.Plan(tree, NP, K.MIXED)
        try:
            plan.set_points(pts, sh)
            for _ in range(warmup):
                plan.run(sh)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(steps):
                plan.run(sh)
            b.record(stream)
            torch.cuda.synchronize()
            ms = a.elapsed_time(b) / steps
            ms_by[str(ppb)] = ms
            if best is None or ms < best[1]:
                pot = plan.potentials(sh)[ids]
                best = (ppb, ms, float(np.linalg.norm(pot - direct) / np.linalg.norm(direct)),
                        tree.desc.num_nodes)
        finally:
            plan.close()
            tree.close()
    n = len(pts["sx"])
    return sig({"ms_by_ppb": ms_by, "best_ppb": best[0], "best_ms": best[1],
                "best_Mpts_s": n / best[1] / 1e3, "best_rel_l2_err": best[2],
                "best_nodes": best[3]}, 4)


def time_plan(K, plan, sh, stream, steps, warmup, barrier, world, dev):
    """Device time per kfmm_run (max over ranks), phase and kernel-group
    breakdown of one run, and the near-field kernel alone (the dominant
    launch) on its launch stream."""
    import torch
    for _ in range(warmup):
        plan.run(sh)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        plan.run(sh)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = reduce_max(e0.elapsed_time(e1) / steps, world, dev)
    plan.enable_timing(True)
    kt = {k: [] for k in K.Plan.KERNEL_PHASES}
    ph = {}
    for _ in range(3):
        plan.run(sh)
        for k, v in plan.kernel_times().items():
            kt[k].append(v)
        ph = plan.phase_times()
    plan.enable_timing(False)
    kernels = {k: statistics.median(v) for k, v in kt.items()}
    nf_ms = []
    for _ in range(3):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        K.check(K.lib().kfmm_ulist_calc(plan.handle, sh), "ulist")
        b.record(stream)
        torch.cuda.synchronize()
        nf_ms.append(a.elapsed_time(b))
    return ms, ph, kernels, statistics.median(nf_ms)


def time_batched(K, count, stream, steps, warmup):
    """The batched workload in both forms: device time of one graph launch
    (all solves), Mpts/s, and per-solve distance of the mixed form to the
    plain one."""
    import torch
    import json as _json
    from kifmm_b200 import autotune, batched
    sp = batched.specs(count)
    out = {"solves": count, "points": sum(s["n"] for s in sp)}
    sh = stream.cuda_stream
    pots = {}
    table = autotune.ConfigTable(candidates=BATCH_LEAF_CANDIDATES)
    if os.path.exists(BATCH_TABLE):
        with open(BATCH_TABLE) as f:
            table.picks = _json.load(f)
    for name, prec in (("mixed", K.MIXED), ("fp64", K.PLAIN_FP64)):
        B = batched.BatchedSolves(K, sp, prec, table=table, nstreams=16)
        for _ in range(warmup):
            B.launch(sh)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            B.launch(sh)
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / steps
        pots[name] = B.potentials(sh)
        out[name] = {"ms": ms, "Mpts_s": B.total_points / (ms * 1e-3) / 1e6}
        B.close()
    rel = [float(np.linalg.norm(m - p) / np.linalg.norm(p)) for m, p in zip(pots["mixed"],
                                                                            pots["fp64"])]
    out["mixed_over_fp64"] = out["fp64"]["ms"] / out["mixed"]["ms"]
    out["rel_l2_mixed_vs_fp64_max"] = max(rel)
    return out


def phase_rooflines(K, st, kern_mixed, pipes, hbm_gbs):
    """Per-kernel-group rooflines of one mixed solve: achieved rate, the
    bound's peak and the fraction, plus the whole solve's roofline time (sum
    of the per-group bound times) against the measured solve time."""
    P, F = st["P"], st["F"]
    fpad = (F + 31) // 32 * 32
    nspec = st["spectra_bytes"] / (16.0 * F)  # boxes with a source or a target spectrum
    mufu = pipes["fp32_rsqrt_tops"] * 1e12
    fma32 = pipes["fp32_fma_tflops"] * 1e12
    dmma = pipes["fp64_dmma_tflops"] * 1e12
    hbm = hbm_gbs * 1e9
    ms = kern_mixed
    out = {}
    bound_s = 0.0

    def put(name, t_ms, achieved, peak, unit, bound_t):
        nonlocal bound_s
        out[name] = {"ms": t_ms, "achieved": achieved, "peak": peak, "unit": unit,
                     "frac": achieved / peak if peak else None}
        bound_s += bound_t

    nf = st["u_pairs"] / (ms["near_field"] * 1e-3)
    put("near_field", ms["near_field"], nf / 1e12, mufu / 1e12, "Tpair/s MUFU",
        st["u_pairs"] / mufu)
    s2m = st["s2m_pairs"] / max(ms["s2m"] * 1e-3, 1e-9)
    put("s2m", ms["s2m"], s2m / 1e12, mufu / 1e12, "Tpair/s MUFU", st["s2m_pairs"] / mufu)
    gemm_s = (ms["up_gemm"] + ms["down_gemm"]) * 1e-3
    put("level_gemms", ms["up_gemm"] + ms["down_gemm"], st["gemm_flops"] / gemm_s / 1e12,
        dmma / 1e12, "TF/s DMMA", st["gemm_flops"] / dmma)
    # V list against HBM: each kernel's compulsory bytes (spectra as complex
    # FP32, one pass; the FFTs also read or write the P-value surfaces)
    half = nspec / 2.0
    b_fft = half * fpad * 8.0 + st["num_nodes"] * P * 8.0
    b_had = 2.0 * half * fpad * 8.0
    for name, b in (("fft_src", b_fft), ("ifft_trg", b_fft)):
        put(name, ms[name], b / (ms[name] * 1e-3) / 1e9, hbm_gbs, "GB/s HBM", b / hbm)
    had_flops = st["hadamard_cmacs"] * FLOPS_PER_CMAC
    out["hadamard"] = {"ms": ms["hadamard"],
                       "achieved": b_had / (ms["hadamard"] * 1e-3) / 1e9, "peak": hbm_gbs,
                       "unit": "GB/s HBM", "frac": b_had / (ms["hadamard"] * 1e-3) / hbm,
                       "fma_frac": had_flops / (ms["hadamard"] * 1e-3) / fma32}
    bound_s += max(b_had / hbm, had_flops / fma32)
    # the V list as a whole (forward FFT, Hadamard, inverse FFT): compulsory
    # bytes over its time against HBM, beside the reference's own per-pair
    # byte model of the V list (fmm/driver.cc:120-136: per target box its
    # FP64 effective values, per V pair a source spectrum and a translation
    # vector, eff_data_size = (2np+2)(2np)^2 reals, fmm/trans.cc:107-115)
    eff = (2 * NP + 2) * (2 * NP) ** 2
    ref_bytes = 8.0 * eff * st["num_nodes"] + 16.0 * eff * st["v_pairs"]
    v_ms = ms["fft_src"] + ms["hadamard"] + ms["ifft_trg"]
    v_bytes = 2 * b_fft + b_had
    out["vlist"] = {"ms": v_ms, "achieved": v_bytes / (v_ms * 1e-3) / 1e9, "peak": hbm_gbs,
                    "unit": "GB/s HBM", "frac": v_bytes / (v_ms * 1e-3) / hbm,
                    "compulsory_GB": v_bytes / 1e9, "ref_model_GB": ref_bytes / 1e9,
                    "ref_model_rate_GBps": ref_bytes / (v_ms * 1e-3) / 1e9}
    total_ms = sum(ms.values())
    out["solve"] = {"roofline_ms": bound_s * 1e3, "measured_ms": total_ms,
                    "frac": bound_s * 1e3 / total_ms}
    return sig(out, 3)


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    import ctypes

    import torch
    import __graft_entry__

    K = __graft_entry__.load_package()
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    n = args.n

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # ---- setup (untimed): points, tree + lists, plans (operators, device arrays)
    pts = K.generate_points(n, DIST, 0, replica_seed(rank), 1000)
    targs = [pts[k] for k in ("sx", "sy", "sz", "tx", "ty", "tz")]
    t0 = time.time()
    tree = K.Tree(*targs, PPB)
    tree_host_s = time.time() - t0
    tree_device_s = None
    if not args.only:
        K.Tree(*targs, PPB, device=True).close()  # CUDA start-up and first-call costs
        t0 = time.time()
        K.Tree(*targs, PPB, device=True).close()
        tree_device_s = time.time() - t0
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream
    if args.only:
        pl = K.Plan(tree, NP, K.MIXED if args.only == "mixed" else K.PLAIN_FP64,
                    tuning={"had_tensor": 2} if args.had_tensor else None)
        pl.set_points(pts, sh)
        for _ in range(args.warmup + args.steps):
            pl.run(sh)
        torch.cuda.synchronize()
        print(json.dumps({"profile_only": args.only, "n": n}))
        return
    plans = {"mixed": K.Plan(tree, NP, K.MIXED), "fp64": K.Plan(tree, NP, K.PLAIN_FP64)}
    for pl in plans.values():
        pl.set_points(pts, sh)
    st = plans["fp64"].stats()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.5)
    res = {}
    for name, pl in plans.items():
        res[name] = time_plan(K, pl, sh, stream, args.steps, args.warmup, barrier, world, dev)
    clk = clocks.stop()
    pots = {name: pl.potentials(sh) for name, pl in plans.items()}

    # ---- the mixed form replayed as a one-plan batch (one CUDA graph launch
    # per solve), against the plain form's direct launches
    graph_ms = {}
    for name, pl in plans.items():
        bt = K.Batch([pl], 1)
        for _ in range(args.warmup):
            bt.launch(sh)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            bt.launch(sh)
        b.record(stream)
        torch.cuda.synchronize()
        bt.wait(sh)
        graph_ms[name] = reduce_max(a.elapsed_time(b) / args.steps, world, dev)
        bt.close()

    # ---- the reference's check: rel-L2 vs an FP64 direct sum on 1000 targets
    ids = pts["check_ids"]
    dsrc = [torch.tensor(pts[k], device=dev) for k in ("sx", "sy", "sz", "den")]
    dtrg = [torch.tensor(pts[k][ids], device=dev) for k in ("tx", "ty", "tz")]
    direct = torch.zeros(len(ids), dtype=torch.float64, device=dev)
    K.check(K.lib().kfmm_direct_evaluation(len(ids), *[x.data_ptr() for x in dtrg],
                                           direct.data_ptr(), n, *[x.data_ptr() for x in dsrc],
                                           sh), "direct")
    torch.cuda.synchronize()
    direct = direct.cpu().numpy()
    err = {k: float(np.linalg.norm(v[ids] - direct) / np.linalg.norm(direct))
           for k, v in pots.items()}
    mixed_vs_fp64 = float(np.linalg.norm(pots["mixed"] - pots["fp64"]) /
                          np.linalg.norm(pots["fp64"]))

    # ---- e2e through the C ABI from pinned host buffers (mixed form): every
    # step copies its points and densities host->device and its potentials
    # back.  Steps are queued back to back with kfmm_evaluate_async, so one
    # step's copies overlap the previous step's solve; the timed region ends
    # when the last step's potentials are in host memory.  The synchronous
    # kfmm_evaluate (one call, one wait) is timed beside it as `sync_ms`.
    hp = {k: torch.from_numpy(pts[k]).pin_memory() for k in ("sx", "sy", "sz", "den", "tx", "ty",
                                                           "tz")}
    hout = torch.empty(n, dtype=torch.float64).pin_memory()
    fp = ctypes.POINTER(ctypes.c_double)
    cargs = [ctypes.cast(hp[k].data_ptr(), fp) for k in ("sx", "sy", "sz", "den", "tx", "ty",
                                                          "tz")] + [ctypes.cast(hout.data_ptr(), fp)]
    plan = plans["mixed"]
    L = K.lib()
    for _ in range(max(1, args.warmup)):
        K.check(L.kfmm_evaluate(plan.handle, *cargs, sh), "evaluate")
    barrier()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        K.check(L.kfmm_evaluate(plan.handle, *cargs, sh), "evaluate")
    b.record(stream)
    torch.cuda.synchronize()
    e2e_sync_ms = reduce_max(a.elapsed_time(b) / args.steps, world, dev)
    assert np.array_equal(hout.numpy(), pots["mixed"]), "e2e potentials differ from the resident run"
    hout.fill_(0.0)
    barrier()
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(args.steps):
        K.check(L.kfmm_evaluate_async(plan.handle, *cargs, sh), "evaluate_async")
    K.check(L.kfmm_evaluate_join(plan.handle, sh), "evaluate_join")
    b.record(stream)
    K.check(L.kfmm_evaluate_wait(plan.handle, sh), "evaluate_wait")
    torch.cuda.synchronize()
    e2e_ms = reduce_max(a.elapsed_time(b) / args.steps, world, dev)
    assert np.array_equal(hout.numpy(), pots["mixed"]), "e2e potentials differ from the resident run"

    # ---- the same workload at the sweep-best leaf size (one GPU only: the
    # replicas of a multi-GPU run report the metric's 512 alone)
    sweep_res = None
    if world == 1 and not args.no_sweep:
        sweep_res = leaf_sweep(K, pts, sh, stream, max(1, min(args.steps, 5)),
                               max(1, min(args.warmup, 2)), ids, direct)

    peaks = measured_peaks()
    hbm_gbs = peaks.get("hbm_gbs") or 6650.0
    pipes = K.measure_peaks()
    pairs = st["u_pairs"]

    def roof(name, nf_ms):
        rate = pairs / (nf_ms * 1e-3)
        ceil = pipes["fp32_rsqrt_tops" if name == "mixed" else "fp64_rsqrt_tops"] * 1e12
        # 11 flops per pair (fmm/driver.cc:60) x pairs per launch / launch time;
        # peak = one pair per measured reciprocal square root
        return {"bound": "fp32 rsqrt (MUFU)" if name == "mixed" else "fp64 rsqrt",
                "kernel": f"p2p_warp_kernel<{name}>",
                "achieved": FLOPS_PER_PAIR * rate / 1e12, "peak": FLOPS_PER_PAIR * ceil / 1e12,
                "unit": "TFLOP/s", "frac": rate / ceil,
                "traffic": NEAR_FIELD_DRAM_BYTES[name] if n == N_POINTS else None,
                "algorithmic_bytes": 32.0 * n + 32.0 * n + 8.0 * n + 8.0 * st["num_nodes"] * st["P"],
                "launch_ms": nf_ms}

    batched_res = None
    if not args.no_batched and args.batch > 0:
        batched_res = time_batched(K, args.batch, stream, max(1, min(args.steps, 5)),
                                   max(1, args.warmup))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            r = run_reference_cpu(n, 3, 0, CPU_BASELINE_BUDGET_S)
            if r:
                cpu = {k: r[k] for k in ("value", "unit", "cores", "kind", "sample",
                                         "precompute_s", "value_with_precompute", "runs",
                                         "cpu_model")}
        except Exception as ex:  # reported, not fatal
            cpu = {"value": None, "error": str(ex)[:200]}

    ms_mixed, ph_mixed, kern_mixed, nf_mixed = res["mixed"]
    ms_fp64, ph_fp64, kern_fp64, nf_fp64 = res["fp64"]
    rl = roof("mixed", nf_mixed)
    phr = phase_rooflines(K, st, kern_mixed, pipes, hbm_gbs)
    # The line: the standard keys first, then the extras, ordered so that the
    # most-read figures (the plain form, the ratio, the errors) close it.
    line = {
        "metric": METRIC, "value": aggregate_mpts(n, world, ms_mixed), "unit": "Mpts/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64 (mixed)", "data": "synthetic",
        "config": dict(config_of(n), parallelism=f"replicas x{world}" if world > 1 else "single"),
        "roofline": rl,
        "cpu_baseline": cpu,
        "e2e": {"value": aggregate_mpts(n, world, e2e_ms), "unit": "Mpts/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": 7 * 8 * n, "d2h_bytes_per_step": 8 * n,
                "api": "kfmm_evaluate_async back to back", "sync_ms": e2e_sync_ms},
        "gpu_launches": int(plans["mixed"].stats()["launches"]) * args.steps,  # kfmm_run steps
        "clocks": clk,
        "tree": {"nodes": st["num_nodes"], "u_pairs": pairs, "v_pairs": st["v_pairs"],
                 "build_s_host": tree_host_s, "build_s_device": tree_device_s},
        "batched": batched_res,
        "leaf_sweep": sweep_res,
        "graph_4m": {"mixed_ms": graph_ms["mixed"], "fp64_ms": graph_ms["fp64"],
                     "mixed_over_fp64_direct": ms_fp64 / graph_ms["mixed"]},
        "phase_roofline": {k: ({"ms": v["ms"], "frac": v["frac"], "of": v["unit"].split()[-1]}
                               if "ms" in v and k not in ("solve", "vlist") else
                               {kk: vv for kk, vv in v.items() if kk not in ("peak", "unit")}
                               if k == "vlist" else v) for k, v in phr.items()},
        "phases_ms": {"mixed": ph_mixed, "fp64": ph_fp64},
        "fp64": {"value": aggregate_mpts(n, world, ms_fp64), "ms_per_step": ms_fp64,
                 "rel_l2_err": err["fp64"], "near_field_frac": roof("fp64", nf_fp64)["frac"]},
        "rel_l2_err": err["mixed"], "rel_l2_vs_fp64": mixed_vs_fp64,
        "mixed_over_fp64": ms_fp64 / ms_mixed,
    }
    if rank == 0:
        print(json.dumps(sig(line)))
    for pl in plans.values():
        pl.close()
    tree.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
