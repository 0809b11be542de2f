#!/usr/bin/env python
"""Throughput benchmark: converged BFGS runs per second on one B200 (or N
replicas under torchrun, one per GPU, weak scaling).

A step is one full optimisation call on the workload: PSO seeding (or
uniform starts when the workload has PSO off), every BFGS run, and the
argmin/census reduction, with inputs resident in HBM.  `value` counts the
runs that finish with status 1 (||grad|| < tol) per second of device time;
`e2e` is the same metric through the public host-buffer calls -- the batch
plan zeus_batch_plan_run for batched workloads, zeus_optimize otherwise --
with the host inputs (starts, objective data) copied in and every class's
best run, coordinates and census copied back inside the timed region.

  python bench.py [--workload W] [--steps K] [--warmup W] [--gpus N]
  python bench.py --impl reference ...   # the reference's own sequential
                                         # BFGS on the host cores
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# transcendental functions (sin, cos, exp, log, pow, lgamma, sqrt) are
# counted as this many FP64 flops in the algorithmic work model
TRANSCENDENTAL_FLOPS = 20


# ---------------------------------------------------------------- work model
def flops_per_eval(kind: int, dim: int, nbins: int = 100) -> float:
    """Algorithmic flops of one f(x) (fast path) including the trial point
    x + alpha p (2 dim)."""
    T = TRANSCENDENTAL_FLOPS
    base = 2 * dim
    if kind == 0:  # Rosenbrock: 8 per term
        return base + 8 * (dim - 1)
    if kind == 1:  # Rastrigin: cos + 4 per coordinate
        return base + (T + 4) * dim
    if kind == 2:  # Ackley: cos + 3 per coordinate, 2 exp + sqrt + 10
        return base + (T + 3) * dim + 3 * T + 10
    if kind == 3:  # Gaussian: C x (2 dim^2) + x.(Cx) (2 dim)
        return base + 2 * dim * dim + 2 * dim
    if kind == 4:  # Poisson NLL: exp + 10 per bin, log a
        return base + (T + 10) * nbins + T
    raise ValueError(kind)


def flops_per_grad(kind: int, dim: int, gradient: str, nbins: int = 100) -> float:
    T = TRANSCENDENTAL_FLOPS
    if gradient == "adjoint":
        if kind == 0:
            return 13 * (dim - 1)
        if kind == 1:
            return (2 * T + 6) * dim
        if kind == 2:
            return (2 * T + 6) * dim + 3 * T + 12
        if kind == 3:
            # CTA layout (dim > 32): the accepted trial's value pass formed
            # C x already; otherwise C x (2 dim^2) and x.(Cx)
            return 2 * dim if dim > 32 else 2 * dim * dim + 2 * dim
        if kind == 4:
            return (T + 18) * nbins + T + 1
    # dual: dim forward passes of the dual-number body
    if kind == 0:
        per = 24 * (dim - 1)
    elif kind == 1:
        per = (2 * T + 18) * dim
    elif kind == 2:
        per = (3 * T + 16) * dim + 4 * T + 20
    elif kind == 3:
        per = 10 * dim * dim + 4
    else:
        per = (8 * T + 40) * nbins
    return dim * per


def flops_per_iteration(dim: int) -> float:
    """Fast-mode linear algebra per BFGS iteration: p = -H g and u = H y
    (2 dim^2 each), the symmetric rank-2 update (4 per packed element) and
    the O(dim) dot products / vector updates."""
    return 6 * dim * dim + 15 * dim


def algorithmic_flops(jobs_counters) -> float:
    total = 0.0
    for (kind, dim, gradient, nbins), cnt in jobs_counters:
        it, ev, gr = cnt[:, 0].sum(), cnt[:, 1].sum(), cnt[:, 2].sum()
        total += (it * flops_per_iteration(dim) + ev * flops_per_eval(kind, dim, nbins)
                  + gr * flops_per_grad(kind, dim, gradient, nbins))
    return float(total)


# ---------------------------------------------------------------- traffic
# DRAM bytes (read + write) of one launch of the dominant kernel, from ncu
# captures summarised under profiles/:
#  * mixed: the batch kernel on the 1/8-size mixed batch (551 KB read, no
#    bytes written: the results stay in L2), scaled to the full batch by its
#    runs (the bytes are the starts read and the results written, in
#    proportion to the runs);
#  * gaussian150: the CTA-layout BFGS kernel at full size (1.50 MB read: C,
#    the starts and the first touch of the outputs).
MEASURED_TRAFFIC = {
    "mixed": (8 * (600064 + 1024), "1/8-size capture x 8, batch kernel"),
    "gaussian150": (1503232, "full-size capture"),
}


def traffic_of(workload: str) -> dict:
    t = MEASURED_TRAFFIC.get(workload)
    if t is None:
        return {"traffic": None}
    return {"traffic": t[0], "traffic_unit": "bytes per launch",
            "traffic_source": f"ncu dram__bytes_read.sum + dram__bytes_write.sum, {t[1]} "
                              "(ncu summaries under profiles/)"}


# ---------------------------------------------------------------- ranks
def job_totals(units: float, ms: float, world: int, device) -> tuple[float, float]:
    """Whole-job (units summed over ranks, step time = the slowest rank's).
    Every rank calls it at the same point (two collectives)."""
    if world <= 1:
        return units, ms
    import torch

    t_units = torch.tensor([units], dtype=torch.float64, device=device)
    t_ms = torch.tensor([ms], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t_units, op=torch.distributed.ReduceOp.SUM)
    torch.distributed.all_reduce(t_ms, op=torch.distributed.ReduceOp.MAX)
    return float(t_units[0]), float(t_ms[0])


# ---------------------------------------------------------------- workloads
class Job:
    """One class of a workload: objective, runs, bounds, PSO iterations (<0:
    uniform starts), BFGS settings, and the layout used when the class runs
    in a persistent batch."""

    def __init__(self, name, obj_fn, n, lo, hi, pso_iter, max_iter, required, tol=1e-8,
                 runs_per_instance=0, ref_runs=64):
        self.name, self.obj_fn, self.n = name, obj_fn, n
        self.lo, self.hi, self.pso_iter = lo, hi, pso_iter
        self.max_iter, self.required, self.tol = max_iter, required, tol
        self.runs_per_instance = runs_per_instance
        # whole runs of this class in each step of the reference's timed
        # sample (0: the class is too heavy for the reference to finish a
        # run inside a step; it enters only the whole-workload estimate)
        self.ref_runs = ref_runs
        self.n_full = n  # before --scale: the objective's data holds n_full / rpi instances

    def make_objective(self):
        """The class's objective; a scaled-down class with per-instance data
        keeps only the instances its runs use."""
        obj = self.obj_fn()
        rpi = self.runs_per_instance
        if rpi and obj.idata is not None and self.n != self.n_full:
            import zeus_b200 as zb

            nb = len(obj.idata) // (self.n_full // rpi)
            used = (self.n + rpi - 1) // rpi
            obj = zb.PoissonNLL(obj.idata[:used * nb], obj.data[:used * nb])
        return obj


def dijet_objective(toys=512, nbins=100, seed=7):
    """512 Poisson toy spectra of the dijet shape, stored one after another
    (the batch's per-instance data): 100 log-spaced bins in x = m/13000 over
    [0.085, 0.54], lambda = p0 (1-x)^p1 / x^(p2 + p3 ln x), p = (1e6, 10, 5,
    0.1) scaled to 1e6 events."""
    import zeus_b200 as zb

    edges = np.geomspace(0.085, 0.54, nbins + 1)
    x = 0.5 * (edges[1:] + edges[:-1])
    lam = (1 - x) ** 10.0 / x ** (5.0 + 0.1 * np.log(x))
    lam *= 1e6 / lam.sum()
    rng = np.random.default_rng(seed)
    k = rng.poisson(np.tile(lam, (toys, 1))).astype(np.int32)
    obj = zb.PoissonNLL(k.reshape(-1), np.tile(x, toys))
    return obj


def workloads():
    import zeus_b200 as zb

    return {
        "mixed": dict(
            desc="uneven persistent batch: 8192 runs, Rosenbrock D in {2,8,32,64,128} "
                 "(1366,1366,1365,1365,1365) + Ackley-30 (1365), uniform starts "
                 "(Philox, seed 42 + class), PSO off, <=10000 iters, tol 1e-8, "
                 "stop-early off",
            batch=True,
            # the reference's O(D^4) update: ~0.2 s per 128-D iteration and
            # ~12 ms per 64-D iteration on one host core, minutes to half an
            # hour per run, so those two classes are estimated, not sampled
            jobs=[Job("rosenbrock128", lambda: zb.Rosenbrock(128), 1365, -5.0, 5.0, -1,
                      10000, 1 << 30, ref_runs=0),
                  Job("rosenbrock64", lambda: zb.Rosenbrock(64), 1365, -5.0, 5.0, -1,
                      10000, 1 << 30, ref_runs=0),
                  Job("ackley30", lambda: zb.Ackley(30), 1365, -32.768, 32.768, -1,
                      10000, 1 << 30),
                  Job("rosenbrock32", lambda: zb.Rosenbrock(32), 1365, -5.0, 5.0, -1,
                      10000, 1 << 30),
                  Job("rosenbrock8", lambda: zb.Rosenbrock(8), 1366, -5.0, 5.0, -1,
                      10000, 1 << 30),
                  Job("rosenbrock2", lambda: zb.Rosenbrock(2), 1366, -5.0, 5.0, -1,
                      10000, 1 << 30)]),
        "gaussian150": dict(
            desc="150-D Gaussian 0.5 x^T C x, C_ii = 75.5, C_ij = 0.5, 1024 starts, "
                 "PSO 10, <=10000 iters, tol 1e-8, stop-early off",
            batch=False,
            jobs=[Job("gaussian150", lambda: zb.Gaussian(zb.gaussian_matrix(150)), 1024,
                      -5.0, 5.0, 10, 10000, 1 << 30, ref_runs=16)]),
        "multimodal": dict(
            desc="Rastrigin-10 (A=10) 16384 starts in +-5.12 and Ackley-30 16384 starts "
                 "in +-32.768, PSO 20 each (CUDA graph), <=10000 iters, tol 1e-8, "
                 "stop-early off; both classes in one persistent batch",
            batch=True,
            jobs=[Job("ackley30", lambda: zb.Ackley(30), 16384, -32.768, 32.768, 20, 10000,
                      1 << 30),
                  Job("rastrigin10", lambda: zb.Rastrigin(10), 16384, -5.12, 5.12, 20,
                      10000, 1 << 30)]),
        "dijet": dict(
            desc="512 Poisson toy dijet spectra x 256 uniform starts in [0,10]^4, "
                 "4-parameter NLL, one persistent batch of 131072 runs, <=10000 iters, "
                 "tol 1e-8, stop-early off; then d(fit)/d(counts) of each toy's best "
                 "fit (implicit-function adjoint, one extra launch)",
            batch=True,
            jobs=[Job("dijet", lambda: dijet_objective(), 131072, 0.0, 10.0, -1, 10000,
                      1 << 30, runs_per_instance=256)]),
        "rosenbrock2": dict(
            desc="2-D Rosenbrock, 1024 starts, PSO 10, <=10000 BFGS iters, "
                 "required_convergences 100, tol 1e-8, seed 42",
            batch=False,
            jobs=[Job("rosenbrock2", lambda: zb.Rosenbrock(2), 1024, -5.0, 5.0, 10,
                      10000, 100)]),
    }


METRIC = "converged runs/s at ||grad||<1e-8"


def workload_config(args, wl, world):
    """The workload the metric is quoted on; the same dict in both arms."""
    return {"workload": args.workload, "description": wl["desc"],
            "runs_per_step": sum(j.n for j in wl["jobs"]) * world,
            "l2": "1 GiB buffer written between timed steps (GPU arm)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def wait_samples(self, n, timeout=3.0):
        t0 = time.time()
        while self.proc is not None and len(self.rows) < n and time.time() - t0 < timeout:
            time.sleep(0.02)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- GPU arm
def measure_fp64_peak(torch, zb):
    """Measured FP64 FMA throughput of this GPU (TFLOP/s), best of 5."""
    import ctypes as C

    g, b = C.c_int32(), C.c_int32()
    zb.lib().zeus_probe_fp64_shape(C.byref(g), C.byref(b))
    sink = torch.empty(g.value * b.value, dtype=torch.float64, device="cuda")
    iters = 20000
    st = torch.cuda.current_stream()
    best = 0.0
    for _ in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        zb.check(zb.lib().zeus_probe_fp64(iters, sink.data_ptr(), st.cuda_stream))
        e1.record(st)
        torch.cuda.synchronize()
        fl = g.value * b.value * iters * 8 * 2
        best = max(best, fl / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


def run_gpu(args, rank, world, local_rank):
    import ctypes as C

    import torch

    import zeus_b200 as zb
    from zeus_b200.device import Batch, BatchJob, BfgsRun, DeviceProblem

    torch.cuda.set_device(local_rank)
    wl = workloads()[args.workload]
    jobs = wl["jobs"]
    if args.scale != 1.0:
        for j in jobs:
            per = j.runs_per_instance or 1
            j.n = max(per, int(round(j.n * args.scale / per)) * per)
    dev = torch.device("cuda", local_rank)
    # a dedicated (non-legacy) stream: the PSO loop is captured into a CUDA
    # graph on it
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    seed = args.seed + 1000003 * rank
    L = zb.lib()

    state = []
    for ci, j in enumerate(jobs):
        obj = j.make_objective()
        dp = DeviceProblem(obj, dev)
        d = obj.dim
        starts = torch.empty((j.n, d), dtype=torch.float64, device=dev)
        s = dict(job=j, obj=obj, dp=dp, starts=starts, seed=seed + ci,
                 cen=torch.zeros((6,), dtype=torch.int32, device=dev),
                 nbins=0 if obj.idata is None else len(obj.idata) // max(
                     1, (j.n + j.runs_per_instance - 1) // j.runs_per_instance
                     if j.runs_per_instance else 1))
        if j.pso_iter >= 0:
            pws = L.zeus_pso_workspace_size(j.n, d)
            s["pso"] = dict(pbf=torch.empty((j.n,), dtype=torch.float64, device=dev),
                            gb=torch.empty((d + 1,), dtype=torch.float64, device=dev),
                            ws=torch.empty((max(pws, 1),), dtype=torch.uint8, device=dev),
                            wsz=pws)
        s["bj"] = BatchJob(dp, starts, required=j.required, runs_per_instance=j.runs_per_instance)
        if j.runs_per_instance and obj.kind == 4:
            # d(fitted parameters)/d(bin counts) of every toy's best fit
            toys = j.n // j.runs_per_instance
            s["sens"] = (torch.empty((toys, 6), dtype=torch.float64, device=dev),
                         torch.empty((toys, 4, s["nbins"]), dtype=torch.float64, device=dev))
        if not j.runs_per_instance:
            cfg_fast = zb.make_config(j.max_iter, j.required, j.tol, "fast", "adjoint")
            s["run"] = BfgsRun(dp, j.n, cfg_fast, device=dev)
        state.append(s)
    # layout autotuner: every class that is not CTA-sized gets its fastest
    # built layout recorded before anything is timed (the batch and the
    # standalone launches read the table)
    tuned = {}
    if not args.no_autotune:
        for s in state:
            j, obj = s["job"], s["obj"]
            if obj.dim > 32 and not (obj.dim % 32 == 0 and obj.kind in (0, 1, 2)):
                continue
            ns = min(j.n, 16384)
            if j.runs_per_instance:
                ns = max(j.runs_per_instance, ns // j.runs_per_instance * j.runs_per_instance)
                # one data instance is enough to tune on
                prob_obj = zb.PoissonNLL(obj.idata[:s["nbins"]], obj.data[:s["nbins"]])
            else:
                prob_obj = obj
            # full-length runs: a class's time in the batch is set as much by
            # its longest runs (those iterating to MAX_ITER) as by its bulk
            lay, tile, ms = zb.autotune(prob_obj, n_sample=ns, max_iter=j.max_iter,
                                        tol=j.tol, lower=j.lo, upper=j.hi, device=dev)
            tuned[j.name] = {"layout": ["auto", "thread", "tile", "cta", "rows"][lay], "tile": tile,
                             "sample_ms": ms}
    batch = Batch([s["bj"] for s in state], jobs[0].max_iter, jobs[0].tol) if wl["batch"] else None
    # row classes of D >= 128 run beside the batch kernel as a companion
    # launch of the standalone row kernel (zeus_batch_device)
    companions = sum(1 for s in state if tuned.get(s["job"].name, {}).get("layout") == "rows"
                     and s["obj"].dim >= 128) if batch is not None else 0

    def gen_starts(s):
        j, prob = s["job"], s["dp"].c()
        if j.pso_iter >= 0:
            p = s["pso"]
            zb.check(L.zeus_pso_device(C.byref(prob), s["seed"], j.n, j.lo, j.hi, j.pso_iter,
                                       0.5, 1.2, 1.5, s["starts"].data_ptr(),
                                       p["pbf"].data_ptr(), p["gb"].data_ptr(),
                                       p["ws"].data_ptr(), p["wsz"], sh))
            return 2 + j.pso_iter
        zb.check(L.zeus_starts_uniform(s["seed"], j.n, s["obj"].dim, j.lo, j.hi,
                                       s["starts"].data_ptr(), sh))
        return 1

    def census(s, out):
        zb.check(L.zeus_census_device(out.fval.data_ptr(), out.status.data_ptr(),
                                      out.x.data_ptr(), s["job"].n, s["obj"].dim, None,
                                      s["cen"].data_ptr(), sh))
        return 1

    def step_fast():
        """The adjoint + persistent-batched form; returns (events, launches)."""
        launches = sum(gen_starts(s) for s in state)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if batch is not None:
            batch.launch(stream)
            launches += 1 + companions + sum(1 for s in state if s["nbins"])
            outs = [s["bj"] for s in state]
        else:
            for s in state:
                s["run"].launch(s["starts"], stream=stream)
                launches += 1 + (1 if s["nbins"] else 0)
            outs = [s["run"] for s in state]
        e1.record(stream)
        for s, o in zip(state, outs):
            launches += census(s, o)
            if "sens" in s:
                best, sens = s["sens"]
                prob = s["bj"].c().problem
                zb.check(L.zeus_nll_sensitivity_device(
                    C.byref(prob), best.shape[0], s["job"].runs_per_instance,
                    o.fval.data_ptr(), o.x.data_ptr(), best.data_ptr(), sens.data_ptr(), sh))
                launches += 1
        return (e0, e1), launches, outs

    flush = torch.empty(256 * 1024 * 1024, dtype=torch.float32, device=dev)

    for _ in range(args.warmup):
        step_fast()
    torch.cuda.synchronize()

    clocks = ClockSampler(local_rank)
    if rank == 0:
        clocks.start()
        clocks.wait_samples(1)
    times, kern_ms, conv, launches = [], [], [], 0
    outs = None
    for k in range(args.steps):
        flush.zero_()  # 1 GiB written: larger than the 126 MB L2
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        (e0, e1), nl, outs = step_fast()
        t1.record(stream)
        torch.cuda.synchronize()
        launches += nl
        times.append(t0.elapsed_time(t1))
        kern_ms.append(e0.elapsed_time(e1))
        conv.append(sum(int(s["cen"][1].item()) for s in state))
    if rank == 0:
        clocks.wait_samples(len(clocks.rows) + 1)
        clocks.stop()
    counters = [((s["obj"].kind, s["obj"].dim, "adjoint", max(s["nbins"], 100)),
                 o.counters.cpu().numpy()) for s, o in zip(state, outs)]
    step_ms = float(np.mean(times))
    conv_mean = float(np.mean(conv))
    conv_all, step_ms_all = job_totals(conv_mean, step_ms, world, dev)
    value = conv_all / (step_ms_all * 1e-3)

    flops = algorithmic_flops(counters)
    kms = float(np.mean(kern_ms))
    achieved = flops / (kms * 1e-3) / 1e12
    peak = measure_fp64_peak(torch, zb) if rank == 0 else None

    # the plain form: dual-number gradients, one standalone launch per class
    plain = None
    if not args.no_plain:
        pl_runs = []
        for s in state:
            j = s["job"]
            if j.runs_per_instance:
                pj = BatchJob(s["dp"], s["starts"], required=j.required,
                              runs_per_instance=j.runs_per_instance)
                pl_runs.append(("batchjob", pj))
            else:
                cfg_pl = zb.make_config(j.max_iter, j.required, j.tol, "fast", "dual")
                pl_runs.append(("run", BfgsRun(s["dp"], j.n, cfg_pl, device=dev)))
        pl_t, pl_c = [], []
        for k in range(1 + args.plain_steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for s in state:
                gen_starts(s)
            for s, (kind, r) in zip(state, pl_runs):
                if kind == "run":
                    r.launch(s["starts"], stream=stream)
                    census(s, r)
                else:
                    # per-instance data: standalone launches cannot carry it,
                    # the batch kernel's single class with dual gradients
                    # would be needed; dijet has no plain form here
                    pass
            t1.record(stream)
            torch.cuda.synchronize()
            if k >= 1:
                pl_t.append(t0.elapsed_time(t1))
                pl_c.append(sum(int(s["cen"][1].item()) for s, (kd, _) in
                                zip(state, pl_runs) if kd == "run"))
        if all(kd == "run" for kd, _ in pl_runs):
            pv = float(np.mean(pl_c)) / (float(np.mean(pl_t)) * 1e-3)
            plain = {"value": pv, "unit": "runs/s", "ms_per_step": float(np.mean(pl_t)),
                     "converged_per_step": float(np.mean(pl_c)),
                     "form": "dual-number gradients, one standalone launch per class, "
                             "default layout by dimension",
                     "speedup_of_headline": value / pv if pv > 0 else None}

    # e2e: through the public host-buffer calls -- a batch plan
    # (zeus_batch_plan_run: host starts and objective data in, every class's
    # best run, coordinates and census out, one synchronisation) for batched
    # workloads, zeus_optimize (the zeus::Zeus of one objective) otherwise --
    # with the host inputs in pinned memory and every copy inside the timed
    # region
    e2e_ms, e2e_conv = [], []
    h2d = d2h = 0
    e2e_api = None
    if batch is not None:
        specs = []
        for s in state:
            j, obj = s["job"], s["obj"]
            hobj = zb.Objective(obj.kind, obj.dim, name=obj.name)
            if s["dp"].data is not None:
                hobj.data = s["dp"].data.cpu().pin_memory().numpy()
            if s["dp"].idata is not None:
                hobj.idata = s["dp"].idata.cpu().pin_memory().numpy()
            spec = dict(obj=hobj, n=j.n, runs_per_instance=j.runs_per_instance,
                        required=j.required)
            if j.pso_iter < 0:
                spec["starts"] = s["starts"].cpu().pin_memory().numpy()
            else:
                spec.update(seed=s["seed"], lower=j.lo, upper=j.hi, pso_iter=j.pso_iter)
            specs.append(spec)
        plan = zb.BatchPlan(specs, jobs[0].max_iter, jobs[0].tol)
        e2e_api = "zeus_batch_plan_run"
        for k in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            t_a = time.perf_counter()
            res = plan.run(stream=stream)
            t_b = time.perf_counter()
            if k >= args.warmup:
                e2e_ms.append((t_b - t_a) * 1e3)
                e2e_conv.append(sum(r.c.claimed for r in res))
        h2d, d2h = plan.traffic()
        plan.close()
    else:
        e2e_api = "zeus_optimize"
        hprobs = []
        for s in state:
            obj = s["obj"]
            hobj = zb.Objective(obj.kind, obj.dim, name=obj.name)
            if s["dp"].data is not None:
                hobj.data = s["dp"].data.cpu().pin_memory().numpy()
            if s["dp"].idata is not None:
                hobj.idata = s["dp"].idata.cpu().pin_memory().numpy()
            hprobs.append(hobj)
        for k in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            t_a = time.perf_counter()
            conv_k = 0
            for s, hobj in zip(state, hprobs):
                j = s["job"]
                cfg = zb.make_config(j.max_iter, j.required, j.tol, "fast", "adjoint")
                best, cen = zb.CResult(), zb.CCensus()
                bx = np.zeros(hobj.dim)
                prob = hobj.host_problem()
                zb.check(L.zeus_optimize(C.byref(prob), j.lo, j.hi, j.n, j.max_iter,
                                         j.pso_iter, j.required, j.tol, s["seed"],
                                         C.byref(cfg), C.byref(best), bx.ctypes.data,
                                         C.byref(cen), None, None, sh))
                conv_k += cen.claimed
            t_b = time.perf_counter()
            if k >= args.warmup:
                e2e_ms.append((t_b - t_a) * 1e3)
                e2e_conv.append(conv_k)
        h2d = sum(0 if h.data is None else h.data.nbytes + (0 if h.idata is None
                                                              else h.idata.nbytes)
                  for h in hprobs)
        d2h = len(state) * (C.sizeof(zb.CResult) + C.sizeof(zb.CCensus)) + \
            sum(8 * h.dim for h in hprobs)
    e2e_units, e2e_ms_all = job_totals(float(np.mean(e2e_conv)), float(np.mean(e2e_ms)),
                                       world, dev)
    e2e_val = e2e_units / (e2e_ms_all * 1e-3)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "runs/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": step_ms_all,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": workload_config(args, wl, world),
            "form": {"gradient": "adjoint", "mode": "fast", "batched": bool(wl["batch"]),
                     "autotuned_layouts": tuned},
            "converged_per_step": conv_all,
            "plain_dual": plain,
            "roofline": {"bound": "fp64",
                         "kernel": ("bfgs_batch_kernel" + (" + bfgs_rows_kernel (companion)"
                                                           if companions else ""))
                         if batch is not None else "bfgs (standalone launches)",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": (achieved / peak) if peak else None,
                         "peak_source": "measured FP64 FMA probe on this GPU "
                                        "(zeus_probe_fp64)",
                         "flops_per_step": flops, "kernel_ms": kms,
                         **traffic_of(args.workload)},
            "e2e": {"value": e2e_val, "unit": "runs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms_all,
                    "api": e2e_api},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
        }
        return line
    return None


def extra_summary(line: dict) -> dict:
    """The figures of a second workload's line that sit beside the default
    one's (its own value, plain form, roofline, e2e and CPU baseline)."""
    keys = ("metric", "value", "unit", "ms_per_step", "converged_per_step", "config",
            "plain_dual", "roofline", "e2e", "gpu_launches", "clocks", "cpu_baseline")
    return {k: line.get(k) for k in keys}


# ---------------------------------------------------------------- CPU side
class _QuietStdout:
    """Silences C-level stdout (the reference's host build prints from its
    convergence check) so this process prints only its JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def _ref_lib():
    from tests import _oracle as O

    if not O.ref_available():
        return None, "oracle/_ref/libzeus_ref.so not built"
    return O, None


PARITY_FIXTURE = ROOT / "tests" / "golden" / "parity_mixed.npz"


def _class_data(obj, job):
    """The objective data of the class's first instance (the runs sampled
    from a per-instance class all use that instance)."""
    data, idata = obj.data, obj.idata
    if job.runs_per_instance and idata is not None:
        nb = len(idata) // max(1, (job.n + job.runs_per_instance - 1) // job.runs_per_instance)
        data, idata = data[:nb], idata[:nb]
    return data, idata


def _ref_classes(O, wl, seed):
    """(job, objective, host starts) of every class of the workload: the
    oracle's Philox starts (equal to the GPU's bit for bit) or, with PSO, the
    oracle's synchronous PSO from the same seed."""
    out = []
    for ci, j in enumerate(wl["jobs"]):
        obj = j.make_objective()
        data, idata = _class_data(obj, j)
        if j.pso_iter >= 0:
            st, _, _, _ = O.oracle_pso(obj.kind, obj.dim, seed + ci, j.n, j.lo, j.hi,
                                       j.pso_iter, data=data, idata=idata)
        else:
            m = j.runs_per_instance or j.n
            st = O.oracle_starts(seed + ci, m, obj.dim, j.lo, j.hi)
        out.append((j, obj, np.ascontiguousarray(st)))
    return out


def _ref_step(O, classes, k, cores):
    """One step of the reference's timed sample: runs k*s .. k*s+s-1
    (wrapping) of every sampled class, s = job.ref_runs, each run to
    completion on the reference's sequential BFGS (host build), the classes
    concurrently with the host threads split among them.  Returns
    (converged runs, wall seconds, runs, statuses per class)."""
    live = [c for c in classes if c[0].ref_runs > 0]
    if not live:
        return 0, 0.0, 0, []
    per = max(1, cores // len(live))
    res = [None] * len(live)

    def work(ci):
        j, obj, st = live[ci]
        s = j.ref_runs
        idx = (np.arange(s) + k * s) % len(st)
        data, idata = _class_data(obj, j)
        res[ci] = O.ref_bfgs(obj.kind, obj.dim, st[idx], max_iter=j.max_iter,
                             required=j.required, tol=j.tol, data=data, idata=idata,
                             lower=j.lo, upper=j.hi, nthreads=per)

    with _QuietStdout():
        t0 = time.perf_counter()
        th = [threading.Thread(target=work, args=(ci,)) for ci in range(len(live))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        wall = time.perf_counter() - t0
    conv = int(sum((r["status"] == 1).sum() for r in res))
    return conv, wall, int(sum(len(r["status"]) for r in res)), \
        {j.name: r["status"] for (j, _, _), r in zip(live, res)}


def _ref_estimate(O, classes, conv_by_class, core_s_by_class, cores, workload):
    """Whole-workload estimate for the reference: sampled classes scaled from
    their measured runs; unsampled (heavy) classes from a measured
    per-iteration time (a few iterations of `cores` runs at once) times the
    reference's own per-run iteration counts and statuses -- those of the
    oracle, which follows the reference's arithmetic bit for bit
    (tests/golden/parity_mixed.npz) -- scaled to the class's runs."""
    total_conv, total_core_s, parts = 0.0, 0.0, []
    fx = np.load(PARITY_FIXTURE) if PARITY_FIXTURE.exists() and workload == "mixed" else None
    for j, obj, st in classes:
        if j.ref_runs > 0:
            runs = max(1, conv_by_class[j.name][1])
            total_conv += conv_by_class[j.name][0] * j.n / runs
            total_core_s += core_s_by_class[j.name] * j.n / runs
            parts.append(f"{j.name}: sampled")
            continue
        if fx is None or f"{j.name}/iter" not in fx:
            return None
        m_it = 3
        k = min(cores, len(st))
        data, idata = _class_data(obj, j)
        with _QuietStdout():
            t0 = time.perf_counter()
            O.ref_bfgs(obj.kind, obj.dim, st[:k], max_iter=m_it, required=1 << 30, tol=j.tol,
                       data=data, idata=idata, lower=j.lo, upper=j.hi, nthreads=cores)
            t_iter = (time.perf_counter() - t0) / m_it  # per iteration per core
        it = fx[f"{j.name}/iter"].astype(np.float64)
        stt = fx[f"{j.name}/status"]
        scale = j.n / len(it)
        total_core_s += float(np.maximum(it, 1).sum()) * t_iter * scale
        total_conv += float((stt == 1).sum()) * scale
        parts.append(f"{j.name}: {t_iter * 1e3:.1f} ms per iteration per core x the "
                     f"reference's {int(it.sum())} iterations over {len(it)} runs, "
                     f"scaled by {scale:.2f}")
    wall = total_core_s / cores
    return {"value": total_conv / wall, "unit": "runs/s",
            "seconds_for_workload": wall, "method": "; ".join(parts)}


def measure_reference(args, steps, warmup, cores):
    """The reference's own sequential BFGS (host build, all host threads) on
    a bounded sample of the workload: per step, whole runs of every sampled
    class (the same starts as the GPU arm).  Returns the measured record and
    the whole-workload estimate, or (None, why)."""
    O, why = _ref_lib()
    if O is None:
        return None, why
    wl = workloads()[args.workload]
    classes = _ref_classes(O, wl, args.seed)
    live = [j for j, _, _ in classes if j.ref_runs > 0]
    if not live:
        return None, "no class of this workload finishes a reference run inside a step"
    for k in range(warmup):  # untimed: one run of each sampled class
        small = [(j, o, st) for j, o, st in classes]
        saved = [j.ref_runs for j, _, _ in small]
        for j, _, _ in small:
            j.ref_runs = min(j.ref_runs, 1)
        _ref_step(O, small, k, cores)
        for (j, _, _), r in zip(small, saved):
            j.ref_runs = r
    conv, wall, runs = [], [], 0
    by_class, core_s = {j.name: [0, 0] for j in live}, {j.name: 0.0 for j in live}
    for k in range(steps):
        c, w, r, st = _ref_step(O, classes, k, cores)
        conv.append(c)
        wall.append(w)
        runs += r
        for name, v in st.items():
            by_class[name][0] += int((v == 1).sum())
            by_class[name][1] += len(v)
            core_s[name] += w * cores / len(st)
    value = float(np.sum(conv)) / float(np.sum(wall))
    sample = (f"{steps} steps x whole runs of the classes " +
              ", ".join(f"{j.name} ({j.ref_runs} runs/step)" for j in live) +
              f", {cores} host threads; {runs} runs, {int(np.sum(conv))} converged")
    skipped = [j.name for j, _, _ in classes if j.ref_runs == 0]
    if skipped:
        sample += ("; not in the timed sample (one reference run takes minutes): " +
                   ", ".join(skipped))
    est = _ref_estimate(O, classes, by_class, core_s, cores, args.workload)
    return {"value": value, "ms_per_step": float(np.mean(wall)) * 1e3,
            "converged_per_step": float(np.mean(conv)), "sample": sample,
            "by_class": {k: {"converged": v[0], "runs": v[1]} for k, v in by_class.items()},
            "estimate_full_workload": est}, None


def cpu_baseline(args):
    """The reference's sequential BFGS (host build, all host threads) on one
    step's bounded sample of this workload, on the GPU arm's starts."""
    cores = os.cpu_count() or 1
    rec, why = measure_reference(args, 2, 0, cores)
    if rec is None:
        return {"value": None, "unit": "runs/s", "cores": 0, "kind": "reference",
                "sample": why}
    return {"value": rec["value"], "unit": "runs/s", "cores": cores, "kind": "reference",
            "sample": rec["sample"], "estimate_full_workload": rec["estimate_full_workload"]}


def run_reference(args, rank, world):
    """The reference's own CPU implementation of the path (its sequential BFGS
    built for the host, oracle/_ref) on this workload: each step runs whole
    reference runs of a rotating sample of every class that can finish a run
    inside a step, on all host threads; `value` is their converged runs per
    second of wall time, measured.  The whole-workload estimate (heavy
    classes from measured per-iteration times) is reported beside it."""
    if rank != 0:
        return
    wl = workloads()[args.workload]
    cores = os.cpu_count() or 1
    rec, why = measure_reference(args, args.steps, args.warmup, cores)
    if rec is None:
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
        return
    v = rec["value"]
    print(json.dumps({
        "impl": "reference",
        "metric": METRIC,
        "value": v, "unit": "runs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": rec["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, wl, world),
        "converged_per_step": rec["converged_per_step"],
        "by_class": rec["by_class"],
        "estimate_full_workload": rec["estimate_full_workload"],
        "cpu_baseline": {"value": v, "unit": "runs/s", "cores": cores, "kind": "reference",
                         "sample": rec["sample"]},
        "e2e": {"value": v, "unit": "runs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


# ---------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="zeus_b200", choices=["zeus_b200", "reference"])
    ap.add_argument("--workload", default="mixed")
    ap.add_argument("--gradient", default="adjoint", choices=["adjoint", "dual"])
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the Gaussian-150 measurement the default run adds")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain dual-AD comparison")
    ap.add_argument("--plain-steps", type=int, default=1)
    ap.add_argument("--scale", type=float, default=1.0,
                    help="multiply every class's run count (small cases for profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group(
            "nccl", timeout=datetime.timedelta(seconds=120),
            device_id=torch.device("cuda", local_rank))
    try:
        line = run_gpu(args, rank, world, local_rank)
        # the default run also measures the 150-D Gaussian (the other
        # workload the adjoint + batched target names) on one GPU
        if (world == 1 and args.workload == "mixed" and not args.no_extra):
            import copy

            args2 = copy.copy(args)
            args2.workload = "gaussian150"
            line2 = run_gpu(args2, rank, world, local_rank)
            if line is not None and line2 is not None:
                line["extra_workloads"] = {"gaussian150": extra_summary(line2)}
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
