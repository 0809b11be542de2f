#!/usr/bin/env python
"""Throughput benchmark: converged BFGS runs per second on one B200 (or N
replicas under torchrun, one per GPU, weak scaling).

A step is one full optimisation call on the workload: PSO seeding (or
uniform starts when the workload has PSO off), every BFGS run, and the
argmin/census reduction, with inputs resident in HBM.  `value` counts the
runs that finish with status 1 (||grad|| < tol) per second of device time;
`e2e` is the same metric through the host-buffer C-ABI call zeus_optimize
(host inputs in, host result out, copies inside the timed region).

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
            return 2 * dim * dim + 2 * dim
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


# ---------------------------------------------------------------- workloads
class Job:
    def __init__(self, name, obj_fn, n, lo, hi, pso_iter, max_iter, required, tol=1e-8):
        self.name, self.obj_fn, self.n = name, obj_fn, n
        self.lo, self.hi, self.pso_iter = lo, hi, pso_iter
        self.max_iter, self.required, self.tol = max_iter, required, tol


def workloads():
    import zeus_b200 as zb

    return {
        "rosenbrock2": dict(
            desc="2-D Rosenbrock, 1024 starts, PSO 10, <=10000 BFGS iters, "
                 "required_convergences 100, tol 1e-8, seed 42",
            jobs=[Job("rosenbrock2", lambda: zb.Rosenbrock(2), 1024, -5.0, 5.0, 10,
                      10000, 100)]),
        "rosenbrock2-nostop": dict(
            desc="2-D Rosenbrock, 1024 starts, PSO 10, <=10000 BFGS iters, "
                 "stop-early off, tol 1e-8, seed 42",
            jobs=[Job("rosenbrock2", lambda: zb.Rosenbrock(2), 1024, -5.0, 5.0, 10,
                      10000, 1025)]),
    }


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
    import torch
    import zeus_b200 as zb
    from zeus_b200.device import DeviceProblem, BfgsRun, _stream_handle
    import ctypes as C

    torch.cuda.set_device(local_rank)
    wl = workloads()[args.workload]
    jobs = wl["jobs"]
    dev = torch.device("cuda", local_rank)
    # a dedicated (non-legacy) stream: the PSO loop is captured into a CUDA
    # graph on it
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    seed = args.seed + 1000003 * rank

    # per job: device problem, buffers
    state = []
    for j in jobs:
        obj = j.obj_fn()
        dp = DeviceProblem(obj, dev)
        cfg = zb.make_config(j.max_iter, j.required, j.tol, "fast", args.gradient)
        run = BfgsRun(dp, j.n, cfg, device=dev, counters=True)
        pws = zb.lib().zeus_pso_workspace_size(j.n, obj.dim)
        pso = dict(pbx=torch.empty((j.n, obj.dim), dtype=torch.float64, device=dev),
                   pbf=torch.empty((j.n,), dtype=torch.float64, device=dev),
                   gb=torch.empty((obj.dim + 1,), dtype=torch.float64, device=dev),
                   ws=torch.empty((max(pws, 1),), dtype=torch.uint8, device=dev), wsz=pws)
        cen = torch.zeros((6,), dtype=torch.int32, device=dev)
        nbins = 0 if obj.idata is None else len(obj.idata)
        state.append(dict(job=j, obj=obj, dp=dp, run=run, pso=pso, cen=cen, nbins=nbins))

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step(timing):
        ev = []
        launches = 0
        for s in state:
            j, run, p = s["job"], s["run"], s["pso"]
            prob = s["dp"].c()
            if j.pso_iter >= 0:
                zb.check(zb.lib().zeus_pso_device(
                    C.byref(prob), seed, j.n, j.lo, j.hi, j.pso_iter, 0.5, 1.2, 1.5,
                    p["pbx"].data_ptr(), p["pbf"].data_ptr(), p["gb"].data_ptr(),
                    p["ws"].data_ptr(), p["wsz"], sh))
                launches += 2 + j.pso_iter
                starts = p["pbx"]
            else:
                zb.check(zb.lib().zeus_starts_uniform(seed, j.n, s["obj"].dim, j.lo, j.hi,
                                                      p["pbx"].data_ptr(), sh))
                launches += 1
                starts = p["pbx"]
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run.launch(starts, stream=stream)
            e1.record(stream)
            launches += 1 + (1 if s["nbins"] else 0)
            ev.append((e0, e1))
            zb.check(zb.lib().zeus_census_device(
                run.fval.data_ptr(), run.status.data_ptr(), run.x.data_ptr(), j.n,
                s["obj"].dim, None, s["cen"].data_ptr(), sh))
            launches += 1
        return ev, launches

    # warm-up
    for _ in range(args.warmup):
        step(False)
    torch.cuda.synchronize()

    clocks = ClockSampler(local_rank)
    if rank == 0:
        clocks.start()
        clocks.wait_samples(1)
    times, kern_ms, conv, launches = [], [], [], 0
    counters = []
    for k in range(args.steps):
        flush.zero_()  # write 1 GiB: larger than the 126 MB L2
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        ev, nl = step(True)
        t1.record(stream)
        torch.cuda.synchronize()
        launches += nl
        times.append(t0.elapsed_time(t1))
        kern_ms.append(sum(a.elapsed_time(b) for a, b in ev))
        conv.append(sum(int(s["cen"][1].item()) for s in state))
        counters = [((s["obj"].kind, s["obj"].dim, args.gradient, s["nbins"]),
                     s["run"].counters.cpu().numpy()) for s in state]
    if rank == 0:
        n0 = len(clocks.rows)
        clocks.wait_samples(n0 + 1)  # one sample after the last timed step
        clocks.stop()

    step_ms = float(np.mean(times))
    conv_mean = float(np.mean(conv))
    if world > 1:
        t = torch.tensor([step_ms, conv_mean], dtype=torch.float64, device=dev)
        mx = t.clone()
        torch.distributed.all_reduce(mx, op=torch.distributed.ReduceOp.MAX)
        sm = t.clone()
        torch.distributed.all_reduce(sm, op=torch.distributed.ReduceOp.SUM)
        step_ms_all, conv_all = float(mx[0]), float(sm[1])
    else:
        step_ms_all, conv_all = step_ms, conv_mean
    value = conv_all / (step_ms_all * 1e-3)

    # roofline: the BFGS kernel, FP64 work per launch / its event time
    flops = algorithmic_flops(counters)
    kms = float(np.mean(kern_ms))
    achieved = flops / (kms * 1e-3) / 1e12
    peak = measure_fp64_peak(torch, zb) if rank == 0 else None

    # e2e through the host-buffer C-ABI call
    e2e_ms, e2e_conv = [], []
    h2d = sum(0 if s["obj"].data is None else s["obj"].data.nbytes +
              (0 if s["obj"].idata is None else s["obj"].idata.nbytes) for s in state)
    d2h = sum(24 + 24 + 8 * s["obj"].dim for s in state)
    for k in range(args.warmup + args.steps):
        t_a = time.perf_counter()
        cc = 0
        for s in state:
            j = s["job"]
            r = zb.Zeus(s["obj"], j.lo, j.hi, j.n, j.max_iter, j.pso_iter, j.required,
                        j.name, j.tol, seed, 0, gradient=args.gradient,
                        stream=sh)
            cc += r.c.claimed
        t_b = time.perf_counter()
        if k >= args.warmup:
            e2e_ms.append((t_b - t_a) * 1e3)
            e2e_conv.append(cc)
    e2e_val = float(np.mean(e2e_conv)) / (float(np.mean(e2e_ms)) * 1e-3)
    if world > 1:
        t = torch.tensor([e2e_val], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
        e2e_val = float(t[0])

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, state, torch)

    if rank == 0:
        line = {
            "metric": "converged runs/s at ||grad||<1e-8 (adjoint+batched form)",
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
            "config": {"workload": args.workload, "description": wl["desc"],
                       "gradient": args.gradient, "mode": "fast",
                       "converged_per_step": conv_all,
                       "l2": "1 GiB buffer written between timed steps",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "roofline": {"bound": "fp64", "kernel": "bfgs (all BFGS launches of a step)",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": (achieved / peak) if peak else None,
                         "peak_source": "measured FP64 FMA probe on this GPU "
                                        "(zeus_probe_fp64)",
                         "flops_per_step": flops, "kernel_ms": kms,
                         "traffic": None},
            "e2e": {"value": e2e_val, "unit": "runs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": float(np.mean(e2e_ms))},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)


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


def cpu_baseline(args, state, torch):
    """The reference's sequential BFGS (host build) on the same starts as the
    GPU's last step, all host threads."""
    O, why = _ref_lib()
    if O is None:
        return {"value": None, "unit": "runs/s", "cores": 0, "kind": "reference",
                "sample": why}
    cores = os.cpu_count() or 1
    total_t, total_conv, sample = 0.0, 0, []
    for s in state:
        j, obj = s["job"], s["obj"]
        starts = s["pso"]["pbx"].cpu().numpy()
        with _QuietStdout():
            t0 = time.perf_counter()
            r = O.ref_bfgs(obj.kind, obj.dim, starts, max_iter=j.max_iter,
                           required=j.required, tol=j.tol, data=obj.data, idata=obj.idata,
                           lower=j.lo, upper=j.hi, nthreads=cores)
            total_t += time.perf_counter() - t0
        total_conv += int((r["status"] == 1).sum())
        sample.append(f"{j.name}: all {j.n} runs from the GPU's PSO starts")
    return {"value": total_conv / total_t, "unit": "runs/s", "cores": cores,
            "kind": "reference", "sample": "; ".join(sample), "seconds": total_t}


def run_reference(args, rank, world):
    if rank != 0:
        return
    O, why = _ref_lib()
    wl = workloads()[args.workload]
    if O is None:
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
        return
    cores = os.cpu_count() or 1
    # starts: the oracle's synchronous PSO restatement with the same seed
    sts = []
    for j in wl["jobs"]:
        obj = j.obj_fn()
        if j.pso_iter >= 0:
            pbx, _, _, _ = O.oracle_pso(obj.kind, obj.dim, args.seed, j.n, j.lo, j.hi,
                                        j.pso_iter, data=obj.data, idata=obj.idata)
        else:
            pbx = O.oracle_starts(args.seed, j.n, obj.dim, j.lo, j.hi)
        sts.append((j, obj, pbx))
    times, convs = [], []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        c = 0
        for j, obj, pbx in sts:
            with _QuietStdout():
                r = O.ref_bfgs(obj.kind, obj.dim, pbx, max_iter=j.max_iter,
                               required=j.required, tol=j.tol, data=obj.data,
                               idata=obj.idata, lower=j.lo, upper=j.hi, nthreads=cores)
            c += int((r["status"] == 1).sum())
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
            convs.append(c)
    v = float(np.mean(convs)) / float(np.mean(times))
    print(json.dumps({
        "impl": "reference",
        "metric": "converged runs/s at ||grad||<1e-8 (adjoint+batched form)",
        "value": v, "unit": "runs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": float(np.mean(times)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "description": wl["desc"]},
        "cpu_baseline": {"value": v, "unit": "runs/s", "cores": cores, "kind": "reference",
                         "sample": "whole workload per step; starts from the synchronous "
                                   "PSO restatement (same seed)"},
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
    ap.add_argument("--workload", default="rosenbrock2")
    ap.add_argument("--gradient", default="adjoint", choices=["adjoint", "dual"])
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
        run_gpu(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
