"""Device-buffer entry points: the C ABI called with CUDA tensors.

torch supplies device memory and streams (plumbing only); every kernel that
runs is in libzeus_b200.so.  Inputs must already be on the GPU.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import (BatchClass, BfgsConfig, Objective, RunOutputs, check, lib, make_config,
               prng_code, LAYOUT_AUTO, PRNG_PHILOX, GRADPATH_QUADRATIC, _GRADS)


def _stream_handle(stream: Optional[torch.cuda.Stream]) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _ptr(t: Optional[torch.Tensor]):
    return None if t is None else t.data_ptr()


class DeviceProblem:
    """An Objective with its data copied to the GPU."""

    def __init__(self, obj: Objective, device="cuda"):
        self.obj = obj
        self.data = None if obj.data is None else torch.from_numpy(
            np.ascontiguousarray(obj.data)).to(device)
        self.idata = None if obj.idata is None else torch.from_numpy(
            np.ascontiguousarray(obj.idata)).to(device)

    def c(self):
        return self.obj.problem(_ptr(self.data), _ptr(self.idata))


def _as_problem(obj, device):
    return obj if isinstance(obj, DeviceProblem) else DeviceProblem(obj, device)


def starts(seed: int, n: int, dim: int, lower: float, upper: float, prng=PRNG_PHILOX,
           device="cuda", stream=None) -> torch.Tensor:
    """Starts (n, dim) in [lower, upper) from generator `prng` (a PRNGType,
    its name or value): Philox uniforms, or Sobol' points for SOBOL."""
    out = torch.empty((n, dim), dtype=torch.float64, device=device)
    check(lib().zeus_starts(seed, prng_code(prng), n, dim, lower, upper, _ptr(out),
                            _stream_handle(stream)))
    return out


def starts_uniform(seed: int, n: int, dim: int, lower: float, upper: float,
                   device="cuda", stream=None) -> torch.Tensor:
    """Philox uniform starts (n, dim) in [lower, upper)."""
    out = torch.empty((n, dim), dtype=torch.float64, device=device)
    check(lib().zeus_starts_uniform(seed, n, dim, lower, upper, _ptr(out),
                                    _stream_handle(stream)))
    return out


def pso_device(obj, seed: int, n: int, lower: float, upper: float, iters: int,
               w: float = 0.5, c1: float = 1.2, c2: float = 1.5, device="cuda",
               stream=None, prng=PRNG_PHILOX):
    """PSO seeding; returns (pbest_x (n, dim), pbest_f (n,), gbest (dim+1,)).
    `prng` picks the initial positions' generator (Sobol' for SOBOL)."""
    dp = _as_problem(obj, device)
    dim = dp.obj.dim
    pbx = torch.empty((n, dim), dtype=torch.float64, device=device)
    pbf = torch.empty((n,), dtype=torch.float64, device=device)
    gb = torch.empty((dim + 1,), dtype=torch.float64, device=device)
    wsz = lib().zeus_pso_workspace_size(n, dim)
    ws = torch.empty((max(wsz, 1),), dtype=torch.uint8, device=device)
    prob = dp.c()
    check(lib().zeus_pso_device_prng(C.byref(prob), seed, prng_code(prng), n, lower,
                                     upper, iters, w, c1, c2, _ptr(pbx), _ptr(pbf),
                                     _ptr(gb), _ptr(ws), wsz, _stream_handle(stream)))
    return pbx, pbf, gb


class BfgsRun:
    """Preallocated outputs + workspace for repeated BFGS launches."""

    def __init__(self, obj, n: int, cfg: BfgsConfig, device="cuda",
                 traj: bool = False, counters: bool = True, cycles: bool = False):
        self.dp = _as_problem(obj, device)
        self.n, self.cfg = n, cfg
        dim = self.dp.obj.dim
        f64 = dict(dtype=torch.float64, device=device)
        i32 = dict(dtype=torch.int32, device=device)
        self.fval = torch.empty((n,), **f64)
        self.status = torch.empty((n,), **i32)
        self.iter = torch.empty((n,), **i32)
        self.gnorm = torch.empty((n,), **f64)
        self.x = torch.empty((n, dim), **f64)
        self.counters = torch.zeros((n, 3), dtype=torch.int64, device=device) if counters else None
        # per run {gradient, update, whole-run} clock64 cycles (sampled only
        # when asked for)
        self.cycles = torch.zeros((n, 3), dtype=torch.int64, device=device) if cycles else None
        self.control = torch.zeros((2,), **i32)
        self.traj = None
        if traj:
            T = cfg.max_iter
            self.traj = dict(
                x=torch.full((T, dim, n), float("nan"), **f64),
                f=torch.full((T, n), float("nan"), **f64),
                g=torch.full((T, n), float("nan"), **f64),
                status=torch.full((T, n), -1, dtype=torch.int8, device=device))
        self.prob = self.dp.c()
        self.wsz = lib().zeus_bfgs_workspace_size(C.byref(self.prob), C.byref(cfg), n)
        self.ws = torch.empty((max(self.wsz, 1),), dtype=torch.uint8, device=device)
        t = self.traj or {}
        self.out = RunOutputs(_ptr(self.fval), _ptr(self.status), _ptr(self.iter),
                              _ptr(self.gnorm), _ptr(self.x), _ptr(self.counters),
                              _ptr(t.get("x")), _ptr(t.get("f")), _ptr(t.get("g")),
                              _ptr(t.get("status")), _ptr(self.cycles))

    def launch(self, starts: torch.Tensor, stream=None, reset_control=True):
        if starts.dtype != torch.float64 or not starts.is_cuda or not starts.is_contiguous():
            raise ValueError("starts must be a contiguous float64 CUDA tensor")
        if starts.shape != (self.n, self.dp.obj.dim):
            raise ValueError(f"starts must have shape {(self.n, self.dp.obj.dim)}")
        if reset_control:
            self.control.zero_()
        check(lib().zeus_bfgs_device(C.byref(self.prob), C.byref(self.cfg),
                                     _ptr(starts), self.n, C.byref(self.out),
                                     _ptr(self.control), _ptr(self.ws), self.wsz,
                                     _stream_handle(stream)))
        return self


def bfgs_device(obj, starts: torch.Tensor, max_iter: int = 10000,
                required: Optional[int] = None, tol: float = 1e-8,
                mode: str = "fast", gradient: str = "adjoint",
                layout: int = LAYOUT_AUTO, tile: int = 0, block: int = 0,
                traj: bool = False, stream=None, flags: int = 0,
                cycles: bool = False) -> BfgsRun:
    """One BFGS per row of ``starts``; returns the BfgsRun with its outputs."""
    n = starts.shape[0]
    if required is None:
        required = n + 1  # stop-early off
    cfg = make_config(max_iter, required, tol, mode, gradient, layout, tile, block, flags)
    r = BfgsRun(obj, n, cfg, device=starts.device, traj=traj, cycles=cycles)
    return r.launch(starts, stream=stream)


def gradient_device(obj, x: torch.Tensor, path: int, gradient: str = "adjoint",
                    width: int = 0, p: Optional[torch.Tensor] = None, alpha: float = 0.0,
                    stream=None):
    """f and grad f at the rows of ``x`` (n, dim) through one gradient path of
    the BFGS layouts (GRADPATH_*: thread, tile / tile gradient-only of
    ``width`` lanes, CTA / CTA gradient-only of ``width`` threads, or the
    quadratic form's carried point x + alpha p).  Returns (f (n,), g (n, dim))."""
    dp = _as_problem(obj, x.device)
    dim = dp.obj.dim
    if x.dtype != torch.float64 or not x.is_cuda or x.dim() != 2 or x.shape[1] != dim:
        raise ValueError(f"x must be a float64 CUDA tensor of shape (n, {dim})")
    x = x.contiguous()
    if path == GRADPATH_QUADRATIC:
        if p is None or p.shape != x.shape:
            raise ValueError("the quadratic path needs directions p shaped like x")
        p = p.contiguous()
    n = x.shape[0]
    fo = torch.empty((n,), dtype=torch.float64, device=x.device)
    go = torch.empty((n, dim), dtype=torch.float64, device=x.device)
    prob = dp.c()
    wsz = lib().zeus_gradient_workspace_size(C.byref(prob))
    ws = torch.empty((max(wsz, 1),), dtype=torch.uint8, device=x.device)
    check(lib().zeus_gradient_device(C.byref(prob), path, _GRADS[gradient], width, _ptr(x),
                                     _ptr(p), alpha, n, _ptr(fo), _ptr(go), _ptr(ws), wsz,
                                     _stream_handle(stream)))
    return fo, go


def tile_widths(kind: int, dim: int) -> list[int]:
    """Lanes per run the tile layout is built with for (kind, dim)."""
    m = lib().zeus_tile_widths(kind, dim)
    return [1 << k for k in range(1, 6) if (m >> k) & 1]


def census_device(fval: torch.Tensor, status: torch.Tensor, x: Optional[torch.Tensor],
                  dim: int, known_min=None, stream=None) -> dict:
    out = torch.zeros((6,), dtype=torch.int32, device=fval.device)
    km = None
    if known_min is not None:
        km = np.ascontiguousarray(np.asarray(known_min, dtype=np.float64))
    check(lib().zeus_census_device(
        _ptr(fval), _ptr(status), _ptr(x), fval.shape[0], dim,
        None if km is None else km.ctypes.data, _ptr(out), _stream_handle(stream)))
    v = out.cpu().tolist()
    return dict(actual=v[0], claimed=v[1], surrendered=v[2], stopped=v[3],
                best_idx=v[4])


class BatchJob:
    """One class of a persistent batch: an objective (optionally with several
    data instances stored one after another), its starts on the GPU and its
    own outputs and stop-early control."""

    def __init__(self, obj, starts: torch.Tensor, required: Optional[int] = None,
                 layout: int = LAYOUT_AUTO, tile: int = 0, runs_per_instance: int = 0,
                 counters: bool = True, cycles: bool = False):
        self.dp = obj if isinstance(obj, DeviceProblem) else DeviceProblem(obj, starts.device)
        if starts.dtype != torch.float64 or not starts.is_cuda or not starts.is_contiguous():
            raise ValueError("starts must be a contiguous float64 CUDA tensor")
        self.starts = starts
        self.n = starts.shape[0]
        self.required = self.n + 1 if required is None else required
        self.layout, self.tile, self.rpi = layout, tile, runs_per_instance
        dev = starts.device
        dim = self.dp.obj.dim
        self.fval = torch.empty((self.n,), dtype=torch.float64, device=dev)
        self.status = torch.empty((self.n,), dtype=torch.int32, device=dev)
        self.iter = torch.empty((self.n,), dtype=torch.int32, device=dev)
        self.gnorm = torch.empty((self.n,), dtype=torch.float64, device=dev)
        self.x = torch.empty((self.n, dim), dtype=torch.float64, device=dev)
        self.counters = (torch.zeros((self.n, 3), dtype=torch.int64, device=dev)
                         if counters else None)
        self.cycles = (torch.zeros((self.n, 3), dtype=torch.int64, device=dev)
                       if cycles else None)
        self.control = torch.zeros((2,), dtype=torch.int32, device=dev)

    def c(self) -> BatchClass:
        out = RunOutputs(_ptr(self.fval), _ptr(self.status), _ptr(self.iter),
                         _ptr(self.gnorm), _ptr(self.x), _ptr(self.counters),
                         None, None, None, None, _ptr(self.cycles))
        prob = self.dp.c()
        if self.rpi and self.dp.idata is not None:
            # ndata is per instance
            ninst = max(1, (self.n + self.rpi - 1) // self.rpi)
            prob.ndata = self.dp.idata.numel() // ninst
        return BatchClass(prob, self.n, self.rpi, _ptr(self.starts), out,
                          _ptr(self.control), self.required, self.layout, self.tile, 0)


class Batch:
    """A persistent-batch launch with preallocated workspace."""

    def __init__(self, jobs, max_iter: int = 10000, tol: float = 1e-8, flags: int = 0,
                 block: int = 0):
        self.jobs = list(jobs)
        self.cfg = make_config(max_iter, 1, tol, "fast", "adjoint", block=block, flags=flags)
        self.arr = (BatchClass * len(self.jobs))(*[j.c() for j in self.jobs])
        self.wsz = lib().zeus_batch_workspace_size(self.arr, len(self.jobs))
        dev = self.jobs[0].starts.device
        self.ws = torch.empty((max(self.wsz, 1),), dtype=torch.uint8, device=dev)

    def launch(self, stream=None, reset=True):
        if reset:
            for j in self.jobs:
                j.control.zero_()
        check(lib().zeus_batch_device(self.arr, len(self.jobs), C.byref(self.cfg),
                                      _ptr(self.ws), self.wsz, _stream_handle(stream)))
        return self


def batch_device(jobs, max_iter: int = 10000, tol: float = 1e-8, flags: int = 0,
                 stream=None, block: int = 0) -> Batch:
    """Runs every BatchJob in one persistent kernel launch (block: 512 or 384
    threads, 0 = chosen by the library)."""
    return Batch(jobs, max_iter, tol, flags, block).launch(stream)


def autotune(obj, n_sample: int = 2048, max_iter: int = 10000, tol: float = 1e-8,
             lower: float = -5.0, upper: float = 5.0, seed: int = 1,
             gradient: str = "adjoint", device="cuda", stream=None):
    """Times every built layout for `obj` and records the fastest; returns
    (layout, tile, ms)."""
    dp = _as_problem(obj, device)
    cfg = make_config(max_iter, n_sample + 1, tol, "fast", gradient)
    lay, til, ms = C.c_int32(), C.c_int32(), C.c_float()
    prob = dp.c()
    check(lib().zeus_autotune(C.byref(prob), C.byref(cfg), n_sample, seed, lower, upper,
                              C.byref(lay), C.byref(til), C.byref(ms),
                              _stream_handle(stream)))
    return lay.value, til.value, ms.value


def nll_sensitivity(job: "BatchJob", stream=None):
    """d(fitted parameters)/d(bin counts) for every toy of a Poisson NLL batch
    class: returns (best (toys, 6): fval, a, b, c, d, run; sens (toys, 4,
    nbins))."""
    if not job.rpi or job.n % job.rpi:
        raise ValueError("the class must have runs_per_instance > 0 dividing its runs")
    toys = job.n // job.rpi
    prob = job.c().problem
    dev = job.fval.device
    best = torch.empty((toys, 6), dtype=torch.float64, device=dev)
    sens = torch.empty((toys, 4, prob.ndata), dtype=torch.float64, device=dev)
    check(lib().zeus_nll_sensitivity_device(C.byref(prob), toys, job.rpi,
                                            _ptr(job.fval), _ptr(job.x), _ptr(best),
                                            _ptr(sens), _stream_handle(stream)))
    return best, sens


METRIC_NAMES = ("ms_per_call", "calls_per_thread_mean", "fraction_of_thread", "block95",
                "serialized", "fraction_of_kernel", "avg_cycles_per_thread",
                "avg_ms_per_thread")


def cycle_metrics(cycles, counters, ms_opt: float, sm_clock_khz: float,
                  runs_per_block: int = 128) -> dict:
    """The reference's AD and BFGS timer summaries
    (bfgs_sequential.cuh:236-373) from per-run cycles and counters ((n, 3)
    int64 arrays or tensors, host or device) of one launch of ms_opt ms:
    {"ad": {...}, "bfgs": {...}} with METRIC_NAMES keys (the first five in
    the order the results file writes them)."""
    cyc = np.ascontiguousarray(_host_i64(cycles))
    cnt = np.ascontiguousarray(_host_i64(counters))
    if cyc.shape != cnt.shape or cyc.ndim != 2 or cyc.shape[1] != 3:
        raise ValueError("cycles and counters must both be (n, 3)")
    out = {}
    for which, name in ((0, "ad"), (1, "bfgs")):
        m = (C.c_double * 8)()
        check(lib().zeus_cycle_metrics(cyc.ctypes.data, cnt.ctypes.data, cyc.shape[0], which,
                                       float(sm_clock_khz), float(ms_opt), runs_per_block, m))
        out[name] = dict(zip(METRIC_NAMES, list(m)))
    return out


def _host_i64(a):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return np.asarray(a, dtype=np.int64)
