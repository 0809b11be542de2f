"""Device-buffer entry points: the C ABI called with CUDA tensors.

torch supplies device memory and streams (plumbing only); every kernel that
runs is in libzeus_b200.so.  Inputs must already be on the GPU.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import (BfgsConfig, Objective, RunOutputs, check, lib, make_config,
               LAYOUT_AUTO)


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


def starts_uniform(seed: int, n: int, dim: int, lower: float, upper: float,
                   device="cuda", stream=None) -> torch.Tensor:
    """Philox uniform starts (n, dim) in [lower, upper)."""
    out = torch.empty((n, dim), dtype=torch.float64, device=device)
    check(lib().zeus_starts_uniform(seed, n, dim, lower, upper, _ptr(out),
                                    _stream_handle(stream)))
    return out


def pso_device(obj, seed: int, n: int, lower: float, upper: float, iters: int,
               w: float = 0.5, c1: float = 1.2, c2: float = 1.5, device="cuda",
               stream=None):
    """PSO seeding; returns (pbest_x (n, dim), pbest_f (n,), gbest (dim+1,))."""
    dp = _as_problem(obj, device)
    dim = dp.obj.dim
    pbx = torch.empty((n, dim), dtype=torch.float64, device=device)
    pbf = torch.empty((n,), dtype=torch.float64, device=device)
    gb = torch.empty((dim + 1,), dtype=torch.float64, device=device)
    wsz = lib().zeus_pso_workspace_size(n, dim)
    ws = torch.empty((max(wsz, 1),), dtype=torch.uint8, device=device)
    prob = dp.c()
    check(lib().zeus_pso_device(C.byref(prob), seed, n, lower, upper, iters, w,
                                c1, c2, _ptr(pbx), _ptr(pbf), _ptr(gb), _ptr(ws),
                                wsz, _stream_handle(stream)))
    return pbx, pbf, gb


class BfgsRun:
    """Preallocated outputs + workspace for repeated BFGS launches."""

    def __init__(self, obj, n: int, cfg: BfgsConfig, device="cuda",
                 traj: bool = False, counters: bool = True):
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
                              _ptr(t.get("status")))

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
                traj: bool = False, stream=None, flags: int = 0) -> BfgsRun:
    """One BFGS per row of ``starts``; returns the BfgsRun with its outputs."""
    n = starts.shape[0]
    if required is None:
        required = n + 1  # stop-early off
    cfg = make_config(max_iter, required, tol, mode, gradient, layout, tile, block, flags)
    r = BfgsRun(obj, n, cfg, device=starts.device, traj=traj)
    return r.launch(starts, stream=stream)


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
