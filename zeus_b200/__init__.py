"""zeus_b200: B200 (sm_100a) FP64 global optimiser behind the zeus::Zeus API.

Host-side Python mirror of the reference's entry point
``zeus::Zeus(f, lower, upper, N, MAX_ITER, PSO_ITER, requiredConverged,
fun_name, tolerance, seed, run, parallel, prng, trajectory_file, nzerosteps)``
(include/zeus.cuh:341-375 in the reference), bound to the C ABI in
include/zeus_b200.h through ctypes.  The compute path is the CUDA library
``libzeus_b200.so`` built in-tree by ``zeus_b200/build.py``; there is no CPU
fallback: if the library is missing or a call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import enum
import time
import os
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libzeus_b200.so"

# ---- constants mirrored from include/zeus_b200.h -------------------------
OK = 0
E_INVALID, E_UNSUPPORTED, E_CUDA, E_NOMEM, E_WORKSPACE = -1, -2, -3, -4, -5
STATUS_SURRENDER, STATUS_CONVERGED, STATUS_STOPPED = 0, 1, 2
STATUS_NOMEM, STATUS_KERNEL, STATUS_NONFINITE = 3, 4, 5
OBJ_ROSENBROCK, OBJ_RASTRIGIN, OBJ_ACKLEY, OBJ_GAUSSIAN, OBJ_POISSON_NLL = range(5)
PROBLEM_SYMMETRIC = 1
MODE_EXACT, MODE_FAST = 0, 1
GRAD_DUAL, GRAD_ADJOINT = 0, 1
LAYOUT_AUTO, LAYOUT_THREAD, LAYOUT_TILE, LAYOUT_CTA, LAYOUT_ROWS = 0, 1, 2, 3, 4
FLAG_NO_FIXED_POINT = 1
(GRADPATH_THREAD, GRADPATH_TILE, GRADPATH_TILE_GRAD, GRADPATH_CTA, GRADPATH_CTA_GRAD,
 GRADPATH_QUADRATIC) = range(6)
PRNG_XORWOW, PRNG_PHILOX, PRNG_SOBOL = 0, 1, 2


class PRNGType(enum.IntEnum):
    """The reference's PRNGType (traits.hpp:67-71).  XORWOW and PHILOX both
    draw from Philox4x32-10 here; SOBOL places the starts (and the PSO's
    initial swarm) on a digitally shifted Sobol' sequence."""
    XORWOW = PRNG_XORWOW
    PHILOX = PRNG_PHILOX
    SOBOL = PRNG_SOBOL


def prng_code(prng) -> int:
    """ZEUS_PRNG_* for a PRNGType, its int value, its name, or None (the
    reference's default, XORWOW)."""
    if prng is None:
        return PRNG_XORWOW
    if isinstance(prng, str):
        return int(PRNGType[prng.upper()])
    return int(PRNGType(int(prng)))

_MODES = {"exact": MODE_EXACT, "fast": MODE_FAST}
_GRADS = {"dual": GRAD_DUAL, "adjoint": GRAD_ADJOINT}


class ZeusError(RuntimeError):
    """A C-ABI call returned an error code."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"zeus_b200 error {code}: {msg}")
        self.code = code


class Problem(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("dim", C.c_int32),
        ("data", C.c_void_p),
        ("idata", C.c_void_p),
        ("ndata", C.c_int32),
        ("flags", C.c_int32),
    ]


class BfgsConfig(C.Structure):
    _fields_ = [
        ("max_iter", C.c_int32),
        ("required_converged", C.c_int32),
        ("tolerance", C.c_double),
        ("mode", C.c_int32),
        ("gradient", C.c_int32),
        ("layout", C.c_int32),
        ("tile", C.c_int32),
        ("block", C.c_int32),
        ("flags", C.c_int32),
        ("prng", C.c_int32),
    ]


class RunOutputs(C.Structure):
    _fields_ = [
        ("fval", C.c_void_p),
        ("status", C.c_void_p),
        ("iter", C.c_void_p),
        ("gnorm", C.c_void_p),
        ("x", C.c_void_p),
        ("counters", C.c_void_p),
        ("traj_x", C.c_void_p),
        ("traj_f", C.c_void_p),
        ("traj_g", C.c_void_p),
        ("traj_status", C.c_void_p),
        ("cycles", C.c_void_p),
    ]


class CResult(C.Structure):
    _fields_ = [
        ("idx", C.c_int32),
        ("status", C.c_int32),
        ("fval", C.c_double),
        ("gradient_norm", C.c_double),
        ("iter", C.c_int32),
        ("reserved", C.c_int32),
    ]


class CCensus(C.Structure):
    _fields_ = [
        ("actual", C.c_int32),
        ("claimed", C.c_int32),
        ("surrendered", C.c_int32),
        ("stopped", C.c_int32),
        ("best_idx", C.c_int32),
        ("reserved", C.c_int32),
    ]


class BatchClass(C.Structure):
    _fields_ = [
        ("problem", Problem),
        ("n", C.c_int64),
        ("runs_per_instance", C.c_int64),
        ("d_starts", C.c_void_p),
        ("out", RunOutputs),
        ("d_control", C.c_void_p),
        ("required_converged", C.c_int32),
        ("layout", C.c_int32),
        ("tile", C.c_int32),
        ("reserved", C.c_int32),
    ]


class HostClass(C.Structure):
    _fields_ = [
        ("problem", Problem),
        ("n", C.c_int64),
        ("runs_per_instance", C.c_int64),
        ("starts", C.c_void_p),
        ("seed", C.c_uint64),
        ("lower", C.c_double),
        ("upper", C.c_double),
        ("pso_iter", C.c_int32),
        ("required_converged", C.c_int32),
        ("layout", C.c_int32),
        ("tile", C.c_int32),
    ]


# Every symbol include/zeus_b200.h declares: (name, restype, argtypes).
_P = C.c_void_p
SIGNATURES = {
    "zeus_last_error": (C.c_char_p, []),
    "zeus_version": (C.c_char_p, []),
    "zeus_supported": (C.c_int, [C.c_int32] * 4),
    "zeus_starts": (
        C.c_int,
        [C.c_uint64, C.c_int32, C.c_int64, C.c_int32, C.c_double, C.c_double, _P, _P],
    ),
    "zeus_starts_uniform": (
        C.c_int,
        [C.c_uint64, C.c_int64, C.c_int32, C.c_double, C.c_double, _P, _P],
    ),
    "zeus_sobol_directions": (C.c_int, [C.c_int32, _P]),
    "zeus_sobol_device_table": (C.c_int, [C.POINTER(C.c_void_p)]),
    "zeus_pso_workspace_size": (C.c_size_t, [C.c_int64, C.c_int32]),
    "zeus_pso_device": (
        C.c_int,
        [C.POINTER(Problem), C.c_uint64, C.c_int64, C.c_double, C.c_double,
         C.c_int32, C.c_double, C.c_double, C.c_double, _P, _P, _P, _P,
         C.c_size_t, _P],
    ),
    "zeus_pso_device_prng": (
        C.c_int,
        [C.POINTER(Problem), C.c_uint64, C.c_int32, C.c_int64, C.c_double, C.c_double,
         C.c_int32, C.c_double, C.c_double, C.c_double, _P, _P, _P, _P,
         C.c_size_t, _P],
    ),
    "zeus_pso_device_noalloc": (
        C.c_int,
        [C.POINTER(Problem), C.c_uint64, C.c_int64, C.c_double, C.c_double,
         C.c_int32, C.c_double, C.c_double, C.c_double, _P, _P, _P, _P],
    ),
    "zeus_bfgs_workspace_size": (
        C.c_size_t, [C.POINTER(Problem), C.POINTER(BfgsConfig), C.c_int64]),
    "zeus_bfgs_device": (
        C.c_int,
        [C.POINTER(Problem), C.POINTER(BfgsConfig), _P, C.c_int64,
         C.POINTER(RunOutputs), _P, _P, C.c_size_t, _P],
    ),
    "zeus_gradient_workspace_size": (C.c_size_t, [C.POINTER(Problem)]),
    "zeus_gradient_device": (
        C.c_int,
        [C.POINTER(Problem), C.c_int32, C.c_int32, C.c_int32, _P, _P, C.c_double,
         C.c_int64, _P, _P, _P, C.c_size_t, _P]),
    "zeus_tile_widths": (C.c_uint32, [C.c_int32, C.c_int32]),
    "zeus_census_device": (
        C.c_int, [_P, _P, _P, C.c_int64, C.c_int32, _P, _P, _P]),
    "zeus_optimize": (
        C.c_int,
        [C.POINTER(Problem), C.c_double, C.c_double, C.c_int64, C.c_int32,
         C.c_int32, C.c_int32, C.c_double, C.c_uint64, C.POINTER(BfgsConfig),
         C.POINTER(CResult), _P, C.POINTER(CCensus), _P, _P, _P],
    ),
    "zeus_batch_workspace_size": (C.c_size_t, [C.POINTER(BatchClass), C.c_int32]),
    "zeus_batch_device": (
        C.c_int, [C.POINTER(BatchClass), C.c_int32, C.POINTER(BfgsConfig), _P, C.c_size_t,
                  _P]),
    "zeus_batch_plan_create": (
        C.c_int, [C.POINTER(HostClass), C.c_int32, C.POINTER(BfgsConfig),
                  C.POINTER(C.c_void_p)]),
    "zeus_batch_plan_run": (
        C.c_int, [C.c_void_p, C.POINTER(HostClass), C.POINTER(CResult), _P,
                  C.POINTER(CCensus), _P]),
    "zeus_batch_plan_traffic": (
        C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "zeus_batch_plan_destroy": (C.c_int, [C.c_void_p]),
    "zeus_nll_sensitivity_device": (
        C.c_int, [C.POINTER(Problem), C.c_int64, C.c_int64, _P, _P, _P, _P, _P]),
    "zeus_write_trajectory_tsv": (
        C.c_int, [C.c_char_p, _P, _P, _P, _P, _P, C.c_int64, C.c_int32, C.c_int32]),
    "zeus_euclidean_error": (C.c_double, [C.c_char_p, _P, C.c_int32]),
    "zeus_append_results_tsv": (
        C.c_int, [C.c_char_p, C.c_char_p, C.c_int32, C.c_int64, C.c_int32, C.c_float,
                  C.c_float, C.c_float, C.c_float, C.c_int32, C.c_int32, C.c_double,
                  C.POINTER(CResult), C.POINTER(CCensus), _P, _P]),
    "zeus_cycle_metrics": (
        C.c_int, [_P, _P, C.c_int64, C.c_int32, C.c_double, C.c_float, C.c_int32, _P]),
    "zeus_autotune": (
        C.c_int,
        [C.POINTER(Problem), C.POINTER(BfgsConfig), C.c_int64, C.c_uint64, C.c_double,
         C.c_double, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_float), _P]),
    "zeus_autotune_lookup": (
        C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                  C.POINTER(C.c_int32)]),
    "zeus_autotune_record": (C.c_int, [C.c_int32] * 5),
    "zeus_probe_fp64_shape": (None, [C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "zeus_probe_fp64": (C.c_int, [C.c_int64, _P, _P]),
}

_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """The loaded CUDA library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python zeus_b200/build.py` "
                "(the CUDA library is the only compute path)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().zeus_last_error().decode()


def check(rc: int) -> None:
    if rc != OK:
        raise ZeusError(rc, last_error())


def supported(kind: int, dim: int, mode: str = "fast", gradient: str = "adjoint") -> bool:
    return bool(lib().zeus_supported(kind, dim, _MODES[mode], _GRADS[gradient]))


# ---- objectives ------------------------------------------------------------
@dataclasses.dataclass
class Objective:
    """A built-in objective: kind, dimension and host-side data."""

    kind: int
    dim: int
    data: Optional[np.ndarray] = None   # Gaussian C / NLL bin centres
    idata: Optional[np.ndarray] = None  # NLL counts
    name: str = ""

    def problem(self, data_ptr=None, idata_ptr=None, flags=None) -> Problem:
        """C struct with the given (device or host) data pointers."""
        nd = 0 if self.idata is None else len(self.idata)
        if flags is None:
            flags = 0
            if self.kind == OBJ_GAUSSIAN and self.data is not None and np.array_equal(
                    self.data, self.data.T):
                flags = PROBLEM_SYMMETRIC
        return Problem(self.kind, self.dim, data_ptr, idata_ptr, nd, flags)

    def host_problem(self) -> Problem:
        d = None if self.data is None else self.data.ctypes.data
        i = None if self.idata is None else self.idata.ctypes.data
        return self.problem(d, i)

    @property
    def known_minimum(self) -> Optional[np.ndarray]:
        if self.kind == OBJ_ROSENBROCK:
            return np.ones(self.dim)
        return None


def Rosenbrock(dim: int) -> Objective:
    """examples/rosenbrock.hpp: sum (1-x_i)^2 + 100 (x_{i+1}-x_i^2)^2."""
    return Objective(OBJ_ROSENBROCK, dim, name="rosenbrock")


def Rastrigin(dim: int) -> Objective:
    """examples/rastrigin.hpp: 10 D + sum x_i^2 - 10 cos(2 pi x_i)."""
    return Objective(OBJ_RASTRIGIN, dim, name="rastrigin")


def Ackley(dim: int) -> Objective:
    """examples/ackley.hpp (a=20, b=0.2, c=2 pi)."""
    return Objective(OBJ_ACKLEY, dim, name="ackley")


def Gaussian(C_matrix) -> Objective:
    """examples/gaussian.hpp: 0.5 x^T C x with dense C (D x D)."""
    Cm = np.ascontiguousarray(np.asarray(C_matrix, dtype=np.float64))
    if Cm.ndim != 2 or Cm.shape[0] != Cm.shape[1]:
        raise ValueError("C must be square")
    return Objective(OBJ_GAUSSIAN, Cm.shape[0], data=Cm, name="gaussian")


def PoissonNLL(counts, centres) -> Objective:
    """simulation/fitting/LogLikelihood.h: binned Poisson NLL, 4 parameters."""
    k = np.ascontiguousarray(np.asarray(counts, dtype=np.int32))
    x = np.ascontiguousarray(np.asarray(centres, dtype=np.float64))
    if k.shape != x.shape or k.ndim != 1 or len(k) == 0:
        raise ValueError("counts and centres must be equal-length 1-D arrays")
    return Objective(OBJ_POISSON_NLL, 4, data=x, idata=k, name="poisson")


def gaussian_matrix(dim: int, off: float = 0.5) -> np.ndarray:
    """C_ii = 1 + (dim-1) off, C_ij = off: the reference's Gaussian example
    (C_ii = 1 + 149 * 0.5 = 75.5 at dim 150)."""
    C_m = np.full((dim, dim), off)
    np.fill_diagonal(C_m, 1.0 + (dim - 1) * off)
    return C_m


# ---- the reference's result types -----------------------------------------
@dataclasses.dataclass
class Convergence:
    """util.hpp:27-32."""

    actual: int = 0
    claimed: int = 0
    surrendered: int = 0
    stopped: int = 0


@dataclasses.dataclass
class Result:
    """zeus::Result<D> (util.hpp:36-54)."""

    idx: int = -1
    status: int = -1
    fval: float = 37.0
    gradientNorm: float = 0.0
    coordinates: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
    iter: int = 0
    c: Convergence = dataclasses.field(default_factory=Convergence)
    per_run_fval: Optional[np.ndarray] = None
    per_run_status: Optional[np.ndarray] = None


def make_config(max_iter: int, required: int, tol: float, mode: str = "fast",
                gradient: str = "adjoint", layout: int = LAYOUT_AUTO, tile: int = 0,
                block: int = 0, flags: int = 0, prng=None) -> BfgsConfig:
    return BfgsConfig(max_iter, required, tol, _MODES[mode], _GRADS[gradient],
                      layout, tile, block, flags, prng_code(prng))


def Zeus(f: Objective, lower: float, upper: float, N: int, MAX_ITER: int,
         PSO_ITER: int, requiredConverged: int, fun_name: str = "",
         tolerance: float = 1e-8, seed: int = 42, run: int = 0,
         parallel: bool = True, prng=None, trajectory_file: str = "",
         nzerosteps: int = 0, *, mode: str = "fast", gradient: str = "adjoint",
         per_run: bool = False, stream=None) -> Result:
    """The reference's zeus::Zeus on a built-in objective, host buffers in and
    out.  ``prng`` (a PRNGType, its name or value; None = XORWOW) picks the
    start positions' generator: Philox for XORWOW and PHILOX, Sobol' for
    SOBOL.  ``parallel``/``nzerosteps`` are accepted for signature
    compatibility: the layout is chosen by dimension, and the zero-step limit
    cannot trigger because the reference's line search never returns 0
    (utils.cuh:395-411).  A ``trajectory_file``
    (``.tsv``) runs the BFGS in exact mode, which records every iteration,
    and writes the reference's trajectory file (zeus.cuh:62-103, 189-239).
    Like the reference (zeus.cuh:170-183), every call with N > 0 appends its
    row to zeus_<D>d_results.tsv in the current directory; here the row's
    `kernel` and `time` are the call's wall time in ms (no separate PSO
    timing)."""
    del parallel, nzerosteps
    if N < 0:
        raise ValueError("N must be >= 0")
    prng = prng_code(prng)
    t0 = time.perf_counter()
    if trajectory_file:
        r = _zeus_with_trajectories(f, lower, upper, N, MAX_ITER, PSO_ITER,
                                    requiredConverged, tolerance, seed,
                                    trajectory_file, per_run, stream, prng)
        _append_results(f, fun_name, run, N, MAX_ITER, PSO_ITER, r, t0)
        return r
    cfg = make_config(MAX_ITER, requiredConverged, tolerance, mode, gradient, prng=prng)
    best = CResult()
    census = CCensus()
    bx = np.zeros(f.dim)
    pf = np.zeros(max(N, 1)) if per_run else None
    ps = np.zeros(max(N, 1), dtype=np.int32) if per_run else None
    rc = lib().zeus_optimize(
        C.byref(f.host_problem()), lower, upper, N, MAX_ITER, PSO_ITER,
        requiredConverged, tolerance, seed & 0xFFFFFFFFFFFFFFFF, C.byref(cfg),
        C.byref(best), bx.ctypes.data, C.byref(census),
        None if pf is None else pf.ctypes.data,
        None if ps is None else ps.ctypes.data, stream)
    r = Result(idx=best.idx, status=best.status, fval=best.fval,
               gradientNorm=best.gradient_norm, coordinates=bx, iter=best.iter,
               c=Convergence(census.actual, census.claimed, census.surrendered,
                             census.stopped))
    if per_run and N > 0:
        r.per_run_fval, r.per_run_status = pf[:N], ps[:N]
    if rc != OK:
        if rc in (E_NOMEM, E_CUDA):
            return r  # status 3 / 4 as the reference reports them
        check(rc)
    _append_results(f, fun_name, run, N, MAX_ITER, PSO_ITER, r, t0)
    return r


def sobol_directions(ndim: int) -> np.ndarray:
    """The library's Sobol' direction numbers (host): (ndim, 32) uint32,
    row d = v_1..v_32 of dimension d as 32-bit fractions."""
    out = np.zeros((ndim, 32), dtype=np.uint32)
    check(lib().zeus_sobol_directions(ndim, out.ctypes.data))
    return out


def _append_results(f, fun_name, run, N, MAX_ITER, PSO_ITER, r, t0) -> None:
    """The reference's per-call results row (util::appendResultsToTsv) and
    its census line on stdout."""
    if N == 0:
        return  # the reference returns before its results file (zeus.cuh:58-60)
    ms = (time.perf_counter() - t0) * 1e3
    x = np.ascontiguousarray(r.coordinates, dtype=np.float64)
    err = lib().zeus_euclidean_error(fun_name.encode(), x.ctypes.data, f.dim)
    best = CResult(r.idx, r.status, r.fval, r.gradientNorm, r.iter, 0)
    cen = CCensus(r.c.actual, r.c.claimed, r.c.surrendered, r.c.stopped, r.idx, 0)
    check(lib().zeus_append_results_tsv(None, fun_name.encode(), run, N, f.dim, 0.0, 0.0,
                                        ms, 0.0, MAX_ITER, PSO_ITER, err, C.byref(best),
                                        C.byref(cen), x.ctypes.data, None))
    print(f"claimed: {r.c.claimed}\tactual : {r.c.actual}\tsurrendered: "
          f"{r.c.surrendered}\tstopped: {r.c.stopped}")


def write_trajectory_tsv(path: str, traj: dict, alpha=None) -> None:
    """Writes an exact-mode run's trajectory buffers (BfgsRun.traj) in the
    reference's TSV layout (src/utils.cu:128-176)."""
    host = {k: np.ascontiguousarray(v.cpu().numpy()) for k, v in traj.items()}
    T, dim, n = host["x"].shape
    a = None if alpha is None else np.ascontiguousarray(alpha, dtype=np.float64)
    check(lib().zeus_write_trajectory_tsv(
        str(path).encode(), host["x"].ctypes.data, host["f"].ctypes.data,
        host["g"].ctypes.data, host["status"].ctypes.data,
        None if a is None else a.ctypes.data, n, T, dim))


def _zeus_with_trajectories(f, lower, upper, N, MAX_ITER, PSO_ITER, required, tol, seed,
                            path, per_run, stream, prng=PRNG_XORWOW) -> "Result":
    """Zeus with a trajectory file: PSO (or uniform) starts, exact-mode BFGS
    recording every iteration, the census, then the file."""
    import torch

    from .device import bfgs_device, census_device, pso_device, starts

    if not str(path).endswith(".tsv"):
        check(lib().zeus_write_trajectory_tsv(str(path).encode(), None, None, None, None,
                                              None, 0, 0, f.dim))
    if N == 0:
        return Result()
    if PSO_ITER >= 0:
        x0, _, _ = pso_device(f, seed & 0xFFFFFFFFFFFFFFFF, N, lower, upper, PSO_ITER,
                              prng=prng)
    else:
        x0 = starts(seed & 0xFFFFFFFFFFFFFFFF, N, f.dim, lower, upper, prng=prng)
    r = bfgs_device(f, x0, max_iter=MAX_ITER, required=required, tol=tol,
                    mode="exact", gradient="dual", traj=True, stream=stream)
    cen = census_device(r.fval, r.status, r.x, f.dim,
                        np.ones(f.dim) if f.kind == OBJ_ROSENBROCK else None)
    torch.cuda.synchronize()
    write_trajectory_tsv(path, r.traj)
    idx = int(cen["best_idx"])
    out = Result(idx=idx, status=int(r.status[idx]), fval=float(r.fval[idx]),
                 gradientNorm=float(r.gnorm[idx]), coordinates=r.x[idx].cpu().numpy(),
                 iter=int(r.iter[idx]),
                 c=Convergence(cen["actual"], cen["claimed"], cen["surrendered"],
                               cen["stopped"]))
    if per_run:
        out.per_run_fval = r.fval.cpu().numpy()
        out.per_run_status = r.status.cpu().numpy()
    return out


from .device import (bfgs_device, pso_device, starts, starts_uniform,  # noqa: E402
                     census_device, batch_device, autotune, BatchJob)

__all__ = [
    "Zeus", "write_trajectory_tsv", "Result", "Convergence", "Objective", "Rosenbrock", "Rastrigin",
    "Ackley", "Gaussian", "PoissonNLL", "gaussian_matrix", "bfgs_device",
    "pso_device", "starts", "starts_uniform", "census_device", "lib", "supported",
    "PRNGType", "sobol_directions",
    "batch_device", "autotune", "BatchJob",
]


class BatchPlan:
    """Several objectives in one persistent kernel launch, host buffers in and
    out: zeus_batch_plan_* (the batch form of zeus::Zeus).

    ``classes`` is a list of dicts: ``obj`` (an Objective whose data/idata
    hold every instance), ``n``, and either ``starts`` (host (n, dim) float64
    array) or ``seed`` / ``lower`` / ``upper`` / ``pso_iter`` (starts drawn
    on the device: PSO for pso_iter >= 0, else uniform Philox); optional
    ``runs_per_instance``, ``required`` (stop-early threshold, default off),
    ``layout``, ``tile``.  Device memory is allocated once, on the current
    device; ``run()`` copies the host inputs in and returns one Result per
    class, synchronously.  Pass pinned arrays (e.g. torch ``pin_memory()``
    views) for asynchronous copies."""

    def __init__(self, classes, max_iter: int = 10000, tol: float = 1e-8,
                 block: int = 0, flags: int = 0):
        self.specs = [dict(c) for c in classes]
        self.cfg = make_config(max_iter, 1, tol, "fast", "adjoint", block=block, flags=flags)
        self._keep = []
        arr = self._host_classes(self.specs)
        h = C.c_void_p()
        check(lib().zeus_batch_plan_create(arr, len(self.specs), C.byref(self.cfg),
                                           C.byref(h)))
        self.handle = h
        self.dims = [c["obj"].dim for c in self.specs]

    def _host_classes(self, specs):
        keep = []
        arr = (HostClass * len(specs))()
        for i, c in enumerate(specs):
            obj = c["obj"]
            d = None if obj.data is None else np.ascontiguousarray(obj.data, np.float64)
            k = None if obj.idata is None else np.ascontiguousarray(obj.idata, np.int32)
            keep += [d, k]
            prob = obj.problem(None if d is None else d.ctypes.data,
                               None if k is None else k.ctypes.data)
            rpi = int(c.get("runs_per_instance", 0))
            if rpi and k is not None:
                prob.ndata = len(k) // max(1, (c["n"] + rpi - 1) // rpi)
            st = c.get("starts")
            if st is not None:
                st = np.ascontiguousarray(st, np.float64)
                if st.shape != (c["n"], obj.dim):
                    raise ValueError(f"class {i}: starts must have shape {(c['n'], obj.dim)}")
                keep.append(st)
            arr[i] = HostClass(prob, c["n"], rpi, None if st is None else st.ctypes.data,
                               int(c.get("seed", 0)), float(c.get("lower", 0.0)),
                               float(c.get("upper", 0.0)), int(c.get("pso_iter", -1)),
                               int(c.get("required", c["n"] + 1)),
                               int(c.get("layout", LAYOUT_AUTO)), int(c.get("tile", 0)))
        self._keep = keep
        return arr

    def run(self, classes=None, stream=None):
        """Runs the batch (optionally with new host inputs of the same
        shapes); returns a list of Result, one per class."""
        if classes is not None:
            self.specs = [dict(c) for c in classes]
        arr = self._host_classes(self.specs)
        nc = len(self.specs)
        best = (CResult * nc)()
        cen = (CCensus * nc)()
        bx = np.zeros(sum(self.dims))
        sh = 0 if stream is None else int(getattr(stream, "cuda_stream", stream))
        check(lib().zeus_batch_plan_run(self.handle, arr, best, bx.ctypes.data, cen, sh))
        out, off = [], 0
        for i, d in enumerate(self.dims):
            b, c = best[i], cen[i]
            out.append(Result(idx=b.idx, status=b.status, fval=b.fval,
                              gradientNorm=b.gradient_norm,
                              coordinates=bx[off:off + d].copy(), iter=b.iter,
                              c=Convergence(c.actual, c.claimed, c.surrendered, c.stopped)))
            off += d
        return out

    def traffic(self):
        """(host-to-device bytes of the last run, device-to-host bytes of a run)."""
        h, d = C.c_size_t(), C.c_size_t()
        check(lib().zeus_batch_plan_traffic(self.handle, C.byref(h), C.byref(d)))
        return h.value, d.value

    def close(self):
        if getattr(self, "handle", None):
            lib().zeus_batch_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
