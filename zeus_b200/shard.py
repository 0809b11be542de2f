"""Sharded call across GPUs: one process per GPU (torchrun), the runs of one
zeus::Zeus-style call (zeus.cuh:341-375) split into contiguous per-rank
shards, the best run and the census merged across ranks.

Runs are independent once their starts are fixed, so the shards share no
data while they run: each rank computes the starts of ALL n runs (uniform
Philox starts, or the whole PSO swarm, which is cheap next to BFGS and
would otherwise need a gbest exchange every PSO iteration), keeps its slice
[start, start + count) and runs BFGS on it.  The only exchange is the
reduction the reference does on one GPU (bfgs_common.cuh:280-319,
util.hpp:151-200), here across ranks after the kernels end:

  * census counts: one all-reduce (sum) of {actual, claimed, surrendered,
    stopped};
  * argmin: one all-reduce (min) of the best run's fval as a totally ordered
    int64 key (NaN above +inf), one all-reduce (min) of the global index
    among the ranks holding that key (lowest index on ties, as on one GPU),
    and one broadcast of that run's result row from the rank that owns it.

With stop-early off (required_converged > n) the merged result equals the
one-GPU call run for run.  Stop-early has no cross-GPU flag here: each rank
stops at its share, ceil(required * count / n), of the required count.

The merge itself (`merge`) takes any per-rank local census, so the same code
runs over NCCL between GPUs and over gloo between CPU processes.
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np
import torch
import torch.distributed as dist

_I64_MAX = (1 << 63) - 1


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous shard of n runs for `rank` of `world`: (start, count); the
    first n % world ranks take one run more."""
    if world <= 0 or not 0 <= rank < world or n < 0:
        raise ValueError("need n >= 0 and 0 <= rank < world")
    base, rem = divmod(n, world)
    return rank * base + min(rank, rem), base + (1 if rank < rem else 0)


def owner_of(idx: int, n: int, world: int) -> int:
    """The rank whose shard holds global run `idx`."""
    for r in range(world):
        s, c = shard_range(n, r, world)
        if s <= idx < s + c:
            return r
    raise ValueError(f"run {idx} is outside 0..{n - 1}")


def order_key(f: float) -> int:
    """fval as a signed int64 ordered like the doubles, NaN above +inf (it
    never wins a min); the device census uses the same order."""
    if math.isnan(f):
        return _I64_MAX
    u = struct.unpack("<Q", struct.pack("<d", f))[0]
    u = (~u & 0xFFFFFFFFFFFFFFFF) if (u >> 63) else (u | (1 << 63))
    return u - (1 << 63)  # unsigned order -> signed order


@dataclass
class LocalCensus:
    """One rank's census of its shard (zeus_census fields), its best run's
    LOCAL index (-1 if it has no runs) and that run's result row."""
    actual: int = 0
    claimed: int = 0
    surrendered: int = 0
    stopped: int = 0
    best_local: int = -1
    fval: float = float("nan")
    status: int = -1
    iter: int = 0
    gnorm: float = 0.0
    x: Optional[np.ndarray] = None


@dataclass
class MergedResult:
    """The call's best run (global index) and census over all ranks."""
    idx: int
    status: int
    fval: float
    gnorm: float
    iter: int
    x: np.ndarray
    actual: int
    claimed: int
    surrendered: int
    stopped: int


def census_host(fval, status, x, known_min=None) -> LocalCensus:
    """The census of runs held in host arrays, by the rules of
    zeus_census_device: claimed = status 1, stopped = status 2, surrendered =
    the rest, actual = claimed and within 0.5 of the known minimum (origin
    when None), best = argmin fval, lowest index on ties, NaN never wins."""
    fval = np.asarray(fval, dtype=np.float64)
    status = np.asarray(status)
    n = fval.shape[0]
    c = LocalCensus()
    if n == 0:
        return c
    c.claimed = int((status == 1).sum())
    c.stopped = int((status == 2).sum())
    c.surrendered = n - c.claimed - c.stopped
    if x is not None:
        x = np.asarray(x, dtype=np.float64).reshape(n, -1)
        km = np.zeros(x.shape[1]) if known_min is None else np.asarray(known_min, np.float64)
        dist_ = np.sqrt(((x - km) ** 2).sum(axis=1))
        c.actual = int(((status == 1) & (dist_ < 0.5)).sum())
    keys = [order_key(float(v)) for v in fval]
    c.best_local = int(min(range(n), key=lambda i: (keys[i], i)))
    return c


def merge(local: LocalCensus, start: int, n: int, dim: int,
          group=None) -> MergedResult:
    """Merges the ranks' local censuses of one call of n runs (this rank's
    shard starts at global run `start`); every rank of `group` calls it and
    gets the same result.  Works on any backend: tensors live on the current
    CUDA device for NCCL, on the host otherwise."""
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    dev = torch.device("cpu")
    if dist.is_initialized() and dist.get_backend(group) == "nccl":
        dev = torch.device("cuda", torch.cuda.current_device())
    counts = torch.tensor([local.actual, local.claimed, local.surrendered, local.stopped],
                          dtype=torch.int64, device=dev)
    mine = local.best_local >= 0
    key = torch.tensor([order_key(local.fval) if mine else _I64_MAX], dtype=torch.int64,
                       device=dev)
    if world > 1:
        dist.all_reduce(counts, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(key, op=dist.ReduceOp.MIN, group=group)
    gidx = start + local.best_local if mine else _I64_MAX
    kmin = int(key.item())
    cand = torch.tensor([gidx if (mine and order_key(local.fval) == kmin) else _I64_MAX],
                        dtype=torch.int64, device=dev)
    if world > 1:
        dist.all_reduce(cand, op=dist.ReduceOp.MIN, group=group)
    best = int(cand.item())
    row = torch.zeros(4 + dim, dtype=torch.float64, device=dev)
    if best == _I64_MAX:  # no runs anywhere, or every fval NaN and no run
        best = -1
    if best >= 0 and mine and start + local.best_local == best:
        row[0], row[1], row[2], row[3] = local.fval, local.status, local.iter, local.gnorm
        if local.x is not None:
            row[4:] = torch.as_tensor(np.asarray(local.x, dtype=np.float64), device=dev)
    if world > 1 and best >= 0:
        dist.broadcast(row, src=_global_rank(owner_of(best, n, world), group), group=group)
    r = row.cpu().numpy()
    c = counts.cpu().numpy()
    if best < 0:
        return MergedResult(-1, -1, float("nan"), 0.0, 0, np.zeros(dim), *map(int, c))
    return MergedResult(best, int(r[1]), float(r[0]), float(r[3]), int(r[2]), r[4:].copy(),
                        *map(int, c))


def _global_rank(group_rank: int, group) -> int:
    if group is None:
        return group_rank
    return dist.get_global_rank(group, group_rank)


def sharded_call(n: int, dim: int, local_fn: Callable[[int, int], LocalCensus],
                 group=None) -> MergedResult:
    """Runs `local_fn(start, count)` on this rank's shard of n runs and merges
    the ranks' results."""
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    start, count = shard_range(n, rank, world)
    return merge(local_fn(start, count), start, n, dim, group)


def sharded_optimize(obj, n: int, lower: float, upper: float, max_iter: int,
                     pso_iter: int, required_converged: int, tolerance: float,
                     seed: int, known_min=None, group=None,
                     gradient: str = "adjoint", layout: int = 0) -> MergedResult:
    """zeus::Zeus on a built-in objective across the ranks of `group`, each on
    its current CUDA device: starts of all n runs on every rank (PSO with
    pso_iter iterations when pso_iter >= 0, else uniform Philox starts), BFGS
    on this rank's shard, census and argmin merged across ranks."""
    from .device import (DeviceProblem, bfgs_device, census_device, pso_device,
                         starts_uniform)

    dev = torch.device("cuda", torch.cuda.current_device())
    dp = DeviceProblem(obj, dev)
    dim = dp.obj.dim

    def local(start: int, count: int) -> LocalCensus:
        if pso_iter >= 0:
            allst, _, _ = pso_device(dp, seed, n, lower, upper, pso_iter, device=dev)
        else:
            allst = starts_uniform(seed, n, dim, lower, upper, device=dev)
        if count == 0:
            return LocalCensus()
        st = allst[start:start + count].contiguous()
        req = count + 1 if required_converged > n else \
            max(1, math.ceil(required_converged * count / n))
        r = bfgs_device(dp, st, max_iter=max_iter, required=req, tol=tolerance,
                        gradient=gradient, layout=layout)
        c = census_device(r.fval, r.status, r.x, dim, known_min)
        b = int(c["best_idx"])
        out = LocalCensus(c["actual"], c["claimed"], c["surrendered"], c["stopped"], b)
        if b >= 0:
            out.fval = float(r.fval[b].item())
            out.status = int(r.status[b].item())
            out.iter = int(r.iter[b].item())
            out.gnorm = float(r.gnorm[b].item())
            out.x = r.x[b].cpu().numpy()
        return out

    return sharded_call(n, dim, local, group)
