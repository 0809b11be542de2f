"""Generates the oracle fixtures of the benchmarked workloads
(tests/golden/parity_mixed.npz, tests/golden/parity_gaussian150.npz).

For every class of the mixed-dimension batch (Rosenbrock D = 128, 64, 32, 8,
2 and Ackley-30, uniform Philox starts with seed 42 + class index, PSO off,
MAX_ITER 10000, tol 1e-8, stop-early off) and for the 150-D Gaussian (1024
PSO starts: seed 42, 10 iterations, w = 0.5, c1 = 1.2, c2 = 1.5), the
oracle's restatement of the reference's sequential BFGS
(bfgs_sequential.cuh:46-234) runs every sampled start to completion.  The
same runs are repeated by the oracle compiled with FMA contraction -- the
reference's algorithm as an FMA-contracting compiler evaluates it -- to give
the share of run outcomes that move with rounding alone.

Stored per run: final fval, status and iteration count (oracle and FMA
oracle).  Starts are not stored: they are the oracle's Philox starts /
synchronous PSO, reproducible from the seed, and equal the GPU's bit for bit.

    python tests/golden/make_parity_fixtures.py [--threads N]

Takes about 15-30 minutes on 8 cores (the 128-D class: O(D^3) per
iteration in the reference's update order).
"""
from __future__ import annotations

import argparse
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from tests import _oracle as O  # noqa: E402

GOLDEN = Path(__file__).resolve().parent
SEED = 42
MAX_ITER = 10000
TOL = 1e-8

# (name, kind, dim, runs in the workload, runs sampled, lower, upper); the
# class index (order) is the bench's: its seed is SEED + index
MIXED = [
    ("rosenbrock128", 0, 128, 1365, 256, -5.0, 5.0),
    ("rosenbrock64", 0, 64, 1365, 1365, -5.0, 5.0),
    ("ackley30", 2, 30, 1365, 1365, -32.768, 32.768),
    ("rosenbrock32", 0, 32, 1365, 1365, -5.0, 5.0),
    ("rosenbrock8", 0, 8, 1366, 1366, -5.0, 5.0),
    ("rosenbrock2", 0, 2, 1366, 1366, -5.0, 5.0),
]


def gaussian_matrix(dim, off=0.5):
    C = np.full((dim, dim), off)
    np.fill_diagonal(C, 1.0 + (dim - 1) * off)
    return C


def _chunk(args):
    fma, kind, dim, starts, lo, hi, data = args
    fn = O.oracle_fma_bfgs if fma else O.oracle_bfgs
    r = fn(kind, dim, starts, max_iter=MAX_ITER, required=1 << 30, tol=TOL, data=data,
           lower=lo, upper=hi)
    return r["fval"], r["status"], r["iter"]


def run_both(kind, dim, starts, lo, hi, threads, data=None):
    """The oracle and the FMA oracle on every start, runs split over a pool
    of processes (stop-early is off, so runs are independent)."""
    import concurrent.futures as cf
    import multiprocessing as mp

    chunks = np.array_split(np.arange(len(starts)), max(1, 4 * threads))
    chunks = [c for c in chunks if len(c)]
    res = []
    with cf.ProcessPoolExecutor(threads, mp_context=mp.get_context("spawn")) as ex:
        for fma in (False, True):
            parts = list(ex.map(_chunk, [(fma, kind, dim, starts[c], lo, hi, data)
                                         for c in chunks]))
            res.append(dict(fval=np.concatenate([p[0] for p in parts]),
                            status=np.concatenate([p[1] for p in parts]),
                            iter=np.concatenate([p[2] for p in parts])))
    return res[0], res[1]


def mixed(threads):
    out = {}
    for ci, (name, kind, dim, n, m, lo, hi) in enumerate(MIXED):
        t0 = time.time()
        st = O.oracle_starts(SEED + ci, n, dim, lo, hi)[:m]
        a, b = run_both(kind, dim, st, lo, hi, threads)
        out[f"{name}/fval"] = a["fval"]
        out[f"{name}/status"] = a["status"].astype(np.int8)
        out[f"{name}/iter"] = a["iter"].astype(np.int32)
        out[f"{name}/fma_fval"] = b["fval"]
        out[f"{name}/fma_status"] = b["status"].astype(np.int8)
        out[f"{name}/meta"] = np.array([kind, dim, n, m, SEED + ci], dtype=np.int64)
        out[f"{name}/bounds"] = np.array([lo, hi])
        print(f"{name}: {m} runs, {time.time() - t0:.0f} s, converged "
              f"{(a['status'] == 1).sum()} (FMA {(b['status'] == 1).sum()}), status "
              f"agreement oracle/FMA {(a['status'] == b['status']).mean():.3f}", flush=True)
    np.savez_compressed(GOLDEN / "parity_mixed.npz", **out)


def gaussian150(threads):
    t0 = time.time()
    C = gaussian_matrix(150)
    pbx, _, _, _ = O.oracle_pso(3, 150, SEED, 1024, -5.0, 5.0, 10, data=C)
    a, b = run_both(3, 150, pbx, -5.0, 5.0, threads, data=C)
    np.savez_compressed(GOLDEN / "parity_gaussian150.npz", fval=a["fval"],
                        status=a["status"].astype(np.int8), iter=a["iter"].astype(np.int32),
                        fma_fval=b["fval"], fma_status=b["status"].astype(np.int8),
                        meta=np.array([3, 150, 1024, 1024, SEED], dtype=np.int64))
    print(f"gaussian150: 1024 runs, {time.time() - t0:.0f} s, converged "
          f"{(a['status'] == 1).sum()}, mean iterations {a['iter'].mean():.2f}", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only", choices=["mixed", "gaussian150"], default=None)
    args = ap.parse_args()
    if args.only in (None, "gaussian150"):
        gaussian150(args.threads)
    if args.only in (None, "mixed"):
        mixed(args.threads)


if __name__ == "__main__":
    main()
