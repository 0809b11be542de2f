"""The benchmarked workloads against the oracle, run for run.

tests/golden/make_parity_fixtures.py ran the oracle (the reference's
sequential BFGS restated, bfgs_sequential.cuh:46-234) on the bench's own
starts: every class of the mixed-dimension batch (Philox starts, seed 42 +
class index; all runs of each class, the first 256 of the 128-D class) and
the 150-D Gaussian's 1024 PSO starts, all to completion (MAX_ITER 10000,
tol 1e-8, stop-early off).  The same runs under the oracle compiled with FMA
contraction give the share of outcomes that move with rounding alone.

Here the GPU runs the same workloads through the bench's own calls (one
persistent batch launch for the mixed classes; the CTA-layout BFGS for the
Gaussian), and per run:
  * status agreement with the oracle is at least the FMA oracle's agreement
    less a margin (the fast mode changes rounding in more places than FMA
    contraction: O(D^2) update, adjoint gradients);
  * every run both call converged has the same fval within 1e-8;
  * every run the GPU calls converged has an oracle (dual) gradient norm
    below the tolerance at the GPU's point: its claim holds by the
    reference's own gradient;
  * converged counts agree within binomial noise.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest
import torch

import zeus_b200 as zb
from zeus_b200.device import BatchJob, DeviceProblem, batch_device, bfgs_device, starts_uniform
from tests import _oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = 1e-8
# class order, objectives and bounds of bench.py's mixed workload
MIXED = [("rosenbrock128", zb.Rosenbrock, 128, -5.0, 5.0),
         ("rosenbrock64", zb.Rosenbrock, 64, -5.0, 5.0),
         ("ackley30", zb.Ackley, 30, -32.768, 32.768),
         ("rosenbrock32", zb.Rosenbrock, 32, -5.0, 5.0),
         ("rosenbrock8", zb.Rosenbrock, 8, -5.0, 5.0),
         ("rosenbrock2", zb.Rosenbrock, 2, -5.0, 5.0)]
# status agreement may fall short of the FMA oracle's by this much (absolute)
# plus three binomial standard deviations
AGREE_SLACK = 0.05


def _fixture(name):
    p = GOLDEN / name
    if not p.exists():
        pytest.skip(f"{name} missing: run tests/golden/make_parity_fixtures.py")
    return np.load(p)


def _check_class(name, kind, dim, st_g, f_g, x_g, st_o, f_o, st_fma, report, data=None):
    m = len(st_o)
    agree = float(np.mean(st_g == st_o))
    agree_fma = float(np.mean(st_fma == st_o))
    sd = math.sqrt(max(agree_fma * (1 - agree_fma), 1.0 / m) / m)
    both = (st_g == 1) & (st_o == 1)
    dfv = float(np.abs(f_g[both] - f_o[both]).max()) if both.any() else 0.0
    # the GPU's converged claims, checked by the oracle's dual gradient
    gmax = 0.0
    for i in np.flatnonzero(st_g == 1):
        _, g = O.grad_dual(kind, dim, x_g[i], data)
        gmax = max(gmax, float(np.sqrt(np.dot(g, g))))
    c_g, c_o = int((st_g == 1).sum()), int((st_o == 1).sum())
    report[name] = dict(runs=m, status_agreement=agree, fma_oracle_agreement=agree_fma,
                        converged_gpu=c_g, converged_oracle=c_o,
                        co_converged=int(both.sum()), max_dfval_co_converged=dfv,
                        max_oracle_gradnorm_at_gpu_converged=gmax)
    assert agree >= agree_fma - AGREE_SLACK - 3 * sd, report[name]
    assert dfv <= 1e-8, report[name]
    assert gmax < TOL * (1 + 1e-3), report[name]
    p = c_o / m
    assert abs(c_g - c_o) <= 4 * math.sqrt(m * max(p * (1 - p), 0.25 / m)) + 0.05 * m, \
        report[name]


@pytest.mark.parametrize("block", [0, 384, 512])
def test_mixed_batch_run_for_run(cuda, block):
    fx = _fixture("parity_mixed.npz")
    jobs = []
    for ci, (name, ctor, dim, lo, hi) in enumerate(MIXED):
        kind, _, n, m, seed = fx[f"{name}/meta"]
        assert dim == fx[f"{name}/meta"][1]
        st = starts_uniform(int(seed), int(n), dim, lo, hi)
        jobs.append(BatchJob(ctor(dim), st))
    batch_device(jobs, max_iter=10000, tol=TOL, block=block)
    torch.cuda.synchronize()
    report = {}
    for (name, ctor, dim, lo, hi), j in zip(MIXED, jobs):
        kind, _, n, m, _ = (int(v) for v in fx[f"{name}/meta"])
        _check_class(name, kind, dim, j.status.cpu().numpy()[:m],
                     j.fval.cpu().numpy()[:m], j.x.cpu().numpy()[:m],
                     fx[f"{name}/status"], fx[f"{name}/fval"], fx[f"{name}/fma_status"],
                     report)
    print(f"\nmixed batch (block {block}) vs oracle:", json.dumps(report, indent=1))


def test_gaussian150_run_for_run(cuda):
    fx = _fixture("parity_gaussian150.npz")
    C = zb.gaussian_matrix(150)
    pbx, _, _, _ = O.oracle_pso(3, 150, 42, 1024, -5.0, 5.0, 10, data=C)
    r = bfgs_device(DeviceProblem(zb.Gaussian(C)), torch.from_numpy(pbx).cuda(),
                    max_iter=10000, tol=TOL)
    torch.cuda.synchronize()
    st, fv, x = r.status.cpu().numpy(), r.fval.cpu().numpy(), r.x.cpu().numpy()
    it = r.iter.cpu().numpy()
    report = {}
    _check_class("gaussian150", 3, 150, st, fv, x, fx["status"], fx["fval"],
                 fx["fma_status"], report, data=C)
    report["gaussian150"].update(mean_iterations_gpu=float(it.mean()),
                                 mean_iterations_oracle=float(fx["iter"].mean()))
    print("\ngaussian150 vs oracle:", json.dumps(report, indent=1))
    assert (st == 1).all() and (fx["status"] == 1).all()
    assert np.abs(x).max() < 1e-9
