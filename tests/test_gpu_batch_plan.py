"""The host-buffer batch (zeus_batch_plan_*): host inputs in, each class's
best run, coordinates and census out.  Its results equal the device-buffer
persistent batch (zeus_batch_device) and census on the same starts, run for
run, and a second run of the same plan with new inputs matches a fresh
batch too."""
import numpy as np
import pytest
import torch

import zeus_b200 as zb
from zeus_b200.device import (BatchJob, DeviceProblem, batch_device, census_device,
                              pso_device, starts_uniform)
from tests import _oracle as O

pytestmark = pytest.mark.gpu


def device_reference(jobs):
    """Best (lowest fval, lowest index) and census of each BatchJob."""
    out = []
    for j in jobs:
        cen = census_device(j.fval, j.status, j.x, j.dp.obj.dim,
                            known_min=j.dp.obj.known_minimum)
        b = cen["best_idx"]
        out.append(dict(cen=cen, fval=float(j.fval[b]), status=int(j.status[b]),
                        iter=int(j.iter[b]), gnorm=float(j.gnorm[b]),
                        x=j.x[b].cpu().numpy(), idx=b))
    return out


def check_same(res, ref):
    for r, w in zip(res, ref):
        assert r.idx == w["idx"]
        assert r.status == w["status"] and r.iter == w["iter"]
        assert r.fval == w["fval"] and r.gradientNorm == w["gnorm"]
        np.testing.assert_array_equal(r.coordinates, w["x"])
        assert (r.c.actual, r.c.claimed, r.c.surrendered, r.c.stopped) == (
            w["cen"]["actual"], w["cen"]["claimed"], w["cen"]["surrendered"],
            w["cen"]["stopped"])


def test_plan_equals_device_batch(cuda):
    objs = [(zb.Rosenbrock(64), -5.0, 5.0, 128), (zb.Ackley(30), -32.768, 32.768, 200),
            (zb.Rosenbrock(8), -5.0, 5.0, 300), (zb.Gaussian(zb.gaussian_matrix(32)), -5, 5, 64)]
    specs, jobs = [], []
    for ci, (obj, lo, hi, n) in enumerate(objs):
        st = starts_uniform(7 + ci, n, obj.dim, lo, hi)
        jobs.append(BatchJob(obj, st))
        specs.append(dict(obj=obj, n=n, starts=st.cpu().numpy()))
    batch_device(jobs, max_iter=3000)
    torch.cuda.synchronize()
    ref = device_reference(jobs)
    plan = zb.BatchPlan(specs, max_iter=3000)
    check_same(plan.run(), ref)
    h2d, d2h = plan.traffic()
    assert h2d == sum(s["starts"].nbytes for s in specs) + 32 * 32 * 8
    assert d2h > 0
    # new starts through the same plan
    specs2, jobs2 = [], []
    for ci, (obj, lo, hi, n) in enumerate(objs):
        st = starts_uniform(100 + ci, n, obj.dim, lo, hi)
        jobs2.append(BatchJob(obj, st))
        specs2.append(dict(obj=obj, n=n, starts=st.cpu().numpy()))
    batch_device(jobs2, max_iter=3000)
    torch.cuda.synchronize()
    check_same(plan.run(specs2), device_reference(jobs2))
    plan.close()


def test_plan_device_drawn_starts_and_instances(cuda):
    """A PSO class (starts from the device swarm) and a per-instance NLL
    class (two toys, host starts)."""
    x, k, _ = O.dijet_toy()
    x2 = np.concatenate([x, x])
    k2 = np.concatenate([k, np.random.default_rng(3).poisson(k).astype(np.int32)])
    nll = zb.PoissonNLL(k2, x2)
    rng = np.random.default_rng(4)
    lam = (1 - x) ** 10 / x ** (5 + 0.1 * np.log(x))
    a0 = k.sum() / lam.sum()
    st_nll = np.column_stack([a0 * rng.uniform(0.8, 1.2, 64), rng.uniform(9, 11, 64),
                              rng.uniform(4.5, 5.5, 64), rng.uniform(0.08, 0.12, 64)])
    ras = zb.Rastrigin(10)
    specs = [dict(obj=ras, n=256, seed=11, lower=-5.12, upper=5.12, pso_iter=5),
             dict(obj=nll, n=64, runs_per_instance=32, starts=st_nll)]
    plan = zb.BatchPlan(specs, max_iter=2000)
    res = plan.run()
    pbx, _, _ = pso_device(ras, 11, 256, -5.12, 5.12, 5)
    jobs = [BatchJob(ras, pbx),
            BatchJob(DeviceProblem(nll), torch.from_numpy(st_nll).cuda(),
                     runs_per_instance=32)]
    batch_device(jobs, max_iter=2000)
    torch.cuda.synchronize()
    check_same(res, device_reference(jobs))
    h2d, _ = plan.traffic()
    assert h2d == st_nll.nbytes + x2.nbytes + k2.nbytes
    plan.close()


def test_plan_rejects_changed_shapes(cuda):
    obj = zb.Rosenbrock(2)
    st = np.zeros((16, 2))
    plan = zb.BatchPlan([dict(obj=obj, n=16, starts=st)], max_iter=10)
    with pytest.raises(zb.ZeusError):
        plan.run([dict(obj=obj, n=8, starts=st[:8])])
    with pytest.raises(zb.ZeusError):  # exact mode is not the batch's
        zb.BatchPlan([dict(obj=obj, n=16, starts=st)], max_iter=10, block=0).run(
            [dict(obj=zb.Rosenbrock(4), n=16, starts=np.zeros((16, 4)))])
    plan.close()
