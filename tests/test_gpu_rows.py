"""The row layout (zb_bfgs_rows.cuh): one run per group of warps, each
thread holding a segment of R rows of H in registers (split groups: part
of it in shared memory), several groups per block.  Checked against the
oracle on final results (fast-mode arithmetic), and the persistent batch's
row classes against standalone row launches bit for bit (same per-run
body, same group shape; a 128-D class at 384 threads runs the standalone
kernel itself beside the batch kernel)."""
import numpy as np
import pytest
import torch

import zeus_b200 as zb
from zeus_b200.device import BatchJob, batch_device, bfgs_device, starts_uniform
from tests import _oracle as O

pytestmark = pytest.mark.gpu


def host(r):
    return {k: getattr(r, k).cpu().numpy() for k in ("fval", "status", "iter", "gnorm", "x")}


@pytest.mark.parametrize("dim,n,iters", [(32, 96, 3000), (64, 64, 3000), (128, 24, 1500)])
@pytest.mark.parametrize("grad", ["adjoint", "dual"])
def test_rows_against_oracle(cuda, dim, n, iters, grad):
    st = O.oracle_starts(21 + dim, n, dim, -5.0, 5.0)
    want = O.oracle_bfgs(0, dim, st, max_iter=iters)
    r = bfgs_device(zb.Rosenbrock(dim), torch.from_numpy(st).cuda(), max_iter=iters,
                    gradient=grad, layout=zb.LAYOUT_ROWS)
    torch.cuda.synchronize()
    got = host(r)
    agree = (got["status"] == want["status"]).mean()
    assert agree >= 0.85, agree
    both = (got["status"] == 1) & (want["status"] == 1)
    assert both.sum() >= 0.5 * (want["status"] == 1).sum()
    np.testing.assert_allclose(got["fval"][both], want["fval"][both], atol=1e-8)
    np.testing.assert_allclose(got["x"][both], want["x"][both], atol=1e-5)
    conv = got["status"] == 1
    assert (got["gnorm"][conv] < 1e-8).all()
    for i in np.flatnonzero(conv)[:8]:  # the claim holds by the oracle's gradient
        _, g = O.grad_dual(0, dim, got["x"][i])
        assert np.linalg.norm(g) < 1e-8 * (1 + 1e-3)
    # f(x_out) is the reported fval
    for i in range(0, n, 7):
        assert got["fval"][i] == pytest.approx(O.value(0, dim, got["x"][i]), rel=1e-12,
                                               abs=1e-14)


@pytest.mark.parametrize("block,dims", [(384, (32, 64, 128)), (512, (64,))])
def test_batch_rows_equal_standalone(cuda, block, dims):
    jobs, sts = [], []
    for i, d in enumerate(dims):
        st = starts_uniform(300 + i, 200, d, -5.0, 5.0)
        sts.append(st)
        jobs.append(BatchJob(zb.Rosenbrock(d), st, layout=zb.LAYOUT_ROWS))
    # a warp-sized class beside them, so the batch has both phases
    st8 = starts_uniform(5, 300, 8, -5.0, 5.0)
    jobs.append(BatchJob(zb.Rosenbrock(8), st8, layout=zb.LAYOUT_TILE, tile=8))
    batch_device(jobs, max_iter=800, block=block)
    torch.cuda.synchronize()
    for d, j, st in zip(dims, jobs, sts):
        ref = host(bfgs_device(zb.Rosenbrock(d), st, max_iter=800, layout=zb.LAYOUT_ROWS))
        torch.cuda.synchronize()
        got = host(j)
        for k in got:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"dim {d} {k}")
        assert (j.counters.cpu().numpy()[:, 0] > 0).all()


@pytest.mark.parametrize("block", [384, 512])
def test_batch_rows_dim128_against_oracle(cuda, block):
    """A 128-D class runs in the standalone kernel's split groups beside the
    batch kernel at 384 threads (a companion launch) and in sixteen-warp
    groups inside the 512-thread batch kernel: both against the oracle."""
    st = O.oracle_starts(77, 32, 128, -5.0, 5.0)
    want = O.oracle_bfgs(0, 128, st, max_iter=1500)
    j = BatchJob(zb.Rosenbrock(128), torch.from_numpy(st).cuda(), layout=zb.LAYOUT_ROWS)
    batch_device([j], max_iter=1500, block=block)
    torch.cuda.synchronize()
    got = host(j)
    assert (got["status"] == want["status"]).mean() >= 0.85
    both = (got["status"] == 1) & (want["status"] == 1)
    np.testing.assert_allclose(got["fval"][both], want["fval"][both], atol=1e-8)


def test_rows_stop_early_and_default_layout(cuda):
    st = starts_uniform(11, 300, 64, -2.0, 2.0)
    j = BatchJob(zb.Rosenbrock(64), st, required=10)
    batch_device([j], max_iter=5000)
    torch.cuda.synchronize()
    s = j.status.cpu().numpy()
    assert (s == 1).sum() >= 10 and (s == 2).sum() > 0
    assert j.control.cpu().numpy()[0] == 1
