"""Implicit-function adjoint of the binned Poisson fits (dijet toys) on the
GPU: d(fitted parameters)/d(bin counts) for every toy's best run, against
the numpy formula at the same point (the formula itself is checked against
finite-difference refits in test_fit_math.py)."""
import numpy as np
import pytest
import torch

import zeus_b200 as zb
from zeus_b200.device import BatchJob, batch_device, nll_sensitivity
from tests import _oracle as O

pytestmark = pytest.mark.gpu


def toy_starts(k, x, n, rng):
    lam = (1 - x) ** 10 / x ** (5 + 0.1 * np.log(x))
    a0 = k.sum() / lam.sum()
    return np.column_stack([a0 * rng.uniform(0.9, 1.1, n), rng.uniform(9.5, 10.5, n),
                            rng.uniform(4.8, 5.2, n), rng.uniform(0.09, 0.11, n)])


@pytest.fixture(scope="module")
def fits(cuda):
    rng = np.random.default_rng(4)
    toys, per = 5, 32
    ks, xs, sts = [], [], []
    for t in range(toys):
        x, k, _ = O.dijet_toy(seed=10 + t)
        ks.append(k)
        xs.append(x)
        sts.append(toy_starts(k, x, per, rng))
    obj = zb.PoissonNLL(np.concatenate(ks), np.concatenate(xs))
    j = BatchJob(obj, torch.tensor(np.concatenate(sts)).cuda(), runs_per_instance=per)
    batch_device([j], max_iter=5000)
    best, sens = nll_sensitivity(j)
    torch.cuda.synchronize()
    return ks, xs, j, best.cpu().numpy(), sens.cpu().numpy()


def test_best_run_per_toy(fits):
    ks, xs, j, best, _ = fits
    fv = j.fval.cpu().numpy().reshape(len(ks), -1)
    xr = j.x.cpu().numpy().reshape(len(ks), fv.shape[1], 4)
    for t in range(len(ks)):
        r = int(np.argmin(fv[t]))
        assert best[t, 0] == fv[t].min()
        assert int(best[t, 5]) == t * fv.shape[1] + r
        np.testing.assert_array_equal(best[t, 1:5], xr[t, r])


def test_sensitivity_matches_formula(fits):
    """Kernel (4x4 Cholesky per toy) against numpy's solve at the same
    parameters; the scaled Hessian's condition number is ~1e7, so the two
    fp64 solutions agree to ~1e-9 of each row's scale."""
    ks, xs, _, best, sens = fits
    for t in range(len(ks)):
        ref = O.nll_sensitivity(xs[t], ks[t].astype(np.float64), best[t, 1:5])
        for r in range(4):
            np.testing.assert_allclose(sens[t, r], ref[r], rtol=1e-7,
                                       atol=1e-9 * np.abs(ref[r]).max())


def test_best_fit_is_near_the_minimum(fits):
    """The sensitivities are evaluated at the GPU's best run; it sits close
    to the exact minimum, so they are the fit's own to first order."""
    ks, xs, _, best, sens = fits
    for t in range(len(ks)):
        p = O.nll_newton_fit(xs[t], ks[t], best[t, 1:5])
        th = lambda q: np.array([np.log(q[0]), q[1], q[2], q[3]])
        np.testing.assert_allclose(th(best[t, 1:5]), th(p), rtol=1e-3, atol=1e-4)
        ref = O.nll_sensitivity(xs[t], ks[t].astype(np.float64), p)
        np.testing.assert_allclose(sens[t], ref, rtol=5e-2, atol=1e-3 * np.abs(ref).max())


def test_no_toys_is_a_no_op(cuda):
    x, k, _ = O.dijet_toy(seed=3)
    obj = zb.PoissonNLL(k, x)
    j = BatchJob(obj, torch.zeros((0, 4), dtype=torch.float64, device="cuda"),
                 runs_per_instance=4)
    best, sens = nll_sensitivity(j)
    assert best.shape == (0, 6) and sens.shape[0] == 0
