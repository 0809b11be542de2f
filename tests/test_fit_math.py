"""The implicit-function adjoint formula of the binned Poisson fit, checked
on the CPU: d p_hat / d k_j = H^-1 J_j against central differences of
Newton refits with one bin's count moved by +-1."""
import numpy as np
import pytest

from tests import _oracle as O


@pytest.fixture(scope="module")
def toy():
    x, k, lam = O.dijet_toy(seed=11)
    a0 = k.sum() / ((1 - x) ** 10 / x ** (5 + 0.1 * np.log(x))).sum()
    p = O.nll_newton_fit(x, k, (a0, 10.0, 5.0, 0.1))
    return x, k, p


def test_newton_fit_is_a_minimum(toy):
    x, k, p = toy
    _, _, g, H = O.nll_parts(x, k, p)
    # gradient small against the scale of its terms, Hessian positive definite
    lam, J, _, _ = O.nll_parts(x, k, p)
    scale = np.abs(J) @ (lam + k)
    assert np.all(np.abs(g) <= 1e-9 * scale)
    assert np.all(np.linalg.eigvalsh(H / np.sqrt(np.outer(np.diag(H), np.diag(H)))) > 0)


@pytest.mark.parametrize("b", [0, 37, 99])
def test_sensitivity_matches_finite_difference_refits(toy, b):
    x, k, p = toy
    S = O.nll_sensitivity(x, k, p)
    kp, km = k.astype(np.float64), k.astype(np.float64)
    kp[b] += 1
    km[b] -= 1
    # compared in theta = (ln a, b, c, d), in which the fit is close to linear
    # in the counts (a itself moves by a third of its value per count of the
    # last bin, where sinh makes a central difference in a 2% off)
    th = lambda q: np.array([np.log(q[0]), q[1], q[2], q[3]])
    fd = (th(O.nll_newton_fit(x, kp, p)) - th(O.nll_newton_fit(x, km, p))) / 2.0
    S_theta = S.copy()
    S_theta[0] /= p[0]
    np.testing.assert_allclose(S_theta[:, b], fd, rtol=1e-4)


def test_sensitivities_are_linear_in_counts(toy):
    """sum_j S_j (k_j - lambda_j) = p_hat - p(lambda): the adjoint propagates
    a count shift to first order (here exactly at p, where k -> lambda(p)
    leaves p unchanged)."""
    x, k, p = toy
    lam, _, _, _ = O.nll_parts(x, k, p)
    S = O.nll_sensitivity(x, k, p)
    # refitting the model's own expectation gives back p: zero shift
    p_asimov = O.nll_newton_fit(x, lam, p)
    np.testing.assert_allclose(p_asimov, p, rtol=1e-9)
    # a small shift of all counts moves p by S @ dk to first order
    rng = np.random.default_rng(3)
    dk = rng.normal(0.0, 0.01, size=k.shape)
    dp = O.nll_newton_fit(x, k + dk, p) - p
    np.testing.assert_allclose(dp, S @ dk, rtol=2e-3, atol=1e-6 * np.abs(dp).max())
