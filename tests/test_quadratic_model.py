"""The premise of the Gaussian's quadratic-form line search, on the CPU.

For f(x) = 0.5 x^T C x, f(x + a p) = f(x) + a grad f(x).p + a^2 f(p)
exactly, so the reference's backtracking test (utils.cuh:376-412: alpha =
2^-k, k = 0..19, accept the first with f_k <= f0 + c1 alpha g.p and
f_k < f0, else alpha = 2^-20) can be decided on the model.  Checked here
against the oracle's direct evaluation of f (the reference's operation
order) on random symmetric and non-symmetric C: the chosen trial agrees,
and the model's values agree with the evaluated ones to rounding."""
import numpy as np
import pytest

from tests import _oracle as O

GAU = 3
C1 = 0.1


def first_pass(values, f0, gp):
    for k, fk in enumerate(values):
        a = 2.0 ** -k
        if fk <= f0 + C1 * a * gp and fk < f0:
            return k
    return 20


@pytest.mark.parametrize("symmetric", [True, False])
def test_model_picks_the_evaluated_trial(symmetric):
    rng = np.random.default_rng(11 if symmetric else 12)
    dim = 8
    agree = total = 0
    for _ in range(200):
        A = rng.normal(size=(dim, dim))
        C = A @ A.T + dim * np.eye(dim) if symmetric else \
            np.diag(rng.uniform(1, 50, dim)) + rng.uniform(-0.5, 0.5, (dim, dim))
        x = rng.uniform(-5, 5, dim)
        g = 0.5 * (C + C.T) @ x
        # a quasi-Newton-like direction: -g scaled, sometimes far too long
        p = -g * rng.choice([1.0, 0.1, 0.01, 3.0])
        f0 = O.value(GAU, dim, x, data=C)
        fp = O.value(GAU, dim, p, data=C)
        gp = float(g @ p)
        direct = [O.value(GAU, dim, x + 2.0 ** -k * p, data=C) for k in range(20)]
        model = [f0 + 2.0 ** -k * (gp + 2.0 ** -k * fp) for k in range(20)]
        np.testing.assert_allclose(model, direct, rtol=1e-9,
                                   atol=1e-12 * max(1.0, abs(f0)))
        total += 1
        agree += first_pass(model, f0, gp) == first_pass(direct, f0, gp)
    assert agree == total
