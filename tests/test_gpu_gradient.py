"""Every gradient path of the BFGS layouts, evaluated at points on the GPU
through the C ABI (zeus_gradient_device), against the oracle's forward-mode
dual gradient -- a restatement of dual::calculateGradientUsingAD
(include/duals.cuh:241-266) pinned to the reference's own host build in
tests/test_oracle.py -- and against central differences of the oracle's f.

Paths: the thread layout's adjoint() and dual passes; the tile layout's
cooperative value+gradient and gradient-only forms at every built width; the
CTA layout's (and the persistent batch's) forms at the block sizes the
kernels launch; the CTA line search's carried value and gradient of a
symmetric quadratic form.

Tolerances: gradients within 1e-10 relative to the oracle's dual gradient
(max-norm: max_i |g_i - g_ref_i| <= 1e-10 max_i |g_ref_i|), values within
1e-10 relative; central differences within 1e-6 relative (step 1e-6 |x_i|,
at least 1e-6)."""
import numpy as np
import pytest
import torch

import zeus_b200 as zb
from zeus_b200.device import DeviceProblem, gradient_device, tile_widths
from tests import _oracle as O

pytestmark = pytest.mark.gpu

ROS, RAS, ACK, GAU, NLL = 0, 1, 2, 3, 4
REL = 1e-10
FD_REL = 1e-6
CTA_BLOCKS = (128, 256, 384, 512)  # standalone CTA layout: 256/512; batch: 384/512

CASES = [(ROS, d) for d in (2, 4, 8, 10, 16, 32, 64, 128, 256)] + \
        [(RAS, d) for d in (2, 10, 16)] + [(ACK, d) for d in (2, 10, 30)] + \
        [(GAU, d) for d in (2, 8, 32, 150)] + [(NLL, 4)]


def gaussian_nonsym(dim, seed=3):
    rng = np.random.default_rng(seed)
    C = zb.gaussian_matrix(dim) + 0.25 * rng.normal(size=(dim, dim))
    return C


def problem(kind, dim, sym=True):
    """(Objective, oracle data, oracle idata)."""
    if kind == ROS:
        return zb.Rosenbrock(dim), None, None
    if kind == RAS:
        return zb.Rastrigin(dim), None, None
    if kind == ACK:
        return zb.Ackley(dim), None, None
    if kind == GAU:
        C = zb.gaussian_matrix(dim) if sym else gaussian_nonsym(dim)
        C = np.ascontiguousarray(C)
        return zb.Gaussian(C), C, None
    x, k, _ = O.dijet_toy()
    return zb.PoissonNLL(k, x), x, k


def points(kind, dim, n, seed):
    rng = np.random.default_rng(1000 * kind + dim + seed)
    if kind == NLL:
        x, k, _ = O.dijet_toy()
        base = np.array([1.0, 10.0, 5.0, 0.1])
        shape = (1 - x) ** base[1] / x ** (base[2] + base[3] * np.log(x))
        base[0] = k.sum() / shape.sum()
        th = base * (1.0 + 0.05 * rng.normal(size=(n, 4)))
        return np.ascontiguousarray(th)
    lo, hi = {ROS: (-5, 5), RAS: (-5.12, 5.12), ACK: (-32.768, 32.768),
              GAU: (-5, 5)}[kind]
    return rng.uniform(lo, hi, size=(n, dim))


def oracle_grad(kind, dim, X, data, idata):
    F = np.empty(len(X))
    G = np.empty_like(X)
    for i, x in enumerate(X):
        F[i], G[i] = O.grad_dual(kind, dim, x, data, idata)
    return F, G


def check_close(f, g, F, G, what):
    for i in range(len(F)):
        scale = np.abs(G[i]).max()
        err = np.abs(g[i] - G[i]).max()
        assert err <= REL * scale, f"{what}: point {i}: |dg| {err:.3e} vs |g| {scale:.3e}"
        if np.isfinite(f[i]):  # NaN: the path forms no value (gradient-only)
            assert abs(f[i] - F[i]) <= REL * max(abs(F[i]), 1.0), \
                f"{what}: point {i}: f {f[i]!r} vs {F[i]!r}"


def run_path(obj, X, path, gradient, width=0, P=None, alpha=0.0):
    xd = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    pd = None if P is None else torch.from_numpy(np.ascontiguousarray(P)).cuda()
    f, g = gradient_device(obj, xd, path, gradient, width, pd, alpha)
    torch.cuda.synchronize()
    return f.cpu().numpy(), g.cpu().numpy()


@pytest.mark.parametrize("kind,dim", CASES)
def test_every_path_matches_oracle_dual_gradient(cuda, kind, dim):
    obj, data, idata = problem(kind, dim)
    dp = DeviceProblem(obj)
    n = 6
    X = points(kind, dim, n, 0)
    F, G = oracle_grad(kind, dim, X, data, idata)
    checked = []
    if dim <= 32:
        for grad in ("adjoint", "dual"):
            f, g = run_path(dp, X, zb.GRADPATH_THREAD, grad)
            check_close(f, g, F, G, f"thread {grad}")
            checked.append(f"thread-{grad}")
    for ts in tile_widths(kind, dim):
        for path, grad in ((zb.GRADPATH_TILE, "adjoint"), (zb.GRADPATH_TILE, "dual"),
                           (zb.GRADPATH_TILE_GRAD, "adjoint")):
            f, g = run_path(dp, X, path, grad, ts)
            check_close(f, g, F, G, f"tile {ts} path {path} {grad}")
            checked.append(f"tile{ts}-{path}-{grad}")
    for blk in CTA_BLOCKS:
        for path, grad in ((zb.GRADPATH_CTA, "adjoint"), (zb.GRADPATH_CTA, "dual"),
                           (zb.GRADPATH_CTA_GRAD, "adjoint")):
            f, g = run_path(dp, X, path, grad, blk)
            check_close(f, g, F, G, f"cta {blk} path {path} {grad}")
            checked.append(f"cta{blk}-{path}-{grad}")
    assert checked


@pytest.mark.parametrize("dim", [2, 8, 32, 150])
def test_nonsymmetric_gaussian_paths(cuda, dim):
    obj, data, _ = problem(GAU, dim, sym=False)
    assert not np.array_equal(data, data.T)
    dp = DeviceProblem(obj)
    X = points(GAU, dim, 5, 1)
    F, G = oracle_grad(GAU, dim, X, data, None)
    for ts in tile_widths(GAU, dim):
        f, g = run_path(dp, X, zb.GRADPATH_TILE, "adjoint", ts)
        check_close(f, g, F, G, f"tile {ts}")
    for blk in CTA_BLOCKS:
        f, g = run_path(dp, X, zb.GRADPATH_CTA, "adjoint", blk)
        check_close(f, g, F, G, f"cta {blk}")
    if dim <= 32:
        f, g = run_path(dp, X, zb.GRADPATH_THREAD, "adjoint")
        check_close(f, g, F, G, "thread")
    with pytest.raises(zb.ZeusError):  # the carried form needs C = C^T
        run_path(dp, X, zb.GRADPATH_QUADRATIC, "adjoint", 256, P=X)


@pytest.mark.parametrize("dim", [8, 32, 150])
def test_quadratic_carried_value_and_gradient(cuda, dim):
    """The CTA line search of a symmetric quadratic form steps to x + a p with
    f(x) + a g.p + a^2 f(p) and g + a C p from one pass over C: both equal
    the oracle's f and dual gradient at the accepted point."""
    obj, data, _ = problem(GAU, dim)
    dp = DeviceProblem(obj)
    X = points(GAU, dim, 6, 2)
    P = np.random.default_rng(dim).uniform(-3, 3, size=X.shape)
    for blk in [b for b in CTA_BLOCKS if b >= dim]:
        for k in (0, 1, 7, 20):
            a = 2.0 ** -k
            f, g = run_path(dp, X, zb.GRADPATH_QUADRATIC, "adjoint", blk, P=P, alpha=a)
            Xa = X + a * P  # a power of two: the same bits as fma(a, p, x)
            F, G = oracle_grad(GAU, dim, Xa, data, None)
            check_close(f, g, F, G, f"quadratic block {blk} alpha 2^-{k}")


@pytest.mark.parametrize("kind,dim", [(ROS, 2), (ROS, 32), (ROS, 128), (RAS, 10),
                                      (ACK, 30), (GAU, 150), (NLL, 4)])
def test_adjoint_against_central_differences(cuda, kind, dim):
    obj, data, idata = problem(kind, dim)
    dp = DeviceProblem(obj)
    X = points(kind, dim, 3, 3)
    if dim <= 32:
        _, g = run_path(dp, X, zb.GRADPATH_THREAD, "adjoint")
    else:
        _, g = run_path(dp, X, zb.GRADPATH_CTA_GRAD, "adjoint", 384)
    for i, x in enumerate(X):
        fd = np.empty(dim)
        for d in range(dim):
            h = 1e-6 * max(1.0, abs(x[d]))
            xp, xm = x.copy(), x.copy()
            xp[d] += h
            xm[d] -= h
            fd[d] = (O.value(kind, dim, xp, data, idata) -
                     O.value(kind, dim, xm, data, idata)) / (xp[d] - xm[d])
        err = np.abs(g[i] - fd).max()
        assert err <= FD_REL * np.abs(fd).max(), (i, err, np.abs(fd).max())


def test_ackley_known_gradient_near_origin(cuda):
    """test/fun_tests.cu:75-128: grad Ackley(-1e-17, 1e-17) = (-2, 2)."""
    obj, _, _ = problem(ACK, 2)
    X = np.array([[-1e-17, 1e-17]])
    _, Gd = oracle_grad(ACK, 2, X, None, None)
    np.testing.assert_allclose(Gd[0], [-2.0, 2.0], rtol=1e-12)
    for path, width in ((zb.GRADPATH_THREAD, 0), (zb.GRADPATH_TILE, 2),
                        (zb.GRADPATH_TILE, 8), (zb.GRADPATH_CTA, 128)):
        for grad in ("adjoint", "dual"):
            _, g = run_path(obj, X, path, grad, width)
            np.testing.assert_allclose(g[0], [-2.0, 2.0], rtol=1e-12,
                                       err_msg=f"path {path} width {width} {grad}")


def test_gradient_paths_reject_bad_arguments(cuda):
    obj = zb.Rosenbrock(64)
    X = torch.zeros((2, 64), dtype=torch.float64, device="cuda")
    with pytest.raises(zb.ZeusError):  # the thread path stops at dim 32
        gradient_device(obj, X, zb.GRADPATH_THREAD, "adjoint")
    with pytest.raises(zb.ZeusError):  # no tile layout past dim 32
        gradient_device(obj, X, zb.GRADPATH_TILE, "adjoint", 32)
    with pytest.raises(zb.ZeusError):  # block not a multiple of 32
        gradient_device(obj, X, zb.GRADPATH_CTA, "adjoint", 100)
    with pytest.raises(zb.ZeusError):  # not a quadratic form
        gradient_device(obj, X, zb.GRADPATH_QUADRATIC, "adjoint", 128, p=X)
