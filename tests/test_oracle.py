"""The oracle (C restatement) against the reference's own known-answer tests
and, where the reference's host build is present, bit for bit against it."""
import ctypes as C
import math

import numpy as np
import pytest

from tests import _oracle as O

ROS, RAS, ACK, GAU, NLL = 0, 1, 2, 3, 4
EULER = 0.5772156649015328606


# ---- known answers from test/bfgs_tests.cu --------------------------------
def test_line_search_quadratic_alpha_half():
    """test/bfgs_tests.cu:121-151: x^2 from x=1, p=-2, g=2 -> alpha 0.5."""
    # x^2 is Rosenbrock-free; use the Gaussian 0.5 * x * 2 * x = x^2 in 1-D.
    C1 = np.array([[2.0]])
    o = O.zobj(GAU, 1, C1)
    x, p, g = np.array([1.0]), np.array([-2.0]), np.array([2.0])
    a = O.oracle().zor_line_search(C.byref(o), 1.0, x.ctypes.data, p.ctypes.data,
                                   g.ctypes.data)
    assert a == 0.5


def test_bfgs_update_known_step():
    """test/bfgs_tests.cu:228-264: H=I, s=(1,0), y=(2,0) -> diag(0.5, 1)."""
    H = np.eye(2)
    s, y = np.array([1.0, 0.0]), np.array([2.0, 0.0])
    O.oracle().zor_bfgs_update(2, H.ctypes.data, s.ctypes.data, y.ctypes.data, 2.0)
    np.testing.assert_allclose(H, [[0.5, 0.0], [0.0, 1.0]], atol=1e-12)


def test_bfgs_update_skips_tiny_curvature():
    """utils.cuh:254-255: |s.y| < 1e-14 leaves H untouched."""
    H = np.eye(3) * 2.0
    s, y = np.array([1e-8, 0, 0]), np.array([1e-8, 0, 0])
    O.oracle().zor_bfgs_update(3, H.ctypes.data, s.ctypes.data, y.ctypes.data, 1e-16)
    np.testing.assert_array_equal(H, np.eye(3) * 2.0)


def test_rastrigin_converges_at_iter0_from_origin():
    """test/bfgs_tests.cu:266-329."""
    r = O.oracle_bfgs(RAS, 2, np.zeros((1, 2)), max_iter=10, required=1, tol=1e-6)
    assert r["status"][0] == 1 and r["iter"][0] == 0
    assert abs(r["fval"][0]) <= 1e-6
    np.testing.assert_allclose(r["x"][0], [0, 0], atol=1e-6)


def test_quadratic_from_4p5():
    """test/bfgs_tests.cu:340-389 (x0^2 + x1^2 from (4.5, 4.5))."""
    r = O.oracle_bfgs(GAU, 2, np.array([[4.5, 4.5]]), max_iter=100, required=1,
                      tol=1e-6, data=2.0 * np.eye(2))
    assert r["status"][0] == 1
    assert abs(r["fval"][0]) <= 1e-6
    np.testing.assert_allclose(r["x"][0], [0, 0], atol=1e-6)


def test_rosenbrock_from_4p5():
    """test/bfgs_tests.cu:391-453 (tol 1e-17 there; status 1 at 1e-8 here,
    x within 1e-6 of (1, 1) either way)."""
    r = O.oracle_bfgs(ROS, 2, np.array([[4.5, 4.5]]), max_iter=1000, required=1,
                      tol=1e-8)
    assert r["status"][0] == 1 and r["iter"][0] < 1000
    assert abs(r["fval"][0]) <= 1e-4
    np.testing.assert_allclose(r["x"][0], [1, 1], atol=1e-6)


def test_trajectory_nan_tail():
    """test/bfgs_tests.cu:554-671: slots after convergence stay NaN."""
    r = O.oracle_bfgs(GAU, 2, np.array([[1.0, 1.0]]), max_iter=50, required=1,
                      tol=1e-6, data=2.0 * np.eye(2), traj=True)
    assert r["traj_f"][0, 0] > 0 and not math.isnan(r["traj_f"][0, 0])
    conv = int(np.argmax(r["traj_status"][:, 0] == 1))
    assert r["traj_status"][conv, 0] == 1 and conv < 49
    assert np.isnan(r["traj_f"][conv + 1:, 0]).all()


def test_max_iter_zero_is_surrender():
    r = O.oracle_bfgs(ROS, 2, np.array([[3.0, -3.0]]), max_iter=0)
    assert r["status"][0] == 0 and r["iter"][0] == 0
    assert r["fval"][0] == O.value(ROS, 2, np.array([3.0, -3.0]))


def test_nonfinite_start_is_status5():
    r = O.oracle_bfgs(ROS, 2, np.array([[1e200, 1e200]]), max_iter=10)
    assert r["status"][0] == 5


def test_stop_early_status2():
    rng = np.random.default_rng(3)
    st = rng.uniform(-2, 2, (20, 2))
    r = O.oracle_bfgs(ROS, 2, st, max_iter=5000, required=3)
    assert (r["status"] == 1).sum() == 3
    assert (r["status"] == 2).sum() >= 1


# ---- test/fun_tests.cu:75-128 ----------------------------------------------
def test_values_at_minima():
    assert O.value(RAS, 2, [0.0, 0.0]) == pytest.approx(0.0)
    assert abs(O.value(ACK, 2, [0.0, 0.0])) <= 1e-6
    assert O.value(ROS, 2, [1.0, 1.0]) == 0.0


def test_gradients_at_minima():
    np.testing.assert_allclose(O.grad_dual(RAS, 2, [0.0, 0.0])[1], [0, 0], atol=1e-12)
    np.testing.assert_allclose(O.grad_dual(ROS, 2, [1.0, 1.0])[1], [0, 0], atol=1e-12)
    g = O.grad_dual(ACK, 2, [-1e-17, 1e-17])[1]
    np.testing.assert_allclose(g, [-2.0, 2.0], rtol=1e-6)


def test_ackley_gradient_nan_at_origin():
    """duals.cuh:174-178: sqrt'(0) makes the dual gradient NaN at exactly 0."""
    assert np.isnan(O.grad_dual(ACK, 2, [0.0, 0.0])[1]).all()


# ---- test/dual_tests.cu:511-571 --------------------------------------------
def test_digamma_known_values():
    d = O.oracle().zor_digamma
    assert d(1.0) == pytest.approx(-EULER, rel=1.1e-13, abs=1.1e-13)
    assert d(2.0) == pytest.approx(1 - EULER, rel=1.1e-13, abs=1.1e-13)
    assert d(3.0) == pytest.approx(1.5 - EULER, rel=1.1e-13, abs=1.1e-13)
    assert d(0.5) == pytest.approx(-EULER - 2 * math.log(2), rel=1.1e-13, abs=1.1e-13)


def test_digamma_poles():
    d = O.oracle().zor_digamma
    eps = 1e-9
    for pole in (0.0, -1.0, -2.0):
        assert math.isinf(d(pole))
        assert d(pole + eps) < 0 and d(pole - eps) > 0
        assert d(pole + eps) == pytest.approx(-1 / eps, rel=1.2e-7)
        assert d(pole - eps) == pytest.approx(1 / eps, rel=1.2e-7)


# ---- test/pso_tests.cu:96-277 ----------------------------------------------
def test_pso_inertia_only_step():
    x = np.array([0.0, 1.0, 2.0, 3.0])
    v = np.array([10.0, 20.0, 30.0, 40.0])
    for i in range(4):
        xi, vi = x[i:i + 1].copy(), v[i:i + 1].copy()
        r = np.array([0.3])
        O.oracle().zor_pso_step(1, 0.5, 0.0, 0.0, r.ctypes.data, r.ctypes.data,
                                xi.ctypes.data, vi.ctypes.data, xi.ctypes.data,
                                np.zeros(1).ctypes.data)
        assert vi[0] == 0.5 * v[i] and xi[0] == x[i] + 0.5 * v[i]


def test_pso_zero_coefficients_freeze():
    x, v = np.array([1.5, -2.0]), np.array([0.3, 0.1])
    x0 = x.copy()
    r = np.array([0.4, 0.9])
    O.oracle().zor_pso_step(2, 0.0, 0.0, 0.0, r.ctypes.data, r.ctypes.data,
                            x.ctypes.data, v.ctypes.data, x0.ctypes.data,
                            np.zeros(2).ctypes.data)
    np.testing.assert_array_equal(x, x0)
    np.testing.assert_array_equal(v, [0.0, 0.0])


def test_pso_init_consistency():
    """test/pso_tests.cu:27-94: pBestVal = f(pBestX), gBest = best particle."""
    pbx, pbf, gbx, gbf = O.oracle_pso(RAS, 2, 42, 64, -5.0, 5.0, 0)
    for i in range(64):
        assert pbf[i] == O.value(RAS, 2, pbx[i])
    assert gbf == pbf.min()
    np.testing.assert_array_equal(gbx, pbx[int(np.argmin(pbf))])


def test_pso_improves_and_bounds_starts():
    pbx0, pbf0, _, g0 = O.oracle_pso(RAS, 10, 42, 256, -5.12, 5.12, 0)
    pbx, pbf, _, g = O.oracle_pso(RAS, 10, 42, 256, -5.12, 5.12, 20)
    assert (pbf <= pbf0).all() and g <= g0


# ---- RNG -------------------------------------------------------------------
def test_philox_known_answer():
    """Philox4x32-10 known-answer vectors published with Random123
    (kat_vectors): counter/key all zero and all 0xffffffff."""
    L = O.oracle()
    out = np.zeros(4, np.uint32)
    ctr = np.zeros(4, np.uint32)
    key = np.zeros(2, np.uint32)
    L.zor_philox4x32_10(ctr.ctypes.data, key.ctypes.data, out.ctypes.data)
    assert [hex(v) for v in out] == ["0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]
    ctr[:] = 0xFFFFFFFF
    key[:] = 0xFFFFFFFF
    L.zor_philox4x32_10(ctr.ctypes.data, key.ctypes.data, out.ctypes.data)
    assert [hex(v) for v in out] == ["0x408f276d", "0x41c83b0e", "0xa20bc7c6", "0x6d5451fd"]


def test_uniform_starts_in_range_and_distinct():
    s = O.oracle_starts(42, 1000, 3, -5.0, 5.0)
    assert s.min() >= -5.0 and s.max() < 5.0
    assert abs(s.mean()) < 0.3
    assert len(np.unique(s)) == s.size


# ---- gradients: adjoint maths vs dual vs central differences --------------
@pytest.mark.parametrize("kind,dim", [(ROS, 2), (ROS, 8), (RAS, 10), (ACK, 30), (GAU, 8)])
def test_analytic_gradient_matches_dual(kind, dim):
    rng = np.random.default_rng(kind * 100 + dim)
    data = None
    if kind == GAU:
        A = rng.normal(size=(dim, dim))
        data = A @ A.T + dim * np.eye(dim)
    for _ in range(5):
        x = rng.uniform(-2, 2, dim)
        _, gd = O.grad_dual(kind, dim, x, data)
        _, ga = O.grad_analytic(kind, dim, x, data)
        np.testing.assert_allclose(ga, gd, rtol=1e-10, atol=1e-10 * np.abs(gd).max())


def test_nll_gradient_dual_analytic_fd():
    x, k, _ = O.dijet_toy()
    th = np.array([0.5, 10.0, 5.0, 0.1])  # a in normalised units is scaled below
    # scale a so lambda matches the data's normalisation
    lam = (1 - x) ** th[1] / x ** (th[2] + th[3] * np.log(x))
    th[0] = k.sum() / lam.sum()
    _, gd = O.grad_dual(NLL, 4, th, x, k)
    _, ga = O.grad_analytic(NLL, 4, th, x, k)
    np.testing.assert_allclose(ga, gd, rtol=1e-9, atol=1e-9 * np.abs(gd).max())
    for i in range(4):
        h = 1e-6 * max(1.0, abs(th[i]))
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        fd = (O.value(NLL, 4, tp, x, k) - O.value(NLL, 4, tm, x, k)) / (2 * h)
        assert fd == pytest.approx(gd[i], rel=1e-5, abs=1e-3)


# ---- the pin: oracle == reference host build, bit for bit -----------------
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("kind,dim,lo,hi,n", [
    (ROS, 2, -5, 5, 64), (ROS, 8, -5, 5, 16), (ROS, 32, -5, 5, 4),
    (RAS, 2, -5.12, 5.12, 32), (RAS, 10, -5.12, 5.12, 8),
    (ACK, 2, -32.768, 32.768, 32), (ACK, 30, -32.768, 32.768, 4),
])
def test_oracle_bit_identical_to_reference(kind, dim, lo, hi, n):
    st = O.oracle_starts(42, n, dim, lo, hi)
    a = O.oracle_bfgs(kind, dim, st, max_iter=200, traj=True, lower=lo, upper=hi)
    b = O.ref_bfgs(kind, dim, st, max_iter=200, traj=True, lower=lo, upper=hi)
    for key in ("fval", "status", "iter", "gnorm", "x", "traj_x", "traj_f", "traj_g",
                "traj_status"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)


@needs_ref
def test_oracle_bit_identical_gaussian_and_nll():
    C8 = np.full((8, 8), 0.5) + np.eye(8) * 3.5
    st = O.oracle_starts(1, 6, 8, -5, 5)
    a = O.oracle_bfgs(GAU, 8, st, max_iter=100, data=C8, traj=True)
    b = O.ref_bfgs(GAU, 8, st, max_iter=100, data=C8, traj=True)
    for key in ("fval", "status", "iter", "x", "traj_x", "traj_f"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)
    x, k, _ = O.dijet_toy()
    st = np.array([[0.6, 10.2, 4.9, 0.09], [0.4, 9.5, 5.2, 0.11]])
    st[:, 0] *= 1.0
    a = O.oracle_bfgs(NLL, 4, st, max_iter=60, data=x, idata=k, traj=True)
    b = O.ref_bfgs(NLL, 4, st, max_iter=60, data=x, idata=k, traj=True)
    for key in ("fval", "status", "iter", "x", "traj_x", "traj_f"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)


@needs_ref
def test_reference_known_answers_through_ref_build():
    R = O.ref()
    assert R.zref_linesearch_quadratic(1.0, 1.0, -2.0, 2.0) == 0.5
    H = np.eye(2)
    s, y = np.array([1.0, 0.0]), np.array([2.0, 0.0])
    R.zref_bfgs_update(2, H.ctypes.data, s.ctypes.data, y.ctypes.data, 2.0)
    np.testing.assert_allclose(H, [[0.5, 0], [0, 1]], atol=1e-12)
    for v in (1.0, 2.0, 3.0, 0.5, 1e-9, -1e-9, 7.3, -2.5):
        assert R.zref_digamma(v) == O.oracle().zor_digamma(v)


@needs_ref
def test_update_hoisted_equals_reference_quartic_loop():
    rng = np.random.default_rng(5)
    for dim in (2, 3, 4, 8):
        for _ in range(10):
            A = rng.normal(size=(dim, dim))
            H0 = A @ A.T + np.eye(dim)
            s, y = rng.normal(size=dim), rng.normal(size=dim)
            sy = float(s @ y)
            Ho, Hr = H0.copy(), H0.copy()
            O.oracle().zor_bfgs_update(dim, Ho.ctypes.data, s.ctypes.data, y.ctypes.data, sy)
            O.ref().zref_bfgs_update(dim, Hr.ctypes.data, s.ctypes.data, y.ctypes.data, sy)
            np.testing.assert_array_equal(Ho, Hr)


# ---- the reference's own sensitivity to rounding --------------------------
@pytest.mark.parametrize("kind,dim,lo,hi,n,iters", [
    (RAS, 2, -5.12, 5.12, 256, 3000), (ACK, 30, -32.768, 32.768, 32, 2000),
    (ROS, 8, -5, 5, 96, 2000)])
def test_reference_outcomes_move_with_fma_contraction(kind, dim, lo, hi, n, iters):
    """The same algorithm with and without FMA contraction (the reference
    built by nvcc vs for the host) ends some runs differently: run status is
    not reproducible across compilers, only its statistics and the values of
    runs both sides converge."""
    st = O.oracle_starts(21, n, dim, lo, hi)
    a = O.oracle_bfgs(kind, dim, st, max_iter=iters, lower=lo, upper=hi)
    b = O.oracle_fma_bfgs(kind, dim, st, max_iter=iters, lower=lo, upper=hi)
    agree = (a["status"] == b["status"]).mean()
    both = (a["status"] == 1) & (b["status"] == 1)
    print(f"kind {kind} dim {dim}: status agreement {agree:.1%}")
    assert 0.8 <= agree < 1.0
    assert np.abs(a["fval"][both] - b["fval"][both]).max() <= 1e-8


# ---- the dual gradient pinned to the reference's own ----------------------
def _grad_points(kind, dim, n, seed):
    rng = np.random.default_rng(seed)
    lo, hi = {ROS: (-5, 5), RAS: (-5.12, 5.12), ACK: (-32.768, 32.768),
              GAU: (-5, 5)}[kind]
    return rng.uniform(lo, hi, size=(n, dim))


@needs_ref
@pytest.mark.parametrize("kind,dim", [(ROS, d) for d in (2, 4, 8, 10, 16, 32, 64, 128, 256)]
                         + [(RAS, d) for d in (2, 10, 16)] + [(ACK, d) for d in (2, 10, 30)])
def test_oracle_dual_gradient_bit_identical_to_reference(kind, dim):
    """zor_value_grad_dual equals the reference's dual::calculateGradientUsingAD
    (include/duals.cuh:241-266) from its host build, bit for bit."""
    for x in _grad_points(kind, dim, 8, 17 * dim + kind):
        fo, go = O.grad_dual(kind, dim, x)
        fr, gr = O.ref_grad_dual(kind, dim, x)
        np.testing.assert_array_equal(go, gr)
        assert fo == fr


@needs_ref
@pytest.mark.parametrize("dim,sym", [(2, True), (8, True), (32, True), (150, True),
                                     (8, False), (150, False)])
def test_oracle_dual_gradient_gaussian_bit_identical_to_reference(dim, sym):
    rng = np.random.default_rng(dim)
    C = np.full((dim, dim), 0.5)
    np.fill_diagonal(C, 1.0 + (dim - 1) * 0.5)
    if not sym:
        C = C + 0.25 * rng.normal(size=(dim, dim))
    C = np.ascontiguousarray(C)
    for x in _grad_points(GAU, dim, 4, dim + 1):
        fo, go = O.grad_dual(GAU, dim, x, C)
        fr, gr = O.ref_grad_dual(GAU, dim, x, C)
        np.testing.assert_array_equal(go, gr)
        assert fo == fr


@needs_ref
def test_oracle_dual_gradient_nll_bit_identical_to_reference():
    x, k, _ = O.dijet_toy()
    rng = np.random.default_rng(11)
    base = np.array([1.0, 10.0, 5.0, 0.1])
    shape = (1 - x) ** base[1] / x ** (base[2] + base[3] * np.log(x))
    base[0] = k.sum() / shape.sum()
    for th in base * (1.0 + 0.05 * rng.normal(size=(6, 4))):
        fo, go = O.grad_dual(NLL, 4, th, x, k)
        fr, gr = O.ref_grad_dual(NLL, 4, th, x, k)
        np.testing.assert_array_equal(go, gr)
        assert fo == fr


@needs_ref
def test_reference_ackley_gradient_near_origin():
    """test/fun_tests.cu:75-128 through the reference build and the oracle."""
    for fn in (O.grad_dual, O.ref_grad_dual):
        _, g = fn(ACK, 2, np.array([-1e-17, 1e-17]))
        np.testing.assert_allclose(g, [-2.0, 2.0], rtol=1e-12)


@pytest.mark.skipif(not O.ref_gpu_available(), reason="oracle/_ref GPU build not built")
def test_reference_gpu_build_loads_without_a_gpu():
    """The reference kernel's GPU build (the checker of exact mode on the
    device) loads here and exports its entry point; it runs only under -m gpu."""
    import ctypes

    lib = ctypes.CDLL(str(O.REF_GPU_SO))
    assert hasattr(lib, "zrefg_bfgs")


@needs_ref
@pytest.mark.parametrize("kind,dim,n,iters", [(ROS, 64, 2, 30), (ROS, 128, 1, 8),
                                              (GAU, 150, 1, 5)])
def test_oracle_bit_identical_at_the_benchmarked_dimensions(kind, dim, n, iters):
    """The oracle's hoisted O(D^3) update against the reference's O(D^4) loop
    (utils.cuh:245-287) at the sizes whose run-for-run fixtures the oracle
    wrote (Rosenbrock 64 and 128 of the mixed batch, the 150-D Gaussian):
    every iterate, f, gradient norm and status, bit for bit."""
    data = None
    if kind == GAU:
        data = np.full((dim, dim), 0.5)  # C_ii = 75.5, C_ij = 0.5 at dim 150
        np.fill_diagonal(data, 1.0 + (dim - 1) * 0.5)
    st = O.oracle_starts(42, n, dim, -5.0, 5.0)
    a = O.oracle_bfgs(kind, dim, st, max_iter=iters, data=data, traj=True)
    b = O.ref_bfgs(kind, dim, st, max_iter=iters, data=data, traj=True)
    for key in ("fval", "status", "iter", "gnorm", "x", "traj_x", "traj_f", "traj_g",
                "traj_status"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)
