"""CUDA path vs the oracle, through the C ABI (zeus_b200 -> libzeus_b200.so).

Exact mode reproduces the reference's arithmetic: for polynomial objectives
(Rosenbrock, Gaussian) the GPU trajectories must equal the oracle's bit for
bit; for objectives with cos/exp/log/pow/lgamma the only difference is CUDA's
libm versus glibc (an ulp here and there), and iterates must agree to
1e-10 relative (max-norm over dimensions, per iteration) over the first 50
iterations.  Fast mode uses an O(D^2) update with FMA, so it is checked on
final results: per-run status agreement, final fval to 1e-8 (absolute, plus
1e-10 relative) and final x to 1e-5 where both converged."""
import numpy as np
import pytest
import torch

import zeus_b200 as zb
from zeus_b200.device import DeviceProblem, bfgs_device, pso_device, starts_uniform, census_device
from tests import _oracle as O

pytestmark = pytest.mark.gpu

ROS, RAS, ACK, GAU, NLL = 0, 1, 2, 3, 4
BOUNDS = {ROS: (-5.0, 5.0), RAS: (-5.12, 5.12), ACK: (-32.768, 32.768), GAU: (-5.0, 5.0)}


def make_obj(kind, dim):
    if kind == ROS:
        return zb.Rosenbrock(dim), None, None
    if kind == RAS:
        return zb.Rastrigin(dim), None, None
    if kind == ACK:
        return zb.Ackley(dim), None, None
    if kind == GAU:
        C = zb.gaussian_matrix(dim)
        return zb.Gaussian(C), C, None
    x, k, _ = O.dijet_toy()
    return zb.PoissonNLL(k, x), x, k


def gpu_run(obj, starts, **kw):
    """bfgs_device through the C ABI; host numpy results."""
    st = torch.from_numpy(np.ascontiguousarray(starts)).cuda()
    r = bfgs_device(obj, st, **kw)
    torch.cuda.synchronize()
    out = dict(fval=r.fval.cpu().numpy(), status=r.status.cpu().numpy(),
               iter=r.iter.cpu().numpy(), gnorm=r.gnorm.cpu().numpy(),
               x=r.x.cpu().numpy(), counters=r.counters.cpu().numpy())
    if r.traj is not None:
        out.update(traj_x=r.traj["x"].cpu().numpy(), traj_f=r.traj["f"].cpu().numpy(),
                   traj_g=r.traj["g"].cpu().numpy(),
                   traj_status=r.traj["status"].cpu().numpy())
    return out


def rel_iterate_error(a, b):
    """Per (iteration, run): max_d |a-b| / max_d |b| on trajectory coords
    (NaN where the run had already stopped on both sides)."""
    num = np.max(np.abs(a - b), axis=1)
    den = np.maximum(np.max(np.abs(b), axis=1), 1e-300)
    both_nan = np.isnan(a).all(axis=1) & np.isnan(b).all(axis=1)
    out = num / den
    out[both_nan] = 0.0
    return out


# ---- exact mode: bit-identical trajectories for polynomial objectives ------
@pytest.mark.parametrize("kind,dim,n,iters", [
    (ROS, 2, 256, 200), (ROS, 8, 32, 200), (ROS, 32, 4, 100), (GAU, 8, 16, 100),
    (GAU, 150, 1, 50),
])
def test_exact_mode_bit_identical(cuda, kind, dim, n, iters):
    obj, data, idata = make_obj(kind, dim)
    lo, hi = BOUNDS[kind]
    st = O.oracle_starts(42, n, dim, lo, hi)
    want = O.oracle_bfgs(kind, dim, st, max_iter=iters, data=data, idata=idata, traj=True,
                         lower=lo, upper=hi)
    got = gpu_run(obj, st, max_iter=iters, mode="exact", gradient="dual", traj=True)
    for key in ("status", "iter", "fval", "gnorm", "x", "traj_x", "traj_f", "traj_g",
                "traj_status"):
        np.testing.assert_array_equal(got[key], want[key], err_msg=key)


# ---- exact mode with transcendental objectives: 1e-10 over 50 iterations ---
def nll_starts(n, seed=11):
    """Starts within +-20% of the generating parameters, `a` normalised to
    the toy's event count (a fit's usual starting region)."""
    x, k, _ = O.dijet_toy()
    lam = (1 - x) ** 10 / x ** (5 + 0.1 * np.log(x))
    a0 = k.sum() / lam.sum()
    rng = np.random.default_rng(seed)
    return np.column_stack([a0 * rng.uniform(0.8, 1.2, n), rng.uniform(8, 12, n),
                            rng.uniform(4, 6, n), rng.uniform(0.08, 0.12, n)])


# Measured floor of runs whose 50 exact-mode iterates stay within 1e-10 of the
# reference's: CUDA's cos/exp/log/pow/lgamma differ from glibc's by an ulp now
# and then, and a line-search decision taken on f values that differ in the
# last bit sends the two trajectories apart.  Rounding alone does as much:
# the oracle built with FMA contraction (same libm, only the rounding of
# a*b+c differs) keeps 19% of these NLL runs and 56% of the Rastrigin-10
# runs within 1e-10 of the plain oracle (tests/test_rounding_sensitivity.py).
# On the same libm the exact mode equals the reference's own kernel bit for
# bit on these objectives (tests/test_gpu_reference_gpu_build.py).
MIN_WITHIN = {RAS: 0.75, ACK: 0.75, NLL: 0.25}


@pytest.mark.parametrize("kind,dim,n", [(RAS, 10, 32), (ACK, 30, 8), (RAS, 2, 64),
                                        (ACK, 2, 64), (NLL, 4, 16)])
def test_exact_mode_iterates_within_1e10(cuda, kind, dim, n):
    obj, data, idata = make_obj(kind, dim)
    if kind == NLL:
        st = nll_starts(n)
        lo, hi = 0.0, 10.0
    else:
        lo, hi = BOUNDS[kind]
        st = O.oracle_starts(7, n, dim, lo, hi)
    want = O.oracle_bfgs(kind, dim, st, max_iter=50, data=data, idata=idata, traj=True,
                         lower=lo, upper=hi)
    got = gpu_run(obj, st, max_iter=50, mode="exact", gradient="dual", traj=True)
    rel = rel_iterate_error(got["traj_x"], want["traj_x"])
    worst = np.nanmax(rel, axis=0)
    ok = worst <= 1e-10
    frac = ok.mean()
    print(f"kind {kind} dim {dim}: {ok.sum()}/{n} runs within 1e-10 over 50 iterations; "
          f"worst {np.nanmax(worst):.2e}")
    assert frac >= MIN_WITHIN[kind], f"only {frac:.0%} of runs within 1e-10"


# ---- fast mode: final results --------------------------------------------
@pytest.mark.parametrize("kind,dim,n,grad", [
    (ROS, 2, 512, "dual"), (ROS, 2, 512, "adjoint"), (ROS, 8, 64, "adjoint"),
    (RAS, 10, 64, "adjoint"), (GAU, 8, 32, "adjoint"), (RAS, 2, 256, "dual"),
])
def test_fast_mode_final_results(cuda, kind, dim, n, grad):
    obj, data, idata = make_obj(kind, dim)
    lo, hi = BOUNDS[kind]
    st = O.oracle_starts(42, n, dim, lo, hi)
    want = O.oracle_bfgs(kind, dim, st, max_iter=3000, data=data, idata=idata, lower=lo,
                         upper=hi)
    got = gpu_run(obj, st, max_iter=3000, mode="fast", gradient=grad)
    agree = got["status"] == want["status"]
    # the reference itself agrees with its FMA-contracted build on 88-100% of
    # runs (test_oracle.py); fast mode changes the update and the libm calls
    assert agree.mean() >= 0.75, f"status agreement {agree.mean():.2%}"
    conv_g, conv_w = (got["status"] == 1).sum(), (want["status"] == 1).sum()
    assert abs(int(conv_g) - int(conv_w)) <= max(3, 0.15 * n)
    both = (got["status"] == 1) & (want["status"] == 1)
    assert both.sum() > 0
    df = np.abs(got["fval"][both] - want["fval"][both])
    assert (df <= 1e-8 + 1e-10 * np.abs(want["fval"][both])).all(), df.max()
    dx = np.abs(got["x"][both] - want["x"][both]).max()
    assert dx <= 1e-5, dx
    assert (got["gnorm"][got["status"] == 1] < 1e-8).all()


# ---- starts, PSO -----------------------------------------------------------
def test_uniform_starts_bit_identical(cuda):
    got = starts_uniform(42, 1000, 7, -5.0, 5.0).cpu().numpy()
    np.testing.assert_array_equal(got, O.oracle_starts(42, 1000, 7, -5.0, 5.0))


@pytest.mark.parametrize("kind,dim,n,iters", [(ROS, 2, 1024, 10), (ROS, 8, 777, 5),
                                              (GAU, 8, 300, 4)])
def test_pso_bit_identical(cuda, kind, dim, n, iters):
    obj, data, idata = make_obj(kind, dim)
    lo, hi = BOUNDS[kind]
    pbx, pbf, gb = pso_device(obj, 42, n, lo, hi, iters)
    torch.cuda.synchronize()
    wx, wf, wgx, wgf = O.oracle_pso(kind, dim, 42, n, lo, hi, iters, data=data)
    np.testing.assert_array_equal(pbx.cpu().numpy(), wx)
    np.testing.assert_array_equal(pbf.cpu().numpy(), wf)
    gbv = gb.cpu().numpy()
    assert gbv[0] == wgf
    np.testing.assert_array_equal(gbv[1:], wgx)


def test_pso_rastrigin_close(cuda):
    pbx, pbf, gb = pso_device(zb.Rastrigin(10), 3, 4096, -5.12, 5.12, 20)
    wx, wf, wgx, wgf = O.oracle_pso(RAS, 10, 3, 4096, -5.12, 5.12, 20)
    same = np.isclose(pbf.cpu().numpy(), wf, rtol=1e-12, atol=1e-12)
    assert same.mean() > 0.95


# ---- census / argmin -------------------------------------------------------
def test_census_matches_numpy(cuda):
    rng = np.random.default_rng(0)
    n, dim = 5000, 3
    f = rng.normal(size=n)
    f[17] = np.nan
    f[100] = f[200] = np.nanmin(f) - 1.0  # tie -> lowest index
    s = rng.integers(0, 6, n).astype(np.int32)
    x = rng.normal(size=(n, dim)) * 0.3 + 1.0
    c = census_device(torch.tensor(f).cuda(), torch.tensor(s).cuda(),
                      torch.tensor(x).cuda(), dim, known_min=np.ones(dim))
    assert c["best_idx"] == 100
    assert c["claimed"] == (s == 1).sum() and c["stopped"] == (s == 2).sum()
    assert c["surrendered"] == n - (s == 1).sum() - (s == 2).sum()
    near = np.sqrt(((x - 1) ** 2).sum(1)) < 0.5
    assert c["actual"] == (near & (s == 1)).sum()


# ---- edge cases -------------------------------------------------------------
@pytest.mark.parametrize("mode,grad", [("exact", "dual"), ("fast", "adjoint"), ("fast", "dual")])
def test_edge_cases(cuda, mode, grad):
    obj = zb.Rosenbrock(2)
    st = np.array([[3.0, -3.0], [1e200, 1e200], [0.5, 0.5]])
    r = gpu_run(obj, st, max_iter=0, mode=mode, gradient=grad)
    assert (r["status"] == 0).all() and (r["iter"] == 0).all()
    assert r["fval"][0] == O.value(ROS, 2, st[0])
    r = gpu_run(obj, st, max_iter=20, mode=mode, gradient=grad)
    assert r["status"][1] == 5
    rng = np.random.default_rng(3)
    st = rng.uniform(-2, 2, (64, 2))
    r = gpu_run(obj, st, max_iter=5000, mode=mode, gradient=grad, required=3)
    assert (r["status"] == 1).sum() >= 3 and (r["status"] == 2).sum() >= 1


# ---- the whole call with host buffers ----------------------------------------
@pytest.mark.parametrize("mode,grad", [("fast", "adjoint"), ("fast", "dual"), ("exact", "dual")])
def test_zeus_rosenbrock_end_to_end(cuda, mode, grad, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)  # Zeus appends zeus_2d_results.tsv here
    r = zb.Zeus(zb.Rosenbrock(2), -5.0, 5.0, 1024, 10000, 10, 100, "rosenbrock", 1e-8, 42,
                0, mode=mode, gradient=grad, per_run=True)
    assert r.status in (1, 2) and r.fval < 1e-10
    np.testing.assert_allclose(r.coordinates, [1.0, 1.0], atol=1e-5)
    assert r.c.claimed >= 100 and r.c.actual >= 100
    assert r.c.claimed + r.c.stopped + r.c.surrendered == 1024
    assert (r.per_run_status == 1).sum() == r.c.claimed
    assert r.per_run_fval[r.idx] == r.per_run_fval.min()
    row = (tmp_path / "zeus_2d_results.tsv").read_text().splitlines()[1].split("\t")
    assert row[0] == "rosenbrock" and int(row[14]) == r.c.claimed
    assert int(row[18]) == r.idx and float(row[24]) == pytest.approx(r.fval, abs=1e-300,
                                                                      rel=1e-5)


def test_zeus_gaussian_and_nll_end_to_end(cuda, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    r = zb.Zeus(zb.Gaussian(zb.gaussian_matrix(8)), -5.0, 5.0, 256, 1000, 10, 1000,
                "gaussian", 1e-8, 1, 0)
    assert r.status == 1 and r.fval < 1e-15
    x, k, _ = O.dijet_toy()
    r = zb.Zeus(zb.PoissonNLL(k, x), 0.0, 10.0, 256, 2000, 10, 1000, "poisson", 1e-8, 5, 0,
                mode="exact", gradient="dual")
    assert r.status in (0, 1) and np.isfinite(r.fval)


# ---- fixed-point shortcut: same final results as iterating to MAX_ITER -----
@pytest.mark.parametrize("kind,dim,n", [(ROS, 2, 256), (ROS, 8, 64), (ROS, 32, 8), (GAU, 8, 16)])
def test_exact_mode_fixed_point_shortcut_is_invisible(cuda, kind, dim, n):
    """Without trajectories the exact kernel ends a run at an exact fixed
    point; final results must still equal the oracle's, which iterates all
    MAX_ITER iterations."""
    obj, data, idata = make_obj(kind, dim)
    lo, hi = BOUNDS[kind]
    st = O.oracle_starts(9, n, dim, lo, hi)
    want = O.oracle_bfgs(kind, dim, st, max_iter=1500, data=data, idata=idata, lower=lo,
                         upper=hi)
    got = gpu_run(obj, st, max_iter=1500, mode="exact", gradient="dual")
    full = gpu_run(obj, st, max_iter=1500, mode="exact", gradient="dual",
                   flags=zb.FLAG_NO_FIXED_POINT)
    for key in ("status", "iter", "fval", "gnorm", "x"):
        np.testing.assert_array_equal(got[key], want[key], err_msg=key)
        np.testing.assert_array_equal(full[key], want[key], err_msg=key)
    assert got["counters"][:, 0].sum() <= full["counters"][:, 0].sum()


def test_fast_mode_fixed_point_matches_full_iteration(cuda):
    obj = zb.Rosenbrock(8)
    st = O.oracle_starts(4, 128, 8, -5.0, 5.0)
    a = gpu_run(obj, st, max_iter=4000, mode="fast", gradient="adjoint")
    b = gpu_run(obj, st, max_iter=4000, mode="fast", gradient="adjoint",
                flags=zb.FLAG_NO_FIXED_POINT)
    for key in ("status", "iter", "fval", "gnorm", "x"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)
    assert a["counters"][:, 0].sum() < b["counters"][:, 0].sum()


# ---- tile and CTA layouts ----------------------------------------------------
def _check_final(got, want, min_agree=0.75, dx_tol=1e-5):
    agree = got["status"] == want["status"]
    assert agree.mean() >= min_agree, f"status agreement {agree.mean():.2%}"
    both = (got["status"] == 1) & (want["status"] == 1)
    if both.sum() == 0:
        return
    df = np.abs(got["fval"][both] - want["fval"][both])
    assert (df <= 1e-8 + 1e-10 * np.abs(want["fval"][both])).all(), df.max()
    dx = np.abs(got["x"][both] - want["x"][both]).max()
    assert dx <= dx_tol, dx


@pytest.mark.parametrize("kind,dim,tile,n", [
    (ROS, 8, 2, 96), (ROS, 8, 4, 96), (ROS, 8, 8, 96), (ROS, 16, 8, 48), (ROS, 32, 32, 16),
    (ROS, 32, 16, 16), (RAS, 10, 4, 64), (RAS, 10, 16, 64), (ACK, 30, 32, 32),
    (GAU, 32, 32, 16), (GAU, 8, 8, 32), (ROS, 4, 2, 64), (ROS, 2, 2, 128),
])
@pytest.mark.parametrize("grad", ["adjoint", "dual"])
def test_tile_layout_final_results(cuda, kind, dim, tile, n, grad):
    obj, data, idata = make_obj(kind, dim)
    lo, hi = BOUNDS[kind]
    st = O.oracle_starts(21, n, dim, lo, hi)
    want = O.oracle_bfgs(kind, dim, st, max_iter=2000, data=data, idata=idata, lower=lo,
                         upper=hi)
    got = gpu_run(obj, st, max_iter=2000, mode="fast", gradient=grad,
                  layout=zb.LAYOUT_TILE, tile=tile)
    _check_final(got, want)


def test_tile_layout_nll(cuda):
    obj, x, k = make_obj(NLL, 4)
    rng = np.random.default_rng(2)
    lam = (1 - x) ** 10 / x ** (5 + 0.1 * np.log(x))
    a0 = k.sum() / lam.sum()
    st = np.column_stack([a0 * rng.uniform(0.8, 1.2, 32), rng.uniform(9, 11, 32),
                          rng.uniform(4.5, 5.5, 32), rng.uniform(0.08, 0.12, 32)])
    want = O.oracle_bfgs(NLL, 4, st, max_iter=3000, data=x, idata=k, lower=0, upper=10)
    best = np.nanmin(want["fval"])
    for tile in (2, 4, 8):
        for grad in ("adjoint", "dual"):
            got = gpu_run(obj, st, max_iter=3000, mode="fast", gradient=grad,
                          layout=zb.LAYOUT_TILE, tile=tile)
            both = (got["status"] == 1) & (want["status"] == 1)
            np.testing.assert_allclose(got["fval"][both], want["fval"][both], rtol=1e-9)
            # the fit's minimum is found
            assert np.nanmin(got["fval"]) == pytest.approx(best, rel=1e-9)


@pytest.mark.parametrize("kind,dim,n", [(ROS, 64, 16), (ROS, 128, 2), (GAU, 150, 2)])
@pytest.mark.parametrize("grad", ["adjoint", "dual"])
def test_cta_layout_final_results(cuda, kind, dim, n, grad):
    obj, data, idata = make_obj(kind, dim)
    lo, hi = BOUNDS[kind]
    st = O.oracle_starts(13, n, dim, lo, hi)
    iters = 600 if dim == 128 else 1500
    want = O.oracle_bfgs(kind, dim, st, max_iter=iters, data=data, idata=idata, lower=lo,
                         upper=hi)
    got = gpu_run(obj, st, max_iter=iters, mode="fast", gradient=grad,
                  layout=zb.LAYOUT_CTA)
    _check_final(got, want, min_agree=0.5 if dim == 128 else 0.75, dx_tol=1e-4)
    if kind == GAU:
        assert (got["status"] == 1).all()
        assert np.abs(got["x"]).max() < 1e-9


@pytest.mark.parametrize("kind,dim", [(ROS, 2), (ROS, 4), (ROS, 8), (ROS, 10), (ROS, 16),
                                      (ROS, 32), (ROS, 64), (ROS, 128), (RAS, 2), (RAS, 10),
                                      (RAS, 16), (ACK, 2), (ACK, 10), (ACK, 30), (GAU, 2),
                                      (GAU, 8), (GAU, 32), (GAU, 150)])
def test_auto_layout_runs_everywhere(cuda, kind, dim):
    obj, data, idata = make_obj(kind, dim)
    lo, hi = BOUNDS[kind]
    st = O.oracle_starts(5, 40, dim, lo, hi)
    for grad in ("adjoint", "dual"):
        got = gpu_run(obj, st, max_iter=50, mode="fast", gradient=grad)
        assert set(np.unique(got["status"])) <= {0, 1, 5}
        assert np.isfinite(got["fval"]).all()
        # f(x_out) is the reported fval
        for i in range(0, 40, 13):
            assert got["fval"][i] == pytest.approx(O.value(kind, dim, got["x"][i], data),
                                                   rel=1e-12, abs=1e-12)
