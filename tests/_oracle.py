"""ctypes access to the checkers: the C restatement (oracle/libzeus_oracle.so)
and the reference's own sequential BFGS compiled for the host
(oracle/_ref/libzeus_ref.so) and for the GPU (oracle/_ref/libzeus_ref_gpu.so).
Test infrastructure only."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
ORACLE_SO = ROOT / "oracle" / "libzeus_oracle.so"
ORACLE_FMA_SO = ROOT / "oracle" / "libzeus_oracle_fma.so"
REF_SO = ROOT / "oracle" / "_ref" / "libzeus_ref.so"
REF_GPU_SO = ROOT / "oracle" / "_ref" / "libzeus_ref_gpu.so"

_P = C.c_void_p
_BFGS_SIG = [C.c_int, C.c_int, _P, _P, C.c_int, _P, C.c_int, C.c_double, C.c_double,
             C.c_int, C.c_int, C.c_double, _P, _P, _P, _P, _P, _P, _P, _P, _P, C.c_int]


class ZorObjective(C.Structure):
    _fields_ = [("kind", C.c_int), ("dim", C.c_int), ("data", _P), ("idata", _P),
                ("ndata", C.c_int)]


_oracle = None
_ref = None


def oracle():
    global _oracle
    if _oracle is None:
        L = C.CDLL(str(ORACLE_SO))
        L.zor_bfgs.argtypes = _BFGS_SIG
        L.zor_value.restype = C.c_double
        L.zor_value.argtypes = [C.POINTER(ZorObjective), _P]
        L.zor_value_grad_dual.restype = C.c_double
        L.zor_value_grad_dual.argtypes = [C.POINTER(ZorObjective), _P, _P]
        L.zor_value_grad_analytic.restype = C.c_double
        L.zor_value_grad_analytic.argtypes = [C.POINTER(ZorObjective), _P, _P]
        L.zor_digamma.restype = C.c_double
        L.zor_digamma.argtypes = [C.c_double]
        L.zor_line_search.restype = C.c_double
        L.zor_line_search.argtypes = [C.POINTER(ZorObjective), C.c_double, _P, _P, _P]
        L.zor_bfgs_update.argtypes = [C.c_int, _P, _P, _P, C.c_double]
        L.zor_uniform.restype = C.c_double
        L.zor_uniform.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32]
        L.zor_uniform_starts.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_double,
                                         C.c_double, _P]
        L.zor_philox4x32_10.argtypes = [_P, _P, _P]
        L.zor_pso.argtypes = [C.POINTER(ZorObjective), C.c_uint64, C.c_int, C.c_double,
                              C.c_double, C.c_int, C.c_double, C.c_double, C.c_double,
                              _P, _P, _P, _P]
        L.zor_pso_step.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, _P, _P,
                                   _P, _P, _P, _P]
        L.zor_pso_sobol.argtypes = [C.POINTER(ZorObjective), C.c_uint64, _P, C.c_int,
                                    C.c_double, C.c_double, C.c_int, C.c_double,
                                    C.c_double, C.c_double, _P, _P, _P, _P]
        L.zor_sobol_directions.argtypes = [C.c_int, _P, _P, C.c_int, _P]
        L.zor_sobol_params.argtypes = [C.c_int, _P, _P, C.c_int]
        L.zor_sobol01.restype = C.c_double
        L.zor_sobol01.argtypes = [_P, C.c_uint64, C.c_uint64, C.c_uint32]
        L.zor_starts.argtypes = [C.c_uint64, _P, C.c_int, C.c_int, C.c_double,
                                 C.c_double, _P]
        _oracle = L
    return _oracle


_oracle_fma = None


def oracle_fma_bfgs(*a, **k):
    """The oracle compiled with FMA contraction (the reference's algorithm
    under an FMA-contracting compiler)."""
    global _oracle_fma
    if _oracle_fma is None:
        L = C.CDLL(str(ORACLE_FMA_SO))
        L.zor_bfgs.argtypes = _BFGS_SIG
        _oracle_fma = L
    return run_bfgs(_oracle_fma.zor_bfgs, *a, **k)


def ref_available() -> bool:
    return REF_SO.exists()


def ref():
    global _ref
    if _ref is None:
        L = C.CDLL(str(REF_SO))
        L.zref_bfgs.argtypes = _BFGS_SIG
        L.zref_linesearch_quadratic.restype = C.c_double
        L.zref_linesearch_quadratic.argtypes = [C.c_double] * 4
        L.zref_bfgs_update.argtypes = [C.c_int, _P, _P, _P, C.c_double]
        L.zref_digamma.restype = C.c_double
        L.zref_digamma.argtypes = [C.c_double]
        L.zref_value_grad.restype = C.c_double
        L.zref_value_grad.argtypes = [C.c_int, C.c_int, _P, _P]
        L.zref_value_grad_data.restype = C.c_double
        L.zref_value_grad_data.argtypes = [C.c_int, C.c_int, _P, _P, C.c_int, _P, _P]
        _ref = L
    return _ref


def _p(a):
    return None if a is None else a.ctypes.data


def zobj(kind, dim, data=None, idata=None):
    nd = 0 if idata is None else len(idata)
    return ZorObjective(kind, dim, _p(data), _p(idata), nd)


def run_bfgs(fn, kind, dim, starts, max_iter=1000, required=None, tol=1e-8,
             data=None, idata=None, traj=False, lower=-5.0, upper=5.0, nthreads=1):
    """Calls zor_bfgs / zref_bfgs; returns dict of numpy arrays."""
    starts = np.ascontiguousarray(starts, dtype=np.float64)
    n = starts.shape[0]
    if required is None:
        required = n + 1
    out = dict(fval=np.zeros(n), status=np.zeros(n, np.int32), iter=np.zeros(n, np.int32),
               gnorm=np.zeros(n), x=np.zeros((n, dim)))
    tx = tf = tg = ts = None
    if traj:
        tx = np.full((max_iter, dim, n), np.nan)
        tf = np.full((max_iter, n), np.nan)
        tg = np.full((max_iter, n), np.nan)
        ts = np.full((max_iter, n), -1, np.int8)
    nd = 0 if idata is None else len(idata)
    rc = fn(kind, dim, _p(data), _p(idata), nd, _p(starts), n, lower, upper, max_iter,
            required, tol, _p(out["fval"]), _p(out["status"]), _p(out["iter"]),
            _p(out["gnorm"]), _p(out["x"]), _p(tx), _p(tf), _p(tg), _p(ts), nthreads)
    assert rc == 0, f"bfgs returned {rc}"
    if traj:
        out.update(traj_x=tx, traj_f=tf, traj_g=tg, traj_status=ts)
    return out


def oracle_bfgs(*a, **k):
    return run_bfgs(oracle().zor_bfgs, *a, **k)


def ref_bfgs(*a, **k):
    return run_bfgs(ref().zref_bfgs, *a, **k)


_ref_gpu = None


def ref_gpu_available() -> bool:
    return REF_GPU_SO.exists()


def ref_gpu_bfgs(*a, **k):
    """The reference's sequential BFGS kernel run on the GPU (cuda:0), same
    arguments and results as ref_bfgs."""
    global _ref_gpu
    if _ref_gpu is None:
        L = C.CDLL(str(REF_GPU_SO))
        L.zrefg_bfgs.argtypes = _BFGS_SIG
        _ref_gpu = L
    return run_bfgs(_ref_gpu.zrefg_bfgs, *a, **k)


PRNG_XORWOW, PRNG_PHILOX, PRNG_SOBOL = 0, 1, 2
SOBOL_MAXDEG = 16


def sobol_params(ndim):
    """The product's Sobol' polynomials and initial direction numbers."""
    poly = np.zeros(ndim, dtype=np.uint32)
    minit = np.zeros((ndim, SOBOL_MAXDEG), dtype=np.uint32)
    assert oracle().zor_sobol_params(ndim, _p(poly), _p(minit), SOBOL_MAXDEG) == 0
    return poly, minit


def sobol_directions(ndim, poly=None, minit=None):
    """dirs[d, k] = v_(k+1) of dimension d (32-bit fractions)."""
    if poly is None:
        poly, minit = sobol_params(ndim)
    poly = np.ascontiguousarray(poly, dtype=np.uint32)
    minit = np.ascontiguousarray(minit, dtype=np.uint32)
    dirs = np.zeros((ndim, 32), dtype=np.uint32)
    oracle().zor_sobol_directions(ndim, _p(poly), _p(minit), minit.shape[1], _p(dirs))
    return dirs


_SOBOL_DIRS = {}


def _sobol_table(prng, dim):
    if prng != PRNG_SOBOL:
        return None
    if dim not in _SOBOL_DIRS:
        _SOBOL_DIRS[dim] = sobol_directions(dim)
    return _SOBOL_DIRS[dim]


def oracle_starts(seed, n, dim, lower, upper, prng=PRNG_PHILOX):
    out = np.zeros((n, dim))
    dirs = _sobol_table(prng, dim)
    oracle().zor_starts(seed, None if dirs is None else _p(dirs), n, dim, lower, upper,
                        _p(out))
    return out


def oracle_pso(kind, dim, seed, n, lower, upper, iters, w=0.5, c1=1.2, c2=1.5,
               data=None, idata=None, prng=PRNG_PHILOX):
    o = zobj(kind, dim, data, idata)
    pbx = np.zeros((n, dim))
    pbf = np.zeros(n)
    gbx = np.zeros(dim)
    gbf = np.zeros(1)
    dirs = _sobol_table(prng, dim)
    oracle().zor_pso_sobol(C.byref(o), seed, None if dirs is None else _p(dirs), n,
                           lower, upper, iters, w, c1, c2, _p(pbx), _p(pbf), _p(gbx),
                           _p(gbf))
    return pbx, pbf, gbx, gbf[0]


def value(kind, dim, x, data=None, idata=None):
    o = zobj(kind, dim, data, idata)
    x = np.ascontiguousarray(x, dtype=np.float64)
    return oracle().zor_value(C.byref(o), _p(x))


def grad_dual(kind, dim, x, data=None, idata=None):
    o = zobj(kind, dim, data, idata)
    x = np.ascontiguousarray(x, dtype=np.float64)
    g = np.zeros(dim)
    f = oracle().zor_value_grad_dual(C.byref(o), _p(x), _p(g))
    return f, g


def ref_grad_dual(kind, dim, x, data=None, idata=None):
    """The reference's own dual::calculateGradientUsingAD
    (include/duals.cuh:241-266) from its host build: (f, grad)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    g = np.zeros(dim)
    if data is None:
        f = ref().zref_value_grad(kind, dim, _p(x), _p(g))
    else:
        data = np.ascontiguousarray(data, dtype=np.float64)
        idata = None if idata is None else np.ascontiguousarray(idata, dtype=np.int32)
        nd = 0 if idata is None else len(idata)
        f = ref().zref_value_grad_data(kind, dim, _p(data), _p(idata), nd, _p(x), _p(g))
    return f, g


def grad_analytic(kind, dim, x, data=None, idata=None):
    o = zobj(kind, dim, data, idata)
    x = np.ascontiguousarray(x, dtype=np.float64)
    g = np.zeros(dim)
    f = oracle().zor_value_grad_analytic(C.byref(o), _p(x), _p(g))
    return f, g


def dijet_toy(seed=7, nbins=100, total=1e6, p=(1e6, 10.0, 5.0, 0.1)):
    """Synthetic binned dijet spectrum: 100 log-spaced bins in x = m/13000
    over [0.085, 0.54], lambda_i = p0 (1-x)^p1 / x^(p2 + p3 ln x) at bin
    centres rescaled to `total` events, counts ~ Poisson(lambda)."""
    edges = np.geomspace(0.085, 0.54, nbins + 1)
    x = 0.5 * (edges[1:] + edges[:-1])
    lam = p[0] * (1 - x) ** p[1] / x ** (p[2] + p[3] * np.log(x))
    lam *= total / lam.sum()
    rng = np.random.default_rng(seed)
    k = rng.poisson(lam).astype(np.int32)
    return x, k, lam


# ------------------------------------------------------------------ dijet fits
# The implicit-function adjoint of the binned Poisson fit has no counterpart
# in the reference (its dijet example stops at the minimum,
# examples/fit_dijet_spectrum.cu:162-221); these numpy functions are the
# checker for it: NLL = sum_i lambda_i - k_i ln lambda_i (+ const) with
# ln lambda = ln a + b ln(1-x) - (c + d ln x) ln x.
def nll_parts(x, k, p):
    """(lambda, J = d ln lambda / dp (4, nbins), gradient, exact Hessian)."""
    a, b, c, d = p
    lx, l1 = np.log(x), np.log1p(-x)
    lam = np.exp(np.log(a) + b * l1 - (c + d * lx) * lx)
    J = np.stack([np.full_like(x, 1.0 / a), l1, -lx, -lx * lx])
    r = lam - k
    grad = J @ r
    H = (J * lam) @ J.T
    H[0, 0] -= r.sum() / (a * a)
    return lam, J, grad, H


def nll_value(x, k, p):
    a, b, c, d = p
    lx, l1 = np.log(x), np.log1p(-x)
    ll = np.log(a) + b * l1 - (c + d * lx) * lx
    return float(np.sum(np.exp(ll) - k * ll))


def nll_newton_fit(x, k, p0, iters=100):
    """The fit by Newton's method in theta = (ln a, b, c, d), where ln lambda
    is linear in theta (a Poisson log-linear model: the NLL is convex and its
    Hessian sum lambda J J^T positive definite), with step halving; returns
    p = (a, b, c, d)."""
    lx, l1 = np.log(x), np.log1p(-x)
    Jt = np.stack([np.ones_like(x), l1, -lx, -lx * lx])
    k = np.asarray(k, dtype=np.float64)

    def f(t):
        ll = t @ Jt
        return float(np.sum(np.exp(ll) - k * ll))

    t = np.array([np.log(p0[0]), p0[1], p0[2], p0[3]], dtype=np.float64)
    fv = f(t)
    for _ in range(iters):
        lam = np.exp(t @ Jt)
        step = np.linalg.solve((Jt * lam) @ Jt.T, Jt @ (lam - k))
        h = 1.0
        while h > 1e-8 and f(t - h * step) > fv:
            h *= 0.5
        t_new = t - h * step
        f_new = f(t_new)
        done = f_new >= fv and h < 1.0
        if f_new <= fv:
            t, fv = t_new, f_new
        if done or np.all(np.abs(h * step) <= 1e-15 * np.maximum(np.abs(t), 1.0)):
            break
    return np.array([np.exp(t[0]), t[1], t[2], t[3]])


def nll_sensitivity(x, k, p):
    """d p_hat / d k_j = H^-1 J_j for every bin j, shape (4, nbins)."""
    _, J, _, H = nll_parts(x, k, p)
    return np.linalg.solve(H, J)
