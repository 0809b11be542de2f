"""Exact mode against the reference's own kernel on the same GPU.

oracle/_ref/libzeus_ref_gpu.so is the reference's sequential BFGS kernel
(bfgs_sequential.cuh:16-234) compiled for sm_100a from the reference sources,
launched with injected starts and trajectories on (the reference's own test
entry, test/bfgs_tests.cu:297-317).  It runs on CUDA's math library, as the
library's exact mode does, so the glibc-versus-CUDA difference that limits the
CPU oracle comparison for cos/exp/log/pow/lgamma objectives is gone: both sides
are compiled without FMA contraction and keep the reference's operation order,
and every iterate, f, gradient norm and status must agree bit for bit.

The reference's host build differs from its GPU build only in the libm; the
share of runs on which those two agree is printed beside the result (on a
B200: all runs for Rosenbrock, 0-6% for the cos/exp/log/pow/lgamma
objectives -- the whole of the difference the CPU comparison sees)."""
import numpy as np
import pytest

from tests import _oracle as O
from tests.test_gpu_parity import (ACK, BOUNDS, NLL, RAS, ROS, gpu_run, make_obj,
                                   nll_starts)

pytestmark = pytest.mark.gpu

KEYS = ("status", "iter", "fval", "gnorm", "x", "traj_x", "traj_f", "traj_g",
        "traj_status")


def _starts(kind, dim, n):
    if kind == NLL:
        return nll_starts(n), 0.0, 10.0
    lo, hi = BOUNDS[kind]
    return O.oracle_starts(7, n, dim, lo, hi), lo, hi


def _runs_equal(a, b):
    """Per run: every trajectory entry and final value equal (NaN == NaN)."""
    ok = np.ones(a["status"].shape[0], bool)
    for k in KEYS:
        x, y = np.asarray(a[k]), np.asarray(b[k])
        if k.startswith("traj"):
            run_axis = x.ndim - 1  # [iter][dim][run] or [iter][run]
            eq = (x == y) | (np.isnan(x) & np.isnan(y)) if x.dtype.kind == "f" else x == y
            ok &= eq.reshape(-1, x.shape[run_axis]).all(axis=0)
        else:
            eq = (x == y) | (np.isnan(x) & np.isnan(y)) if x.dtype.kind == "f" else x == y
            ok &= eq.reshape(x.shape[0], -1).all(axis=1)
    return ok


@pytest.fixture(scope="module")
def ref_gpu():
    if not O.ref_gpu_available():
        pytest.skip("oracle/_ref/libzeus_ref_gpu.so not built (needs the reference sources)")
    return O.ref_gpu_bfgs


@pytest.mark.parametrize("kind,dim,n,iters", [
    (ROS, 8, 32, 200), (RAS, 2, 64, 50), (RAS, 10, 32, 50), (ACK, 2, 64, 50),
    (ACK, 30, 8, 50), (NLL, 4, 16, 50),
])
def test_exact_mode_equals_reference_kernel(cuda, ref_gpu, kind, dim, n, iters):
    obj, data, idata = make_obj(kind, dim)
    st, lo, hi = _starts(kind, dim, n)
    want = ref_gpu(kind, dim, st, max_iter=iters, data=data, idata=idata, traj=True,
                   lower=lo, upper=hi)
    got = gpu_run(obj, st, max_iter=iters, mode="exact", gradient="dual", traj=True)
    same = _runs_equal(got, want)
    host = O.ref_bfgs(kind, dim, st, max_iter=iters, data=data, idata=idata, traj=True,
                      lower=lo, upper=hi) if O.ref_available() else None
    libm = f"{_runs_equal(host, want).mean():.0%}" if host is not None else "n/a"
    print(f"\nkind {kind} dim {dim}: {same.sum()}/{n} runs bit-identical to the "
          f"reference kernel; reference host build (glibc) vs kernel: {libm}")
    for k in KEYS:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
