"""The CTA layout past D = 160: H (D*D doubles, 512 KB at D = 256) no longer
fits in shared memory and each block keeps it in its slice of the caller's
workspace; checked against the oracle (the reference algorithm) on
Rosenbrock-256 at the fast-mode tolerances."""
import ctypes as C

import numpy as np
import pytest
import torch

import zeus_b200 as zb
from zeus_b200.device import bfgs_device
from tests import _oracle as O

pytestmark = pytest.mark.gpu


def test_rosenbrock256_global_h_matches_oracle(cuda):
    """Both descend to the 256-D minimum from the same starts; near it the
    gradient norm of Rosenbrock-256 floors around 1e-5 in FP64 (the oracle
    too), so the runs end at MAX_ITER and are compared on f and x."""
    rng = np.random.default_rng(8)
    n, d, iters = 2, 256, 200
    st = 1.0 + 0.05 * rng.standard_normal((n, d))
    r = bfgs_device(zb.Rosenbrock(d), torch.tensor(st).cuda(), max_iter=iters, tol=1e-8,
                    layout=zb.LAYOUT_CTA)
    torch.cuda.synchronize()
    assert r.wsz >= 8 * d * d * n  # one H slice per block
    o = O.oracle_bfgs(0, d, st, max_iter=iters)
    f0 = np.array([O.value(0, d, x) for x in st])
    got_f, got_x = r.fval.cpu().numpy(), r.x.cpu().numpy()
    assert (o["fval"] < 1e-7).all() and (got_f < 1e-7).all()
    assert (got_f < 1e-7 * f0).all()
    np.testing.assert_allclose(got_x, o["x"], atol=1e-3)
    np.testing.assert_allclose(got_x, 1.0, atol=1e-3)
    assert set(r.status.cpu().numpy()) <= {0, 1}


def test_global_h_rejects_a_short_workspace(cuda):
    d, n = 256, 4
    st = torch.ones((n, d), dtype=torch.float64, device="cuda")
    cfg = zb.make_config(100, n + 1, 1e-8, "fast", "adjoint", layout=zb.LAYOUT_CTA)
    prob = zb.Problem(zb.OBJ_ROSENBROCK, d, None, None, 0, 0)
    L = zb.lib()
    need = L.zeus_bfgs_workspace_size(C.byref(prob), C.byref(cfg), n)
    assert need == 256 + 8 * d * d * n  # the run queue, then one H slice per block
    out = torch.empty((n,), dtype=torch.float64, device="cuda")
    ws = torch.empty((need // 2,), dtype=torch.uint8, device="cuda")
    outs = zb.RunOutputs(out.data_ptr(), None, None, None, None, None, None, None, None, None)
    ctl = torch.zeros((2,), dtype=torch.int32, device="cuda")
    rc = L.zeus_bfgs_device(C.byref(prob), C.byref(cfg), st.data_ptr(), n, C.byref(outs),
                            ctl.data_ptr(), ws.data_ptr(), ws.numel(), None)
    assert rc == zb.E_WORKSPACE and "workspace" in zb.last_error()
