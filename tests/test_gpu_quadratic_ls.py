"""The Gaussian's line search in the CTA layout: f(x + a p) = f(x) +
a grad f(x).p + a^2 f(p) for the quadratic form 0.5 x^T C x.  For symmetric
C one pass over C per iteration forms C x and C p, decides every trial on
the model and carries f and g = C x + a C p to the accepted point (exact f
and g confirm convergence); otherwise f(p) is evaluated once and then only
the trial the model accepts, instead of one pass over C per trial.
Checked against the oracle (the reference's algorithm, every trial
evaluated) on final results and iteration counts, for a symmetric and a
non-symmetric C, and on the evaluation counters."""
import numpy as np
import pytest
import torch

import zeus_b200 as zb
from zeus_b200.device import bfgs_device
from tests import _oracle as O

pytestmark = pytest.mark.gpu


def _run(C, st, max_iter):
    r = bfgs_device(zb.Gaussian(C), torch.from_numpy(st).cuda(), max_iter=max_iter,
                    layout=zb.LAYOUT_CTA)
    torch.cuda.synchronize()
    return dict(status=r.status.cpu().numpy(), fval=r.fval.cpu().numpy(),
                iter=r.iter.cpu().numpy(), x=r.x.cpu().numpy(),
                counters=r.counters.cpu().numpy())


@pytest.mark.parametrize("dim,symmetric", [(150, True), (150, False)])
def test_quadratic_line_search_matches_the_oracle(cuda, dim, symmetric):
    if symmetric:
        C = zb.gaussian_matrix(dim)
    else:
        rng = np.random.default_rng(dim)
        C = np.diag(np.full(dim, float(dim))) + rng.uniform(-0.5, 0.5, (dim, dim))
    n = 64
    st = O.oracle_starts(17, n, dim, -5.0, 5.0)
    want = O.oracle_bfgs(3, dim, st, max_iter=2000, data=C, lower=-5.0, upper=5.0)
    got = _run(C, st, 2000)
    assert (got["status"] == 1).all() and (want["status"] == 1).all()
    assert np.abs(got["x"]).max() < 1e-9
    if not symmetric:
        # about 250 iterations a run: the line-search decisions are the
        # reference's, run for run
        assert (got["iter"] == want["iter"]).mean() >= 0.9
        assert got["iter"].mean() == pytest.approx(want["iter"].mean(), rel=0.02)
    # (the symmetric case ends at ||g|| ~ 1e-7, where f ~ 1e-17 and the
    # decisions follow rounding: the reference's own arithmetic takes 13
    # iterations on average there, FMA arithmetic with or without this
    # line search 6.6, run for run the same)
    # two evaluations an iteration, rarely more (symmetric C: C x and C p in
    # one pass; otherwise f(p) and the accepted trial), plus the start and,
    # for symmetric C, the exact f and g at the end
    it, ev = got["counters"][:, 0].sum(), got["counters"][:, 1].sum()
    assert ev <= 2.2 * it + 3 * n


def test_unaligned_matrix_takes_the_scalar_pass(cuda):
    """C 8 bytes off a 16-byte boundary: the pass reads C one double at a
    time (the pair form needs 16-byte alignment) with the same results up
    to rounding."""
    import ctypes as C_

    dim, n = 150, 32
    Cm = zb.gaussian_matrix(dim)
    st = O.oracle_starts(23, n, dim, -5.0, 5.0)
    buf = torch.empty(dim * dim + 1, dtype=torch.float64, device="cuda")
    buf[1:] = torch.from_numpy(Cm.ravel()).cuda()
    assert (buf.data_ptr() + 8) % 16 == 8
    prob = zb.Problem(zb.OBJ_GAUSSIAN, dim, buf.data_ptr() + 8, None, 0,
                      zb.PROBLEM_SYMMETRIC)
    cfg = zb.make_config(2000, n + 1, 1e-8, "fast", "adjoint", layout=zb.LAYOUT_CTA)
    L = zb.lib()
    wsz = L.zeus_bfgs_workspace_size(C_.byref(prob), C_.byref(cfg), n)
    ws = torch.empty(max(wsz, 1), dtype=torch.uint8, device="cuda")
    fval = torch.empty(n, dtype=torch.float64, device="cuda")
    status = torch.empty(n, dtype=torch.int32, device="cuda")
    x = torch.empty((n, dim), dtype=torch.float64, device="cuda")
    outs = zb.RunOutputs(fval.data_ptr(), status.data_ptr(), None, None, x.data_ptr(),
                         None, None, None, None, None)
    ctl = torch.zeros(2, dtype=torch.int32, device="cuda")
    d_st = torch.from_numpy(st).cuda()
    zb.check(L.zeus_bfgs_device(C_.byref(prob), C_.byref(cfg), d_st.data_ptr(), n,
                                C_.byref(outs), ctl.data_ptr(), ws.data_ptr(), wsz, None))
    torch.cuda.synchronize()
    aligned = _run(Cm, st, 2000)
    assert (status.cpu().numpy() == 1).all() and (aligned["status"] == 1).all()
    assert x.abs().max().item() < 1e-9
    assert fval.abs().max().item() < 1e-17
