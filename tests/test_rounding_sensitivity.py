"""How far last-bit rounding alone moves the exact-mode trajectories that the
GPU parity test compares (tests/test_gpu_parity.py,
test_exact_mode_iterates_within_1e10): the oracle against the same oracle
compiled with FMA contraction -- the same libm and the same algorithm, only
the rounding of a*b+c differs -- over the same starts and 50 iterations.  The
share of runs that stay within 1e-10 is what the GPU's floors are set
against: the NLL's 25% floor is above what rounding alone leaves (19%), the
transcendental objectives' 75% floors are near or above it."""
import numpy as np
import pytest

from tests import _oracle as O
from tests.test_gpu_parity import (ACK, BOUNDS, MIN_WITHIN, NLL, RAS, make_obj, nll_starts,
                                   rel_iterate_error)

# (kind, dim, n): the GPU test's cases; the rounding-only share measured here
# (CPU, x86-64): Rastrigin-10 0.56, Ackley-30 0.88, Rastrigin-2 0.97,
# Ackley-2 0.97, NLL 0.19
CASES = [(RAS, 10, 32), (ACK, 30, 8), (RAS, 2, 64), (ACK, 2, 64), (NLL, 4, 16)]


def within_share(kind, dim, n):
    obj, data, idata = make_obj(kind, dim)
    if kind == NLL:
        st, lo, hi = nll_starts(n), 0.0, 10.0
    else:
        lo, hi = BOUNDS[kind]
        st = O.oracle_starts(7, n, dim, lo, hi)
    kw = dict(max_iter=50, data=data, idata=idata, traj=True, lower=lo, upper=hi)
    a = O.oracle_bfgs(kind, dim, st, **kw)
    b = O.oracle_fma_bfgs(kind, dim, st, **kw)
    worst = np.nanmax(rel_iterate_error(b["traj_x"], a["traj_x"]), axis=0)
    return float((worst <= 1e-10).mean())


@pytest.mark.parametrize("kind,dim,n", CASES)
def test_rounding_alone_moves_trajectories(kind, dim, n):
    share = within_share(kind, dim, n)
    print(f"kind {kind} dim {dim}: {share:.0%} of runs within 1e-10 under rounding alone")
    # the NLL and Rastrigin-10 trajectories leave 1e-10 under rounding alone
    # for most runs; the 2-D ones rarely do
    if (kind, dim) in ((NLL, 4), (RAS, 10)):
        assert share < 0.75
    # the GPU floor never asks for more agreement than rounding alone gives
    # plus the margin of a libm that differs in more places than FMA does
    assert MIN_WITHIN[kind] <= share + 0.25
