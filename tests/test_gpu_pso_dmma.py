"""PSO on the Gaussian quadratic form (D >= 33): f = 0.5 x^T C x of 8
particles per warp on the FP64 tensor cores (mma.sync m8n8k4 f64).  The
values are checked against numpy on the same positions, and the swarm
against the oracle's PSO."""
import numpy as np
import pytest

import zeus_b200 as zb
from zeus_b200.device import pso_device
from tests import _oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [300, 7])  # a partial last warp and a single warp
def test_dmma_values_match_numpy(cuda, n):
    rng = np.random.default_rng(2)
    C = rng.standard_normal((150, 150))  # not symmetric: f uses C as given
    pbx, pbf, gb = pso_device(zb.Gaussian(C), 11, n, -5.0, 5.0, 0)
    X = pbx.cpu().numpy()
    want = 0.5 * np.einsum("ij,jk,ik->i", X, C, X)
    np.testing.assert_allclose(pbf.cpu().numpy(), want, rtol=1e-12, atol=1e-10)
    g = gb.cpu().numpy()
    k = int(np.argmin(want))
    assert g[0] == pbf.cpu().numpy()[k]
    np.testing.assert_array_equal(g[1:], X[k])


def test_dmma_swarm_matches_oracle(cuda):
    C = zb.gaussian_matrix(150)
    pbx, pbf, gb = pso_device(zb.Gaussian(C), 42, 1024, -5.0, 5.0, 10)
    wx, wf, wgx, wgf = O.oracle_pso(3, 150, 42, 1024, -5.0, 5.0, 10, data=C)
    got = pbf.cpu().numpy()
    close = np.isclose(got, wf, rtol=1e-12, atol=0)
    assert close.mean() > 0.95
    assert gb.cpu().numpy()[0] == pytest.approx(wgf, rel=1e-12)
