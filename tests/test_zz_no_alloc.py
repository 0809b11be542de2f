"""zeus_pso_device_noalloc: PSO seeding for callers that cannot allocate
device memory (their allocator belongs to another framework, or their loop
must not allocate).  It keeps the swarm state in a fixed 8 MiB array inside
the library instead of a caller-provided workspace; its results must equal
zeus_pso_device's exactly, call after call, although every call reuses the
same array.  Collected last (file name) so that a stop at its first failure
has already run everything else."""
import ctypes as C

import numpy as np
import pytest
import torch

import zeus_b200 as zb
from zeus_b200.device import DeviceProblem, pso_device

pytestmark = pytest.mark.gpu


def noalloc(dp, seed, n, lo, hi, iters):
    dim = dp.obj.dim
    pbx = torch.full((n, dim), np.nan, dtype=torch.float64, device="cuda")
    pbf = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
    gb = torch.full((dim + 1,), np.nan, dtype=torch.float64, device="cuda")
    prob = dp.c()
    rc = zb.lib().zeus_pso_device_noalloc(
        C.byref(prob), seed, n, lo, hi, iters, 0.5, 1.2, 1.5, pbx.data_ptr(),
        pbf.data_ptr(), gb.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return rc, pbx, pbf, gb


@pytest.mark.parametrize("first,second", [
    ((zb.Rosenbrock(8), 5000, -5.0, 5.0, 12, 11), (zb.Rosenbrock(2), 1024, -5.0, 5.0, 10, 42)),
    ((zb.Gaussian(zb.gaussian_matrix(32)), 3000, -5.0, 5.0, 6, 3),
     (zb.Rastrigin(10), 4096, -5.12, 5.12, 20, 7)),
])
def test_noalloc_matches_workspace_pso_twice_in_a_row(cuda, first, second):
    for obj, n, lo, hi, iters, seed in (first, second):
        dp = DeviceProblem(obj)
        rc, pbx, pbf, gb = noalloc(dp, seed, n, lo, hi, iters)
        assert rc == zb.OK, zb.last_error()
        wx, wf, wg = pso_device(dp, seed, n, lo, hi, iters)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(pbx.cpu().numpy(), wx.cpu().numpy())
        np.testing.assert_array_equal(pbf.cpu().numpy(), wf.cpu().numpy())
        np.testing.assert_array_equal(gb.cpu().numpy(), wg.cpu().numpy())


def test_noalloc_rejects_more_state_than_the_array_holds(cuda):
    dp = DeviceProblem(zb.Rosenbrock(128))
    n = 8 * 1024  # 2 * 8192 * 128 * 8 bytes of positions and velocities > 8 MiB
    rc, *_ = noalloc(dp, 1, n, -5.0, 5.0, 1)
    assert rc == zb.E_WORKSPACE
    assert "8388608" in zb.last_error()
