"""Sobol' start positions on the GPU (ZEUS_PRNG_SOBOL) against the oracle,
through the C ABI.  Positions are integer work plus one multiply-add
computed without contraction on both sides, so they must agree bit for bit;
PSO values follow the existing PSO parity rules (bit-identical for the
per-thread kernels, 1e-12 relative where the GPU reduces f cooperatively)."""
import ctypes as C

import numpy as np
import pytest
import torch

import zeus_b200 as zb
from zeus_b200.device import bfgs_device, pso_device, starts
from tests import _oracle as O

pytestmark = pytest.mark.gpu

SOBOL = zb.PRNG_SOBOL


class _DeviceArray:
    """A uint32 device array at a raw address, for torch.as_tensor."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": "<u4",
                                         "data": (ptr, False), "version": 3}


@pytest.mark.parametrize("seed,n,dim,lo,hi", [(42, 1000, 7, -5.0, 5.0),
                                              (7, 300, 150, -5.12, 5.12),
                                              (9, 33, 1024, -1.0, 1.0),
                                              (3, 1, 1, 0.0, 1.0)])
def test_sobol_starts_bit_identical(cuda, seed, n, dim, lo, hi):
    got = starts(seed, n, dim, lo, hi, prng=SOBOL).cpu().numpy()
    np.testing.assert_array_equal(got, O.oracle_starts(seed, n, dim, lo, hi,
                                                       prng=O.PRNG_SOBOL))


def test_generator_choice_and_errors(cuda):
    a = starts(5, 64, 4, 0.0, 1.0, prng="philox").cpu().numpy()
    np.testing.assert_array_equal(a, starts(5, 64, 4, 0.0, 1.0, prng="xorwow").cpu().numpy())
    np.testing.assert_array_equal(a, O.oracle_starts(5, 64, 4, 0.0, 1.0))
    assert starts(5, 0, 4, 0.0, 1.0, prng=SOBOL).shape == (0, 4)
    out = torch.empty(8, dtype=torch.float64, device="cuda")
    assert zb.lib().zeus_starts(1, 3, 2, 4, 0.0, 1.0, out.data_ptr(), None) == zb.E_INVALID
    big = torch.empty(1025, dtype=torch.float64, device="cuda")
    assert zb.lib().zeus_starts(1, SOBOL, 1, 1025, 0.0, 1.0, big.data_ptr(),
                                None) == zb.E_UNSUPPORTED
    p = C.c_void_p()
    assert zb.lib().zeus_sobol_device_table(C.byref(p)) == zb.OK and p.value
    table = torch.as_tensor(_DeviceArray(p.value, (1024, 32)), device="cuda")
    np.testing.assert_array_equal(table.cpu().numpy(), O.sobol_directions(1024))


@pytest.mark.parametrize("kind,dim,n,iters", [(0, 2, 1024, 10), (0, 8, 777, 5),
                                              (3, 8, 300, 4)])
def test_sobol_pso_bit_identical(cuda, kind, dim, n, iters):
    data = zb.gaussian_matrix(dim) if kind == 3 else None
    obj = zb.Gaussian(data) if kind == 3 else zb.Rosenbrock(dim)
    pbx, pbf, gb = pso_device(obj, 42, n, -5.0, 5.0, iters, prng=SOBOL)
    torch.cuda.synchronize()
    wx, wf, wgx, wgf = O.oracle_pso(kind, dim, 42, n, -5.0, 5.0, iters, data=data,
                                    prng=O.PRNG_SOBOL)
    np.testing.assert_array_equal(pbx.cpu().numpy(), wx)
    np.testing.assert_array_equal(pbf.cpu().numpy(), wf)
    gbv = gb.cpu().numpy()
    assert gbv[0] == wgf
    np.testing.assert_array_equal(gbv[1:], wgx)


@pytest.mark.parametrize("kind,dim", [(0, 64), (3, 150)])  # warp-cooperative, DMMA
def test_sobol_initial_swarm_of_the_wide_kernels(cuda, kind, dim):
    data = zb.gaussian_matrix(dim) if kind == 3 else None
    obj = zb.Gaussian(data) if kind == 3 else zb.Rosenbrock(dim)
    pbx, pbf, gb = pso_device(obj, 11, 200, -5.0, 5.0, 0, prng=SOBOL)
    wx, wf, _, wgf = O.oracle_pso(kind, dim, 11, 200, -5.0, 5.0, 0, data=data,
                                  prng=O.PRNG_SOBOL)
    np.testing.assert_array_equal(pbx.cpu().numpy(), wx)
    np.testing.assert_allclose(pbf.cpu().numpy(), wf, rtol=1e-12)
    assert gb.cpu().numpy()[0] == pytest.approx(wgf, rel=1e-12)


def test_zeus_passes_the_generator_through(cuda, tmp_path, monkeypatch):
    """zeus_optimize with config.prng = SOBOL and PSO off runs the BFGS from
    the oracle's Sobol' starts: per-run results equal a direct BFGS launch
    on those starts."""
    monkeypatch.chdir(tmp_path)
    n = 512
    r = zb.Zeus(zb.Rosenbrock(8), -5.0, 5.0, n, 3000, -1, n + 1, "rosenbrock", 1e-8, 21,
                0, prng=zb.PRNGType.SOBOL, per_run=True)
    st = torch.from_numpy(O.oracle_starts(21, n, 8, -5.0, 5.0, prng=O.PRNG_SOBOL)).cuda()
    d = bfgs_device(zb.Rosenbrock(8), st, max_iter=3000, required=n + 1)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(r.per_run_status, d.status.cpu().numpy())
    np.testing.assert_array_equal(r.per_run_fval, d.fval.cpu().numpy())
    rp = zb.Zeus(zb.Rosenbrock(8), -5.0, 5.0, n, 3000, -1, n + 1, "rosenbrock", 1e-8, 21,
                 0, per_run=True)
    assert not np.array_equal(rp.per_run_fval, r.per_run_fval)
    rs = zb.Zeus(zb.Rosenbrock(2), -5.0, 5.0, 1024, 10000, 10, 100, "rosenbrock", 1e-8,
                 42, 0, prng="sobol")
    assert rs.status in (1, 2) and rs.fval < 1e-10
