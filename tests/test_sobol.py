"""Sobol' start positions (the reference's PRNGType::SOBOL, traits.hpp:67-71,
in own construction) on the CPU.

The oracle's construction is pinned to scipy's Sobol' generator (Joe and
Kuo's direction numbers, installed with scipy; read at test time, not copied
into the repository):
  * the oracle's primitive polynomials, in order of degree then value, are
    scipy's polynomial list for the first 1024 dimensions;
  * the oracle's Bratley-Fox recurrence, fed scipy's initial direction
    numbers, reproduces scipy's unscrambled points bit for bit (scipy emits
    them in Gray-code order: its k-th point is natural-order point k ^ k>>1).
The library's own table (zeus_sobol_directions, host code of
libzeus_b200.so) must equal the oracle's bit for bit, and the point sets
keep the net properties every Sobol' sequence has."""
import os

import numpy as np
import pytest

import zeus_b200 as zb
from tests import _oracle as O

scipy = pytest.importorskip("scipy")
from scipy.stats import qmc  # noqa: E402


def _scipy_table():
    path = os.path.join(os.path.dirname(scipy.__file__), "stats",
                        "_sobol_direction_numbers.npz")
    if not os.path.exists(path):
        pytest.skip("scipy's Sobol' direction numbers are not installed")
    z = np.load(path)
    return z["poly"], z["vinit"]


def _points(dirs, n):
    """Unshifted natural-order points 0..n-1 as uint32, (n, ndim)."""
    k = np.arange(n, dtype=np.uint64)
    out = np.zeros((n, dirs.shape[0]), dtype=np.uint64)
    for b in range(int(n - 1).bit_length()):
        sel = ((k >> np.uint64(b)) & np.uint64(1)).astype(bool)
        out[sel] ^= dirs[:, b].astype(np.uint64)
    return out


def test_polynomials_are_the_standard_order():
    poly, _ = O.sobol_params(1024)
    ref_poly, _ = _scipy_table()
    np.testing.assert_array_equal(poly[1:], ref_poly[1:1024])


@pytest.mark.parametrize("ndim,m", [(2, 12), (40, 10), (300, 8)])
def test_recurrence_reproduces_scipy(ndim, m):
    ref_poly, ref_init = _scipy_table()
    dirs = O.sobol_directions(ndim, ref_poly[:ndim].astype(np.uint32),
                              ref_init[:ndim].astype(np.uint32))
    n = 1 << m
    got = _points(dirs, n)
    want = (qmc.Sobol(ndim, scramble=False, bits=32).random(n) * 2.0 ** 32).astype(np.uint64)
    k = np.arange(n)
    np.testing.assert_array_equal(got[k ^ (k >> 1)], want)


def test_library_table_equals_the_oracle():
    np.testing.assert_array_equal(zb.sobol_directions(1024), O.sobol_directions(1024))
    np.testing.assert_array_equal(zb.sobol_directions(3), O.sobol_directions(1024)[:3])


def test_initial_numbers_are_valid():
    poly, minit = O.sobol_params(1024)
    for d in range(1, 1024):
        s = int(poly[d]).bit_length() - 1
        m = minit[d, :s].astype(np.int64)
        assert (m & 1).all() and (m < (1 << np.arange(1, s + 1))).all()
        assert (minit[d, s:] == 0).all()


@pytest.mark.parametrize("seed", [42, 7])
def test_every_coordinate_is_stratified(seed):
    """Any 2^m consecutive points starting at a multiple of 2^m put one
    point in each interval [j/2^m, (j+1)/2^m) of every coordinate; the
    digital shift permutes the intervals."""
    dim, m = 64, 9
    n = 1 << m
    for start in (0, n):
        x = O.oracle_starts(seed, 2 * n, dim, 0.0, 1.0, prng=O.PRNG_SOBOL)[start:start + n]
        cells = np.floor(x * n).astype(int)
        for d in range(dim):
            assert len(np.unique(cells[:, d])) == n


def test_first_two_dimensions_form_a_net():
    """Dimensions 0 and 1 (van der Corput and x + 1) make a (0, m, 2)-net:
    every elementary interval of area 2^-m holds one of the first 2^m
    points, shifted or not."""
    m = 8
    n = 1 << m
    x = O.oracle_starts(3, n, 2, 0.0, 1.0, prng=O.PRNG_SOBOL)
    for a in range(m + 1):
        b = m - a
        cell = np.floor(x[:, 0] * (1 << a)).astype(int) * (1 << b) + \
            np.floor(x[:, 1] * (1 << b)).astype(int)
        assert len(np.unique(cell)) == n


def test_shift_depends_on_the_seed_and_points_stay_inside():
    a = O.oracle_starts(1, 256, 5, -2.0, 3.0, prng=O.PRNG_SOBOL)
    b = O.oracle_starts(2, 256, 5, -2.0, 3.0, prng=O.PRNG_SOBOL)
    assert not np.array_equal(a, b)
    assert (a > -2.0).all() and (a < 3.0).all()
    # the unshifted point 0 is the origin: shifted, it is the shift itself
    dirs = O.sobol_directions(5)
    u0 = np.array([O.oracle().zor_sobol01(dirs.ctypes.data, 1, 0, d) for d in range(5)])
    np.testing.assert_array_equal(a[0], -2.0 + 5.0 * u0)


def test_prng_names_map_to_the_abi():
    assert zb.prng_code(None) == zb.PRNG_XORWOW
    assert zb.prng_code("sobol") == zb.prng_code(zb.PRNGType.SOBOL) == zb.PRNG_SOBOL
    assert zb.prng_code(1) == zb.PRNG_PHILOX
    with pytest.raises(ValueError):
        zb.prng_code(7)
