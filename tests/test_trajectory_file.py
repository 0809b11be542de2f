"""Trajectory files (the reference's util::writeTrajectoryDataTSV,
src/utils.cu:128-176): the library's writer checked on the CPU against a
Python restatement of the reference's format, on the oracle's trajectories
of the reference algorithm."""
import math

import numpy as np
import pytest

import zeus_b200 as zb
from tests import _oracle as O


def reference_tsv(tx, tf, tg, ts, alpha=None):
    """The reference's TSV text: header, then for every run i and every step
    it: i, it, fval, grad, status, alpha, x0..; doubles in C++ scientific
    with precision 17 (printf %.17e), NaN written "NaN" for fval, grad and
    coordinates (src/utils.cu:137-171)."""
    T, D, N = tx.shape
    alpha = np.zeros((T, N)) if alpha is None else alpha
    lines = ["traj\tstep\tfval\tgrad\tstatus\talpha" + "".join(f"\tx{d}" for d in range(D))]

    def v(x):
        return "NaN" if math.isnan(x) else "%.17e" % x

    for i in range(N):
        for it in range(T):
            row = [str(i), str(it), v(tf[it, i]), v(tg[it, i]), str(int(ts[it, i])),
                   "%.17e" % alpha[it, i]]
            row += [v(tx[it, d, i]) for d in range(D)]
            lines.append("\t".join(row))
    return "\n".join(lines) + "\n"


def _write(path, tx, tf, tg, ts, alpha=None):
    arrs = [np.ascontiguousarray(a) for a in (tx, tf, tg, ts)]
    a = None if alpha is None else np.ascontiguousarray(alpha)
    return zb.lib().zeus_write_trajectory_tsv(
        str(path).encode(), arrs[0].ctypes.data, arrs[1].ctypes.data, arrs[2].ctypes.data,
        arrs[3].ctypes.data, None if a is None else a.ctypes.data, tx.shape[2], tx.shape[0],
        tx.shape[1])


@pytest.mark.parametrize("kind,dim,n,iters", [(0, 2, 6, 40), (1, 10, 3, 25)])
def test_writer_matches_reference_format_on_oracle_trajectories(tmp_path, kind, dim, n, iters):
    lo, hi = (-5.0, 5.0) if kind == 0 else (-5.12, 5.12)
    st = O.oracle_starts(42, n, dim, lo, hi)
    r = O.oracle_bfgs(kind, dim, st, max_iter=iters, traj=True, lower=lo, upper=hi)
    path = tmp_path / "traj.tsv"
    assert _write(path, r["traj_x"], r["traj_f"], r["traj_g"], r["traj_status"]) == zb.OK
    want = reference_tsv(r["traj_x"], r["traj_f"], r["traj_g"], r["traj_status"])
    assert path.read_text() == want


def test_writer_alpha_column_and_nan_tail(tmp_path):
    T, D, N = 3, 2, 2
    tx = np.full((T, D, N), np.nan)
    tx[0] = [[1.5, -2.0], [0.25, 1e-300]]
    tf = np.full((T, N), np.nan)
    tf[0] = [3.0, -0.0]
    tg = np.full((T, N), np.nan)
    tg[0] = [1e100, 2.5]
    ts = np.full((T, N), -1, np.int8)
    ts[0] = [1, 0]
    alpha = np.full((T, N), 0.5)
    path = tmp_path / "t.tsv"
    assert _write(path, tx, tf, tg, ts, alpha) == zb.OK
    text = path.read_text()
    assert text == reference_tsv(tx, tf, tg, ts, alpha)
    rows = text.splitlines()
    assert rows[1] == "0\t0\t3.00000000000000000e+00\t1.00000000000000002e+100\t1\t" \
                      "5.00000000000000000e-01\t1.50000000000000000e+00\t2.50000000000000000e-01"
    assert rows[2].split("\t")[2:4] == ["NaN", "NaN"]


def test_writer_rejects_other_extensions(tmp_path):
    z = np.zeros((1, 1, 1))
    s = np.zeros((1, 1), np.int8)
    rc = _write(tmp_path / "t.nc", z, z[0], z[0], s)
    assert rc == zb.E_UNSUPPORTED and "NetCDF" in zb.last_error()
