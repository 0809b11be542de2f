"""Trajectory files end to end on the GPU: zeus_b200.Zeus(...,
trajectory_file=...) records every iteration in exact mode and writes the
reference's TSV; for the polynomial Rosenbrock the file equals, byte for
byte, the reference format of the oracle's trajectories."""
import numpy as np
import pytest

import zeus_b200 as zb
from tests import _oracle as O
from tests.test_trajectory_file import reference_tsv

pytestmark = pytest.mark.gpu


def test_zeus_trajectory_file_equals_oracle(cuda, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    n, iters, seed = 12, 60, 42
    path = tmp_path / "rosen.tsv"
    r = zb.Zeus(zb.Rosenbrock(2), -5.0, 5.0, n, iters, -1, 1000, "rosenbrock", 1e-8, seed,
                0, trajectory_file=str(path))
    st = O.oracle_starts(seed, n, 2, -5.0, 5.0)
    o = O.oracle_bfgs(0, 2, st, max_iter=iters, traj=True, lower=-5.0, upper=5.0)
    assert path.read_text() == reference_tsv(o["traj_x"], o["traj_f"], o["traj_g"],
                                             o["traj_status"])
    best = int(np.argmin(o["fval"]))
    assert r.idx == best and r.fval == o["fval"][best] and r.status == o["status"][best]


def test_zeus_trajectory_file_with_pso_starts(cuda, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    path = tmp_path / "ras.tsv"
    r = zb.Zeus(zb.Rastrigin(2), -5.12, 5.12, 8, 30, 5, 1000, "rastrigin", 1e-8, 3, 0,
                trajectory_file=str(path))
    rows = path.read_text().splitlines()
    assert rows[0].split("\t") == ["traj", "step", "fval", "grad", "status", "alpha", "x0", "x1"]
    assert len(rows) == 1 + 8 * 30
    body = [row.split("\t") for row in rows[1:]]
    # run r's rows are steps 0..29 in order; step 0 is recorded for every run
    assert [int(b[0]) for b in body] == [i for i in range(8) for _ in range(30)]
    assert all(b[2] != "NaN" for b in body[::30])
    assert r.status in (0, 1, 5) and np.isfinite(r.fval)


def test_zeus_trajectory_file_rejects_netcdf(cuda, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    with pytest.raises(zb.ZeusError):
        zb.Zeus(zb.Rosenbrock(2), -5.0, 5.0, 4, 10, -1, 10, "rosenbrock", 1e-8, 1, 0,
                trajectory_file=str(tmp_path / "t.nc"))
