"""The C++ drop-in (include/zeus.cuh: zeus::Zeus, Matrix, Result) used as code
written for the reference uses it: tests/cpp/dropin_test.cu, built by
zeus_b200/build.py into zeus_b200/_bin/dropin_test."""
import json
import subprocess

import numpy as np
import pytest

from zeus_b200 import build as zbuild

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def workdir(tmp_path_factory):
    return tmp_path_factory.mktemp("dropin")


@pytest.fixture(scope="module")
def traj_path(workdir):
    return workdir / "traj.tsv"


@pytest.fixture(scope="module")
def sobol_traj_path(workdir):
    return workdir / "traj_sobol.tsv"


@pytest.fixture(scope="module")
def results(cuda, traj_path, sobol_traj_path, workdir):
    exe = zbuild.DROPIN_BIN
    if not exe.exists():
        pytest.fail(f"{exe} is missing: run zeus_b200/build.py (build_dropin_test)")
    out = subprocess.run([str(exe), str(traj_path), str(sobol_traj_path)],
                         capture_output=True, text=True, timeout=300, cwd=str(workdir))
    assert out.returncode == 0, out.stderr
    return {d["case"]: d for d in (json.loads(l) for l in out.stdout.splitlines()
                                   if l.startswith("{"))}


def test_trajectory_file_from_the_drop_in(results, traj_path):
    """Zeus(..., trajectory_file) writes the reference's TSV: every run's
    MAX_ITER steps, step 0 at the injected start."""
    from tests import _oracle as O

    rows = traj_path.read_text().splitlines()
    assert rows[0].split("\t") == ["traj", "step", "fval", "grad", "status", "alpha",
                                    "x0", "x1"]
    assert len(rows) == 1 + 6 * 40
    st = O.oracle_starts(42, 6, 2, -5.0, 5.0)
    for i in range(6):
        r0 = rows[1 + 40 * i].split("\t")
        assert (int(r0[0]), int(r0[1])) == (i, 0)
        np.testing.assert_array_equal([float(r0[6]), float(r0[7])], st[i])
        f0 = (1 - st[i, 0]) ** 2 + 100 * (st[i, 1] - st[i, 0] ** 2) ** 2
        np.testing.assert_allclose(float(r0[2]), f0, rtol=1e-13)
    r = results["traj"]
    assert r["status"] in (0, 1)


def test_sobol_starts_from_the_drop_in(results, sobol_traj_path):
    """PRNGType::SOBOL: step 0 of each run's trajectory is its start, point i
    of the oracle's shifted Sobol' sequence."""
    from tests import _oracle as O

    rows = sobol_traj_path.read_text().splitlines()
    st = O.oracle_starts(42, 6, 2, -5.0, 5.0, prng=O.PRNG_SOBOL)
    assert not np.array_equal(st, O.oracle_starts(42, 6, 2, -5.0, 5.0))
    for i in range(6):
        r0 = rows[1 + 40 * i].split("\t")
        np.testing.assert_array_equal([float(r0[6]), float(r0[7])], st[i])
    r = results["sphere16_sobol"]
    assert r["status"] == 1 and r["gnorm"] < 1e-8
    np.testing.assert_allclose(r["x"], [0.5] * 16, atol=1e-8)


def test_rosenbrock_functor(results):
    r = results["rosenbrock"]
    assert r["status"] in (1, 2) and r["fval"] < 1e-12
    np.testing.assert_allclose(r["x"], [1.0, 1.0], atol=1e-6)
    assert r["claimed"] >= 100 and r["claimed"] + r["stopped"] + r["surrendered"] == 1024


def test_functor_template_dimension_and_tile_layout(results):
    r = results["sphere16"]
    assert r["status"] == 1 and r["gnorm"] < 1e-8
    np.testing.assert_allclose(r["x"], [0.5] * 16, atol=1e-8)


def test_matrix_backed_objective(results):
    r = results["gaussian8"]
    assert r["status"] == 1 and abs(r["fval"]) < 1e-15
    np.testing.assert_allclose(r["x"], [0.0] * 8, atol=1e-8)


def test_adjoint_member_and_uniform_starts(results):
    r = results["adjoint4"]
    assert r["status"] == 1 and r["fval"] < 1e-16


def test_cta_layout_from_template(results):
    r = results["sphere40"]
    assert r["status"] == 1
    np.testing.assert_allclose(r["x"], [0.5] * 40, atol=1e-8)


def test_zero_runs_default_result(results):
    r = results["empty"]
    assert r["status"] == -1 and r["fval"] == 37.0 and r["idx"] == -1


def test_results_files_like_the_reference(results, workdir):
    """Every call with N > 0 appends its row to zeus_<D>d_results.tsv in the
    working directory (zeus.cuh:170-183, util.hpp:79-136)."""
    rows = (workdir / "zeus_2d_results.tsv").read_text().splitlines()
    assert rows[0].startswith("fun\trun\tN\tkernel\t")
    assert rows[0].endswith("\tcoord_0\tcoord_1")
    # "rosenbrock", "traj" and "traj_sobol"; the N == 0 call writes nothing
    assert len(rows) == 4
    for row, case in zip(rows[1:], ("rosenbrock", "traj", "traj_sobol")):
        f = row.split("\t")
        r = results[case]
        assert f[0] == "rosenbrock" and int(f[19]) == r["status"]
        assert float(f[24]) == pytest.approx(r["fval"], rel=1e-5, abs=1e-300)
        assert int(f[14]) == r["claimed"]
    for d in (16, 8, 4, 40, 200):
        assert (workdir / f"zeus_{d}d_results.tsv").exists()


def test_cycle_metrics_like_the_reference(results, workdir):
    """Every call samples the reference's AD / BFGS / total cycle timers
    (bfgs_sequential.cuh:93-97, 150-174, 229-232) and reports their summary
    (report_metrics_and_cleanup, :236-373) in Result::ad / ::bfgs and in the
    results row's ten metric columns."""
    for case in ("rosenbrock", "sphere16", "gaussian8", "sphere40", "sphere200", "traj"):
        r = results[case]
        ad, bf = r["ad"], r["bfgs"]  # ms/call, calls, kernel frac, p95, serialized, thread frac
        assert ad[0] > 0 and bf[0] > 0, case
        assert ad[1] >= 1.0 and bf[1] >= 0.0, case  # the first gradient counts
        assert ad[1] == pytest.approx(bf[1] + 1.0, abs=1e-9), case
        for m in (ad, bf):
            assert 0.0 < m[5] < 1.0 and m[2] > 0 and m[3] > 0 and m[4] > 0, (case, m)
        assert ad[5] + bf[5] < 1.0, case  # parts of the run
    rows = (workdir / "zeus_2d_results.tsv").read_text().splitlines()
    f = rows[1].split("\t")
    ad = [float(v) for v in f[4:9]]
    bf = [float(v) for v in f[9:14]]
    r = results["rosenbrock"]
    # file order: ms_per_call, calls_per_thread_mean, fraction_of_thread, block95, serialized
    assert ad[0] == pytest.approx(r["ad"][0], rel=1e-5)
    assert ad[1] == pytest.approx(r["ad"][1], rel=1e-5)
    assert ad[2] == pytest.approx(r["ad"][5], rel=1e-5)
    assert bf[4] == pytest.approx(r["bfgs"][4], rel=1e-5)


def test_cta_layout_with_h_in_global_memory(results):
    """D = 200: H (320 KB) does not fit in shared memory; each block streams
    its own slice of a global workspace."""
    r = results["sphere200"]
    assert r["status"] == 1 and r["fval"] < 1e-12
    assert r["claimed"] == 40
