"""The reference's own example programs, compiled unmodified against this
library's include/ (zeus_b200/build.py: build_reference_examples), run on
the GPU and checked against the oracle on the same starts.

  optimize_rosenbrock / optimize_rastrigin / optimize_ackley
      examples/optimize_*.cu + optimization_utils.cc: util::setStackSize(),
      zeus::Zeus on the examples' 2-D functors (rosenbrock.hpp, rastrigin.hpp,
      ackley.hpp written against the reference's duals.cuh), print_result.
  fit_dijet_spectrum
      examples/fit_dijet_spectrum.cu: LogLikelihood.h fitted to
      ../examples/simulation/dijet_spectrum.tsv (absent from the reference:
      a synthetic spectrum of the dijet shape is written there).
  ref_objectives_test
      tests/cpp/ref_objectives_test.cu: the reference's Gaussian class
      (examples/gaussian.hpp, Matrix<double> member) at D = 8 and 150, and
      LogLikelihood.h on synthetic toy counts.

The drop-in's PSO equals the oracle's synchronous PSO bit for bit, so the
oracle runs BFGS from the same starts; the best run's status, value and
coordinates are compared (to the printed precision where the program
prints rounded values)."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import zeus_b200 as zb
from tests import _oracle as O

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
BIN = ROOT / "zeus_b200" / "_bin" / "ref_examples"
ROS, RAS, ACK, GAU, NLL = 0, 1, 2, 3, 4

needs_bin = pytest.mark.skipif(
    not (BIN / "optimize_rosenbrock").exists(),
    reason="reference examples not built (build() builds them where the reference "
           "checkout is present)")


def run(prog, *args, cwd=None, timeout=300):
    r = subprocess.run([str(BIN / prog), *map(str, args)], capture_output=True, text=True,
                       cwd=cwd, timeout=timeout)
    assert r.returncode in (0, 2), (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


def parse_example(out):
    """print_result of optimization_utils.cc."""
    st = int(re.search(r"Status: (-?\d+)", out).group(1))
    fv = float(re.search(r"Function value: (\S+)", out).group(1))
    it = int(re.search(r"Iterations: (\d+)", out).group(1))
    xs = re.search(r"Best coordinates: \(([^)]*)\)", out).group(1)
    return st, fv, it, np.array([float(v) for v in xs.split(",")])


def parse_result_line(out):
    f = re.search(r"^RESULT (.*)$", out, re.M).group(1).split()
    return int(f[0]), float(f[1]), float(f[2]), int(f[3]), np.array([float(v) for v in f[4:]])


def oracle_best(kind, dim, n, lo, hi, pso_iter, max_iter, seed=42, data=None, idata=None,
                pso_data=None):
    """Oracle PSO starts, oracle BFGS on every start (stop-early off), and the
    run with the lowest fval (lowest index on ties, NaN never)."""
    pbx, _, _, _ = O.oracle_pso(kind, dim, seed, n, lo, hi, pso_iter,
                                data=data if pso_data is None else pso_data, idata=idata)
    r = O.oracle_bfgs(kind, dim, pbx, max_iter=max_iter, data=data, idata=idata,
                      lower=lo, upper=hi)
    f = np.where(np.isnan(r["fval"]), np.inf, r["fval"])
    i = int(np.argmin(f))
    return r["status"][i], r["fval"][i], r["x"][i], r


@needs_bin
@pytest.mark.parametrize("prog,kind,lo,hi", [
    ("optimize_rosenbrock", ROS, -5.0, 5.0),
    ("optimize_rastrigin", RAS, -5.12, 5.12),
    ("optimize_ackley", ACK, -32.768, 32.768)])
def test_reference_example_programs(cuda, tmp_path, prog, kind, lo, hi):
    n, pso, max_iter = 512, 10, 10000
    # <lower> <upper> <max_iter> <pso_iters> <converged> <N> <tol> <seed> <run>;
    # required > N: no stop-early, so every run's outcome is timing-free
    out = run(prog, lo, hi, max_iter, pso, n + 1, n, 1e-8, 42, 0, cwd=tmp_path)
    st, fv, _, x = parse_example(out)
    ost, ofv, ox, _ = oracle_best(kind, 2, n, lo, hi, pso, max_iter)
    assert st == ost
    assert fv == pytest.approx(ofv, rel=1e-5, abs=1e-12)
    np.testing.assert_allclose(x, ox, rtol=1e-8, atol=1e-6)
    # the reference's results row is appended in the working directory
    assert (tmp_path / "zeus_2d_results.tsv").exists()


def dijet_spectrum_rows(seed=5, nbins=100, sqrt_s=13.6):
    """Synthetic spectrum in the reference's dijet_spectrum.tsv layout
    (bin_low bin_high counts, masses in TeV, x = m / 13.6 over [0.085,
    0.54]); lambda = a (1-x)^10 / x^(5 + 0.1 ln x) normalised so the
    amplitude a of the fit is about 3."""
    edges = np.geomspace(0.085, 0.54, nbins + 1) * sqrt_s
    lo, hi = edges[:-1], edges[1:]
    x = 0.5 * (lo + hi) / sqrt_s
    shape = (1 - x) ** 10.0 / x ** (5.0 + 0.1 * np.log(x))
    k = np.random.default_rng(seed).poisson(3.0 * shape).astype(np.int32)
    return lo, hi, k, x


@needs_bin
def test_reference_dijet_fit_program(cuda, tmp_path):
    lo, hi, k, x = dijet_spectrum_rows()
    data = tmp_path / "examples" / "simulation"
    data.mkdir(parents=True)
    with open(data / "dijet_spectrum.tsv", "w") as fh:
        fh.write("bin_low\tbin_high\tcounts\n")
        for a, b, c in zip(lo, hi, k):
            fh.write(f"{float(a)!r}\t{float(b)!r}\t{int(c)}\n")
    work = tmp_path / "run"
    work.mkdir()
    n, max_iter = 64, 1000
    out = run("fit_dijet_spectrum", n, max_iter, 0, cwd=work)
    assert "Loaded 100 bins" in out
    fv = float(re.search(r"best NLL: (\S+)", out).group(1))
    pars = [float(v) for v in re.search(
        r"a=(\S+)\s+b=(\S+)\s+c=(\S+)\s+d=(\S+)", out).groups()]
    assert (work / "dijet_fit_vs_data.tsv").exists()
    # the program's centres: 0.5 (low + high) / 13.6 from the values it read
    xc = 0.5 * (lo + hi) / 13.6
    _, ofv, ox, r = oracle_best(NLL, 4, n, 0.0, 10.0, 10, max_iter, data=xc, idata=k)
    # printed to 6 significant digits; stop-early at 100 converged runs makes
    # the set of finished runs timing-dependent, but every run ends in the
    # same basin
    assert fv == pytest.approx(ofv, rel=2e-6)
    np.testing.assert_allclose(pars, ox, rtol=1e-4)


@needs_bin
@pytest.mark.parametrize("dim,n,pso,max_iter", [(8, 64, 5, 1000), (150, 128, 10, 10000)])
def test_reference_gaussian_class(cuda, dim, n, pso, max_iter):
    out = run("ref_objectives_test", "gaussian", dim, n, pso, max_iter, 42)
    st, fv, gn, it, x = parse_result_line(out)
    C = zb.gaussian_matrix(dim)
    ost, ofv, ox, r = oracle_best(GAU, dim, n, -5.0, 5.0, pso, max_iter, data=C)
    assert st == ost == 1
    assert (r["status"] == 1).all()
    assert gn < 1e-8 and abs(fv) < 1e-15 and abs(ofv) < 1e-15
    assert np.abs(x).max() < 1e-9 and np.abs(ox).max() < 1e-9


@needs_bin
def test_reference_loglikelihood_class(cuda, tmp_path):
    xk, k, _ = O.dijet_toy()
    f = tmp_path / "bins.txt"
    f.write_text("".join(f"{int(c)} {float(v)!r}\n" for c, v in zip(k, xk)))
    n, pso, max_iter = 64, 10, 1000
    out = run("ref_objectives_test", "nll", f, n, pso, max_iter, 42)
    st, fv, gn, it, x = parse_result_line(out)
    ost, ofv, ox, r = oracle_best(NLL, 4, n, 0.0, 10.0, pso, max_iter, data=xk, idata=k)
    assert np.isfinite(fv)
    assert fv == pytest.approx(ofv, rel=1e-9)
    np.testing.assert_allclose(x, ox, rtol=1e-5)
