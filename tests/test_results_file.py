"""The per-call results file (util::appendResultsToTsv, src/util.cpp:44-108)
and the error it reports (util::calculateEuclideanError, src/util.cpp:12-41),
checked on the CPU against a restatement of the reference's stream output:
default float format (%g, precision 6) up to `time`, then std::scientific
(%e) for error, fval, norm and the coordinates."""
import ctypes as C
import math

import numpy as np

import zeus_b200 as zb

HEADER = ("fun\trun\tN\tkernel\tad_ms_per_call\tad_calls_per_thread_mean\tad_fraction"
          "\tad_block95\tad_serialized\tbfgs_ms_per_call\tbfgs_calls_per_thread_mean"
          "\tbfgs_fraction\tbfgs_block95\tbfgs_serialized\tclaimed\tactual\tsurrender"
          "\tstopped\tidx\tstatus\tbfgs_iter\tpso_iter\ttime\terror\tfval\tnorm")


def reference_row(fun, run, n, ms_init, ms_pso, ms_opt, ms_rand, max_iter, pso_iter, error,
                  best, census, x):
    f32 = lambda v: float(np.float32(v))  # the reference passes the times as float
    t = (f32(ms_init) + f32(ms_pso) + f32(ms_opt) + f32(ms_rand) if pso_iter > 0
         else f32(ms_opt) + f32(ms_rand))
    fields = [fun, str(run), str(n), "%g" % f32(ms_opt)] + ["%g" % 0.0] * 10 + [
        str(census[1]), str(census[0]), str(census[2]), str(census[3]), str(best[0]),
        str(best[1]), str(max_iter), str(pso_iter), "%g" % t, "%e" % error, "%e" % best[2],
        "%e" % best[3]]
    return "\t".join(fields) + "\t" + "\t".join("%e" % v for v in x) + "\n"


def _append(tmp_path, fun, run, n, ms, max_iter, pso_iter, err, best, census, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    cb = zb.CResult(best[0], best[1], best[2], best[3], best[4], 0)
    cc = zb.CCensus(census[0], census[1], census[2], census[3], best[0], 0)
    return zb.lib().zeus_append_results_tsv(
        str(tmp_path).encode(), fun.encode(), run, n, len(x), ms[0], ms[1], ms[2], ms[3],
        max_iter, pso_iter, err, C.byref(cb), C.byref(cc), x.ctypes.data, None)


def test_results_rows_and_header(tmp_path):
    x = np.array([1.0000001, 0.99999])
    best = (17, 1, 3.25e-15, 7.5e-9, 42)
    census = (900, 950, 70, 4)  # actual, claimed, surrendered, stopped
    err = zb.lib().zeus_euclidean_error(b"rosenbrock", x.ctypes.data, 2)
    assert err == math.sqrt((x[0] - 1) ** 2 + (x[1] - 1) ** 2)
    ms = (0.125, 2.5, 12.345678, 0.0)
    assert _append(tmp_path, "rosenbrock", 3, 1024, ms, 10000, 10, err, best, census, x) == 0
    assert _append(tmp_path, "rosenbrock", 4, 1024, ms, 10000, -1, err, best, census, x) == 0
    lines = (tmp_path / "zeus_2d_results.tsv").read_text().splitlines(keepends=True)
    assert lines[0] == HEADER + "\tcoord_0\tcoord_1\n"
    assert lines[1] == reference_row("rosenbrock", 3, 1024, *ms, 10000, 10, err, best,
                                     census, x)
    assert lines[2] == reference_row("rosenbrock", 4, 1024, *ms, 10000, -1, err, best,
                                     census, x)
    assert len(lines) == 3


def test_euclidean_error_by_name():
    L = zb.lib()
    x = np.array([3.0, 4.0])
    assert L.zeus_euclidean_error(b"ackley", x.ctypes.data, 2) == 5.0
    assert L.zeus_euclidean_error(b"goldstein_price", x.ctypes.data, 2) == math.hypot(3, 5)
    x3 = np.zeros(3)
    assert math.isnan(L.zeus_euclidean_error(b"goldstein_price", x3.ctypes.data, 3))
