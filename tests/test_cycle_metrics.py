"""zeus_cycle_metrics against a plain restatement of the reference's
report_metrics_and_cleanup (bfgs_sequential.cuh:236-373) on synthetic
per-run timer values (host only)."""
import math

import numpy as np
import pytest

from zeus_b200.device import METRIC_NAMES, cycle_metrics


def reference_metrics(cyc, calls, total, ms_opt, khz, tpb):
    """The reference's formulas, one timer, a run standing for a thread."""
    n = len(cyc)
    hz = khz * 1000.0
    sum_cycles, sum_calls = int(np.sum(cyc)), int(np.sum(calls))
    avg_cycles = sum_cycles / n
    avg_calls = sum_calls / n if sum_calls > 0 else 0.0
    per_call = avg_cycles / avg_calls if avg_calls > 0 else 0.0
    ms_thread = avg_cycles / hz * 1e3
    frac_kernel = ms_thread / ms_opt if ms_thread > 0 and ms_opt > 0 else 0.0
    serialized = (sum_cycles / hz * 1e3) / ms_opt if ms_opt > 0 else 0.0
    fr = [c / t for c, t in zip(cyc, total) if t > 0]
    frac_thread = float(np.mean(fr)) if fr else 0.0
    nb = (n + tpb - 1) // tpb
    fb = sorted((sum(cyc[b * tpb:(b + 1) * tpb]) / hz * 1e3) / ms_opt for b in range(nb))
    i95 = min(len(fb) - 1, math.ceil(0.95 * len(fb)) - 1)
    return dict(ms_per_call=per_call / hz * 1e3, calls_per_thread_mean=avg_calls,
                fraction_of_thread=frac_thread, block95=fb[i95], serialized=serialized,
                fraction_of_kernel=frac_kernel, avg_cycles_per_thread=avg_cycles,
                avg_ms_per_thread=ms_thread)


@pytest.mark.parametrize("n,tpb", [(1, 128), (300, 128), (1000, 7), (4096, 256)])
def test_cycle_metrics_match_the_reference_formulas(n, tpb):
    rng = np.random.default_rng(n)
    grads = rng.integers(1, 400, n)
    counters = np.stack([grads - 1, 3 * grads, grads], axis=1).astype(np.int64)
    g = rng.integers(1_000, 5_000_000, n)
    u = rng.integers(1_000, 9_000_000, n)
    tot = g + u + rng.integers(0, 2_000_000, n)
    tot[::17] = 0  # runs with no total are left out of the thread fraction
    cycles = np.stack([g, u, tot], axis=1).astype(np.int64)
    khz, ms = 1_965_000.0, 12.5
    got = cycle_metrics(cycles, counters, ms, khz, runs_per_block=tpb)
    want_ad = reference_metrics(g, grads, tot, ms, khz, tpb)
    want_bf = reference_metrics(u, grads - 1, tot, ms, khz, tpb)
    for name in METRIC_NAMES:
        assert got["ad"][name] == pytest.approx(want_ad[name], rel=1e-12, abs=1e-15), name
        assert got["bfgs"][name] == pytest.approx(want_bf[name], rel=1e-12, abs=1e-15), name


def test_cycle_metrics_rejects_bad_arguments():
    with pytest.raises(Exception):
        cycle_metrics(np.zeros((3, 3), np.int64), np.zeros((2, 3), np.int64), 1.0, 1e6)
    with pytest.raises(Exception):
        cycle_metrics(np.zeros((3, 3), np.int64), np.zeros((3, 3), np.int64), 1.0, 0.0)
