"""Per-run cycle timers (zeus_run_outputs.cycles): the reference's AD / BFGS
/ total clock64 spans (bfgs_sequential.cuh:93-97, 150-174, 229-232), sampled
in every layout when asked for, without changing any result."""
import numpy as np
import pytest
import torch

import zeus_b200 as zb
from zeus_b200.device import (BatchJob, batch_device, bfgs_device, cycle_metrics,
                              starts_uniform)

pytestmark = pytest.mark.gpu


def host(r):
    return {k: getattr(r, k).cpu().numpy() for k in ("fval", "status", "iter", "gnorm", "x",
                                                      "counters")}


CASES = [  # (objective, dim, mode, layout, tile)
    (zb.Rosenbrock(4), "fast", zb.LAYOUT_THREAD, 0),
    (zb.Rosenbrock(8), "fast", zb.LAYOUT_TILE, 8),
    (zb.Rosenbrock(64), "fast", zb.LAYOUT_CTA, 0),
    (zb.Rosenbrock(32), "fast", zb.LAYOUT_ROWS, 0),
    (zb.Rosenbrock(128), "fast", zb.LAYOUT_ROWS, 0),
    (zb.Rosenbrock(4), "exact", zb.LAYOUT_AUTO, 0),
]


@pytest.mark.parametrize("obj,mode,layout,tile", CASES)
def test_cycles_sampled_without_changing_results(cuda, obj, mode, layout, tile):
    st = starts_uniform(5, 96, obj.dim, -5.0, 5.0)
    kw = dict(max_iter=600, mode=mode, layout=layout, tile=tile,
              gradient="dual" if mode == "exact" else "adjoint")
    plain = host(bfgs_device(obj, st, **kw))
    r = bfgs_device(obj, st, cycles=True, **kw)
    torch.cuda.synchronize()
    got = host(r)
    for k in plain:
        np.testing.assert_array_equal(got[k], plain[k], err_msg=k)
    cyc = r.cycles.cpu().numpy()
    assert (cyc[:, 0] > 0).all() and (cyc[:, 1] > 0).all()
    assert (cyc[:, 2] >= cyc[:, 0] + cyc[:, 1]).all()
    m = cycle_metrics(cyc, got["counters"], ms_opt=1.0, sm_clock_khz=1.9e6)
    assert m["ad"]["calls_per_thread_mean"] == pytest.approx(
        m["bfgs"]["calls_per_thread_mean"] + 1.0)
    assert 0 < m["ad"]["fraction_of_thread"] < 1 and 0 < m["bfgs"]["fraction_of_thread"] < 1


def test_batch_rejects_cycles(cuda):
    """The batch kernel is built without the timers: a class asking for
    cycles is refused, not silently left unsampled."""
    j = BatchJob(zb.Rosenbrock(8), starts_uniform(7, 16, 8, -5.0, 5.0), cycles=True)
    with pytest.raises(zb.ZeusError):
        batch_device([j], max_iter=100)
