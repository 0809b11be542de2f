"""The sharded call (zeus_b200/shard.py) on one GPU, as a world of one: it
must return what the one-GPU call zeus::Zeus returns (zeus_optimize), run
for run, with stop-early off.  The split and the cross-rank merge are
covered over gloo ranks on the CPU (tests/test_shard.py)."""
import numpy as np
import pytest

import zeus_b200 as zb
from zeus_b200.shard import sharded_optimize

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("obj,n,pso", [(zb.Rosenbrock(8), 512, 10), (zb.Rosenbrock(64), 96, -1)])
def test_world_of_one_equals_the_one_gpu_call(cuda, tmp_path, monkeypatch, obj, n, pso):
    monkeypatch.chdir(tmp_path)  # Zeus appends its results row in the cwd
    dim = obj.dim
    ref = zb.Zeus(obj, -5.0, 5.0, n, 3000, pso, n + 1, "rosenbrock", 1e-8, 42, 0)
    m = sharded_optimize(obj, n, -5.0, 5.0, 3000, pso, n + 1, 1e-8, 42,
                         known_min=np.ones(dim))
    assert m.idx == ref.idx and m.status == ref.status
    assert m.fval == ref.fval and m.iter == ref.iter
    np.testing.assert_array_equal(m.x, np.asarray(ref.coordinates))
    assert (m.actual, m.claimed, m.surrendered, m.stopped) == (
        ref.c.actual, ref.c.claimed, ref.c.surrendered, ref.c.stopped)
