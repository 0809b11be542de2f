"""The persistent batch kernel and the layout autotuner, through the C ABI.

Every batch class runs the same per-run body as the standalone layout
kernels, so with the same layout (and, for the CTA layout, the same block
size) its results must equal the standalone launch's bit for bit."""
import numpy as np
import pytest
import torch

import zeus_b200 as zb
from zeus_b200.device import BatchJob, DeviceProblem, batch_device, bfgs_device, starts_uniform
from tests import _oracle as O

pytestmark = pytest.mark.gpu

ROS, RAS, ACK, GAU, NLL = 0, 1, 2, 3, 4


def host(r):
    return {k: getattr(r, k).cpu().numpy() for k in ("fval", "status", "iter", "gnorm", "x")}


MIX = [  # (objective, n, layout, tile, bounds)
    (lambda: zb.Rosenbrock(2), 700, zb.LAYOUT_THREAD, 0, (-5, 5)),
    (lambda: zb.Rosenbrock(8), 300, zb.LAYOUT_TILE, 4, (-5, 5)),
    (lambda: zb.Rosenbrock(32), 200, zb.LAYOUT_TILE, 32, (-5, 5)),
    (lambda: zb.Ackley(30), 200, zb.LAYOUT_TILE, 32, (-32.768, 32.768)),
    (lambda: zb.Rosenbrock(128), 160, zb.LAYOUT_CTA, 0, (-5, 5)),
    (lambda: zb.Rosenbrock(64), 160, zb.LAYOUT_CTA, 0, (-5, 5)),
]


def test_batch_equals_standalone_launches(cuda):
    jobs, sts = [], []
    for i, (mk, n, lay, tile, (lo, hi)) in enumerate(MIX):
        st = starts_uniform(100 + i, n, mk().dim, lo, hi)
        sts.append(st)
        jobs.append(BatchJob(mk(), st, layout=lay, tile=tile))
    # 512-thread blocks: the standalone CTA kernel's block at dim 128
    b = batch_device(jobs, max_iter=600, block=512)
    torch.cuda.synchronize()
    for (mk, n, lay, tile, _), j, st in zip(MIX, jobs, sts):
        ref = bfgs_device(mk(), st, max_iter=600, layout=lay, tile=tile)
        torch.cuda.synchronize()
        got, want = host(j), host(ref)
        if lay == zb.LAYOUT_CTA and mk().dim == 64:
            # the standalone CTA kernel uses 256 threads at dim 64, the batch
            # 512: the H sweeps sum in a different order
            agree = (got["status"] == want["status"]).mean()
            assert agree > 0.8
            both = (got["status"] == 1) & (want["status"] == 1)
            np.testing.assert_allclose(got["fval"][both], want["fval"][both], atol=1e-8)
        else:
            for k in got:
                np.testing.assert_array_equal(got[k], want[k], err_msg=f"{mk().dim} {k}")
        assert (j.counters.cpu().numpy()[:, 0] > 0).all()


def test_batch_refills_slots_beyond_concurrency(cuda):
    # 148 SMs x 16 warps = 2368 concurrent 32-lane tiles: 6000 runs need refills
    st = starts_uniform(7, 6000, 32, -5.0, 5.0)
    j = BatchJob(zb.Rosenbrock(32), st, layout=zb.LAYOUT_TILE, tile=32)
    batch_device([j], max_iter=300)
    ref = bfgs_device(zb.Rosenbrock(32), st, max_iter=300, layout=zb.LAYOUT_TILE, tile=32)
    torch.cuda.synchronize()
    for k, v in host(j).items():
        np.testing.assert_array_equal(v, host(ref)[k], err_msg=k)


def test_batch_per_instance_nll_toys(cuda):
    toys, per = 4, 16
    xs, ks = [], []
    for t in range(toys):
        x, k, _ = O.dijet_toy(seed=t)
        xs.append(x)
        ks.append(k)
    obj = zb.PoissonNLL(np.concatenate(ks), np.concatenate(xs))
    obj.dim = 4
    st = starts_uniform(3, toys * per, 4, 0.0, 10.0)
    j = BatchJob(obj, st, runs_per_instance=per)
    batch_device([j], max_iter=2000)
    torch.cuda.synchronize()
    got = host(j)
    for t in range(toys):
        one = bfgs_device(zb.PoissonNLL(ks[t], xs[t]), st[t * per:(t + 1) * per].contiguous(),
                          max_iter=2000, layout=j.layout if j.layout else zb.LAYOUT_THREAD)
        torch.cuda.synchronize()
        w = host(one)
        for k in got:
            np.testing.assert_array_equal(got[k][t * per:(t + 1) * per], w[k], err_msg=k)


def test_batch_block_sizes_agree_on_tile_classes(cuda):
    """The 384- and 512-thread kernels run the same per-run tile bodies."""
    st = starts_uniform(9, 500, 8, -5.0, 5.0)
    outs = []
    for block in (384, 512):
        j = BatchJob(zb.Rosenbrock(8), st, layout=zb.LAYOUT_TILE, tile=8)
        batch_device([j], max_iter=800, block=block)
        torch.cuda.synchronize()
        outs.append(host(j))
    for k in outs[0]:
        np.testing.assert_array_equal(outs[0][k], outs[1][k], err_msg=k)


def test_batch_stop_early_per_class(cuda):
    st2 = starts_uniform(1, 512, 2, -2.0, 2.0)
    st8 = starts_uniform(2, 256, 8, -2.0, 2.0)
    a = BatchJob(zb.Rosenbrock(2), st2, required=5)
    b = BatchJob(zb.Rosenbrock(8), st8)
    batch_device([a, b], max_iter=5000)
    torch.cuda.synchronize()
    sa, sb = a.status.cpu().numpy(), b.status.cpu().numpy()
    assert (sa == 1).sum() >= 5 and (sa == 2).sum() > 0
    assert (sb == 2).sum() == 0
    assert a.control.cpu().numpy()[0] == 1 and b.control.cpu().numpy()[0] == 0


def test_batch_rejects_bad_input(cuda):
    st = starts_uniform(1, 8, 3, -1.0, 1.0)
    with pytest.raises(zb.ZeusError):
        batch_device([BatchJob(zb.Objective(ROS, 3), st)])
    st = starts_uniform(1, 8, 32, -1.0, 1.0)  # 16 H rows of 32 per lane: not built
    with pytest.raises(zb.ZeusError):
        batch_device([BatchJob(zb.Rosenbrock(32), st, layout=zb.LAYOUT_TILE, tile=2)])


@pytest.mark.parametrize("obj,lo,hi", [(zb.Rosenbrock(8), -5, 5), (zb.Rastrigin(10), -5.12, 5.12),
                                       (zb.Rosenbrock(64), -5, 5)])
def test_autotune_records_a_built_layout(cuda, obj, lo, hi):
    lay, tile, ms = zb.autotune(obj, n_sample=256, max_iter=300, lower=lo, upper=hi)
    assert lay in (zb.LAYOUT_THREAD, zb.LAYOUT_TILE, zb.LAYOUT_CTA, zb.LAYOUT_ROWS) and ms > 0
    import ctypes as C
    l2, t2 = C.c_int32(), C.c_int32()
    assert zb.lib().zeus_autotune_lookup(obj.kind, obj.dim, zb.GRAD_ADJOINT, C.byref(l2),
                                         C.byref(t2)) == 1
    assert (l2.value, t2.value) == (lay, tile)
    st = starts_uniform(9, 128, obj.dim, lo, hi)
    auto = host(bfgs_device(obj, st, max_iter=300))
    expl = host(bfgs_device(obj, st, max_iter=300, layout=lay, tile=tile))
    torch.cuda.synchronize()
    for k in auto:
        np.testing.assert_array_equal(auto[k], expl[k], err_msg=k)


def test_batch_with_companion_in_a_cuda_graph(cuda):
    """A batch whose 128-D row class runs as a companion launch (a second
    stream forked from and joined back into the caller's) captured into a
    CUDA graph and replayed gives the same runs as the direct launch."""
    from zeus_b200.device import Batch, BatchJob, starts_uniform

    jobs = [BatchJob(zb.Rosenbrock(128), starts_uniform(3, 40, 128, -5.0, 5.0),
                     layout=zb.LAYOUT_ROWS),
            BatchJob(zb.Rosenbrock(8), starts_uniform(4, 200, 8, -5.0, 5.0))]
    b = Batch(jobs, max_iter=600)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        b.launch(s)  # direct: also makes the library's side stream
    torch.cuda.synchronize()
    want = [(j.fval.clone(), j.status.clone(), j.x.clone()) for j in jobs]
    for j in jobs:
        j.fval.fill_(float("nan"))
        j.status.fill_(-7)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s, capture_error_mode="thread_local"):
        b.launch(s, reset=False)
    for j in jobs:
        j.control.zero_()
    g.replay()
    torch.cuda.synchronize()
    for j, (f, st, x) in zip(jobs, want):
        assert torch.equal(j.status, st)
        assert torch.equal(j.fval, f)
        assert torch.equal(j.x, x)
