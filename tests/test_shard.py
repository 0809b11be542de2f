"""The sharded call's split and cross-rank merge (zeus_b200/shard.py): two
and three gloo processes on the CPU, each running the oracle's BFGS on its
shard of the runs, merge their censuses and best runs over the same
collectives the GPUs issue over NCCL; the merged result must equal the
census of all runs computed in one process."""
import math
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from zeus_b200.shard import (LocalCensus, census_host, merge, order_key, owner_of,
                             shard_range, sharded_call)

KIND, DIM, LO, HI, SEED, MAX_ITER = 0, 4, -5.0, 5.0, 42, 400
KNOWN_MIN = np.ones(DIM)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_range_covers_every_run_once():
    for n in (0, 1, 2, 7, 37, 1000):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                s, c = shard_range(n, r, world)
                seen.extend(range(s, s + c))
                assert c in (n // world, n // world + 1)
            assert seen == list(range(n))
            for i in range(n):
                s, c = shard_range(n, owner_of(i, n, world), world)
                assert s <= i < s + c


def test_order_key_orders_like_the_doubles():
    vals = [-math.inf, -1e300, -2.0, -1e-300, -0.0, 0.0, 1e-300, 3.0, 1e300, math.inf]
    keys = [order_key(v) for v in vals]
    assert keys == sorted(keys) and len(set(keys)) == len(keys)
    assert order_key(math.nan) > order_key(math.inf)


def _oracle_local(n, known_min):
    from tests import _oracle as O

    def local(start, count):
        if count == 0:
            return LocalCensus()
        st = O.oracle_starts(SEED, n, DIM, LO, HI)[start:start + count]
        r = O.oracle_bfgs(KIND, DIM, st, max_iter=MAX_ITER)
        c = census_host(r["fval"], r["status"], r["x"], known_min)
        b = c.best_local
        c.fval, c.status, c.iter, c.gnorm = (float(r["fval"][b]), int(r["status"][b]),
                                             int(r["iter"][b]), float(r["gnorm"][b]))
        c.x = r["x"][b]
        return c
    return local


def _synthetic_local(fvals):
    """Per-rank fixed fvals (ties and NaN planted on the host)."""
    def local(start, count):
        f = np.asarray(fvals[start:start + count], dtype=np.float64)
        st = np.where(np.isnan(f), 5, 1).astype(np.int32)
        x = np.tile(np.arange(start, start + count, dtype=np.float64)[:, None], (1, DIM))
        c = census_host(f, st, x, KNOWN_MIN)
        if c.best_local >= 0:
            b = c.best_local
            c.fval, c.status, c.iter, c.gnorm, c.x = float(f[b]), int(st[b]), 7, 0.5, x[b]
        return c
    return local


def _worker(rank, world, port, q, case, n, payload):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = _oracle_local(n, KNOWN_MIN) if case == "oracle" else _synthetic_local(payload)
        m = sharded_call(n, DIM, local)
        q.put((rank, m.idx, m.status, m.fval, m.gnorm, m.iter, m.x.tolist(), m.actual,
               m.claimed, m.surrendered, m.stopped))
    finally:
        dist.destroy_process_group()


def _run(world, case, n, payload=None):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, case, n, payload))
             for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank holds the same merged result
    for g in got[1:]:
        assert g[1:] == got[0][1:]
    return got[0][1:]


@pytest.mark.parametrize("world,n", [(2, 37), (3, 20)])
def test_merged_oracle_runs_equal_the_single_process_census(world, n):
    from tests import _oracle as O

    r = O.oracle_bfgs(KIND, DIM, O.oracle_starts(SEED, n, DIM, LO, HI), max_iter=MAX_ITER)
    want = census_host(r["fval"], r["status"], r["x"], KNOWN_MIN)
    idx, status, fval, gnorm, it, x, actual, claimed, surr, stopped = _run(world, "oracle", n)
    b = want.best_local
    assert (actual, claimed, surr, stopped) == (want.actual, want.claimed, want.surrendered,
                                                want.stopped)
    assert claimed > 0 and actual > 0
    assert idx == b and fval == r["fval"][b] and status == r["status"][b]
    assert it == r["iter"][b] and gnorm == r["gnorm"][b]
    np.testing.assert_array_equal(np.asarray(x), r["x"][b])


def test_ties_go_to_the_lowest_global_index_and_nan_never_wins():
    # shards of 5 runs over 2 ranks: [0..2] on rank 0, [3..4] on rank 1; the
    # minimum 1.0 sits at 1 and 3, NaN at 0 and 4
    f = [math.nan, 1.0, 2.0, 1.0, math.nan]
    idx, status, fval, *_ , actual, claimed, surr, stopped = _run(2, "synthetic", 5, f)
    assert idx == 1 and fval == 1.0 and status == 1
    assert (claimed, surr, stopped) == (3, 2, 0)


def test_rank_without_runs():
    # one run over two ranks: rank 1 holds nothing
    idx, status, fval, *_ = _run(2, "synthetic", 1, [4.0])
    assert idx == 0 and fval == 4.0


def test_single_process_merge_is_the_local_census():
    local = _synthetic_local([3.0, 2.0, 2.0, 9.0])
    m = merge(local(0, 4), 0, 4, DIM)
    assert (m.idx, m.fval, m.claimed, m.surrendered) == (1, 2.0, 4, 0)
