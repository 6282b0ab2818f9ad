"""Multi-rank work split on CPU: gloo ranks count their shards and all-reduce; the sum must equal
the single-rank count bit for bit.

Each rank splits the centres (the endpoint with the larger out-degree of the edge each triangle
is found on) into contiguous ranges with the library's own split rule (tc_shard_ranges, the
function the GPU count applies to its device-side prefix), over the predicted work per centre,
and counts its range with the oracle. The ranges must also balance the predicted work."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _graph(kind):
    from custingeralg_b200 import generators as G
    if kind == "rmat":
        return G.rmat(12, 16, seed=2)
    return G.barabasi_albert(3000, 8, seed=3)


def _prefix(cost):
    return np.concatenate([[0], np.cumsum(cost, dtype=np.int64)])


def _worker(rank, world, port, kind, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from custingeralg_b200 import api
    from oracle import pyoracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = _graph(kind)
        lo = api.shard_ranges(_prefix(O.centre_cost(g.n, g.off, g.ind, nthreads=1)), world)
        tot, pv = O.fast_count_range(g.n, g.off, g.ind, int(lo[rank]), int(lo[rank + 1]), nthreads=1)
        t = torch.tensor([tot], dtype=torch.int64)
        p = torch.from_numpy(pv.astype(np.int32))
        dist.all_reduce(t)
        dist.all_reduce(p)
        if rank == 0:
            q.put((int(t.item()), p.numpy().copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,kind", [(2, "rmat"), (3, "rmat"), (4, "ba")])
def test_sharded_counts_sum_to_full(world, kind):
    from oracle import pyoracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, kind, q)) for r in range(world)]
    for p in procs:
        p.start()
    tot, pv = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = _graph(kind)
    ft, fpv = O.fast_count(g.n, g.off, g.ind)
    assert tot == ft
    assert np.array_equal(pv, fpv)


@pytest.mark.parametrize("world", [2, 4, 8])
def test_split_rule_balances_predicted_work(world):
    """Contiguous ranges that cover every centre once; no shard's predicted work exceeds the mean
    by more than the costliest single centre (the rule cuts at prefix quantiles)."""
    from custingeralg_b200 import api, generators as G
    from oracle import pyoracle as O
    g = G.rmat(14, 16, seed=2)
    cost = O.centre_cost(g.n, g.off, g.ind)
    pre = _prefix(cost)
    lo = api.shard_ranges(pre, world)
    assert lo[0] == 0 and lo[-1] == g.n and np.all(np.diff(lo) >= 0)
    work = pre[lo[1:]] - pre[lo[:-1]]
    assert work.sum() == pre[-1]
    assert work.max() <= pre[-1] / world + cost.max()


def test_split_rule_edge_cases():
    from custingeralg_b200 import api
    assert list(api.shard_ranges(np.zeros(1, np.int64), 3)) == [0, 0, 0, 0]          # no centres
    assert list(api.shard_ranges(np.array([0, 0, 0, 0]), 2)) == [0, 0, 3]            # no work
    assert list(api.shard_ranges(np.array([0, 5, 5, 10]), 2)) == [0, 1, 3]
    assert list(api.shard_ranges(np.array([0, 10]), 4)) == [0, 1, 1, 1, 1]           # one centre
