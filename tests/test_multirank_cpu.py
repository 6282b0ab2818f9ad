"""Multi-rank work split on CPU: two gloo ranks count their shards (the split the GPU kernel
uses: c % nshards over the centre c of the edge each triangle is found on) and all-reduce; the
sum must equal the single-rank count bit for bit."""
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


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from custingeralg_b200 import generators as G
    from oracle import pyoracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = G.rmat(12, 16, seed=2)
        tot, pv = O.fast_count_shard(g.n, g.off, g.ind, rank, world, nthreads=1)
        t = torch.tensor([tot], dtype=torch.int64)
        p = torch.from_numpy(pv.astype(np.int32))
        dist.all_reduce(t)
        dist.all_reduce(p)
        if rank == 0:
            q.put((int(t.item()), p.numpy().copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_counts_sum_to_full(world):
    from custingeralg_b200 import generators as G
    from oracle import pyoracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    tot, pv = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = G.rmat(12, 16, seed=2)
    ft, fpv = O.fast_count(g.n, g.off, g.ind)
    assert tot == ft
    assert np.array_equal(pv, fpv)
