"""bench.py's host logic on CPU: the launcher's checks and the reference arm's graph loading.

The reference arm reads its graph from the library's binary CSR cache with numpy alone (so its
process maps no library of this repository); that reader must give back the generator's CSR.
The launcher must refuse rank counts it cannot honour instead of silently running one rank."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_binary_cache_reader_matches_the_generator(tmp_path):
    from custingeralg_b200 import generators as G
    g = G.rmat(12, 16, seed=5)
    path = str(tmp_path / "g.tccsr")
    bench.generate_in_child(["rmat", "--scale", "12", "--edge-factor", "16", "--seed", "5"], path)
    h = bench.read_tccsr(path)
    assert h.n == g.n and h.m == g.m
    assert np.array_equal(h.off, g.off) and np.array_equal(h.ind, g.ind)
    assert bench.edges_intersected_host(h) == bench.edges_intersected_host(g)


def test_workload_config_is_the_same_in_both_arms():
    a = bench.workload_config(20, 16, 2, 1 << 20, 31401752, 15561271)
    b = bench.workload_config(20, 16, 2, 1 << 20, 31401752, 15561271)
    assert a == b and "scheduler" not in a


def _run(args, env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, capture_output=True, text=True,
                          env=env, timeout=300)


def test_launcher_refuses_a_rank_count_it_cannot_honour():
    # the launcher started a different number of ranks than --gpus asks for
    r = _run(["--gpus", "2"], {"WORLD_SIZE": "1", "RANK": "0", "LOCAL_RANK": "0"})
    assert r.returncode != 0 and "launcher started 1 ranks" in (r.stdout + r.stderr)
    r = _run(["--gpus", "0"], {})
    assert r.returncode != 0
    # more ranks than visible devices (none here): refused, not run as one rank
    r = _run(["--gpus", "2"], {"CUDA_VISIBLE_DEVICES": ""})
    assert r.returncode != 0 and "CUDA devices are visible" in (r.stdout + r.stderr)


class _GlooCtx:
    """The part of bench.Ctx that rmat_graph uses, over a gloo process group."""

    def __init__(self, rank, world):
        self.rank, self.world = rank, world

    def barrier(self):
        import torch.distributed as dist
        dist.barrier()


def _shared_graph_worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench as B
    from custingeralg_b200 import generators as G
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = B.rmat_graph(_GlooCtx(rank, world), 11, 16, 3)
        ref = G.rmat(11, 16, seed=3)
        q.put((rank, g.n == ref.n and np.array_equal(g.off, ref.off) and np.array_equal(g.ind, ref.ind)))
    finally:
        dist.destroy_process_group()


def test_ranks_share_one_generated_graph():
    """With several ranks, rank 0 generates each bench graph once and the others read it back
    from a binary file: every rank must hold the generator's CSR, and the file is removed."""
    import socket
    import tempfile

    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shared_graph_worker, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    assert all(p.exitcode == 0 for p in procs)
    got = dict(q.get(timeout=5) for _ in procs)
    assert got == {0: True, 1: True, 2: True}
    assert not os.path.exists(os.path.join(tempfile.gettempdir(), f"tc_bench_{port}_rmat11_16_3.tccsr"))


def test_stream_plan_round_trips_through_a_bench_line(tmp_path):
    """--stream-plan reads the bins a bench line recorded back into the pipeline plan they came
    from: capacities, the bin serving each one and its tile shape."""
    bins = [{"capacity": 1024, "served_by_capacity": 4096, "delta_ctas_per_sm": 6, "plan_ctas_per_sm": 0,
             "split_min": 128, "chunk": 64},
            {"capacity": 2048, "served_by_capacity": 4096, "delta_ctas_per_sm": 6, "plan_ctas_per_sm": 0,
             "split_min": 128, "chunk": 64},
            {"capacity": 4096, "served_by_capacity": 4096, "delta_ctas_per_sm": 6, "plan_ctas_per_sm": 0,
             "split_min": 256, "chunk": 128},
            {"capacity": 8192, "served_by_capacity": 8192, "delta_ctas_per_sm": 6,
             "split_min": 512, "chunk": 256}]
    path = tmp_path / "line.json"
    path.write_text("noise before the line\n" + __import__("json").dumps({"streaming": {"bins": bins}}) + "\n")
    p = bench.plan_from_bench(str(path))
    assert p.nbins == 4
    assert list(p.bin_cap)[:4] == [1024, 2048, 4096, 8192]
    assert list(p.serve)[:4] == [2, 2, 2, 3]
    assert list(p.split_min)[:4] == [128, 128, 256, 512] and list(p.chunk)[:4] == [64, 64, 128, 256]
    assert list(p.ctas_per_sm)[:4] == [0, 0, 0, 0]
