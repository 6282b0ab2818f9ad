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
