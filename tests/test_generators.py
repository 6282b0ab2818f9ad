"""Generator invariants: symmetric, sorted, no self-loops or duplicates, deterministic."""
import numpy as np
import pytest

from custingeralg_b200 import generators as G


def check_simple_symmetric(g):
    off, ind = g.off, g.ind
    assert off[0] == 0 and np.all(np.diff(off) >= 0) and off[-1] == ind.size
    src = np.repeat(np.arange(g.n), np.diff(off))
    assert np.all(src != ind)
    for v in range(g.n):
        lst = ind[off[v]:off[v + 1]]
        assert np.all(np.diff(lst) > 0)
    a = set(zip(src.tolist(), ind.tolist()))
    assert all((d, s) in a for s, d in a)


@pytest.mark.parametrize("make", [
    lambda nt: G.rmat(8, 8, seed=3, nthreads=nt),
    lambda nt: G.rmat(8, 8, seed=3, noise=True, nthreads=nt),
    lambda nt: G.erdos_renyi(500, 0.02, seed=4, nthreads=nt),
    lambda nt: G.barabasi_albert(400, 4, seed=5, nthreads=nt),
    lambda nt: G.grid_rewired(20, 0.05, seed=6, nthreads=nt),
])
def test_invariants_and_thread_independence(make):
    a = make(1)
    b = make(4)
    check_simple_symmetric(a)
    assert np.array_equal(a.off, b.off) and np.array_equal(a.ind, b.ind)


def test_rmat_sizes():
    g = G.rmat(10, 16, seed=2)
    assert g.n == 1024 and 0 < g.m <= 2 * 16 * 1024
    deg = g.degrees()
    assert deg.max() > 10 * deg.mean()  # heavy-tailed


def test_er_density():
    n = 1 << 14
    g = G.erdos_renyi(n, 16.0 / n, seed=1)
    assert abs(g.m / n - 16.0) < 0.5
