"""CPU oracle checks: restatement vs the reference's own counter and the golden fixtures."""
import numpy as np
import pytest

from custingeralg_b200 import generators as G
from oracle import pyoracle as O
from tests.util import digest, golden_graph, load_golden, random_graph

GOLD = load_golden()["graphs"]


@pytest.mark.parametrize("name", sorted(GOLD))
def test_oracle_matches_golden(name):
    rec = GOLD[name]
    g = golden_graph(name)
    assert digest(g.off) + digest(g.ind) == rec["graph_digest"], "generator drift"
    tot, tri = O.host_count_triangles(g.n, g.off, g.ind, per_edge=True)
    assert tot == rec["ref_all_triangles"]
    assert digest(tri) == rec["triNE_digest"]
    pv = O.static_per_vertex(g.n, g.off, g.ind)
    cpv = O.csr_per_vertex(g.n, g.off, g.ind)
    assert digest(pv) == rec["per_vertex_handle_digest"]
    assert digest(cpv) == rec["per_vertex_csr_digest"]
    assert int(pv.astype(np.int64).sum()) == 6 * rec["triangles"]
    assert int(cpv.astype(np.int64).sum()) == 3 * rec["triangles"]
    ft, fpv = O.fast_count(g.n, g.off, g.ind)
    assert ft == rec["ref_all_triangles"] and np.array_equal(fpv, pv)


def test_known_answers():
    for n in (3, 4, 5, 6, 10, 20):
        g = G.complete(n)
        assert O.host_count_triangles(g.n, g.off, g.ind)[0] == 6 * (n * (n - 1) * (n - 2) // 6)
    assert O.host_count_triangles(*(lambda g: (g.n, g.off, g.ind))(G.star(50)))[0] == 0


@pytest.mark.skipif(not O.ref_available(), reason="reference counter not built (no reference sources)")
@pytest.mark.parametrize("seed", range(6))
def test_restatement_vs_reference_random(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 300))
    g = random_graph(rng, n, int(rng.integers(0, 4 * n)))
    a, ta = O.host_count_triangles(g.n, g.off, g.ind, per_edge=True)
    b, tb = O.ref_host_count_triangles(g.n, g.off, g.ind, per_edge=True)
    assert a == b and np.array_equal(ta, tb)
    assert O.ref_host_count_triangles_omp(g.n, g.off, g.ind) == b
    for i in range(min(g.n, 20)):
        for j in range(min(g.n, 20)):
            la, lb = g.ind[g.off[i]:g.off[i + 1]], g.ind[g.off[j]:g.off[j + 1]]
            x = O.lib().oracle_single_intersection(la.size, la.ctypes.data if la.size else None, lb.size,
                                                   lb.ctypes.data if lb.size else None)
            y = O.ref().ref_host_single_intersection(i, la.size, la.ctypes.data if la.size else None, j, lb.size,
                                                    lb.ctypes.data if lb.size else None)
            assert x == y == len(np.intersect1d(la, lb))


@pytest.mark.parametrize("seed", range(8))
def test_streaming_identity(seed):
    """K1 + K2 - K3 per vertex == static(after) - static(before) (tests/cct_upd.cpp:407-414)."""
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(5, 120))
    base = random_graph(rng, n, int(rng.integers(0, 3 * n)))
    k = int(rng.integers(1, 2 * n))
    s = rng.integers(0, n, k, dtype=np.int32)
    d = rng.integers(0, n, k, dtype=np.int32)
    # in-batch duplicates and edges already present, like tests/cct_upd.cpp:313-332
    if base.m:
        e = rng.integers(0, base.m, 5)
        src_of = np.repeat(np.arange(n, dtype=np.int32), np.diff(base.off))
        s = np.concatenate([s, s[:3], src_of[e]]).astype(np.int32)
        d = np.concatenate([d, d[:3], base.ind[e]]).astype(np.int32)
    bs = np.concatenate([s, d]).astype(np.int32)   # symmetric batch (tests/cct_upd.cpp:337-341)
    bd = np.concatenate([d, s]).astype(np.int32)
    ss, sd, boff, dup = O.sort_batch(n, base.off, base.ind, bs, bd)
    after = G.from_pairs(n, np.concatenate([np.repeat(np.arange(n, dtype=np.int32), np.diff(base.off)), ss]),
                         np.concatenate([base.ind, sd]))
    delta = O.new_triangles(n, after.off, after.ind, ss, sd, boff, dup)
    before_pv = O.static_per_vertex(n, base.off, base.ind)
    after_pv = O.static_per_vertex(n, after.off, after.ind)
    assert np.array_equal(delta, (after_pv.astype(np.int64) - before_pv).astype(np.int32))
