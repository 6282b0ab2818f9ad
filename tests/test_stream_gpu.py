"""Streaming updates on the GPU: structure and triangle deltas against the CPU oracle."""
import ctypes

import numpy as np
import pytest

from custingeralg_b200 import api, generators as G, native as N
from oracle import pyoracle as O
from tests.util import random_graph

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def edge_set(g):
    src = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(g.off))
    keep = src < g.ind
    return set(zip(src[keep].tolist(), g.ind[keep].tolist()))


def expected_after(n, edges, s, d, dele):
    """Set semantics: per undirected pair, deletions apply before insertions; self-loops ignored."""
    ops = {}
    for a, b, x in zip(s.tolist(), d.tolist(), dele.tolist()):
        if a == b:
            continue
        k = (min(a, b), max(a, b))
        dl, ins = ops.get(k, (False, False))
        ops[k] = (dl or bool(x), ins or not bool(x))
    out = set(edges)
    for k, (dl, ins) in ops.items():
        if dl and not ins:
            out.discard(k)
        if ins:
            out.add(k)
    if out:
        a = np.array(sorted(out), dtype=np.int32)
        return G.from_pairs(n, a[:, 0], a[:, 1])
    return G.from_pairs(n, [], [])


def random_batch(rng, g, k, del_frac=0.3):
    n = g.n
    s = rng.integers(0, n, k, dtype=np.int32)
    d = rng.integers(0, n, k, dtype=np.int32)
    dele = (rng.random(k) < del_frac).astype(np.uint8)
    if g.m:
        # deletions mostly of existing edges, plus repeats and self-loops
        src_of = np.repeat(np.arange(n, dtype=np.int32), np.diff(g.off))
        idx = rng.integers(0, g.m, k)
        pick = dele.astype(bool) & (rng.random(k) < 0.8)
        s[pick] = src_of[idx[pick]]
        d[pick] = g.ind[idx[pick]]
    if k > 4:
        s[-2], d[-2] = s[0], d[0]        # repeat
        s[-1] = d[-1] = s[1]             # self-loop
    return s, d, dele


@pytest.mark.parametrize("seed", range(12))
def test_apply_batch_random(seed):
    torch = _torch()
    rng = np.random.default_rng(seed)
    n = int(rng.integers(8, 2000))
    g = random_graph(rng, n, int(rng.integers(0, 12 * n)))
    slack = [0.0, 0.25, 1.0][seed % 3]
    graph = api.Graph.from_csr(g, slack=slack)
    pv = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    delta = torch.zeros(1, dtype=torch.int64, device="cuda")
    cur = g
    for step in range(4):
        k = int(rng.integers(1, 4 * n))
        s, d, dele = random_batch(rng, cur, k)
        before_pv = O.static_per_vertex(n, cur.off, cur.ind)
        before_T = O.host_count_triangles(n, cur.off, cur.ind)[0] // 6
        exp = expected_after(n, edge_set(cur), s, d, dele)
        info = graph.apply_batch(s, d, dele, per_vertex=pv, delta_dev=delta)
        off, ind = graph.export()
        assert np.array_equal(off, exp.off) and np.array_equal(ind, exp.ind), "structure mismatch"
        after_pv = O.static_per_vertex(n, exp.off, exp.ind)
        after_T = O.host_count_triangles(n, exp.off, exp.ind)[0] // 6
        assert info.triangles_added - info.triangles_removed == after_T - before_T
        assert info.inserted - info.deleted == (exp.m - cur.m) // 2
        # per-vertex running delta equals the per-vertex recount difference since the start
        want = (after_pv.astype(np.int64) - O.static_per_vertex(n, g.off, g.ind)).astype(np.int32)
        assert np.array_equal(pv[:n].cpu().numpy(), want)
        assert int(delta.item()) == after_T - O.host_count_triangles(n, g.off, g.ind)[0] // 6
        T, _ = graph.count(N.TC_PV_HANDLE, torch.zeros(n + 1, dtype=torch.int32, device="cuda"))
        assert T == after_T
        cur = exp
    graph.validate()


def test_apply_batch_device_arrays_and_edge_cases():
    torch = _torch()
    g = G.complete(6)
    graph = api.Graph.from_csr(g, slack=0.0)
    # empty batch
    info = graph.apply_batch(np.zeros(0, np.int32), np.zeros(0, np.int32))
    assert info.inserted == info.deleted == 0
    # delete and re-insert the same edge in one batch: no structural change, no delta
    s = torch.tensor([0, 0], dtype=torch.int32, device="cuda")
    d = torch.tensor([1, 1], dtype=torch.int32, device="cuda")
    dl = torch.tensor([1, 0], dtype=torch.uint8, device="cuda")
    info = graph.apply_batch(s, d, dl)
    assert info.inserted == 0 and info.deleted == 0
    # delete an absent edge, insert a present one: ignored
    info = graph.apply_batch(np.array([0, 2], np.int32), np.array([6 - 1, 3], np.int32), np.array([0, 0], np.uint8))
    assert info.inserted == 0
    # ids out of range are rejected
    with pytest.raises(N.TcError) as e:
        graph.apply_batch(np.array([0], np.int32), np.array([99], np.int32))
    assert e.value.status == N.TC_ERR_INVALID_ARG
    # removing every edge of K6 removes all 20 triangles
    src = np.repeat(np.arange(6, dtype=np.int32), np.diff(g.off))
    info = graph.apply_batch(src, g.ind, np.ones(g.m, np.uint8))
    assert info.deleted == 15 and info.triangles_removed == 20
    assert graph.info()[1] == 0
    # and inserting them back (into zero-capacity lists: every list moves) restores them
    info = graph.apply_batch(src, g.ind)
    assert info.inserted == 15 and info.triangles_added == 20
    off, ind = graph.export()
    assert np.array_equal(off, g.off) and np.array_equal(ind, g.ind)


def test_pool_growth_many_insertions():
    rng = np.random.default_rng(7)
    n = 3000
    g = random_graph(rng, n, 2 * n)
    graph = api.Graph.from_csr(g, slack=0.0)
    cur = g
    for _ in range(3):
        s = rng.integers(0, n, 40 * n, dtype=np.int32)
        d = rng.integers(0, n, 40 * n, dtype=np.int32)
        exp = expected_after(n, edge_set(cur), s, d, np.zeros(s.size, np.uint8))
        info = graph.apply_batch(s, d)
        off, ind = graph.export()
        assert np.array_equal(off, exp.off) and np.array_equal(ind, exp.ind)
        assert info.triangles_added == (O.host_count_triangles(n, exp.off, exp.ind)[0]
                                        - O.host_count_triangles(n, cur.off, cur.ind)[0]) // 6
        cur = exp


def _cus_batch(n, s, d, graph):
    """cuStinger-style steps through the C ABI: sort, then return device arrays."""
    torch = _torch()
    ds = torch.from_numpy(np.ascontiguousarray(s, np.int32)).cuda()
    dd = torch.from_numpy(np.ascontiguousarray(d, np.int32)).cuda()
    off = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    dup = torch.zeros(max(len(s), 1), dtype=torch.int32, device="cuda")
    N.check(N.lib().tc_batch_sort(n, ds.data_ptr(), dd.data_ptr(), len(s), off.data_ptr(), dup.data_ptr(), None))
    return ds, dd, off, dup


@pytest.mark.parametrize("strategy", [None, 0, 1, 2])
@pytest.mark.parametrize("seed", range(8))
def test_custinger_path_matches_reference_kernels(seed, strategy):
    """sortDeviceBUD + edgeInsertionsSorted + callDeviceNewTriangles == K1 + K2 - K3 (oracle),
    with the default rule and with every degree cell forced to one intersection strategy
    (0 search, 1 merge, 2 staged in shared memory)."""
    from custingeralg_b200 import sched_learn as L
    sched = None if strategy is None else L.forced(strategy)
    sp = None if sched is None else ctypes.byref(sched)
    torch = _torch()
    rng = np.random.default_rng(50 + seed)
    n = int(rng.integers(8, 800))
    base = random_graph(rng, n, int(rng.integers(n, 10 * n)))
    k = int(rng.integers(1, 3 * n))
    s = rng.integers(0, n, k, dtype=np.int32)
    d = rng.integers(0, n, k, dtype=np.int32)
    if base.m:
        e = rng.integers(0, base.m, 6)
        src_of = np.repeat(np.arange(n, dtype=np.int32), np.diff(base.off))
        s = np.concatenate([s, s[:3], src_of[e]]).astype(np.int32)
        d = np.concatenate([d, d[:3], base.ind[e]]).astype(np.int32)
    bs = np.concatenate([s, d]).astype(np.int32)
    bd = np.concatenate([d, s]).astype(np.int32)
    graph = api.Graph.from_csr(base, slack=0.5)
    ds, dd, off, dup = _cus_batch(n, bs, bd, graph)
    # oracle: sort, flag against the graph before insertion, K1 + K2 - K3 after insertion
    ss, sd, boff, odup = O.sort_batch(n, base.off, base.ind, bs, bd)
    assert np.array_equal(ds.cpu().numpy(), ss) and np.array_equal(dd.cpu().numpy(), sd)
    assert np.array_equal(off.cpu().numpy(), boff.astype(np.int32))
    moved = ctypes.c_int64()
    N.check(N.lib().tc_insert_sorted(graph.handle, ds.data_ptr(), dd.data_ptr(), bs.size, dup.data_ptr(),
                                     ctypes.byref(moved), None))
    assert np.array_equal(dup.cpu().numpy()[: bs.size], odup)
    after = G.from_pairs(n, np.concatenate([np.repeat(np.arange(n, dtype=np.int32), np.diff(base.off)), ss]),
                         np.concatenate([base.ind, sd]))
    o2, i2 = graph.export()
    assert np.array_equal(o2, after.off) and np.array_equal(i2, after.ind)
    pv = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    delta = torch.zeros(1, dtype=torch.int64, device="cuda")
    N.check(N.lib().tc_count_batch(graph.handle, ds.data_ptr(), dd.data_ptr(), off.data_ptr(), dup.data_ptr(),
                                   bs.size, 1, pv.data_ptr(), delta.data_ptr(), sp, None))
    want = O.new_triangles(n, after.off, after.ind, ss, sd, boff, odup)
    assert np.array_equal(pv[:n].cpu().numpy(), want)
    assert int(delta.item()) == (O.host_count_triangles(n, after.off, after.ind)[0]
                                 - O.host_count_triangles(n, base.off, base.ind)[0]) // 6
    # deletion of the same batch: count before, then delete, back to the base graph
    pv2 = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    N.check(N.lib().tc_count_batch(graph.handle, ds.data_ptr(), dd.data_ptr(), off.data_ptr(), dup.data_ptr(),
                                   bs.size, -1, pv2.data_ptr(), None, sp, None))
    # dup now flags the pre-existing entries, so exactly the inserted edges go away
    N.check(N.lib().tc_delete_sorted(graph.handle, ds.data_ptr(), dd.data_ptr(), dup.data_ptr(), bs.size, None))
    o3, i3 = graph.export()
    assert np.array_equal(o3, base.off) and np.array_equal(i3, base.ind)
    assert np.array_equal(pv2[:n].cpu().numpy(), (-want.astype(np.int64)).astype(np.int32))


@pytest.mark.parametrize("strategy", [None, 2])
def test_custinger_path_splits_hub_hub_intersections(strategy):
    """callDeviceNewTriangles on hub-hub edges (both lists > 2048, counted in queued chunks)
    equals the reference's K1 + K2 - K3 on the oracle, per vertex; the deletion count of the same
    edges gives the negative. Strategy 2 stages every intersection in shared memory."""
    from custingeralg_b200 import sched_learn as L
    sp = None if strategy is None else ctypes.byref(L.forced(strategy))
    torch = _torch()
    rng = np.random.default_rng(91)
    n, hubs = 9000, 4
    pool = rng.choice(np.arange(hubs, n), 4000, replace=False).astype(np.int32)
    src = np.concatenate([np.full(3000, h, np.int32) for h in range(hubs)] + [rng.integers(0, n, 8000).astype(np.int32)])
    dst = np.concatenate([rng.choice(pool, 3000, replace=False) for _ in range(hubs)] +
                         [rng.integers(0, n, 8000).astype(np.int32)])
    base = G.from_pairs(n, src, dst)
    pairs = np.array([(a, b) for a in range(hubs) for b in range(a + 1, hubs)], np.int32)
    s = np.concatenate([pairs[:, 0], rng.integers(0, n, 50).astype(np.int32)])
    d = np.concatenate([pairs[:, 1], rng.integers(0, n, 50).astype(np.int32)])
    bs = np.concatenate([s, d]).astype(np.int32)
    bd = np.concatenate([d, s]).astype(np.int32)
    graph = api.Graph.from_csr(base, slack=0.5)
    ds, dd, off, dup = _cus_batch(n, bs, bd, graph)
    ss, sd, boff, odup = O.sort_batch(n, base.off, base.ind, bs, bd)
    N.check(N.lib().tc_insert_sorted(graph.handle, ds.data_ptr(), dd.data_ptr(), bs.size, dup.data_ptr(), None, None))
    after = G.from_pairs(n, np.concatenate([np.repeat(np.arange(n, dtype=np.int32), np.diff(base.off)), ss]),
                         np.concatenate([base.ind, sd]))
    assert min(np.diff(after.off)[:hubs]) > 2048
    pv = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    delta = torch.zeros(1, dtype=torch.int64, device="cuda")
    N.check(N.lib().tc_count_batch(graph.handle, ds.data_ptr(), dd.data_ptr(), off.data_ptr(), dup.data_ptr(),
                                   bs.size, 1, pv.data_ptr(), delta.data_ptr(), sp, None))
    want = O.new_triangles(n, after.off, after.ind, ss, sd, boff, odup)
    assert np.array_equal(pv[:n].cpu().numpy(), want)
    t_after = O.host_count_triangles(n, after.off, after.ind)[0] // 6
    t_base = O.host_count_triangles(n, base.off, base.ind)[0] // 6
    assert int(delta.item()) == t_after - t_base > 0
    pv2 = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    delta2 = torch.zeros(1, dtype=torch.int64, device="cuda")
    N.check(N.lib().tc_count_batch(graph.handle, ds.data_ptr(), dd.data_ptr(), off.data_ptr(), dup.data_ptr(),
                                   bs.size, -1, pv2.data_ptr(), delta2.data_ptr(), sp, None))
    assert np.array_equal(pv2[:n].cpu().numpy(), -want)
    assert int(delta2.item()) == -(t_after - t_base)
