"""Captured streaming pipeline (tc_pipeline_*): the same results as tc_apply_batch, batch by batch.

Every batch goes through the pipeline on one graph and through tc_apply_batch on a twin graph;
after each batch the running totals, the per-vertex deltas and a full static recount must agree,
bit for bit. Batch sizes span several bins (1 .. 20000 updates), so several captured graphs run.
"""
import numpy as np
import pytest

from custingeralg_b200 import api, generators as G, native as N
from tests.test_stream_gpu import edge_set, expected_after, random_batch

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _recount(graph, n):
    torch = _torch()
    out = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    T, _ = graph.count(N.TC_PV_HANDLE, out)
    return T, out[:n].clone()


def _dev(torch, s, d, x):
    return (torch.from_numpy(np.ascontiguousarray(s)).cuda(), torch.from_numpy(np.ascontiguousarray(d)).cuda(),
            torch.from_numpy(np.ascontiguousarray(x)).cuda())


@pytest.mark.parametrize("slack", [0.0, 0.25])
def test_pipeline_matches_apply_batch(slack):
    torch = _torch()
    rng = np.random.default_rng(7)
    base = G.rmat(13, 16, seed=11)
    g_pipe = api.Graph.from_csr(base, slack=slack)
    g_ref = api.Graph.from_csr(base, slack=slack)
    n = base.n
    T0, pv0 = _recount(g_pipe, n)
    pipe = api.Pipeline(g_pipe, 1 << 15)
    pv_p = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    pv_r = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    dp = torch.zeros(1, dtype=torch.int64, device="cuda")
    dr = torch.zeros(1, dtype=torch.int64, device="cuda")
    cur = base
    for k in [1, 3, 37, 600, 5000, 20000, 2, 1500, 9000, 64]:
        s, d, x = random_batch(rng, cur, k)
        ts, td, tx = _dev(torch, s, d, x)
        pipe.apply(ts, td, tx, per_vertex=pv_p, delta_dev=dp)
        info = pipe.sync()
        ref = g_ref.apply_batch(ts, td, tx, per_vertex=pv_r, delta_dev=dr)
        assert (info.inserted, info.deleted, info.triangles_added, info.triangles_removed) == \
            (ref.inserted, ref.deleted, ref.triangles_added, ref.triangles_removed)
        assert int(dp.item()) == int(dr.item())
        assert torch.equal(pv_p, pv_r)
        T, pv = _recount(g_pipe, n)
        assert T == T0 + int(dp.item())
        assert torch.equal(pv, (pv0.to(torch.int64) + pv_p[:n].to(torch.int64)).to(torch.int32))
        off, ind = g_pipe.export()
        cur = G.Csr(n, off, ind)
    pipe.close()


def test_pipeline_autotune_keeps_counts_and_picks_a_grid():
    torch = _torch()
    rng = np.random.default_rng(3)
    base = G.rmat(12, 16, seed=5)
    graph = api.Graph.from_csr(base, slack=0.25)
    n = base.n
    T0, _ = _recount(graph, n)
    pipe = api.Pipeline(graph, 1 << 12)
    pipe.autotune(12)
    delta = torch.zeros(1, dtype=torch.int64, device="cuda")
    for i in range(16):
        s, d, x = random_batch(rng, base, int(rng.integers(1, 4000)))
        pipe.apply(*_dev(torch, s, d, x), delta_dev=delta)
    pipe.sync()
    T, _ = _recount(graph, n)
    assert T == T0 + int(delta.item())
    bins = pipe.info()
    assert [c for c, _ in bins] == [1 << 10, 1 << 11, 1 << 12]
    assert all(1 <= b <= 16 for _, b in bins)
    plan = pipe.plan()
    assert plan.nbins == 3
    for i in range(3):
        assert i <= plan.serve[i] < 3 and (i == 0 or plan.serve[i] >= plan.serve[i - 1])
        assert plan.split_min[i] == 2 * plan.chunk[i]
    pipe.close()


def _apply_both(torch, pipe, g_ref, batches, n):
    """Run the batches through the pipeline and through tc_apply_batch on a twin; compare."""
    pv_p = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    pv_r = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    dp = torch.zeros(1, dtype=torch.int64, device="cuda")
    dr = torch.zeros(1, dtype=torch.int64, device="cuda")
    for s, d, x in batches:
        ts, td, tx = _dev(torch, s, d, x)
        pipe.apply(ts, td, tx, per_vertex=pv_p, delta_dev=dp)
        pipe.sync()
        g_ref.apply_batch(ts, td, tx, per_vertex=pv_r, delta_dev=dr)
    assert int(dp.item()) == int(dr.item())
    assert torch.equal(pv_p, pv_r)
    return int(dp.item())


@pytest.mark.parametrize("shape", [(0, 1024, 2048), (0, 512, 1024), (0, 256, 512), (0, 128, 256),
                                   (0, 64, 128)])
def test_every_tile_shape_counts_the_same(shape):
    """Each candidate tile shape of the persistent delta kernel (CTAs per SM, split-item size,
    split threshold), set through a plan, gives tc_apply_batch's results on hub-heavy batches
    (hub lists of 3000-6000 entries, so hub-hub intersections are split at every threshold)."""
    torch = _torch()
    rng = np.random.default_rng(40)
    n = 9000
    hubs = np.arange(6, dtype=np.int32)
    src, dst = [], []
    for h in hubs:
        nb = rng.choice(np.arange(6, n), int(rng.integers(3000, 6000)), replace=False).astype(np.int32)
        src.append(np.full(nb.size, h, np.int32))
        dst.append(nb)
    src.append(rng.integers(0, n, 30000).astype(np.int32))
    dst.append(rng.integers(0, n, 30000).astype(np.int32))
    base = G.from_pairs(n, np.concatenate(src), np.concatenate(dst))
    g_pipe = api.Graph.from_csr(base, slack=0.25)
    g_ref = api.Graph.from_csr(base, slack=0.25)
    pipe = api.Pipeline(g_pipe, 1 << 13)
    plan = pipe.plan()
    for i in range(plan.nbins):
        plan.serve[i] = i
        plan.ctas_per_sm[i], plan.chunk[i], plan.split_min[i] = shape
    pipe.set_plan(plan)
    batches = []
    for k in [40, 900, 5000]:
        # hub-hub edges (both endpoints hubs) and edges into the hubs' neighbourhoods
        s = np.concatenate([rng.choice(hubs, k // 4), rng.integers(0, n, k - k // 4)]).astype(np.int32)
        d = np.concatenate([rng.choice(hubs, k // 4), rng.integers(0, n, k - k // 4)]).astype(np.int32)
        x = (rng.random(k) < 0.3).astype(np.uint8)
        batches.append((s, d, x))
    T0, _ = _recount(g_pipe, n)
    delta = _apply_both(torch, pipe, g_ref, batches, n)
    T, _ = _recount(g_pipe, n)
    assert T == T0 + delta
    pipe.close()


def test_plan_carries_over_to_a_second_pipeline():
    """Tune on one graph, carry the plan to a pipeline on a twin graph: same shapes, same counts."""
    torch = _torch()
    rng = np.random.default_rng(9)
    base = G.rmat(12, 16, seed=8)
    n = base.n
    g_tune = api.Graph.from_csr(base, slack=0.25)
    tuner = api.Pipeline(g_tune, 1 << 13)
    tuner.autotune(30)
    for i in range(30):
        s, d, x = random_batch(rng, base, int(np.exp(rng.uniform(0, np.log(8000)))))
        tuner.apply(*_dev(torch, s, d, x))
    tuner.sync()
    plan = tuner.plan()
    tuner.close()
    g_pipe = api.Graph.from_csr(base, slack=0.25)
    g_ref = api.Graph.from_csr(base, slack=0.25)
    pipe = api.Pipeline(g_pipe, 1 << 13)
    pipe.set_plan(plan)
    got = pipe.plan()
    for i in range(plan.nbins):
        assert (got.serve[i], got.ctas_per_sm[i], got.chunk[i], got.split_min[i]) == \
            (plan.serve[i], plan.ctas_per_sm[i], plan.chunk[i], plan.split_min[i])
    T0, _ = _recount(g_pipe, n)
    batches = [random_batch(rng, base, k) for k in (5, 300, 2500, 7000)]
    delta = _apply_both(torch, pipe, g_ref, batches, n)
    T, _ = _recount(g_pipe, n)
    assert T == T0 + delta
    pipe.close()


def test_delta_kernel_wait_bound_reports_timeout_and_device_stays_usable():
    """The persistent delta kernel's wait for queued work is bounded. Made to wait for a warp
    that never finishes its entry pass (one beyond the grid), the waiting warps give up after the
    bound (1 ms here), the batch reports TC_ERR_TIMEOUT, and the device keeps working: the
    structure update completed, a recount runs, and later batches count right again with the
    normal bound."""
    torch = _torch()
    rng = np.random.default_rng(12)
    base = G.rmat(11, 16, seed=3)
    n = base.n
    graph = api.Graph.from_csr(base, slack=0.25)
    pipe = api.Pipeline(graph, 1 << 12)
    pipe.set_wait_bound(1_000_000, 1)
    s, d, x = random_batch(rng, base, 800)
    pipe.apply(*_dev(torch, s, d, x))
    with pytest.raises(N.TcError) as ei:
        pipe.sync()
    assert ei.value.status == N.TC_ERR_TIMEOUT
    pipe.set_wait_bound(2_000_000_000, 0)
    T1, _ = _recount(graph, n)
    delta = torch.zeros(1, dtype=torch.int64, device="cuda")
    off, ind = graph.export()
    cur = G.Csr(n, off, ind)
    for k in (3, 500, 3000):
        s, d, x = random_batch(rng, cur, k)
        pipe.apply(*_dev(torch, s, d, x), delta_dev=delta)
        pipe.sync()
    T2, _ = _recount(graph, n)
    assert T2 == T1 + int(delta.item())
    pipe.close()


def test_streaming_shards_add_up():
    """Two ranks' shares of the delta count (the changed edges whose key hashes to 0 and to 1), run
    one after the other on twin graphs, add up to the unsharded count, totals and per-vertex."""
    torch = _torch()
    rng = np.random.default_rng(14)
    base = G.rmat(12, 16, seed=6)
    n = base.n
    batches = [random_batch(rng, base, k) for k in (7, 700, 4000)]
    parts = []
    for shard in range(2):
        g = api.Graph.from_csr(base, slack=0.25)
        sch = N.default_sched()
        sch.shard, sch.nshards = shard, 2
        pipe = api.Pipeline(g, 1 << 12, sched=sch)
        pv = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
        dl = torch.zeros(1, dtype=torch.int64, device="cuda")
        for s, d, x in batches:
            pipe.apply(*_dev(torch, s, d, x), per_vertex=pv, delta_dev=dl)
            pipe.sync()
        parts.append((int(dl.item()), pv.clone()))
        pipe.close()
    g_full = api.Graph.from_csr(base, slack=0.25)
    pv_f = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    d_f = torch.zeros(1, dtype=torch.int64, device="cuda")
    for s, d, x in batches:
        g_full.apply_batch(*_dev(torch, s, d, x), per_vertex=pv_f, delta_dev=d_f)
    assert parts[0][0] + parts[1][0] == int(d_f.item())
    assert torch.equal(parts[0][1] + parts[1][1], pv_f)


def test_pipeline_rejects_oversize_batch_and_recaptures_on_new_outputs():
    torch = _torch()
    rng = np.random.default_rng(5)
    base = G.rmat(11, 8, seed=2)
    graph = api.Graph.from_csr(base)
    n = base.n
    T0, _ = _recount(graph, n)
    pipe = api.Pipeline(graph, 1000)   # one bin of 1024
    s, d, x = random_batch(rng, base, 1500)
    with pytest.raises(N.TcError):
        pipe.apply(*_dev(torch, s, d, x))
    total = 0
    for i in range(3):
        delta = torch.zeros(1, dtype=torch.int64, device="cuda")   # a new output array each time
        s, d, x = random_batch(rng, base, 500)
        pipe.apply(*_dev(torch, s, d, x), delta_dev=delta)
        pipe.sync()
        total += int(delta.item())
    T, _ = _recount(graph, n)
    assert T == T0 + total
    pipe.close()


@pytest.mark.parametrize("path", ["pipeline", "apply"])
def test_long_lists_insert_and_delete(path):
    """Hub lists above 2048 entries take the long-list kernels (k_long_plan/stage/write, k_compact_long)."""
    torch = _torch()
    rng = np.random.default_rng(21)
    n = 12000
    hub_nb = rng.choice(np.arange(1, n), 5000, replace=False).astype(np.int32)
    ru = rng.integers(0, n, 40000).astype(np.int32)
    rv = rng.integers(0, n, 40000).astype(np.int32)
    src = np.concatenate([np.zeros(hub_nb.size, np.int32), ru, np.full(2500, 7, np.int32)])
    dst = np.concatenate([hub_nb, rv, rng.integers(0, n, 2500).astype(np.int32)])
    base = G.from_pairs(n, src, dst)
    assert np.diff(base.off).max() > 2048
    graph = api.Graph.from_csr(base, slack=0.1)
    T0, pv0 = _recount(graph, n)
    pipe = api.Pipeline(graph, 1 << 14) if path == "pipeline" else None
    pv = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    delta = torch.zeros(1, dtype=torch.int64, device="cuda")
    cur = base
    for it in range(4):
        k = 6000
        s = np.where(rng.random(k) < 0.5, 0, rng.integers(0, n, k)).astype(np.int32)  # half touch the hub
        d = rng.integers(0, n, k).astype(np.int32)
        x = np.zeros(k, np.uint8)
        src_of = np.repeat(np.arange(n, dtype=np.int32), np.diff(cur.off))
        hub_edges = np.nonzero(src_of == 0)[0]
        pick = rng.choice(hub_edges, 1500, replace=False)
        s[:1500], d[:1500], x[:1500] = 0, cur.ind[pick], 1    # delete 1500 hub edges
        ts, td, tx = _dev(torch, s, d, x)
        if pipe is not None:
            pipe.apply(ts, td, tx, per_vertex=pv, delta_dev=delta)
            pipe.sync()
        else:
            graph.apply_batch(ts, td, tx, per_vertex=pv, delta_dev=delta)
        want = expected_after(n, edge_set(cur), s, d, x)
        off, ind = graph.export()
        assert np.array_equal(off, want.off) and np.array_equal(ind, want.ind)
        cur = G.Csr(n, off, ind)
        T, pvn = _recount(graph, n)
        assert T == T0 + int(delta.item())
        assert torch.equal(pvn, (pv0.to(torch.int64) + pv[:n].to(torch.int64)).to(torch.int32))
    if pipe is not None:
        pipe.close()


def test_custinger_path_long_lists_round_trip():
    """edgeInsertionsSorted then edgeDeletionsSorted of the same batch on hub lists > 2048."""
    torch = _torch()
    rng = np.random.default_rng(33)
    n = 9000
    nb = rng.choice(np.arange(1, n), 4000, replace=False).astype(np.int32)
    base = G.from_pairs(n, np.concatenate([np.zeros(nb.size, np.int32), rng.integers(0, n, 20000).astype(np.int32)]),
                        np.concatenate([nb, rng.integers(0, n, 20000).astype(np.int32)]))
    graph = api.Graph.from_csr(base, slack=0.0)
    k = 3000
    u = np.where(rng.random(k) < 0.6, 0, rng.integers(0, n, k)).astype(np.int32)
    v = rng.integers(0, n, k).astype(np.int32)
    s = np.concatenate([u, v])
    d = np.concatenate([v, u])
    ds = torch.from_numpy(s).cuda()
    dd = torch.from_numpy(d).cuda()
    off = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    dup = torch.zeros(s.size, dtype=torch.int32, device="cuda")
    N.check(N.lib().tc_batch_sort(n, ds.data_ptr(), dd.data_ptr(), s.size, off.data_ptr(), dup.data_ptr(), None))
    N.check(N.lib().tc_insert_sorted(graph.handle, ds.data_ptr(), dd.data_ptr(), s.size, dup.data_ptr(), None, None))
    want = expected_after(n, edge_set(base), u, v, np.zeros(k, np.uint8))
    o1, i1 = graph.export()
    assert np.array_equal(o1, want.off) and np.array_equal(i1, want.ind)
    N.check(N.lib().tc_delete_sorted(graph.handle, ds.data_ptr(), dd.data_ptr(), dup.data_ptr(), s.size, None))
    o2, i2 = graph.export()
    assert np.array_equal(o2, base.off) and np.array_equal(i2, base.ind)


def _hub_graph(rng, n, hubs, per_hub, pool_size, extra):
    """Hubs 0 .. hubs-1, each adjacent to per_hub vertices of one shared pool (so two hubs share
    most of their neighbours and every hub-hub edge closes thousands of triangles), plus random
    edges."""
    pool = rng.choice(np.arange(hubs, n), pool_size, replace=False).astype(np.int32)
    src, dst = [], []
    for h in range(hubs):
        nb = rng.choice(pool, per_hub, replace=False)
        src.append(np.full(per_hub, h, np.int32))
        dst.append(nb)
    src.append(rng.integers(0, n, extra).astype(np.int32))
    dst.append(rng.integers(0, n, extra).astype(np.int32))
    return G.from_pairs(n, np.concatenate(src), np.concatenate(dst))


def _strategy_sched(strategy):
    """None: the default rule; "staged": every degree cell staged (the longer list copied into
    shared memory piece by piece, the shorter list's entries searched there); "staged_per_edge":
    the same with the hub count off, so every changed edge, hub-hub ones included, is staged."""
    if strategy is None:
        return None
    from custingeralg_b200 import sched_learn as L
    s = L.forced(2)
    if strategy == "staged_per_edge":
        s.stream_hub_min = 0
    return s


@pytest.mark.parametrize("strategy", [None, "staged", "staged_per_edge"])
@pytest.mark.parametrize("path", ["pipeline", "apply"])
def test_split_intersections_between_hubs(path, strategy):
    """Edges whose both lists exceed 2048 entries are split into queued chunks (k_delta_split):
    inserting and deleting hub-hub edges must still give the recount, total and per vertex, with
    each intersection strategy."""
    torch = _torch()
    rng = np.random.default_rng(77)
    n, hubs = 16000, 6
    base = _hub_graph(rng, n, hubs, 6000, 8000, 30000)
    assert np.sort(np.diff(base.off))[-hubs] > 2048
    graph = api.Graph.from_csr(base, slack=0.25)
    T0, pv0 = _recount(graph, n)
    sched = _strategy_sched(strategy)
    pipe = api.Pipeline(graph, 1 << 14, sched=sched) if path == "pipeline" else None
    pv = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    delta = torch.zeros(1, dtype=torch.int64, device="cuda")
    cur = base
    es = edge_set(base)
    hub_pairs = [(a, b) for a in range(hubs) for b in range(a + 1, hubs)]
    for it in range(4):
        k = 4000
        s = rng.integers(0, n, k).astype(np.int32)
        d = rng.integers(0, n, k).astype(np.int32)
        x = np.zeros(k, np.uint8)
        # hub-hub edges: insert the absent ones, delete the present ones (both lists > 2048)
        for j, (a, b) in enumerate(hub_pairs):
            s[j], d[j] = (a, b) if j % 2 else (b, a)
            x[j] = 1 if (min(a, b), max(a, b)) in es else 0
        # hub - pool edges on both sides of the attribution rule
        m = len(hub_pairs)
        s[m:m + 500] = rng.integers(0, hubs, 500)
        d[m:m + 500] = rng.integers(hubs, n, 500)
        ts, td, tx = _dev(torch, s, d, x)
        if pipe is not None:
            pipe.apply(ts, td, tx, per_vertex=pv, delta_dev=delta)
            pipe.sync()
        else:
            graph.apply_batch(ts, td, tx, per_vertex=pv, delta_dev=delta, sched=sched)
        want = expected_after(n, es, s, d, x)
        off, ind = graph.export()
        assert np.array_equal(off, want.off) and np.array_equal(ind, want.ind)
        cur = G.Csr(n, off, ind)
        es = edge_set(cur)
        T, pvn = _recount(graph, n)
        assert T == T0 + int(delta.item())
        assert torch.equal(pvn, (pv0.to(torch.int64) + pv[:n].to(torch.int64)).to(torch.int32))
    if pipe is not None:
        pipe.close()


def _planted_hubs(rng, n):
    """Hubs 0-3 with 20000, 9000, 3000 and 600 neighbours (hub 0 takes three passes of the hub
    table, 8192 entries each), a dense block among 10..2999 so partner lists are long and share
    many neighbours with the hubs, and a random background."""
    src, dst = [], []
    for h, deg in ((0, 20000), (1, 9000), (2, 3000), (3, 600)):
        src.append(np.full(deg, h, np.int32))
        dst.append(rng.choice(np.arange(10, n, dtype=np.int32), deg, replace=False))
    src.append(rng.integers(10, 3000, 150000).astype(np.int32))
    dst.append(rng.integers(10, 3000, 150000).astype(np.int32))
    src.append(rng.integers(0, n, 80000).astype(np.int32))
    dst.append(rng.integers(0, n, 80000).astype(np.int32))
    return G.from_pairs(n, np.concatenate(src), np.concatenate(dst))


def _hub_batch(rng, cur, n):
    """Insertions and deletions of hub edges (many per hub, so they are counted at the hub) mixed
    with edges inside the dense block, random ones and edges between the hubs, so triangles with
    two or three changed edges are common."""
    src_of = np.repeat(np.arange(n, dtype=np.int32), np.diff(cur.off))
    parts = []
    hubs = rng.integers(0, 4, 2500).astype(np.int32)
    parts.append((hubs, rng.integers(10, 3000, 2500).astype(np.int32), np.zeros(2500, np.uint8)))
    hub_edges = np.flatnonzero(src_of < 4)
    pick = rng.choice(hub_edges, 1200, replace=False)
    parts.append((src_of[pick], cur.ind[pick], np.ones(1200, np.uint8)))
    parts.append((rng.integers(10, 3000, 1500).astype(np.int32), rng.integers(10, 3000, 1500).astype(np.int32),
                  np.zeros(1500, np.uint8)))
    pick = rng.integers(0, cur.m, 1500)
    parts.append((src_of[pick], cur.ind[pick], np.ones(1500, np.uint8)))
    # edges between the hubs: partner lists of thousands of entries (several units of work)
    present = set(zip(src_of[hub_edges].tolist(), cur.ind[hub_edges].tolist()))
    pairs = [(a, b) for a in range(4) for b in range(a + 1, 4)]
    parts.append((np.array([a for a, _ in pairs], np.int32), np.array([b for _, b in pairs], np.int32),
                  np.array([1 if (a, b) in present else 0 for a, b in pairs], np.uint8)))
    s = np.concatenate([p[0] for p in parts])
    d = np.concatenate([p[1] for p in parts])
    x = np.concatenate([p[2] for p in parts])
    perm = rng.permutation(s.size)
    return s[perm], d[perm], x[perm]


@pytest.mark.parametrize("path", ["pipeline", "apply"])
def test_hub_groups_match_the_per_edge_count(path):
    """Changed edges that share their longer endpoint are counted at it (k_delta_hub: the hub's
    list hashed once, in value-range passes when it is longer than one table). Totals and
    per-vertex deltas must equal the per-edge kernel's (stream_hub_min = 0) and the recount,
    batch after batch, for deletions and insertions alike."""
    torch = _torch()
    rng = np.random.default_rng(2024)
    n = 40000
    base = _planted_hubs(rng, n)
    assert np.diff(base.off)[0] > 2 * 8192
    off_hub = N.default_sched()
    off_hub.stream_hub_min = 0
    g_hub = api.Graph.from_csr(base, slack=0.25)
    g_edge = api.Graph.from_csr(base, slack=0.25)
    T0, pv0 = _recount(g_hub, n)
    if path == "pipeline":
        p_hub, p_edge = api.Pipeline(g_hub, 1 << 13), api.Pipeline(g_edge, 1 << 13, sched=off_hub)
    pv_h = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    pv_e = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    d_h = torch.zeros(1, dtype=torch.int64, device="cuda")
    d_e = torch.zeros(1, dtype=torch.int64, device="cuda")
    cur = base
    for it in range(3):
        ts, td, tx = _dev(torch, *_hub_batch(rng, cur, n))
        if path == "pipeline":
            p_hub.apply(ts, td, tx, per_vertex=pv_h, delta_dev=d_h)
            p_hub.sync()
            p_edge.apply(ts, td, tx, per_vertex=pv_e, delta_dev=d_e)
            p_edge.sync()
        else:
            g_hub.apply_batch(ts, td, tx, per_vertex=pv_h, delta_dev=d_h)
            g_edge.apply_batch(ts, td, tx, per_vertex=pv_e, delta_dev=d_e, sched=off_hub)
        assert int(d_h.item()) == int(d_e.item())
        assert torch.equal(pv_h, pv_e)
        T, pvn = _recount(g_hub, n)
        assert T == T0 + int(d_h.item())
        assert torch.equal(pvn, (pv0.to(torch.int64) + pv_h[:n].to(torch.int64)).to(torch.int32))
        off, ind = g_hub.export()
        cur = G.Csr(n, off, ind)
    if path == "pipeline":
        p_hub.close()
        p_edge.close()
