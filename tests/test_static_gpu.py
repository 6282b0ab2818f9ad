"""Static triangle count on the GPU through the C ABI, bit-exact against the oracle/fixtures."""
import functools

import numpy as np
import pytest

from custingeralg_b200 import api, generators as G, native as N
from oracle import pyoracle as O
from tests.util import digest, golden_graph, load_golden, random_graph

pytestmark = pytest.mark.gpu
GOLD = load_golden()["graphs"]


def _torch():
    import torch
    return torch


def sched(**kw):
    s = N.default_sched()
    for k, v in kw.items():
        if k == "table_all":
            s.use_table = 1
            for i in range(16):
                for j in range(16):
                    s.table[i][j] = v
        else:
            setattr(s, k, v)
    return s


SCHEDS = {
    "default": None,
    "lane_walk_up_to_64": dict(lane_max_deg=64),
    "never_lane_walk": dict(lane_max_deg=0),
    "warp2": dict(warp_max_deg=2),
    "warp8_chunk32": dict(warp_max_deg=8, chunk=32),
    "one_block_per_sm": dict(blocks_per_sm=1),
    "packed_up_to_64": dict(lane_max_deg=4, packed_max_deg=64),
    "packed_everywhere": dict(table_all=2),
    "packed_warp2": dict(warp_max_deg=2, lane_max_deg=0, packed_max_deg=1 << 20),
}


def run_handle(g, mode, s=None):
    torch = _torch()
    graph = api.Graph.from_csr(g)
    out = torch.full((g.n + 1,), -7, dtype=torch.int32, device="cuda")
    tri_dev = torch.zeros(1, dtype=torch.int64, device="cuda")
    T, info = graph.count(mode, out if mode != N.TC_PV_NONE else None, tri_dev, sched=s)
    assert int(tri_dev.item()) == T
    assert int(out[g.n].item()) == -7, "entry nv must stay untouched"
    return T, out[: g.n].cpu().numpy(), info


@pytest.mark.parametrize("name", sorted(GOLD))
def test_handle_count_matches_golden(name):
    rec = GOLD[name]
    g = golden_graph(name)
    T, pv, info = run_handle(g, N.TC_PV_HANDLE)
    assert T == rec["triangles"]
    assert 6 * T == rec["ref_all_triangles"]
    assert digest(pv) == rec["per_vertex_handle_digest"]
    assert info.status == N.TC_OK


@pytest.mark.parametrize("name", sorted(GOLD))
def test_csr_count_matches_golden(name):
    torch = _torch()
    rec = GOLD[name]
    g = golden_graph(name)
    off32 = torch.from_numpy(g.off32()).cuda()
    ind = torch.from_numpy(g.ind).cuda() if g.m else torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.full((g.n + 1,), -3, dtype=torch.int32, device="cuda")
    T, info = api.count_all_triangles_csr(g.n, off32, ind, out)
    assert T == rec["triangles"]
    assert digest(out[: g.n].cpu().numpy()) == rec["per_vertex_csr_digest"]
    assert int(out[g.n].item()) == -3
    off64 = torch.from_numpy(g.off).cuda()
    T2, _ = api.count_all_triangles_csr(g.n, off64, ind, out, pv_mode=N.TC_PV_HANDLE)
    assert T2 == rec["triangles"] and digest(out[: g.n].cpu().numpy()) == rec["per_vertex_handle_digest"]


@pytest.mark.parametrize("sname", sorted(SCHEDS))
@pytest.mark.parametrize("name", ["rmat12_ef16_s2", "K70", "ba4096_m8_s1", "er14_d16_s1"])
def test_strategies_agree(name, sname):
    rec = GOLD[name]
    g = golden_graph(name)
    kw = SCHEDS[sname]
    s = sched(**kw) if kw else None
    for mode, key in ((N.TC_PV_HANDLE, "per_vertex_handle_digest"), (N.TC_PV_CSR, "per_vertex_csr_digest")):
        T, pv, _ = run_handle(g, mode, s)
        assert T == rec["triangles"] and digest(pv) == rec[key]
    T, _, _ = run_handle(g, N.TC_PV_NONE, s)
    assert T == rec["triangles"]


def test_large_out_degree_chunking():
    # K_2600: every out-degree up to 2599 > 2048 staged entries, so vertices take several passes.
    n = 2600
    g = G.complete(n)
    T, pv, info = run_handle(g, N.TC_PV_HANDLE)
    assert T == n * (n - 1) * (n - 2) // 6
    assert np.array_equal(pv, np.full(n, (n - 1) * (n - 2), dtype=np.int64).astype(np.int32))
    assert info.max_out_degree == n - 1


@functools.lru_cache(maxsize=1)
def _core_periphery_graph():
    """A dense core of 1200 vertices (edge probability 0.92, so the lowest-ranked core vertices
    have out-degree above the 1024 entries one CTA table holds, and take two value-range passes)
    joined to 6000 sparse periphery vertices, whose short lists of core ids are walked whole in
    each pass, plus a few hundred mid-degree vertices with lists that need the range cut."""
    rng = np.random.default_rng(1200)
    core = 1200
    i, j = np.triu_indices(core, 1)
    keep = rng.random(i.size) < 0.92
    src, dst = [i[keep]], [j[keep]]
    per = np.arange(core, core + 6000)
    for k in range(3):  # every periphery vertex joins three random core vertices
        src.append(per)
        dst.append(rng.integers(0, core, per.size))
    mid = np.arange(core + 6000, core + 6400)
    for k in range(150):  # mid-degree vertices: ~150 core neighbours each
        src.append(mid)
        dst.append(rng.integers(0, core, mid.size))
    src.append(rng.integers(core, core + 6400, 20000))  # sparse edges among the rest
    dst.append(rng.integers(core, core + 6400, 20000))
    return G.from_pairs(core + 6400, np.concatenate(src), np.concatenate(dst), name="core_periphery")


@functools.lru_cache(maxsize=1)
def _core_periphery_oracle():
    g = _core_periphery_graph()
    tot, pv_handle = O.fast_count(g.n, g.off, g.ind)
    return tot, pv_handle, O.csr_per_vertex(g.n, g.off, g.ind)


@pytest.mark.parametrize("sname", ["default", "never_lane_walk", "packed_everywhere", "lane_walk_up_to_64"])
def test_value_range_passes_vs_oracle(sname):
    g = _core_periphery_graph()
    tot, pv_handle, pv_csr = _core_periphery_oracle()
    kw = SCHEDS[sname]
    s = sched(**kw) if kw else None
    T, pv, info = run_handle(g, N.TC_PV_HANDLE, s)
    assert info.max_out_degree > 1024, "the graph must hold centres that take several passes"
    assert 6 * T == tot and np.array_equal(pv, pv_handle)
    T, pv, _ = run_handle(g, N.TC_PV_CSR, s)
    assert 6 * T == tot and np.array_equal(pv, pv_csr)
    T, _, _ = run_handle(g, N.TC_PV_NONE, s)
    assert 6 * T == tot


@pytest.mark.parametrize("seed", range(10))
def test_random_graphs_vs_oracle(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 3000))
    g = random_graph(rng, n, int(rng.integers(0, 20 * n)))
    ref_all, _ = O.host_count_triangles(g.n, g.off, g.ind)
    T, pv, _ = run_handle(g, N.TC_PV_HANDLE)
    assert 6 * T == ref_all
    assert np.array_equal(pv, O.static_per_vertex(g.n, g.off, g.ind))
    T, pv, _ = run_handle(g, N.TC_PV_CSR)
    assert np.array_equal(pv, O.csr_per_vertex(g.n, g.off, g.ind))


def test_rmat16_fast_oracle():
    g = G.rmat(16, 16, seed=5)
    tot, pv_ref = O.fast_count(g.n, g.off, g.ind)
    T, pv, info = run_handle(g, N.TC_PV_HANDLE)
    assert 6 * T == tot and np.array_equal(pv, pv_ref)
    assert info.edges_intersected > 0 and info.oriented_work > 0


def _bad_csr(kind):
    g = G.complete(5)
    off, ind = g.off.copy(), g.ind.copy()
    if kind == "unsorted":
        ind[0], ind[1] = ind[1], ind[0]
    elif kind == "self_loop":
        ind[0] = 0
    elif kind == "range":
        ind[0] = 99
    elif kind == "asym":
        # drop 1 from N(0) without dropping 0 from N(1): rebuild off/ind
        lst = [list(ind[off[v]:off[v + 1]]) for v in range(5)]
        lst[0].remove(1)
        off = np.concatenate([[0], np.cumsum([len(x) for x in lst])]).astype(np.int64)
        ind = np.concatenate([np.array(x, np.int32) for x in lst])
    return g.n, off, ind


@pytest.mark.parametrize("kind,code", [("unsorted", N.TC_ERR_BAD_GRAPH), ("self_loop", N.TC_ERR_BAD_GRAPH),
                                       ("range", N.TC_ERR_BAD_GRAPH), ("asym", N.TC_ERR_NOT_SYMMETRIC)])
def test_bad_graphs_are_rejected(kind, code):
    torch = _torch()
    n, off, ind = _bad_csr(kind)
    with pytest.raises(N.TcError) as e:
        api.Graph(n, off, ind, validate=True)
    assert e.value.status == code
    out = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    with pytest.raises(N.TcError) as e:
        api.count_all_triangles_csr(n, torch.from_numpy(off.astype(np.int32)).cuda(), torch.from_numpy(ind).cuda(), out)
    assert e.value.status == code


def test_invalid_args():
    with pytest.raises(N.TcError) as e:
        api.Graph.from_csr(G.complete(4)).count(N.TC_PV_HANDLE, None)
    assert e.value.status == N.TC_ERR_INVALID_ARG
    with pytest.raises(N.TcError):
        api.Graph.from_csr(G.complete(4)).count(7, None)


def test_export_roundtrip():
    g = G.rmat(10, 8, seed=9)
    graph = api.Graph.from_csr(g, slack=0.5)
    off, ind = graph.export()
    assert np.array_equal(off, g.off) and np.array_equal(ind, g.ind)
    n, used, alloc = graph.info()
    assert n == g.n and used == g.m and alloc >= used


@pytest.mark.parametrize("name,nshards", [("rmat12_ef16_s2", 2), ("rmat12_ef16_s2", 3), ("ba4096_m8_s1", 4),
                                          ("rmat14_ef16_s2", 8)])
def test_shards_sum_to_full(name, nshards):
    """Each shard counts the contiguous range of centres the split rule gives it: the device's
    predicted work per centre equals the oracle's, its range equals the host rule's
    (tc_shard_ranges) on that work, its count equals the oracle's count of the range, and the
    shards add up to the full count (total and per-vertex digest)."""
    torch = _torch()
    g = golden_graph(name)
    rec = GOLD[name]
    graph = api.Graph.from_csr(g)
    cost = O.centre_cost(g.n, g.off, g.ind)
    pre = np.concatenate([[0], np.cumsum(cost, dtype=np.int64)])
    lo = api.shard_ranges(pre, nshards)
    total = 0
    acc = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
    for sh in range(nshards):
        out = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
        T, info = graph.count(N.TC_PV_HANDLE, out, sched=sched(shard=sh, nshards=nshards))
        assert (info.shard_lo, info.shard_hi) == (lo[sh], lo[sh + 1])
        assert info.total_work == pre[-1] and info.shard_work == pre[lo[sh + 1]] - pre[lo[sh]]
        tot_o, pv_o = O.fast_count_range(g.n, g.off, g.ind, int(lo[sh]), int(lo[sh + 1]))
        assert 6 * T == tot_o and np.array_equal(out[: g.n].cpu().numpy(), pv_o)
        total += T
        acc += out
    assert total == rec["triangles"]
    assert digest(acc[: g.n].cpu().numpy()) == rec["per_vertex_handle_digest"]


def test_unsharded_count_reports_no_range():
    g = golden_graph("rmat12_ef16_s2")
    _, _, info = run_handle(g, N.TC_PV_HANDLE)
    assert (info.shard_lo, info.shard_hi) == (0, -1)


@pytest.mark.parametrize("name", ["rmat12_ef16_s2", "K70", "ba4096_m8_s1"])
def test_int64_per_vertex_mode(name):
    """TC_PV_HANDLE64 writes 2 t(v) into int64 entries (no wrap): the oracle's per-vertex counts,
    through the handle and through the raw-CSR entry point; entry nv stays untouched."""
    torch = _torch()
    g = golden_graph(name)
    _, want = O.fast_count(g.n, g.off, g.ind)
    graph = api.Graph.from_csr(g)
    out = torch.full((g.n + 1,), -7, dtype=torch.int64, device="cuda")
    T, _ = graph.count(N.TC_PV_HANDLE64, out)
    assert T == GOLD[name]["triangles"]
    assert np.array_equal(out[: g.n].cpu().numpy(), want.astype(np.int64))
    assert int(out[g.n].item()) == -7
    d_off = torch.from_numpy(g.off.astype(np.int32)).cuda()
    d_ind = torch.from_numpy(g.ind).cuda()
    out2 = torch.zeros(g.n, dtype=torch.int64, device="cuda")
    T2, _ = api.count_all_triangles_csr(g.n, d_off, d_ind, out2, pv_mode=N.TC_PV_HANDLE64)
    assert T2 == T and torch.equal(out2, out[: g.n])
