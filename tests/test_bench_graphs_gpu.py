"""The benchmark graphs at full size against the reference's own answers.

tests/golden/bench_configs.json holds, for R-MAT scale 20 (seed 2) and scale 24 (seed 3), the
reference's hostSingleIntersection over every directed edge (tests/cct.cpp:32-89): its total
(6T) and digests of the per-vertex outputs, int32 2t(v) as the handle kernel writes it
(devicecuStingerAllTriangles, src/static_triangle_counting/cct.cu:216-270) and the forward
counts of the raw-CSR kernel (count_all_trianglesGPU, tests/cct_csr.cu:228-276). Each graph is
counted here through the handle (tc_count_static, the callDeviceAllTriangles path) and through the
raw CSR (tc_count_csr32, the callDeviceAllTrianglesCSR path), under the fixed rule and the learned
table, and must match those answers bit for bit. The digests also record whether any 2t(v)
reaches 2^31 (it does not on these graphs).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from custingeralg_b200 import api, generators as G, native as N

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "bench_configs.json")))


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).astype("<i4").tobytes()).hexdigest()[:32]


def _graph_digest(g):
    d = lambda a: hashlib.sha256(np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<")).tobytes()).hexdigest()[:32]
    return d(g.off) + d(g.ind)


def _scheds(graph):
    out = [("fixed", N.default_sched())]
    from custingeralg_b200 import sched_learn as L
    if os.path.exists(L.WEIGHTS):
        out.append(("learned", L.learned_sched(L.load(L.WEIGHTS), graph)))
    return out


@pytest.mark.parametrize("scale,seed", [(20, 2), (24, 3)], ids=["rmat20_C2", "rmat24_C3"])
def test_full_size_counts_equal_the_reference(scale, seed):
    import torch
    rec = GOLD[f"rmat{scale}_ef16_s{seed}"]
    assert rec["checked_by"].startswith("reference"), rec["checked_by"]
    g = G.rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed)
    assert _graph_digest(g) == rec["graph_digest"] and g.m == rec["m"]
    assert rec["wraps_int32"] == 0 and rec["max_2t"] < 2**31

    # handle path (callDeviceAllTriangles): int32 2t(v)
    graph = api.Graph.from_csr(g)
    out = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
    graph.count(N.TC_PV_HANDLE, out)
    for name, sched in _scheds(graph):
        out.fill_(-1)
        T, info = graph.count(N.TC_PV_HANDLE, out, sched=sched)
        assert info.status == N.TC_OK
        assert T == rec["triangles"], name
        assert _digest(out[:g.n].cpu().numpy()) == rec["per_vertex_handle_digest"], name
    # int64 per-vertex mode: the exact 2t(v)
    out64 = torch.zeros(g.n + 1, dtype=torch.int64, device="cuda")
    graph.count(N.TC_PV_HANDLE64, out64.view(torch.int32))
    pv64 = out64[:g.n].cpu().numpy()
    assert int(pv64.max()) == rec["max_2t"]
    assert hashlib.sha256(pv64.astype("<i8").tobytes()).hexdigest()[:32] == rec["per_vertex_handle64_digest"]
    graph.close()
    del out64

    # raw-CSR path (callDeviceAllTrianglesCSR): forward counts, int32 offsets
    d_off = torch.from_numpy(g.off32()).cuda()
    d_ind = torch.from_numpy(g.ind).cuda()
    fwd = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
    T, info = api.count_all_triangles_csr(g.n, d_off, d_ind, fwd, pv_mode=N.TC_PV_CSR)
    assert info.status == N.TC_OK and T == rec["triangles"]
    assert _digest(fwd[:g.n].cpu().numpy()) == rec["per_vertex_csr_digest"]
    T, _ = api.count_all_triangles_csr(g.n, d_off, d_ind, out, pv_mode=N.TC_PV_HANDLE)
    assert T == rec["triangles"] and _digest(out[:g.n].cpu().numpy()) == rec["per_vertex_handle_digest"]


@pytest.mark.parametrize("scale,seed", [(22, 4)], ids=["rmat22_streaming_base"])
def test_streaming_base_graph_equals_the_reference(scale, seed):
    """The streaming workload's base graph (R-MAT 22, seed 4): total and per-vertex 2t(v)."""
    import torch
    rec = GOLD[f"rmat{scale}_ef16_s{seed}"]
    assert rec["checked_by"].startswith("reference"), rec["checked_by"]
    g = G.rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed)
    graph = api.Graph.from_csr(g, slack=0.25)
    out = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
    T, _ = graph.count(N.TC_PV_HANDLE, out)
    assert T == rec["triangles"]
    assert _digest(out[:g.n].cpu().numpy()) == rec["per_vertex_handle_digest"]
