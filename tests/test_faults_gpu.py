"""Out-of-memory paths, injected on the host (no GPU fault).

tc_debug_alloc_cap makes every device allocation of the library above a size fail the way
cudaMalloc fails when device memory runs out. Each entry point must then return TC_ERR_OOM,
leave what it was given usable, and work again once the cap is lifted: graph creation, the
stateless count's workspace, the batch workspace of a streaming update and the captured
pipeline.
"""
import numpy as np
import pytest

from custingeralg_b200 import api, generators as G, native as N
from oracle import pyoracle as O
from tests.test_stream_gpu import random_batch

pytestmark = pytest.mark.gpu

CAP = 1 << 16   # 64 KiB: far below what any of these graphs needs


@pytest.fixture(autouse=True)
def _lift_cap():
    yield
    N.check(N.lib().tc_debug_alloc_cap(0))


def _count(graph, n):
    import torch
    out = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    T, _ = graph.count(N.TC_PV_HANDLE, out)
    return T, out[:n].cpu().numpy()


def test_graph_creation_reports_oom_then_works():
    g = G.rmat(14, 16, seed=2)
    N.check(N.lib().tc_debug_alloc_cap(CAP))
    with pytest.raises(N.TcError) as ei:
        api.Graph.from_csr(g)
    assert ei.value.status == N.TC_ERR_OOM
    N.check(N.lib().tc_debug_alloc_cap(0))
    graph = api.Graph.from_csr(g)
    T, pv = _count(graph, g.n)
    tot, _ = O.host_count_triangles(g.n, g.off, g.ind)
    assert 6 * T == tot and np.array_equal(pv, O.static_per_vertex(g.n, g.off, g.ind))


def test_stateless_count_reports_oom_then_works():
    import torch
    small = G.rmat(10, 8, seed=3)
    big = G.rmat(15, 16, seed=3)

    def run(g):
        d_off = torch.from_numpy(g.off32()).cuda()
        d_ind = torch.from_numpy(g.ind).cuda()
        out = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
        return api.count_all_triangles_csr(g.n, d_off, d_ind, out, pv_mode=N.TC_PV_CSR), out[:g.n].cpu().numpy()

    N.check(N.lib().tc_workspace_release())   # the library's workspace: none on this device now
    N.check(N.lib().tc_debug_alloc_cap(CAP))
    with pytest.raises(N.TcError) as ei:
        run(big)                      # allocating it fails
    assert ei.value.status == N.TC_ERR_OOM
    (T, _), pv = run(small)           # a graph whose workspace fits under the cap counts right
    tot, _ = O.host_count_triangles(small.n, small.off, small.ind)
    assert 6 * T == tot and np.array_equal(pv, O.csr_per_vertex(small.n, small.off, small.ind))
    with pytest.raises(N.TcError) as ei:
        run(big)                      # growing it fails, and leaves it usable
    assert ei.value.status == N.TC_ERR_OOM
    (T, _), pv = run(small)
    assert 6 * T == tot and np.array_equal(pv, O.csr_per_vertex(small.n, small.off, small.ind))
    N.check(N.lib().tc_debug_alloc_cap(0))
    (T, _), pv = run(big)
    tot, _ = O.host_count_triangles(big.n, big.off, big.ind)
    assert 6 * T == tot and np.array_equal(pv, O.csr_per_vertex(big.n, big.off, big.ind))


@pytest.mark.parametrize("path", ["apply", "pipeline"])
def test_streaming_reports_oom_and_the_graph_stays_consistent(path):
    import torch
    rng = np.random.default_rng(31)
    base = G.rmat(12, 16, seed=9)
    n = base.n
    graph = api.Graph.from_csr(base, slack=0.25)
    T0, pv0 = _count(graph, n)
    pv = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    delta = torch.zeros(1, dtype=torch.int64, device="cuda")

    def dev(s, d, x):
        return (torch.from_numpy(s).cuda(), torch.from_numpy(d).cuda(), torch.from_numpy(x).cuda())

    def apply(pipe, s, d, x):
        if pipe is None:
            graph.apply_batch(*dev(s, d, x), per_vertex=pv, delta_dev=delta)
        else:
            pipe.apply(*dev(s, d, x), per_vertex=pv, delta_dev=delta)
            pipe.sync()

    pipe = None
    if path == "pipeline":
        N.check(N.lib().tc_debug_alloc_cap(CAP))
        with pytest.raises(N.TcError) as ei:
            api.Pipeline(graph, 1 << 14)      # its batch workspace cannot be allocated
        assert ei.value.status == N.TC_ERR_OOM
        N.check(N.lib().tc_debug_alloc_cap(0))
        pipe = api.Pipeline(graph, 1 << 14)
    apply(pipe, *random_batch(rng, base, 300))
    # a batch needing a larger workspace (apply) or fresh captures after pool growth fails cleanly
    N.check(N.lib().tc_debug_alloc_cap(CAP))
    if pipe is None:
        with pytest.raises(N.TcError) as ei:
            apply(None, *random_batch(rng, base, 8000))
        assert ei.value.status == N.TC_ERR_OOM
    N.check(N.lib().tc_debug_alloc_cap(0))
    off, ind = graph.export()
    cur = G.Csr(n, off, ind)
    for k in (50, 3000, 9000):
        s, d, x = random_batch(rng, cur, k)
        apply(pipe, s, d, x)
        off, ind = graph.export()
        cur = G.Csr(n, off, ind)
    T, pv_now = _count(graph, n)
    assert T == T0 + int(delta.item())
    assert np.array_equal(pv_now, (pv0.astype(np.int64) + pv[:n].cpu().numpy()).astype(np.int32))
    tot, _ = O.host_count_triangles(n, cur.off, cur.ind)
    assert 6 * T == tot
    if pipe is not None:
        pipe.close()
