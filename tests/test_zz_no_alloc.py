"""The allocation-free static count (tc_count_csr32_noalloc) through the C ABI.

Some callers must not allocate device memory when they count: their device memory belongs to
another allocator (a framework's caching pool) or was reserved in full at start-up, or they run
latency-sensitive loops where cudaMalloc and cudaFree can synchronise the device.
tc_count_csr32_noalloc serves them with working memory held in a fixed array of the library's
own device image. Its results must equal the allocating entry point's (tc_count_csr32) and the
CPU oracle's, bit for bit, on two calls in a row (the array keeps the previous call's contents),
and a call must leave the device's free memory unchanged.

This file is collected last, so a failure here leaves every other test already run. It passes
alone in a fresh process too: the first call loads the module that holds the array.
"""
import ctypes

import numpy as np
import pytest

from custingeralg_b200 import generators as G, native as N
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu


def _count(fn, g, d_off, d_ind, mode):
    import torch
    out = torch.full((g.n + 1,), -5, dtype=torch.int32, device="cuda")
    tri = torch.zeros(1, dtype=torch.int64, device="cuda")
    info = N.CountInfo()
    N.check(fn(g.n, d_off.data_ptr(), d_ind.data_ptr(), mode, out.data_ptr(), tri.data_ptr(), ctypes.byref(info),
               None, None))
    assert int(tri.item()) == info.triangles
    assert int(out[g.n].item()) == -5   # nothing written past the nv entries
    return info.triangles, out[: g.n].cpu().numpy()


def _oracle(g, mode):
    six_t, _ = O.host_count_triangles(g.n, g.off, g.ind)
    pv = O.static_per_vertex(g.n, g.off, g.ind) if mode == N.TC_PV_HANDLE else O.csr_per_vertex(g.n, g.off, g.ind)
    return six_t // 6, pv


@pytest.mark.parametrize("mode", [N.TC_PV_CSR, N.TC_PV_HANDLE])
@pytest.mark.parametrize("name,make", [("rmat14", lambda: G.rmat(14, 16, seed=2)),
                                       ("er14", lambda: G.erdos_renyi(1 << 14, 16.0 / (1 << 14), seed=1))])
def test_noalloc_matches_allocating_entry_point_and_oracle(mode, name, make):
    import torch
    g = make()
    d_off = torch.from_numpy(g.off32()).cuda()
    d_ind = torch.from_numpy(g.ind).cuda()
    T_ora, pv_ora = _oracle(g, mode)
    T_ref, pv_ref = _count(N.lib().tc_count_csr32, g, d_off, d_ind, mode)
    assert T_ref == T_ora and np.array_equal(pv_ref, pv_ora)
    # two calls in a row: the shared array keeps the previous call's contents
    for _ in range(2):
        T, pv = _count(N.lib().tc_count_csr32_noalloc, g, d_off, d_ind, mode)
        assert T == T_ref == T_ora
        assert np.array_equal(pv, pv_ref)


def test_noalloc_leaves_free_device_memory_unchanged():
    """After one call (which loads the module holding the array), later calls allocate nothing:
    the device's free memory is the same before and after them."""
    import torch
    g = G.rmat(15, 16, seed=4)
    d_off = torch.from_numpy(g.off32()).cuda()
    d_ind = torch.from_numpy(g.ind).cuda()
    out = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
    tri = torch.zeros(1, dtype=torch.int64, device="cuda")
    fn = N.lib().tc_count_csr32_noalloc

    def call():
        N.check(fn(g.n, d_off.data_ptr(), d_ind.data_ptr(), N.TC_PV_HANDLE, out.data_ptr(), tri.data_ptr(), None,
                   None, None))

    call()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        call()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    T, _ = O.fast_count(g.n, g.off, g.ind, per_vertex=False)
    assert int(tri.item()) * 6 == T


def test_noalloc_rejects_graphs_beyond_its_limits():
    import torch
    fn = N.lib().tc_count_csr32_noalloc
    # more vertices than the array holds
    n = N.NOALLOC_MAX_NV + 1
    d_off = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    d_ind = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    assert fn(n, d_off.data_ptr(), d_ind.data_ptr(), N.TC_PV_CSR, out.data_ptr(), None, None, None, None) == \
        N.TC_ERR_CAPACITY
    # more directed edges than the array holds (the offsets alone decide: the call reads d_off[nv]
    # and rejects before anything reads the index array)
    n = 1000
    off = np.zeros(n + 1, np.int32)
    off[-1] = N.NOALLOC_MAX_EDGES + 2
    d_off = torch.from_numpy(off).cuda()
    out = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    st = fn(n, d_off.data_ptr(), d_ind.data_ptr(), N.TC_PV_CSR, out.data_ptr(), None, None, None, None)
    assert st == N.TC_ERR_CAPACITY
    assert b"directed edges" in N.lib().tc_last_error()
