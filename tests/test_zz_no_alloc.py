"""The allocation-free static count (tc_count_csr32_noalloc) against the allocating one.

Some callers cannot allocate device memory when they count: they run inside a captured CUDA
graph region, or under an allocator that forbids device allocation after start-up, or they
budget every byte of device memory up front. tc_count_csr32_noalloc serves them with working
memory held in a fixed array of the library's own device image. This file is collected last
so that a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

from custingeralg_b200 import generators as G, native as N

pytestmark = pytest.mark.gpu


def _count(fn, g, d_off, d_ind, mode):
    import torch
    out = torch.full((g.n + 1,), -5, dtype=torch.int32, device="cuda")
    tri = torch.zeros(1, dtype=torch.int64, device="cuda")
    info = N.CountInfo()
    N.check(fn(g.n, d_off.data_ptr(), d_ind.data_ptr(), mode, out.data_ptr(), tri.data_ptr(), ctypes.byref(info),
               None, None))
    assert int(tri.item()) == info.triangles
    assert int(out[g.n].item()) == -5
    return info.triangles, out[: g.n].cpu().numpy()


@pytest.mark.parametrize("mode", [N.TC_PV_CSR, N.TC_PV_HANDLE])
def test_noalloc_matches_allocating_entry_point(mode):
    import torch
    g = G.rmat(14, 16, seed=2)
    d_off = torch.from_numpy(g.off32()).cuda()
    d_ind = torch.from_numpy(g.ind).cuda()
    T_ref, pv_ref = _count(N.lib().tc_count_csr32, g, d_off, d_ind, mode)
    # two calls in a row: the shared scratch keeps the previous call's contents
    for _ in range(2):
        T, pv = _count(N.lib().tc_count_csr32_noalloc, g, d_off, d_ind, mode)
        assert T == T_ref
        assert np.array_equal(pv, pv_ref)


def test_noalloc_rejects_graphs_beyond_its_limit():
    import torch
    n = N.NOALLOC_MAX_NV + 1
    d_off = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    d_ind = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    st = N.lib().tc_count_csr32_noalloc(n, d_off.data_ptr(), d_ind.data_ptr(), N.TC_PV_CSR, out.data_ptr(), None,
                                        None, None, None)
    assert st == N.TC_ERR_CAPACITY
