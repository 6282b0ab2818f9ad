"""The reference's own raw-CSR GPU counter beside this library's count on the same B200.

The reference kernel is count_all_trianglesGPU / callDeviceAllTrianglesCSR
(tests/cct_csr.cu:228-285), rebuilt for sm_100a from the reference sources by oracle/Makefile
(oracle/_ref/libref_cct_gpu.so). Its per-vertex output uses the forward convention
(out[src] = sum over dest > src of |N(src) ∩ N(dest)|), which this library's TC_PV_CSR mode
reproduces; the tests check them equal entry by entry.

Timing (opt-in, it runs the reference's launch sweep on a large graph):
    TC_REF_GPU_SCALE=20 python -m pytest tests/test_ref_gpu.py -m gpu -s -k timing
prints one JSON line with the best reference configuration and this library's count.
"""
import json
import os

import numpy as np
import pytest

from custingeralg_b200 import api, generators as G, native as N
from oracle import pyoracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_gpu_available(), reason="reference GPU counter not built")]

# The reference's merge-path search reads one entry before and one after a list
# (tests/cct_csr.cu:110-112); the device index array gets guard entries on both sides.
GUARD = 64

# Launch configurations from the reference driver's sweep (tests/cct.cpp:103-106):
# (threads per intersection, shifter, blocks, block size).
SWEEP = [(tsp, sh, 16000, bs) for bs in (32, 64, 96, 128, 192, 256)
         for tsp, sh in ((1, 0), (2, 1), (4, 2), (8, 3), (16, 4), (32, 5))]


def _torch():
    import torch
    return torch


def device_csr(g):
    torch = _torch()
    off = torch.from_numpy(g.off32()).cuda()
    buf = torch.empty(g.m + 2 * GUARD, dtype=torch.int32, device="cuda")
    buf[:GUARD] = np.iinfo(np.int32).min
    buf[GUARD + g.m:] = np.iinfo(np.int32).max
    if g.m:
        buf[GUARD:GUARD + g.m] = torch.from_numpy(np.ascontiguousarray(g.ind, dtype=np.int32)).cuda()
    return off, buf, buf[GUARD:]


def ref_gpu_count(g, off, ind_view, cfg):
    torch = _torch()
    out = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
    tsp, sh, blocks, bs = cfg
    rc = O.ref_gpu().ref_gpu_count_csr(g.n, off.data_ptr(), ind_view.data_ptr(), out.data_ptr(), tsp, sh, blocks, bs)
    assert rc == 0, f"reference launch failed: cudaError {rc}"
    torch.cuda.synchronize()
    return out


def ours_csr(g, off, ind_view, sched=None):
    torch = _torch()
    out = torch.full((g.n + 1,), -7, dtype=torch.int32, device="cuda")
    T, _ = api.count_all_triangles_csr(g.n, off, ind_view[:g.m], out, N.TC_PV_CSR, sched=sched)
    return T, out


CASES = {
    "er14": lambda: G.erdos_renyi(1 << 14, 16.0 / (1 << 14), seed=1),
    "rmat14": lambda: G.rmat(14, 16, seed=2),
    "ba12": lambda: G.barabasi_albert(1 << 12, 8, seed=3),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("cfg", [(1, 0, 16000, 256), (32, 5, 16000, 256), (8, 3, 16000, 128)],
                         ids=["tsp1_bs256", "tsp32_bs256", "tsp8_bs128"])
def test_reference_gpu_per_vertex_matches(case, cfg):
    g = CASES[case]()
    off, _, ind_view = device_csr(g)
    ref = ref_gpu_count(g, off, ind_view, cfg)
    T, ours = ours_csr(g, off, ind_view)
    assert np.array_equal(ref[:g.n].cpu().numpy(), ours[:g.n].cpu().numpy())
    assert int(ref[:g.n].to(dtype=_torch().int64).sum().item()) == 3 * T


@pytest.mark.skipif("TC_REF_GPU_SCALE" not in os.environ, reason="opt-in timing run")
def test_reference_gpu_timing():
    torch = _torch()
    scale = int(os.environ["TC_REF_GPU_SCALE"])
    seed = {20: 2, 22: 4, 24: 3}.get(scale, 2)
    g = G.rmat(scale, 16, seed=seed)
    off, _, ind_view = device_csr(g)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps):
        best = float("inf")
        for _ in range(reps):
            torch.cuda.synchronize()
            ev0.record()
            fn()
            ev1.record()
            torch.cuda.synchronize()
            best = min(best, ev0.elapsed_time(ev1))
        return best

    T, ours = ours_csr(g, off, ind_view)
    out = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
    ours_ms = timed(lambda: api.count_all_triangles_csr(g.n, off, ind_view[:g.m], out, N.TC_PV_CSR, sync=False), 5)
    cfgs = SWEEP if os.environ.get("TC_REF_GPU_FULL_SWEEP") else [c for c in SWEEP if c[3] in (128, 256)]
    rows = []
    for cfg in cfgs:
        ref = ref_gpu_count(g, off, ind_view, cfg)
        same = bool(torch.equal(ref[:g.n], ours[:g.n]))
        tsp, sh, blocks, bs = cfg
        ms = timed(lambda: O.ref_gpu().ref_gpu_count_csr(g.n, off.data_ptr(), ind_view.data_ptr(), out.data_ptr(),
                                                          tsp, sh, blocks, bs), 1)
        rows.append({"tsp": tsp, "blocks": blocks, "block_size": bs, "ms": round(ms, 3), "per_vertex_equal": same})
    best = min(rows, key=lambda r: r["ms"])
    print(json.dumps({"graph": f"rmat{scale} ef16 seed {seed}", "n": g.n, "m": g.m, "triangles": T,
                      "ours_ms": round(ours_ms, 3), "reference_best": best,
                      "speedup_vs_reference_best": round(best["ms"] / ours_ms, 2), "reference_sweep": rows}))
    assert all(r["per_vertex_equal"] for r in rows)
