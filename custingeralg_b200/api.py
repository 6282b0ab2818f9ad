"""Python mirror of the reference's triangle-counting entry points over the C ABI.

  Graph                  the cuStinger handle subset (initializeCuStinger from a CSR)
  count_all_triangles    callDeviceAllTriangles  (include/static_triangle_counting/cct.hpp:15-17)
  count_all_triangles_csr callDeviceAllTrianglesCSR (tests/cct_csr.cu:279-285)

Device buffers are torch CUDA tensors (plumbing only); every count runs in the native library.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import native as N


def _stream_ptr(stream=None) -> Optional[int]:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _ptr(t) -> Optional[int]:
    if t is None:
        return None
    return t.data_ptr()


class Graph:
    """Dynamic graph handle (tc_graph*) built from a symmetric sorted CSR."""

    def __init__(self, n: int, off, ind, slack: float = 0.0, validate: bool = True, stream=None):
        import torch
        self._h = ctypes.c_void_p()
        if isinstance(off, np.ndarray):
            off = np.ascontiguousarray(off, dtype=np.int64)
            ind = np.ascontiguousarray(ind, dtype=np.int32)
            ind_p = ind.ctypes.data if ind.size else None
            st = N.lib().tc_graph_create(n, off.ctypes.data, ind_p, N.TC_MEM_HOST, slack, int(validate),
                                         _stream_ptr(stream), ctypes.byref(self._h))
        else:
            assert off.is_cuda and off.dtype == torch.int64 and ind.dtype == torch.int32
            st = N.lib().tc_graph_create(n, off.data_ptr(), ind.data_ptr() if ind.numel() else None,
                                         N.TC_MEM_DEVICE, slack, int(validate), _stream_ptr(stream),
                                         ctypes.byref(self._h))
        N.check(st)
        self.n = n

    @classmethod
    def from_csr(cls, csr, **kw) -> "Graph":
        return cls(csr.n, csr.off, csr.ind, **kw)

    def close(self):
        if self._h:
            N.lib().tc_graph_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def info(self):
        nv, used, alloc = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        N.check(N.lib().tc_graph_info(self._h, ctypes.byref(nv), ctypes.byref(used), ctypes.byref(alloc)))
        return nv.value, used.value, alloc.value

    def export(self):
        n, m, _ = self.info()
        off = np.zeros(n + 1, np.int64)
        ind = np.zeros(max(m, 1), np.int32)
        N.check(N.lib().tc_graph_export(self._h, off.ctypes.data, ind.ctypes.data))
        return off, ind[:m]

    def validate(self, stream=None):
        N.check(N.lib().tc_graph_validate(self._h, _stream_ptr(stream)))

    def count(self, pv_mode: int = N.TC_PV_HANDLE, per_vertex=None, triangles_dev=None, sched=None,
              sync: bool = True, stream=None):
        """Static count. Returns (T, CountInfo) when sync, else None."""
        info = N.CountInfo() if sync else None
        st = N.lib().tc_count_static(self._h, pv_mode, _ptr(per_vertex), _ptr(triangles_dev),
                                     ctypes.byref(info) if sync else None,
                                     ctypes.byref(sched) if sched is not None else None, _stream_ptr(stream))
        N.check(st)
        return (info.triangles, info) if sync else None


def _apply_batch(self, src, dst, is_delete=None, per_vertex=None, delta_dev=None, sched=None, sync=True,
                 stream=None):
    """tc_apply_batch: undirected updates {src[i], dst[i]}; numpy arrays (host) or CUDA tensors.
    Returns BatchInfo when sync."""
    import torch
    info = N.BatchInfo() if sync else None
    if isinstance(src, np.ndarray):
        s = np.ascontiguousarray(src, dtype=np.int32)
        d = np.ascontiguousarray(dst, dtype=np.int32)
        dl = None if is_delete is None else np.ascontiguousarray(is_delete, dtype=np.uint8)
        b = s.size
        args = (s.ctypes.data if b else None, d.ctypes.data if b else None,
                dl.ctypes.data if (dl is not None and b) else None, b, N.TC_MEM_HOST)
    else:
        assert src.is_cuda and src.dtype == torch.int32 and dst.dtype == torch.int32
        b = src.numel()
        args = (src.data_ptr() if b else None, dst.data_ptr() if b else None,
                is_delete.data_ptr() if (is_delete is not None and b) else None, b, N.TC_MEM_DEVICE)
    st = N.lib().tc_apply_batch(self._h, *args, _ptr(per_vertex), _ptr(delta_dev),
                                ctypes.byref(info) if sync else None,
                                ctypes.byref(sched) if sched is not None else None, _stream_ptr(stream))
    N.check(st)
    return info


Graph.apply_batch = _apply_batch


class Pipeline:
    """tc_pipeline: streaming batches of device updates through one captured CUDA graph per
    batch-size bin (same semantics as Graph.apply_batch)."""

    def __init__(self, graph: Graph, max_batch: int, sched=None):
        self._p = ctypes.c_void_p()
        N.check(N.lib().tc_pipeline_create(graph._h, max_batch, ctypes.byref(sched) if sched is not None else None,
                                           ctypes.byref(self._p)))
        self.graph = graph

    def apply(self, src, dst, is_delete=None, per_vertex=None, delta_dev=None, stream=None):
        """Enqueue one batch (int32 CUDA tensors src/dst, optional uint8 is_delete)."""
        b = src.numel()
        N.check(N.lib().tc_pipeline_apply(self._p, _ptr(src) if b else None, _ptr(dst) if b else None,
                                          _ptr(is_delete) if (is_delete is not None and b) else None, b,
                                          _ptr(per_vertex), _ptr(delta_dev), _stream_ptr(stream)))

    def prepare(self, per_vertex=None, delta_dev=None, stream=None):
        """Reserve pool headroom and capture every bin's graph for these outputs now."""
        N.check(N.lib().tc_pipeline_prepare(self._p, _ptr(per_vertex), _ptr(delta_dev), _stream_ptr(stream)))

    def sync(self):
        info = N.BatchInfo()
        N.check(N.lib().tc_pipeline_sync(self._p, ctypes.byref(info)))
        return info

    def autotune(self, batches: int):
        N.check(N.lib().tc_pipeline_autotune(self._p, batches))

    def info(self):
        """[(bin capacity, delta-kernel CTAs per SM)] per bin."""
        nb = ctypes.c_int32(0)
        caps = (ctypes.c_int64 * 16)()
        blocks = (ctypes.c_int32 * 16)()
        N.check(N.lib().tc_pipeline_info(self._p, ctypes.byref(nb), caps, blocks))
        return [(int(caps[i]), int(blocks[i])) for i in range(nb.value)]

    def plan(self) -> "N.PipelinePlan":
        """The tuned bins (which graph serves each bin) and delta-kernel tile shapes."""
        p = N.PipelinePlan()
        N.check(N.lib().tc_pipeline_plan_get(self._p, ctypes.byref(p)))
        return p

    def set_plan(self, plan) -> None:
        N.check(N.lib().tc_pipeline_plan_set(self._p, ctypes.byref(plan)))

    def profile(self, on: bool = True) -> None:
        """Record the delta kernels' event times and algorithmic bytes (before prepare())."""
        N.check(N.lib().tc_pipeline_profile(self._p, int(on)))

    def stats(self) -> dict:
        b, ms, by = ctypes.c_int64(), ctypes.c_double(), ctypes.c_int64()
        N.check(N.lib().tc_pipeline_stats(self._p, ctypes.byref(b), ctypes.byref(ms), ctypes.byref(by)))
        return {"batches": b.value, "delta_ms": ms.value, "delta_bytes": by.value}

    def set_wait_bound(self, wait_ns: int, extra_arrivals: int = 0) -> None:
        N.check(N.lib().tc_pipeline_set_wait_bound(self._p, wait_ns, extra_arrivals))

    def close(self):
        if self._p:
            N.lib().tc_pipeline_destroy(self._p)
            self._p = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def count_all_triangles(graph: Graph, out, sched=None, stream=None):
    """callDeviceAllTriangles: out[v] = 2 t(v) for v < nv (device int32 tensor, >= nv entries)."""
    return graph.count(N.TC_PV_HANDLE, out, sched=sched, stream=stream)


def count_all_triangles_csr(n: int, d_off, d_ind, out, pv_mode: int = N.TC_PV_CSR, sched=None, sync=True,
                            stream=None, triangles_dev=None):
    """callDeviceAllTrianglesCSR on device CSR tensors (int32 or int64 offsets)."""
    import torch
    info = N.CountInfo() if sync else None
    fn = N.lib().tc_count_csr32 if d_off.dtype == torch.int32 else N.lib().tc_count_csr64
    st = fn(n, d_off.data_ptr(), d_ind.data_ptr() if d_ind.numel() else None, pv_mode, _ptr(out),
            _ptr(triangles_dev), ctypes.byref(info) if sync else None,
            ctypes.byref(sched) if sched is not None else None, _stream_ptr(stream))
    N.check(st)
    return (info.triangles, info) if sync else None


def shard_ranges(prefix, nshards: int):
    """The static count's multi-GPU split rule (tc_shard_ranges, host side): given the exclusive
    prefix of the centres' predicted work (int64[n+1]), the first centre of each of nshards
    shards; shard r counts the centres [lo[r], lo[r+1])."""
    prefix = np.ascontiguousarray(prefix, dtype=np.int64)
    n = prefix.size - 1
    lo = np.zeros(nshards + 1, np.int32)
    N.check(N.lib().tc_shard_ranges(prefix.ctypes.data, n, nshards, lo.ctypes.data))
    return lo
