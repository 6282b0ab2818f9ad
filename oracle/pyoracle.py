"""ctypes bindings for the CPU oracle: TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, as the checker.
  - liboracle.so: the plain-C restatement in tc_oracle.c (always present after build);
  - _ref/libref_cct.so: the reference's own hostCountTriangles (tests/cct.cpp:71-89) compiled
    from the reference sources by oracle/Makefile (present when the reference was available at
    build time; it travels with the repository snapshot, the sources do not);
  - _ref/libref_cct_gpu.so: the reference's own raw-CSR GPU counter (tests/cct_csr.cu:228-285)
    compiled for sm_100a the same way, for side-by-side timing and per-vertex parity.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_ref = None
_ref_gpu = None

_P = ctypes.c_void_p


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: build the oracle (make -f oracle/Makefile)")
        L = ctypes.CDLL(path)
        i32, i64 = ctypes.c_int32, ctypes.c_int64
        L.oracle_single_intersection.argtypes = [i32, _P, i32, _P]
        L.oracle_single_intersection.restype = i32
        L.oracle_host_count_triangles.argtypes = [i32, _P, _P, _P, _P]
        L.oracle_static_per_vertex.argtypes = [i32, _P, _P, _P]
        L.oracle_csr_per_vertex.argtypes = [i32, _P, _P, _P]
        L.oracle_new_triangles.argtypes = [i32, _P, _P, _P, _P]
        L.oracle_sort_batch.argtypes = [i32, _P, _P, i64, _P, _P, _P, _P]
        L.oracle_fast_count.argtypes = [i32, _P, _P, ctypes.c_int, _P, _P]
        L.oracle_fast_count_shard.argtypes = [i32, _P, _P, ctypes.c_int, i32, i32, _P, _P]
        L.oracle_fast_count_shard.restype = None
        L.oracle_fast_count_range.argtypes = [i32, _P, _P, ctypes.c_int, i32, i32, _P, _P]
        L.oracle_fast_count_range.restype = None
        L.oracle_centre_cost.argtypes = [i32, _P, _P, ctypes.c_int, _P]
        L.oracle_centre_cost.restype = None
        L.oracle_host_count_sample.argtypes = [i32, _P, _P, _P, i32, ctypes.c_int]
        L.oracle_host_count_sample.restype = i64
        for f in ("oracle_host_count_triangles", "oracle_static_per_vertex", "oracle_csr_per_vertex",
                  "oracle_new_triangles", "oracle_sort_batch", "oracle_fast_count"):
            getattr(L, f).restype = None
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libref_cct.so"))


def ref():
    global _ref
    if _ref is None:
        path = os.path.join(_HERE, "_ref", "libref_cct.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: the reference was not present at build time")
        L = ctypes.CDLL(path)
        i32 = ctypes.c_int32
        L.ref_host_single_intersection.argtypes = [i32, i32, _P, i32, i32, _P]
        L.ref_host_single_intersection.restype = ctypes.c_int
        L.ref_host_count_triangles.argtypes = [i32, _P, _P, _P, _P]
        L.ref_host_count_triangles.restype = None
        L.ref_host_count_triangles_omp.argtypes = [i32, _P, _P, ctypes.c_int]
        L.ref_host_count_triangles_omp.restype = ctypes.c_int64
        L.ref_host_count_triangles_omp_sample.argtypes = [i32, _P, _P, _P, i32, ctypes.c_int]
        L.ref_host_count_triangles_omp_sample.restype = ctypes.c_int64
        L.ref_host_count_triangles_omp_pervertex.argtypes = [i32, _P, _P, _P, _P, ctypes.c_int]
        L.ref_host_count_triangles_omp_pervertex.restype = ctypes.c_int64
        _ref = L
    return _ref


def ref_gpu_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libref_cct_gpu.so"))


def ref_gpu():
    """The reference's callDeviceAllTrianglesCSR behind ref_gpu_count_csr(nv, d_off, d_ind, d_out,
    threads_per_intersection, shifter, blocks, block_size) -> cudaError_t (launch only, default
    stream). d_ind must have readable guard entries before and after the list array."""
    global _ref_gpu
    if _ref_gpu is None:
        path = os.path.join(_HERE, "_ref", "libref_cct_gpu.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: the reference was not present at build time")
        L = ctypes.CDLL(path)
        i32 = ctypes.c_int32
        L.ref_gpu_count_csr.argtypes = [i32, _P, _P, _P, i32, i32, i32, i32]
        L.ref_gpu_count_csr.restype = ctypes.c_int
        _ref_gpu = L
    return _ref_gpu


class _Batch(ctypes.Structure):
    _fields_ = [("b", ctypes.c_int64), ("src", _P), ("dst", _P), ("boff", _P), ("dup", _P)]


def _g(off, ind):
    off = np.ascontiguousarray(off, dtype=np.int64)
    ind = np.ascontiguousarray(ind, dtype=np.int32)
    if ind.size == 0:
        ind = np.zeros(1, np.int32)
    return off, ind


def host_count_triangles(n, off, ind, per_edge=False):
    """Restatement of hostCountTriangles: (total, triNE or None)."""
    off, ind = _g(off, ind)
    tri = np.zeros(max(int(off[-1]), 1), np.int32) if per_edge else None
    tot = np.zeros(1, np.int64)
    lib().oracle_host_count_triangles(n, _ptr(off), _ptr(ind), _ptr(tri) if per_edge else None, _ptr(tot))
    return int(tot[0]), (tri[: int(off[-1])] if per_edge else None)


def static_per_vertex(n, off, ind):
    off, ind = _g(off, ind)
    out = np.zeros(max(n, 1), np.int32)
    lib().oracle_static_per_vertex(n, _ptr(off), _ptr(ind), _ptr(out))
    return out[:n]


def csr_per_vertex(n, off, ind):
    off, ind = _g(off, ind)
    out = np.zeros(max(n, 1), np.int32)
    lib().oracle_csr_per_vertex(n, _ptr(off), _ptr(ind), _ptr(out))
    return out[:n]


def fast_count(n, off, ind, per_vertex=True, nthreads=0):
    off, ind = _g(off, ind)
    tot = np.zeros(1, np.int64)
    pv = np.zeros(max(n, 1), np.int32) if per_vertex else None
    lib().oracle_fast_count(n, _ptr(off), _ptr(ind), nthreads, _ptr(tot), _ptr(pv) if per_vertex else None)
    return int(tot[0]), (pv[:n] if per_vertex else None)


def sort_batch(n, off, ind, src, dst):
    """Sort a directed batch and flag duplicates against the graph BEFORE insertion.
    Returns (src_sorted, dst_sorted, boff, dup)."""
    off, ind = _g(off, ind)
    s = np.array(src, dtype=np.int32, copy=True)
    d = np.array(dst, dtype=np.int32, copy=True)
    b = s.size
    sb = s if b else np.zeros(1, np.int32)
    db = d if b else np.zeros(1, np.int32)
    boff = np.zeros(n + 1, np.int64)
    dup = np.zeros(max(b, 1), np.int32)
    lib().oracle_sort_batch(n, _ptr(off), _ptr(ind), b, _ptr(sb), _ptr(db), _ptr(boff), _ptr(dup))
    return sb[:b], db[:b], boff, dup[:b]


def new_triangles(n, off_after, ind_after, bsrc, bdst, boff, dup, out=None):
    """K1 + K2 - K3 per-vertex deltas of the streaming kernels, accumulated into out."""
    off, ind = _g(off_after, ind_after)
    out = np.zeros(n, np.int32) if out is None else out
    bs = np.ascontiguousarray(bsrc, np.int32)
    bd = np.ascontiguousarray(bdst, np.int32)
    bo = np.ascontiguousarray(boff, np.int64)
    du = np.ascontiguousarray(dup, np.int32)
    keep = (bs, bd, bo, du)
    bt = _Batch(bs.size, _ptr(bs) if bs.size else None, _ptr(bd) if bd.size else None, _ptr(bo),
                _ptr(du) if du.size else None)
    lib().oracle_new_triangles(n, _ptr(off), _ptr(ind), ctypes.byref(bt), _ptr(out))
    del keep
    return out


def ref_host_count_triangles(n, off, ind, per_edge=False):
    """The reference's own hostCountTriangles (int32 offsets, as its length_t)."""
    off32 = np.ascontiguousarray(off, dtype=np.int32)
    ind = np.ascontiguousarray(ind, dtype=np.int32)
    if ind.size == 0:
        ind = np.zeros(1, np.int32)
    tri = np.zeros(max(int(off32[-1]), 1), np.int32)
    tot = np.zeros(1, np.int64)
    ref().ref_host_count_triangles(n, _ptr(off32), _ptr(ind), _ptr(tri), _ptr(tot))
    return int(tot[0]), (tri[: int(off32[-1])] if per_edge else None)


def ref_host_count_triangles_omp(n, off, ind, nthreads=0):
    off32 = np.ascontiguousarray(off, dtype=np.int32)
    ind = np.ascontiguousarray(ind, dtype=np.int32)
    if ind.size == 0:
        ind = np.zeros(1, np.int32)
    return int(ref().ref_host_count_triangles_omp(n, _ptr(off32), _ptr(ind), nthreads))


def ref_host_count_triangles_pervertex(n, off, ind, nthreads=0):
    """The reference's hostSingleIntersection over every directed edge, each edge's count (its
    triNE entry, tests/cct.cpp:71-89) summed into its source vertex. Returns (6T, int64 2t(v) per
    vertex, int64 forward count per vertex: the sum over edges with dest > src only, the raw-CSR
    GPU counter's convention, tests/cct_csr.cu:246-249)."""
    off32 = np.ascontiguousarray(off, dtype=np.int32)
    ind = np.ascontiguousarray(ind, dtype=np.int32)
    if ind.size == 0:
        ind = np.zeros(1, np.int32)
    pv = np.zeros(max(n, 1), np.int64)
    fw = np.zeros(max(n, 1), np.int64)
    tot = int(ref().ref_host_count_triangles_omp_pervertex(n, _ptr(off32), _ptr(ind), _ptr(pv), _ptr(fw),
                                                           nthreads))
    return tot, pv[:n], fw[:n]


def ref_host_count_triangles_omp_sample(n, off32, ind, verts, nthreads=0):
    """The reference's per-edge intersections for the source vertices in `verts` only."""
    off32 = np.ascontiguousarray(off32, dtype=np.int32)
    ind = np.ascontiguousarray(ind, dtype=np.int32)
    verts = np.ascontiguousarray(verts, dtype=np.int32)
    if ind.size == 0:
        ind = np.zeros(1, np.int32)
    return int(ref().ref_host_count_triangles_omp_sample(n, _ptr(off32), _ptr(ind),
                                                         _ptr(verts) if verts.size else None, verts.size,
                                                         nthreads))


def sample_count(n, off, ind, verts, nthreads=0):
    """Restated per-edge loop over the source vertices in `verts` (sum of per-edge counts)."""
    off, ind = _g(off, ind)
    verts = np.ascontiguousarray(verts, dtype=np.int32)
    return int(lib().oracle_host_count_sample(n, _ptr(off), _ptr(ind), _ptr(verts) if verts.size else None,
                                              verts.size, nthreads))


def fast_count_shard(n, off, ind, shard, nshards, nthreads=0):
    """Total (6T share) and per-vertex counts of one vertex shard of the oriented count."""
    off, ind = _g(off, ind)
    tot = np.zeros(1, np.int64)
    pv = np.zeros(max(n, 1), np.int32)
    lib().oracle_fast_count_shard(n, _ptr(off), _ptr(ind), nthreads, shard, nshards, _ptr(tot), _ptr(pv))
    return int(tot[0]), pv[:n]


def fast_count_range(n, off, ind, lo, hi, nthreads=0):
    """Total (6T share) and per-vertex counts of the centres in [lo, hi) (a contiguous shard)."""
    off, ind = _g(off, ind)
    tot = np.zeros(1, np.int64)
    pv = np.zeros(max(n, 1), np.int32)
    lib().oracle_fast_count_range(n, _ptr(off), _ptr(ind), nthreads, lo, hi, _ptr(tot), _ptr(pv))
    return int(tot[0]), pv[:n]


def centre_cost(n, off, ind, nthreads=0):
    """Predicted work per centre (int32, units of 16) as the multi-GPU split balances it."""
    off, ind = _g(off, ind)
    cost = np.zeros(max(n, 1), np.int32)
    lib().oracle_centre_cost(n, _ptr(off), _ptr(ind), nthreads, _ptr(cost))
    return cost[:n]
