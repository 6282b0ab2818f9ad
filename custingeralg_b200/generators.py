"""Seeded synthetic graphs (ctypes over libtcgen.so, host C++/OpenMP).

Stand-ins for the graph files the reference drivers read (tests/cct.cpp:239-257). Every graph
is symmetric, without self-loops or duplicates, adjacency sorted ascending, int64 offsets and
int32 ids, and a pure function of its parameters.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


class _Csr(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("m", ctypes.c_int64),
                ("off", ctypes.POINTER(ctypes.c_int64)), ("ind", ctypes.POINTER(ctypes.c_int32))]


_lib = None


def _load():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "libtcgen.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run __graft_entry__.build() first")
        lib = ctypes.CDLL(path)
        i32, i64, u64, dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double
        p = ctypes.POINTER(_Csr)
        lib.tcgen_rmat.argtypes = [ctypes.c_int, ctypes.c_int, dbl, dbl, dbl, u64, ctypes.c_int, ctypes.c_int, p]
        lib.tcgen_er.argtypes = [i32, dbl, u64, ctypes.c_int, p]
        lib.tcgen_ba.argtypes = [i32, ctypes.c_int, u64, ctypes.c_int, p]
        lib.tcgen_grid.argtypes = [i32, dbl, u64, ctypes.c_int, p]
        lib.tcgen_from_pairs.argtypes = [i32, i64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, p]
        lib.tcgen_rmat_pairs.argtypes = [ctypes.c_int, i64, dbl, dbl, dbl, u64, ctypes.c_int, u64,
                                         ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        lib.tcgen_read.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, p]
        lib.tcgen_write_binary.argtypes = [ctypes.c_char_p, p]
        lib.tcgen_read.restype = ctypes.c_int
        lib.tcgen_write_binary.restype = ctypes.c_int
        lib.tcgen_free.argtypes = [p]
        for f in ("tcgen_rmat", "tcgen_er", "tcgen_ba", "tcgen_grid", "tcgen_from_pairs", "tcgen_rmat_pairs"):
            getattr(lib, f).restype = ctypes.c_int
        lib.tcgen_free.restype = None
        _lib = lib
    return _lib


@dataclass
class Csr:
    """Host CSR: off int64[n+1], ind int32[m]."""

    n: int
    off: np.ndarray
    ind: np.ndarray
    name: str = ""

    @property
    def m(self) -> int:
        return int(self.off[-1])

    def degrees(self) -> np.ndarray:
        return np.diff(self.off)

    def off32(self) -> np.ndarray:
        if self.m > np.iinfo(np.int32).max:
            raise OverflowError("graph has more than 2^31-1 directed edges; int32 offsets overflow")
        return self.off.astype(np.int32)


def _take(rc: int, g: _Csr, name: str) -> Csr:
    if rc != 0:
        raise ValueError(f"generator failed with code {rc}")
    lib = _load()
    try:
        n = int(g.n)
        off = np.ctypeslib.as_array(g.off, shape=(n + 1,)).copy()
        m = int(off[-1])
        ind = np.ctypeslib.as_array(g.ind, shape=(max(m, 1),))[:m].copy()
    finally:
        lib.tcgen_free(ctypes.byref(g))
    return Csr(n, off, ind, name)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 2, noise: bool = False, nthreads: int = 0) -> Csr:
    g = _Csr()
    rc = _load().tcgen_rmat(scale, edge_factor, a, b, c, seed, int(noise), nthreads, ctypes.byref(g))
    return _take(rc, g, f"rmat{scale}_ef{edge_factor}_s{seed}")


def erdos_renyi(n: int, p: float, seed: int = 1, nthreads: int = 0) -> Csr:
    g = _Csr()
    rc = _load().tcgen_er(n, p, seed, nthreads, ctypes.byref(g))
    return _take(rc, g, f"er{n}_p{p:.3g}_s{seed}")


def barabasi_albert(n: int, m0: int, seed: int = 1, nthreads: int = 0) -> Csr:
    g = _Csr()
    rc = _load().tcgen_ba(n, m0, seed, nthreads, ctypes.byref(g))
    return _take(rc, g, f"ba{n}_m{m0}_s{seed}")


def grid_rewired(side: int, rewire: float = 0.05, seed: int = 1, nthreads: int = 0) -> Csr:
    g = _Csr()
    rc = _load().tcgen_grid(side, rewire, seed, nthreads, ctypes.byref(g))
    return _take(rc, g, f"grid{side}_r{rewire}_s{seed}")


def from_pairs(n: int, src, dst, nthreads: int = 0, name: str = "pairs") -> Csr:
    s = np.ascontiguousarray(src, dtype=np.int32)
    d = np.ascontiguousarray(dst, dtype=np.int32)
    assert s.shape == d.shape
    g = _Csr()
    rc = _load().tcgen_from_pairs(n, s.size, s.ctypes.data, d.ctypes.data, nthreads, ctypes.byref(g))
    return _take(rc, g, name)


def rmat_pairs(scale: int, num_pairs: int, a: float = 0.57, b: float = 0.19, c: float = 0.19,
               seed: int = 4, stream: int = 1, noise: bool = False, nthreads: int = 0):
    """Raw R-MAT endpoint pairs (for update batches)."""
    s = np.empty(num_pairs, np.int32)
    d = np.empty(num_pairs, np.int32)
    rc = _load().tcgen_rmat_pairs(scale, num_pairs, a, b, c, seed, int(noise), stream, nthreads,
                                  s.ctypes.data, d.ctypes.data)
    if rc != 0:
        raise ValueError(f"generator failed with code {rc}")
    return s, d


def complete(n: int) -> Csr:
    """K_n (C(n,3) triangles)."""
    i, j = np.triu_indices(n, 1)
    return from_pairs(n, i, j, name=f"K{n}")


def star(n: int) -> Csr:
    """One centre joined to n-1 leaves (no triangles)."""
    return from_pairs(n, np.zeros(n - 1, np.int32), np.arange(1, n, dtype=np.int32), name=f"star{n}")


FMT_AUTO, FMT_DIMACS, FMT_SNAP, FMT_MTX, FMT_BINARY = 0, 1, 2, 3, 4
ERR_IO, ERR_FORMAT = 3, 4


class ReadError(RuntimeError):
    def __init__(self, code: int, path: str):
        super().__init__(f"{path}: cannot read graph (tcgen error {code})")
        self.code = code


def read_graph(path: str, fmt: int = FMT_AUTO, nthreads: int = 0) -> Csr:
    """Read a DIMACS (.graph), SNAP (.txt), MatrixMarket (.mtx) or binary cache (.tccsr) file into
    the symmetric, sorted, deduplicated CSR without self-loops (tcgen_read)."""
    g = _Csr()
    rc = _load().tcgen_read(os.fsencode(path), fmt, nthreads, ctypes.byref(g))
    if rc != 0:
        raise ReadError(rc, path)
    return _take(rc, g, os.path.basename(path))


def write_binary(g: Csr, path: str) -> None:
    """Write g as the binary CSR cache that read_graph(path) reads back unchanged."""
    off = np.ascontiguousarray(g.off, dtype=np.int64)
    ind = np.ascontiguousarray(g.ind, dtype=np.int32)
    c = _Csr(g.n, g.m, off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
             ind.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    rc = _load().tcgen_write_binary(os.fsencode(path), ctypes.byref(c))
    if rc != 0:
        raise ReadError(rc, path)


def write_dimacs(g: Csr, path: str) -> None:
    """Write g as a METIS / DIMACS-10 adjacency file (.graph): "n m" (m undirected edges), then one
    line per vertex with its 1-based neighbours; read_graph(path) reads it back unchanged."""
    off = np.asarray(g.off, dtype=np.int64)
    ids = (np.asarray(g.ind, dtype=np.int64) + 1).astype(str)
    with open(path, "w") as f:
        f.write(f"{g.n} {int(off[-1]) // 2}\n")
        for v in range(g.n):
            f.write(" ".join(ids[off[v]:off[v + 1]]) + "\n")


def write_snap(g: Csr, path: str) -> None:
    """Write g as a SNAP edge list (.txt): each undirected edge once, "u<TAB>v" with 0-based ids."""
    src = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(np.asarray(g.off, dtype=np.int64)))
    dst = np.asarray(g.ind, dtype=np.int64)
    keep = src < dst
    with open(path, "w") as f:
        f.write(f"# Undirected graph: {g.n} nodes, {int(keep.sum())} edges\n# FromNodeId\tToNodeId\n")
        np.savetxt(f, np.stack([src[keep], dst[keep]], axis=1), fmt="%d", delimiter="\t")


def write_mtx(g: Csr, path: str) -> None:
    """Write g as a MatrixMarket coordinate pattern file (.mtx), symmetric, lower triangle, 1-based."""
    src = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(np.asarray(g.off, dtype=np.int64)))
    dst = np.asarray(g.ind, dtype=np.int64)
    keep = src > dst
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern symmetric\n")
        f.write(f"{g.n} {g.n} {int(keep.sum())}\n")
        np.savetxt(f, np.stack([src[keep] + 1, dst[keep] + 1], axis=1), fmt="%d")


def write_graph(g: Csr, path: str) -> None:
    """Write g in the format its file name names, as the reference drivers pick their reader:
    .graph (DIMACS), .txt (SNAP), .mtx (MatrixMarket), anything else the binary cache."""
    if path.endswith(".graph"):
        write_dimacs(g, path)
    elif path.endswith(".txt"):
        write_snap(g, path)
    elif path.endswith(".mtx"):
        write_mtx(g, path)
    else:
        write_binary(g, path)


def main(argv=None) -> None:
    """python -m custingeralg_b200.generators {rmat,er,ba,grid} [options] --out FILE"""
    import argparse
    ap = argparse.ArgumentParser(description="Write a seeded synthetic graph (symmetric, sorted, no self-loops)")
    ap.add_argument("family", choices=["rmat", "er", "ba", "grid"])
    ap.add_argument("--scale", type=int, default=16, help="rmat: 2^scale vertices")
    ap.add_argument("--edge-factor", type=int, default=16, help="rmat: generated pairs per vertex")
    ap.add_argument("--abc", type=float, nargs=3, default=[0.57, 0.19, 0.19], help="rmat quadrant weights a b c")
    ap.add_argument("--n", type=int, default=1 << 14, help="er, ba: vertices")
    ap.add_argument("--degree", type=float, default=16.0, help="er: average degree")
    ap.add_argument("--m0", type=int, default=8, help="ba: edges per new vertex")
    ap.add_argument("--side", type=int, default=256, help="grid: side x side vertices")
    ap.add_argument("--rewire", type=float, default=0.05, help="grid: rewiring probability")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", required=True, help=".graph, .txt, .mtx or a binary cache (.tccsr)")
    a = ap.parse_args(argv)
    if a.family == "rmat":
        g = rmat(a.scale, a.edge_factor, *a.abc, seed=a.seed)
    elif a.family == "er":
        g = erdos_renyi(a.n, a.degree / a.n, seed=a.seed)
    elif a.family == "ba":
        g = barabasi_albert(a.n, a.m0, seed=a.seed)
    else:
        g = grid_rewired(a.side, a.rewire, seed=a.seed)
    write_graph(g, a.out)
    print(f"{a.out}: n={g.n} directed edges={g.m}")


if __name__ == "__main__":
    main()

