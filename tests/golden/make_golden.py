"""Generate tests/golden/static_tc.json: known answers for the static triangle count.

Run in a container that holds the reference sources (the reference's own CPU counter is built
into oracle/_ref/ from tests/cct.cpp by oracle/Makefile):

    make -f oracle/Makefile REF=<reference tree> && python tests/golden/make_golden.py

For each graph it records a digest of the generated CSR (so generator drift is caught), the
total of the reference's hostCountTriangles (tests/cct.cpp:71-89, = 6T) and digests of the
per-edge counts triNE it writes, plus digests of the two per-vertex outputs the GPU kernels
must reproduce (devicecuStingerAllTriangles: 2 t(v); count_all_trianglesGPU: forward counts).
Tiny graphs also keep the arrays themselves.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from custingeralg_b200 import generators as G  # noqa: E402
from oracle import pyoracle as O  # noqa: E402


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<")).tobytes()).hexdigest()[:32]


def small_graphs():
    tri_pendant = G.from_pairs(4, [0, 1, 0, 2], [1, 2, 2, 3], name="triangle_pendant")
    bowtie = G.from_pairs(5, [0, 1, 0, 2, 3, 2], [1, 2, 2, 3, 4, 4], name="bowtie")
    two_tri = G.from_pairs(6, [0, 1, 0, 3, 4, 3], [1, 2, 2, 4, 5, 5], name="two_triangles")
    path = G.from_pairs(6, [0, 1, 2, 3, 4], [1, 2, 3, 4, 5], name="path6")
    empty = G.from_pairs(5, [], [], name="empty5")
    single = G.from_pairs(2, [0], [1], name="single_edge")
    return [G.complete(3), G.complete(4), G.complete(5), G.complete(8), G.complete(33), G.complete(70),
            G.star(10), tri_pendant, bowtie, two_tri, path, empty, single]


def graph_specs():
    return [
        ("er14_d16_s1", lambda: G.erdos_renyi(1 << 14, 16.0 / (1 << 14), seed=1)),
        ("rmat10_ef16_s2", lambda: G.rmat(10, 16, seed=2)),
        ("rmat12_ef16_s2", lambda: G.rmat(12, 16, seed=2)),
        ("rmat14_ef16_s2", lambda: G.rmat(14, 16, seed=2)),
        ("rmat12_ef16_noise_s7", lambda: G.rmat(12, 16, seed=7, noise=True)),
        ("ba4096_m8_s1", lambda: G.barabasi_albert(4096, 8, seed=1)),
        ("grid64_r05_s1", lambda: G.grid_rewired(64, 0.05, seed=1)),
        # rewired grids whose random edges close triangles (the 5 % grid above has none)
        ("grid128_r05_s1", lambda: G.grid_rewired(128, 0.05, seed=1)),
        ("grid64_r50_s1", lambda: G.grid_rewired(64, 0.5, seed=1)),
    ]


def record(g, keep_arrays: bool):
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libref_cct.so missing: build it with make -f oracle/Makefile REF=<reference tree>")
    ref_total, ref_tri = O.ref_host_count_triangles(g.n, g.off, g.ind, per_edge=True)
    tot, tri = O.host_count_triangles(g.n, g.off, g.ind, per_edge=True)
    assert tot == ref_total and np.array_equal(tri, ref_tri), g.name
    pv = O.static_per_vertex(g.n, g.off, g.ind)
    cpv = O.csr_per_vertex(g.n, g.off, g.ind)
    r = {
        "n": int(g.n), "m": int(g.m),
        "graph_digest": digest(g.off) + digest(g.ind),
        "ref_all_triangles": int(ref_total),
        "triangles": int(ref_total // 6),
        "triNE_digest": digest(ref_tri),
        "per_vertex_handle_digest": digest(pv),
        "per_vertex_csr_digest": digest(cpv),
        "per_vertex_handle_sum": int(pv.astype(np.int64).sum()),
        "per_vertex_csr_sum": int(cpv.astype(np.int64).sum()),
    }
    if keep_arrays:
        r["off"] = g.off.tolist()
        r["ind"] = g.ind.tolist()
        r["per_vertex_handle"] = pv.tolist()
        r["per_vertex_csr"] = cpv.tolist()
    return r


def main():
    out = {"generator": "custingeralg_b200.generators (counter-based splitmix64)",
           "reference_counter": "tests/cct.cpp:71-89 hostCountTriangles, built from the reference sources",
           "graphs": {}}
    for g in small_graphs():
        out["graphs"][g.name] = record(g, keep_arrays=g.n <= 80)
    for name, make in graph_specs():
        g = make()
        g.name = name
        out["graphs"][name] = record(g, keep_arrays=False)
        print(name, out["graphs"][name]["n"], out["graphs"][name]["m"], out["graphs"][name]["triangles"])
    path = os.path.join(HERE, "static_tc.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    main()
