"""Shared helpers for the tests (fixtures, graph zoo, digests)."""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

from custingeralg_b200 import generators as G

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<")).tobytes()).hexdigest()[:32]


def load_golden(name="static_tc.json"):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def small_graphs():
    tri_pendant = G.from_pairs(4, [0, 1, 0, 2], [1, 2, 2, 3], name="triangle_pendant")
    bowtie = G.from_pairs(5, [0, 1, 0, 2, 3, 2], [1, 2, 2, 3, 4, 4], name="bowtie")
    two_tri = G.from_pairs(6, [0, 1, 0, 3, 4, 3], [1, 2, 2, 4, 5, 5], name="two_triangles")
    path = G.from_pairs(6, [0, 1, 2, 3, 4], [1, 2, 3, 4, 5], name="path6")
    empty = G.from_pairs(5, [], [], name="empty5")
    single = G.from_pairs(2, [0], [1], name="single_edge")
    return [G.complete(3), G.complete(4), G.complete(5), G.complete(8), G.complete(33), G.complete(70),
            G.star(10), tri_pendant, bowtie, two_tri, path, empty, single]


GRAPH_SPECS = {
    "er14_d16_s1": lambda: G.erdos_renyi(1 << 14, 16.0 / (1 << 14), seed=1),
    "rmat10_ef16_s2": lambda: G.rmat(10, 16, seed=2),
    "rmat12_ef16_s2": lambda: G.rmat(12, 16, seed=2),
    "rmat14_ef16_s2": lambda: G.rmat(14, 16, seed=2),
    "rmat12_ef16_noise_s7": lambda: G.rmat(12, 16, seed=7, noise=True),
    "ba4096_m8_s1": lambda: G.barabasi_albert(4096, 8, seed=1),
    "grid64_r05_s1": lambda: G.grid_rewired(64, 0.05, seed=1),
    "grid128_r05_s1": lambda: G.grid_rewired(128, 0.05, seed=1),
    "grid64_r50_s1": lambda: G.grid_rewired(64, 0.5, seed=1),
}


def golden_graph(name):
    for g in small_graphs():
        if g.name == name:
            return g
    g = GRAPH_SPECS[name]()
    g.name = name
    return g


def random_graph(rng: np.random.Generator, n: int, k: int):
    s = rng.integers(0, n, k, dtype=np.int32)
    d = rng.integers(0, n, k, dtype=np.int32)
    return G.from_pairs(n, s, d, name=f"rand{n}_{k}")
