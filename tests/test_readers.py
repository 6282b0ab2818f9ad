"""Graph file readers and the binary CSR cache (host code, no GPU).

The reference drivers read their inputs through readGraphDIMACS / readGraphSNAP /
readGraphMatrixMarket (tests/cct.cpp:239-257), from the absent cuStinger core. These readers must
hand the counter the symmetric, sorted, deduplicated CSR without self-loops; every test compares
a hand-written file with the CSR the same edges give through tcgen_from_pairs.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from custingeralg_b200 import generators as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def expect(n, pairs):
    a = np.array(pairs, dtype=np.int32).reshape(-1, 2)
    return G.from_pairs(n, a[:, 0], a[:, 1])


def same(g, h):
    return g.n == h.n and np.array_equal(g.off, h.off) and np.array_equal(g.ind, h.ind)


EDGES = [(0, 1), (0, 2), (1, 2), (2, 3), (3, 4), (1, 4)]


def test_dimacs_plain_and_one_sided(tmp_path):
    p = tmp_path / "g.graph"
    # vertex 5 (1-based) lists 2 but 2 does not list 5: the reader symmetrizes; a self-loop on 4
    p.write_text("% comment\n5 6\n2 3\n1 3 5\n1 2 4\n3 5 4\n4 2\n")
    assert same(G.read_graph(str(p)), expect(5, EDGES))


def test_dimacs_with_weights(tmp_path):
    p = tmp_path / "w.graph"
    # fmt 11: one vertex weight, then (neighbour, edge weight) pairs
    p.write_text("5 6 11\n7 2 1 3 9\n7 1 1 3 2 5 4\n7 1 9 2 2 4 1\n7 3 1 5 3\n7 4 3 2 4\n")
    assert same(G.read_graph(str(p)), expect(5, EDGES))


def test_dimacs_trailing_isolated_vertices(tmp_path):
    p = tmp_path / "iso.graph"
    p.write_text("6 1\n2\n1\n")      # vertices 3..6 have no lines at all
    g = G.read_graph(str(p))
    assert same(g, expect(6, [(0, 1)]))


def test_snap_edge_list(tmp_path):
    p = tmp_path / "e.txt"
    p.write_text("# Directed graph\n# FromNodeId\tToNodeId\n0\t1\n1\t0\n0\t2\n2\t1\n2\t3\n3\t4\n"
                 "4\t1\n3\t3\n0\t1\n")
    assert same(G.read_graph(str(p)), expect(5, EDGES))


@pytest.mark.parametrize("field,sym", [("pattern", "symmetric"), ("real", "general"), ("integer", "general")])
def test_matrix_market(tmp_path, field, sym):
    p = tmp_path / "m.mtx"
    val = {"pattern": "", "real": " 1.5e0", "integer": " 3"}[field]
    lines = [f"{i + 1} {j + 1}{val}" for i, j in EDGES] + [f"4 4{val}"]
    p.write_text(f"%%MatrixMarket matrix coordinate {field} {sym}\n% comment\n5 5 {len(lines)}\n" +
                 "\n".join(lines) + "\n")
    assert same(G.read_graph(str(p)), expect(5, EDGES))


def test_binary_cache_roundtrip_and_auto_format(tmp_path):
    g = G.rmat(10, 8, seed=4)
    p = tmp_path / "r.tccsr"
    G.write_binary(g, str(p))
    h = G.read_graph(str(p))
    assert same(g, h)
    # by name, as the reference driver picks its reader
    q = tmp_path / "r.graph"
    lines = [f"{g.n} {g.m // 2}"]
    for v in range(g.n):
        lines.append(" ".join(str(int(u) + 1) for u in g.ind[g.off[v]:g.off[v + 1]]))
    q.write_text("\n".join(lines) + "\n")
    assert same(G.read_graph(str(q)), g)


def test_errors(tmp_path):
    with pytest.raises(G.ReadError) as e:
        G.read_graph(str(tmp_path / "missing.graph"))
    assert e.value.code == G.ERR_IO
    bad = tmp_path / "bad.mtx"
    bad.write_text("%%MatrixMarket matrix coordinate pattern general\n3 3 2\n1 2\n")  # nnz short
    with pytest.raises(G.ReadError) as e:
        G.read_graph(str(bad))
    assert e.value.code == G.ERR_FORMAT
    bad2 = tmp_path / "bad2.graph"
    bad2.write_text("3 1\n2\n9\n")  # neighbour id out of range
    with pytest.raises(G.ReadError):
        G.read_graph(str(bad2))
    corrupt = tmp_path / "c.tccsr"
    corrupt.write_bytes(b"TCCSRv1\x00" + b"\x01" * 20)
    with pytest.raises(G.ReadError):
        G.read_graph(str(corrupt))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_custinger_reader_entry_points_compile_and_agree(tmp_path):
    """The reference driver's call shape (tests/cct.cpp:235-254) against include/utils.hpp."""
    src = tmp_path / "drv.cpp"
    src.write_text(r'''
#include <cstdio>
#include <cstdlib>
#include "utils.hpp"
int main(int argc, char** argv) {
  length_t nv, ne, *off;
  vertexId_t* adj;
  bool isRmat = false;
  readGraphDIMACS(argv[1], &off, &adj, &nv, &ne, isRmat);
  unsigned long long chk = 0;
  for (length_t v = 0; v < nv; ++v)
    for (length_t k = off[v]; k < off[v + 1]; ++k) chk = chk * 31 + (unsigned long long)(adj[k] + 7 * v);
  printf("%d %d %llu\n", nv, ne, chk);
  free(off);
  free(adj);
  return 0;
}
''')
    exe = tmp_path / "drv"
    cuda_inc = "/usr/local/cuda/include"
    lib_dir = os.path.join(ROOT, "custingeralg_b200")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", cuda_inc, str(src),
                    "-L", lib_dir, "-ltcgen", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    p = tmp_path / "g.graph"
    p.write_text("5 6\n2 3\n1 3 5\n1 2 4\n3 5\n4 2\n")
    out = subprocess.run([str(exe), str(p)], check=True, capture_output=True, text=True).stdout.split()
    g = expect(5, EDGES)
    chk = 0
    for v in range(g.n):
        for k in range(g.off[v], g.off[v + 1]):
            chk = (chk * 31 + int(g.ind[k]) + 7 * v) % (1 << 64)
    assert [int(x) for x in out] == [g.n, g.m, chk]


@pytest.mark.parametrize("ext", [".graph", ".txt", ".mtx", ".tccsr"])
@pytest.mark.parametrize("make", [lambda: G.rmat(10, 8, seed=7), lambda: G.barabasi_albert(500, 3, seed=8),
                                  lambda: G.from_pairs(40, np.array([0, 5], np.int32), np.array([1, 6], np.int32))],
                         ids=["rmat10", "ba500", "sparse_with_isolated"])
def test_writers_round_trip(tmp_path, ext, make):
    """write_graph in every format, read back by name, gives the same CSR, isolated vertices
    included where the format has a vertex count (DIMACS and MatrixMarket headers, the binary
    cache). A SNAP edge list has none: the reader sizes the graph by the largest endpoint."""
    g = make()
    p = tmp_path / f"g{ext}"
    G.write_graph(g, str(p))
    h = G.read_graph(str(p))
    if ext in (".txt",):
        # an edge list holds no vertex count: ids past the largest endpoint are not represented
        last = int(np.max(np.nonzero(np.diff(g.off))[0])) + 1 if g.m else 0
        assert h.n == last
        assert np.array_equal(h.off, g.off[: last + 1]) and np.array_equal(h.ind, g.ind)
    else:
        assert same(g, h)


def test_generator_cli(tmp_path):
    out = tmp_path / "er.graph"
    from custingeralg_b200 import generators as GM
    GM.main(["er", "--n", "2000", "--degree", "6", "--seed", "3", "--out", str(out)])
    assert same(G.read_graph(str(out)), G.erdos_renyi(2000, 6 / 2000, seed=3))
    out2 = tmp_path / "r.tccsr"
    GM.main(["rmat", "--scale", "9", "--edge-factor", "4", "--seed", "5", "--out", str(out2)])
    assert same(G.read_graph(str(out2)), G.rmat(9, 4, seed=5))
