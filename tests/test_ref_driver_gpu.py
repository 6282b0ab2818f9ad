"""The reference's own drivers, unmodified, running on this library (drop-in check).

oracle/Makefile compiles tests/cct.cpp from the reference tree against this repository's
include/ (cuStinger.hpp, update.hpp, utils.hpp, static_triangle_counting/cct.hpp) and links it
with libcustinger_tc.so and libtcgen.so (oracle/_ref/ref_cct_driver). The driver reads a DIMACS
file with readGraphDIMACS, builds a cuStinger handle with initializeCuStinger, then runs its
launch sweep (tests/cct.cpp:103-106, 171-206): for each of the 36 launch configurations it calls
callDeviceAllTrianglesCSR ("!!!" lines) and callDeviceAllTriangles ("###" lines) and prints the
sum of the per-vertex output. Those sums must be 3T (forward convention) and 6T (2 t(v) per
vertex) for every configuration.

oracle/_ref/ref_upd_driver is the reference's streaming driver (tests/cct_upd.cpp), built the
same way. It counts the graph (callDeviceAllTriangles), removes 5 x k random edges, counts the
reduced graph, then reinserts them in 5 symmetric batches that also carry 1000 repeats within the
batch and 1000 edges already in the graph (tests/cct_upd.cpp:282-342): sortDeviceBUD,
edgeInsertionsSorted, callDeviceNewTriangles per batch. It prints the per-vertex sum of the
created triangles and the difference of the two static sums; they must agree, and the first
static sum must be 6T.
"""
import re
import os
import subprocess

import numpy as np
import pytest

from custingeralg_b200 import generators as G
from oracle import pyoracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_cct_driver")
UPD_DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_upd_driver")

pytestmark = pytest.mark.gpu


def write_dimacs(g, path):
    lines = [f"{g.n} {g.m // 2}"]
    for v in range(g.n):
        lines.append(" ".join(str(int(u) + 1) for u in g.ind[g.off[v]:g.off[v + 1]]))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


@pytest.mark.parametrize("name,make", [("rmat12", lambda: G.rmat(12, 16, seed=31)),
                                       ("ba11", lambda: G.barabasi_albert(1 << 11, 12, seed=32))])
@pytest.mark.skipif(not os.path.exists(DRIVER), reason="driver not built")
def test_reference_driver_runs_on_this_library(tmp_path, name, make):
    g = make()
    path = tmp_path / f"{name}.graph"
    write_dimacs(g, str(path))
    tot, _ = O.fast_count(g.n, g.off, g.ind, per_vertex=False)
    T = tot // 6
    r = subprocess.run([DRIVER, str(path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    csr = [ln.split() for ln in r.stdout.splitlines() if ln.startswith("!!!")]
    handle = [ln.split() for ln in r.stdout.splitlines() if ln.startswith("###")]
    assert len(csr) == 36 and len(handle) == 36          # 1 x 6 block sizes x 6 lanes per edge
    # "!!! blocks sps tsp nbl shifter <tab> sum <tab> time"
    assert {int(f[6]) for f in csr} == {3 * T}
    assert {int(f[6]) for f in handle} == {6 * T}
    assert f"Vertices: {g.n}" in r.stdout


@pytest.mark.skipif(not os.path.exists(UPD_DRIVER), reason="driver not built")
@pytest.mark.parametrize("name,make,k", [("rmat14", lambda: G.rmat(14, 16, seed=33), 4000),
                                         ("ba13", lambda: G.barabasi_albert(1 << 13, 10, seed=34), 2000)])
def test_reference_streaming_driver_runs_on_this_library(tmp_path, name, make, k):
    g = make()
    path = tmp_path / f"{name}.graph"          # ".graph": the driver picks readGraphDIMACS by name
    write_dimacs(g, str(path))
    tot, _ = O.fast_count(g.n, g.off, g.ind, per_vertex=False)
    r = subprocess.run([UPD_DRIVER, str(path), str(k)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = r.stdout

    def grab(label):
        m = re.search(re.escape(label) + r"\s*(-?\d+)", out)
        assert m, (label, out[-2000:])
        return int(m.group(1))

    assert grab("Triangles in original graph =") == tot
    reduced = grab("Triangles in new reduced graph =")
    created = grab("Triangles created by batch update =")
    assert created == grab("============ should be") == tot - reduced
    assert 0 < reduced < tot and created % 6 == 0
    assert f"Vertices: {g.n}" in out
