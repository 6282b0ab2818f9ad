"""The reference's own static-count driver, unmodified, running on this library (drop-in check).

oracle/Makefile compiles tests/cct.cpp from the reference tree against this repository's
include/ (cuStinger.hpp, update.hpp, utils.hpp, static_triangle_counting/cct.hpp) and links it
with libcustinger_tc.so and libtcgen.so (oracle/_ref/ref_cct_driver). The driver reads a DIMACS
file with readGraphDIMACS, builds a cuStinger handle with initializeCuStinger, then runs its
launch sweep (tests/cct.cpp:103-106, 171-206): for each of the 36 launch configurations it calls
callDeviceAllTrianglesCSR ("!!!" lines) and callDeviceAllTriangles ("###" lines) and prints the
sum of the per-vertex output. Those sums must be 3T (forward convention) and 6T (2 t(v) per
vertex) for every configuration.
"""
import os
import subprocess

import numpy as np
import pytest

from custingeralg_b200 import generators as G
from oracle import pyoracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_cct_driver")

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not os.path.exists(DRIVER), reason="driver not built")]


def write_dimacs(g, path):
    lines = [f"{g.n} {g.m // 2}"]
    for v in range(g.n):
        lines.append(" ".join(str(int(u) + 1) for u in g.ind[g.off[v]:g.off[v + 1]]))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


@pytest.mark.parametrize("name,make", [("rmat12", lambda: G.rmat(12, 16, seed=31)),
                                       ("ba11", lambda: G.barabasi_albert(1 << 11, 12, seed=32))])
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
