"""Generate tests/golden/bench_configs.json: known answers for the benchmark graphs.

    make -f oracle/Makefile REF=<reference tree>
    python tests/golden/make_bench_golden.py [scale ...]

Every answer comes from the reference's own CPU counter: its unmodified hostSingleIntersection
(tests/cct.cpp:32-69), compiled into oracle/_ref/libref_cct.so, run over every directed edge on
all host cores, with each edge's count (its triNE entry, tests/cct.cpp:71-89) summed into the
edge's source vertex. That gives, per graph:

  all_triangles              the reference's allTriangles (6T)
  per_vertex_handle_digest   digest of int32 2t(v) as the handle kernel writes it (two's-complement
                             wrap where 2t(v) >= 2^31, as the reference's int32 triangle_t does)
  per_vertex_csr_digest      digest of the int32 forward counts (edges with dest > src), the
                             raw-CSR kernel's convention (tests/cct_csr.cu:246-249)
  per_vertex_handle64_digest digest of the exact int64 2t(v)
  max_2t, wraps_int32        the largest 2t(v) and how many vertices wrap in int32

The scaled oracle (oracle_fast_count, an oriented counter) must agree on the total and the
per-vertex 2t(v); it is recorded beside the reference as a cross-check.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from custingeralg_b200 import generators as G  # noqa: E402
from oracle import pyoracle as O  # noqa: E402
from tests.util import digest  # noqa: E402

SPECS = {20: (16, 2), 22: (16, 4), 24: (16, 3), 16: (16, 2), 18: (16, 2)}


def main():
    scales = [int(x) for x in sys.argv[1:]] or [16, 18, 20]
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libref_cct.so missing: make -f oracle/Makefile REF=<reference tree>")
    path = os.path.join(HERE, "bench_configs.json")
    out = json.load(open(path)) if os.path.exists(path) else {}
    for sc in scales:
        ef, seed = SPECS[sc]
        t0 = time.time()
        g = G.rmat(sc, ef, 0.57, 0.19, 0.19, seed=seed)
        t1 = time.time()
        ref_all, pv64, fw64 = O.ref_host_count_triangles_pervertex(g.n, g.off, g.ind)
        t_ref = time.time() - t1
        fast_all, pv_fast = O.fast_count(g.n, g.off, g.ind)
        pv32 = pv64.astype(np.int32)  # two's-complement wrap, as int32 arithmetic gives
        assert ref_all == fast_all, (ref_all, fast_all)
        assert np.array_equal(pv32, pv_fast), "oriented oracle disagrees with the reference per vertex"
        assert int(pv64.sum()) == ref_all and 2 * int(fw64.sum()) == ref_all
        rec = {"n": g.n, "m": g.m, "triangles": ref_all // 6, "all_triangles": ref_all,
               "per_vertex_handle_digest": digest(pv32),
               "per_vertex_csr_digest": digest(fw64.astype(np.int32)),
               "per_vertex_handle64_digest": digest(pv64),
               "max_2t": int(pv64.max()) if g.n else 0,
               "wraps_int32": int((pv64 >= 2**31).sum()),
               "graph_digest": digest(g.off) + digest(g.ind),
               "checked_by": "reference hostSingleIntersection over every directed edge, summed per source vertex "
                             f"({os.cpu_count()} threads, {t_ref:.0f} s); oracle_fast_count agrees"}
        out[f"rmat{sc}_ef{ef}_s{seed}"] = rec
        print(sc, rec["triangles"], rec["max_2t"], rec["wraps_int32"], f"{time.time() - t0:.1f}s", flush=True)
        with open(path, "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
