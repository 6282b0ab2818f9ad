"""Generate tests/golden/bench_configs.json: known answers for the benchmark graphs.

    python tests/golden/make_bench_golden.py [scale ...]

T and the per-vertex 2t(v) digest come from the scaled oracle (oracle_fast_count); where the
reference's own counter is built (oracle/_ref) and the graph is at most R-MAT scale 20, its
total over all directed edges (6T) is computed too and must agree.
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from custingeralg_b200 import generators as G  # noqa: E402
from oracle import pyoracle as O  # noqa: E402
from tests.util import digest  # noqa: E402

SPECS = {20: (16, 2), 22: (16, 4), 24: (16, 3), 16: (16, 2), 18: (16, 2)}


def main():
    scales = [int(x) for x in sys.argv[1:]] or [16, 18, 20]
    path = os.path.join(HERE, "bench_configs.json")
    out = json.load(open(path)) if os.path.exists(path) else {}
    for sc in scales:
        ef, seed = SPECS[sc]
        t0 = time.time()
        g = G.rmat(sc, ef, 0.57, 0.19, 0.19, seed=seed)
        tot, pv = O.fast_count(g.n, g.off, g.ind)
        rec = {"n": g.n, "m": g.m, "triangles": tot // 6, "all_triangles": tot,
               "per_vertex_handle_digest": digest(pv), "graph_digest": digest(g.off) + digest(g.ind),
               "checked_by": "oracle_fast_count"}
        if O.ref_available() and sc <= 20:
            ref_all = O.ref_host_count_triangles_omp(g.n, g.off, g.ind)
            assert ref_all == tot, (ref_all, tot)
            rec["checked_by"] += " + reference hostSingleIntersection over all directed edges"
        out[f"rmat{sc}_ef{ef}_s{seed}"] = rec
        print(sc, rec["triangles"], f"{time.time() - t0:.1f}s", flush=True)
        with open(path, "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
