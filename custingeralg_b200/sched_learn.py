"""Learned scheduler for the static count: per-degree-cell strategy from a trained MLP.

The count kernel intersects each edge at its centre (the endpoint with the larger out-degree
a): the other endpoint's list N+(o), b <= a entries, goes through the centre's shared-memory
hash set by one of two strategies: the warp streams it with coalesced loads (one list at a
time), or one lane walks it (the lanes of a warp walk different short lists at once). The fixed
heuristic picks by a length threshold (lane_max_deg). Here a 3-layer FP32 MLP of width 64
predicts the cost per edge of each strategy from the features of the edge's degree cell
(log2 a, log2 b buckets): mean log2(1 + a), mean log2(1 + b), mean b/a and cell id / 255. The
cell's choice goes into the scheduler table; the fixed rule stays the fallback for cells where
the network does not predict a clear gain (tc_sched_learned). The network only changes which
strategy runs, never what is counted.

Pipeline, all on the GPU through the library's own kernels:

  collect   for each training graph, count once, read its per-cell statistics (tc_cell_stats),
            then time the count kernel with only one cell's edges active (cell_filter) under
            each strategy (a table that forces it), minus the time with no cell active.
            Label: log2 of nanoseconds per edge of that cell.
  train     full-batch Adam through tc_mlp_train (the library's forward/backward kernels,
            whose gradients the tests check against the CPU oracle).
  evaluate  held-out graphs: count with the fixed heuristic and with the learned table;
            the counts must agree; report the time of each.

    python -m custingeralg_b200.sched_learn all --out-dir DIR [--quick]

writes DIR/sched_dataset.npz, DIR/sched_mlp.bin (float32[TC_MLP_PARAMS]) and
DIR/sched_report.json. The committed weights live in custingeralg_b200/data/sched_mlp.bin.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import time

import numpy as np

from . import api, generators as G, native as N

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "data", "sched_mlp.bin")
MIN_CELL_EDGES = 4000   # cells with fewer edges are not timed (their labels would be noise)
MIN_CELL_MS = 0.002     # a cell whose time above the empty launch is below this gets no label


# ---- graphs ---------------------------------------------------------------------------------

def training_specs(quick: bool = False):
    """The 64 seeded training graphs: R-MAT (scale 16-22, a in [0.45, 0.6]), Erdos-Renyi
    (average degree 8-64), 2D grids with 5% rewiring and Barabasi-Albert (m = 4-32)."""
    specs = []
    seed = 100
    for scale in (16, 17, 18, 19, 20, 22):
        for a in (0.45, 0.50, 0.55, 0.60):
            specs.append(("rmat", dict(scale=scale, a=a, seed=seed)))
            seed += 1
    for n_log, deg in [(16, 8), (16, 16), (16, 32), (16, 64), (18, 8), (18, 16), (18, 32), (18, 64),
                       (20, 8), (20, 16), (20, 32), (20, 64), (17, 24), (19, 48)]:
        specs.append(("er", dict(n_log=n_log, deg=deg, seed=seed)))
        seed += 1
    for side in (256, 384, 512, 768, 1024, 1280, 1536, 1792, 2048, 2560):
        specs.append(("grid", dict(side=side, seed=seed)))
        seed += 1
    for n_log, m0 in [(16, 4), (16, 8), (16, 16), (16, 32), (18, 4), (18, 8), (18, 16), (18, 32),
                      (20, 4), (20, 8), (20, 16), (20, 32), (17, 12), (19, 24), (17, 6), (19, 10)]:
        specs.append(("ba", dict(n_log=n_log, m0=m0, seed=seed)))
        seed += 1
    assert len(specs) == 64
    if quick:
        specs = [s for s in specs if _size_log(s) <= 17][:12]
    return specs


HELD_OUT = [("rmat", dict(scale=23, a=0.57, seed=23)), ("ba", dict(n_log=22, m0=16, seed=22)),
            ("rmat", dict(scale=20, a=0.57, seed=2))]
HELD_OUT_QUICK = [("rmat", dict(scale=16, a=0.57, seed=23)), ("ba", dict(n_log=16, m0=16, seed=22))]


def _size_log(spec):
    kind, p = spec
    if kind == "rmat":
        return p["scale"]
    if kind == "grid":
        return int(math.log2(p["side"] * p["side"]))
    return p["n_log"]


def spec_name(spec) -> str:
    kind, p = spec
    return kind + "_" + "_".join(f"{k}{v}" for k, v in p.items())


def make_graph(spec):
    kind, p = spec
    if kind == "rmat":
        a = p["a"]
        b = c = (1.0 - a - 0.05) / 2.0
        return G.rmat(p["scale"], 16, a, b, c, seed=p["seed"])
    if kind == "er":
        n = 1 << p["n_log"]
        return G.erdos_renyi(n, p["deg"] / n, seed=p["seed"])
    if kind == "grid":
        return G.grid_rewired(p["side"], 0.05, seed=p["seed"])
    if kind == "ba":
        return G.barabasi_albert(1 << p["n_log"], p["m0"], seed=p["seed"])
    raise ValueError(kind)


# ---- measurement ----------------------------------------------------------------------------

def cell_stats(graph: api.Graph) -> np.ndarray:
    """[256, 4] per-cell sums (edges, sum log2(1+a), sum log2(1+b), sum min/max ratio) of the
    graph's last count."""
    import torch
    out = np.zeros(1024, dtype=np.float64)
    N.check(N.lib().tc_cell_stats(graph._h, out.ctypes.data, torch.cuda.current_stream().cuda_stream))
    return out.reshape(256, 4)


def cell_features(stats: np.ndarray) -> np.ndarray:
    """[256, 4] float32 MLP inputs; cells without edges get their nominal degrees."""
    feat = np.zeros((256, 4), dtype=np.float32)
    for c in range(256):
        cnt = stats[c, 0]
        if cnt > 0:
            feat[c] = (stats[c, 1] / cnt, stats[c, 2] / cnt, stats[c, 3] / cnt, c / 255.0)
        else:
            a, b = 1.5 * (1 << (c // 16)), 1.5 * (1 << (c % 16))
            feat[c] = (math.log2(1 + a), math.log2(1 + b), min(a, b) / max(a, b), c / 255.0)
    return feat


def forced(strategy: int, cell_filter: int = -1):
    s = N.default_sched()
    s.use_table = 1
    for i in range(16):
        for j in range(16):
            s.table[i][j] = strategy
    s.cell_filter = cell_filter
    return s


def count_ms(graph: api.Graph, out, sched, reps: int) -> tuple[float, int]:
    """Best count-kernel time (ms) over reps timed counts after one warm-up, and T."""
    N.lib().tc_profile_enable(1)
    best, T = float("inf"), None
    for r in range(reps + 1):
        T, _ = graph.count(N.TC_PV_HANDLE, out, sched=sched)
        pt = N.PhaseTimes()
        N.check(N.lib().tc_profile_last(ctypes.byref(pt)))
        if r > 0:
            best = min(best, pt.count_ms)
    return best, T


def collect_graph(spec, reps: int = 5):
    """Rows (features, strategy, label) of one graph."""
    import torch
    g = make_graph(spec)
    graph = api.Graph.from_csr(g)
    out = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
    graph.count(N.TC_PV_HANDLE, out)
    stats = cell_stats(graph)
    feat = cell_features(stats)
    t_none, _ = count_ms(graph, out, forced(0, -2), reps)
    rows = []
    for c in range(256):
        cnt = stats[c, 0]
        if cnt < MIN_CELL_EDGES:
            continue
        ts = [count_ms(graph, out, forced(strategy, c), reps)[0] - t_none for strategy in (0, 1)]
        if min(ts) < MIN_CELL_MS:
            continue  # below the timing resolution: no label
        for strategy in (0, 1):
            rows.append((feat[c], strategy, math.log2(ts[strategy] * 1e6 / cnt), c, cnt))
    graph.close()
    return rows, dict(n=g.n, m=g.m, t_none_ms=t_none, cells=int((stats[:, 0] >= MIN_CELL_EDGES).sum()))


def collect(specs, reps: int = 5, log=print):
    X, S, Y, meta = [], [], [], []
    for i, spec in enumerate(specs):
        t0 = time.time()
        rows, info = collect_graph(spec, reps)
        for f, s, y, c, cnt in rows:
            X.append(f)
            S.append(s)
            Y.append(y)
            meta.append((i, c, cnt))
        log(f"[collect] {i + 1}/{len(specs)} {spec_name(spec)} n={info['n']} m={info['m']} "
            f"cells={info['cells']} rows={len(rows)} {time.time() - t0:.1f}s")
    return (np.asarray(X, np.float32).reshape(-1, 4), np.asarray(S, np.int32), np.asarray(Y, np.float32),
            np.asarray(meta, np.float64).reshape(-1, 3))


# ---- training -------------------------------------------------------------------------------

def train(X, S, Y, epochs: int = 4000, lr: float = 3e-3, seed: int = 7):
    """Full-batch Adam on the GPU (tc_mlp_train). Returns (host params, final loss)."""
    import torch
    params = np.zeros(N.MLP_PARAMS, dtype=np.float32)
    N.check(N.lib().tc_mlp_init(params.ctypes.data, seed))
    d_params = torch.from_numpy(params).cuda()
    d_x = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    d_s = torch.from_numpy(np.ascontiguousarray(S)).cuda()
    d_y = torch.from_numpy(np.ascontiguousarray(Y)).cuda()
    loss = ctypes.c_float(0.0)
    stream = torch.cuda.current_stream().cuda_stream
    N.check(N.lib().tc_mlp_train(d_params.data_ptr(), d_x.data_ptr(), d_s.data_ptr(), d_y.data_ptr(), len(Y),
                                 epochs, ctypes.c_float(lr), ctypes.byref(loss), stream))
    return d_params.cpu().numpy(), float(loss.value)


def mse(params: np.ndarray, X, S, Y) -> float:
    import torch
    d_params = torch.from_numpy(params).cuda()
    d_x = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    d_out = torch.empty((len(Y), N.MLP_OUT), dtype=torch.float32, device="cuda")
    N.check(N.lib().tc_mlp_forward(d_params.data_ptr(), d_x.data_ptr(), len(Y), d_out.data_ptr(),
                                   torch.cuda.current_stream().cuda_stream))
    pred = d_out.cpu().numpy()[np.arange(len(Y)), S]
    return float(np.mean((pred - Y) ** 2))


def save(params: np.ndarray, path: str = WEIGHTS) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.asarray(params, dtype=np.float32).tofile(path)


def load(path: str = WEIGHTS) -> np.ndarray:
    p = np.fromfile(path, dtype=np.float32)
    if p.size != N.MLP_PARAMS:
        raise ValueError(f"{path}: {p.size} floats, expected {N.MLP_PARAMS}")
    return p


# ---- use ------------------------------------------------------------------------------------

def learned_sched(params: np.ndarray, graph: api.Graph, base=None):
    """Scheduler for `graph` from the trained network: its last count's cell statistics give
    the features; tc_sched_learned writes the table (fixed rule as the fallback)."""
    import torch
    feat = cell_features(cell_stats(graph))
    s = base if base is not None else N.default_sched()
    d_params = torch.from_numpy(np.ascontiguousarray(params, dtype=np.float32)).cuda()
    N.check(N.lib().tc_sched_learned(d_params.data_ptr(), 0, feat.ctypes.data, ctypes.byref(s),
                                     torch.cuda.current_stream().cuda_stream))
    return s


def evaluate_graph(params, spec, reps: int = 5):
    """Fixed heuristic vs learned table on one graph: median count-kernel times and counts."""
    import torch
    g = make_graph(spec)
    graph = api.Graph.from_csr(g)
    out_fixed = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
    out_learned = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
    graph.count(N.TC_PV_HANDLE, out_fixed)
    ls = learned_sched(params, graph)
    N.lib().tc_profile_enable(1)

    def times(sched, out):
        ts, T = [], None
        for r in range(reps + 1):
            T, _ = graph.count(N.TC_PV_HANDLE, out, sched=sched)
            pt = N.PhaseTimes()
            N.check(N.lib().tc_profile_last(ctypes.byref(pt)))
            if r:
                ts.append(pt.count_ms)
        return statistics.median(ts), T

    t_fixed, T_fixed = times(None, out_fixed)
    t_learned, T_learned = times(ls, out_learned)
    same = bool(torch.equal(out_fixed, out_learned)) and T_fixed == T_learned
    t_warp, T_warp = times(forced(0), out_learned)
    t_lane, T_lane = times(forced(1), out_learned)
    same = same and T_warp == T_fixed and T_lane == T_fixed
    changed = int(sum(ls.table[i][j] != forced_rule_choice(i, j) for i in range(16) for j in range(16)))
    graph.close()
    return dict(graph=spec_name(spec), n=g.n, m=g.m, triangles=T_fixed, fixed_ms=round(t_fixed, 4),
                learned_ms=round(t_learned, 4), gain=round(t_fixed / t_learned, 4),
                always_warp_ms=round(t_warp, 4), always_lane_ms=round(t_lane, 4), counts_equal=same,
                cells_departing_from_rule=changed)


def forced_rule_choice(i: int, j: int, lane_max: int = None) -> int:
    """The fixed rule's choice for a cell at its nominal degrees (for reporting only)."""
    if lane_max is None:
        lane_max = N.default_sched().lane_max_deg
    return 1 if round(1.5 * (1 << j)) <= lane_max else 0


# ---- driver ---------------------------------------------------------------------------------

def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("cmd", choices=["collect", "train", "evaluate", "all"])
    ap.add_argument("--out-dir", default=".")
    ap.add_argument("--quick", action="store_true", help="12 small training graphs (smoke run)")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--epochs", type=int, default=4000)
    ap.add_argument("--weights", default=None, help="weights to evaluate (default: trained or committed)")
    a = ap.parse_args(argv)
    os.makedirs(a.out_dir, exist_ok=True)
    ds_path = os.path.join(a.out_dir, "sched_dataset.npz")
    w_path = os.path.join(a.out_dir, "sched_mlp.bin")
    report = {}
    if a.cmd in ("collect", "all"):
        specs = training_specs(a.quick)
        X, S, Y, meta = collect(specs, a.reps)
        np.savez(ds_path, X=X, S=S, Y=Y, meta=meta, graphs=np.array([spec_name(s) for s in specs]))
        report["dataset"] = dict(graphs=len(specs), rows=int(len(Y)))
    if a.cmd in ("train", "all"):
        d = np.load(ds_path)
        X, S, Y, meta = d["X"], d["S"], d["Y"], d["meta"]
        # graph-level split: every 8th training graph is validation
        val = (meta[:, 0].astype(int) % 8) == 7
        params, loss = train(X[~val], S[~val], Y[~val], epochs=a.epochs)
        save(params, w_path)
        report["train"] = dict(rows=int((~val).sum()), val_rows=int(val.sum()), train_mse=round(loss, 4),
                               val_mse=round(mse(params, X[val], S[val], Y[val]), 4) if val.any() else None,
                               epochs=a.epochs)
        print(json.dumps(report["train"]), flush=True)
    if a.cmd in ("evaluate", "all"):
        wp = a.weights or (w_path if os.path.exists(w_path) else WEIGHTS)
        params = load(wp)
        report["held_out"] = []
        for spec in (HELD_OUT_QUICK if a.quick else HELD_OUT):
            r = evaluate_graph(params, spec)
            report["held_out"].append(r)
            print(json.dumps(r), flush=True)
    with open(os.path.join(a.out_dir, "sched_report.json"), "w") as f:
        json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
