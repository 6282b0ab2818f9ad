"""Learned scheduler for the static count: per-degree-cell strategy from a trained MLP.

The count kernel intersects each edge at its centre (the endpoint with the larger out-degree
a): the other endpoint's list N+(o), b <= a entries, goes through the centre's shared-memory
hash set by one of three strategies: the warp streams it with coalesced loads (one list at a
time), one lane walks it (the lanes of a warp walk different short lists at once), or the warp
walks all such lists of a group of 32 neighbours concatenated (packed). The fixed heuristic
picks by length thresholds (lane_max_deg, packed_max_deg). Here a 3-layer FP32 MLP of width 64
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
STREAM_WEIGHTS = os.path.join(HERE, "data", "sched_mlp_stream.bin")
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
            ("rmat", dict(scale=20, a=0.57, seed=2)), ("er", dict(n_log=20, deg=32, seed=20))]
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


STRATEGIES = (0, 1, 2)  # static table entries (= network outputs): warp, lane, packed


def two_rule_sched():
    """The fixed rule before packed walks existed: lane walks up to lane_max_deg, else warp."""
    s = N.default_sched()
    s.packed_max_deg = 0
    return s


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
        ts = [count_ms(graph, out, forced(strategy, c), reps)[0] - t_none for strategy in STRATEGIES]
        if min(ts) < MIN_CELL_MS:
            continue  # below the timing resolution: no label
        for strategy in STRATEGIES:
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
    st = cell_stats(graph)
    stats_n = st[:, 0]
    stats_b = np.where(st[:, 0] > 0, np.exp2(st[:, 2] / np.maximum(st[:, 0], 1)) - 1, 0)
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
    t_two, T_two = times(two_rule_sched(), out_learned)
    t_warp, T_warp = times(forced(0), out_learned)
    t_lane, T_lane = times(forced(1), out_learned)
    t_pack, T_pack = times(forced(2), out_learned)
    same = same and T_warp == T_fixed and T_lane == T_fixed and T_pack == T_fixed and T_two == T_fixed
    changed = int(sum(ls.table[c // 16][c % 16] != rule_choice(stats_b[c])
                      for c in range(256) if stats_n[c] > 0))
    graph.close()
    return dict(graph=spec_name(spec), n=g.n, m=g.m, triangles=T_fixed, fixed_ms=round(t_fixed, 4),
                learned_ms=round(t_learned, 4), gain=round(t_fixed / t_learned, 4),
                two_rule_ms=round(t_two, 4), gain_vs_two_rule=round(t_two / t_learned, 4),
                always_warp_ms=round(t_warp, 4), always_lane_ms=round(t_lane, 4),
                always_packed_ms=round(t_pack, 4), counts_equal=same, cells_with_edges_off_the_rule=changed)


def rule_choice(mean_b: float, lane_max: int = None, packed_max: int = None) -> int:
    """The fixed rule's choice for a cell whose lists have mean length mean_b (reporting only)."""
    d = N.default_sched()
    lane_max = d.lane_max_deg if lane_max is None else lane_max
    packed_max = d.packed_max_deg if packed_max is None else packed_max
    b = round(max(mean_b, 1.0))
    return 1 if b <= lane_max else 2 if b <= packed_max else 0



# ---- streaming delta count ------------------------------------------------------------------
#
# The delta kernel intersects the full lists N(x), N(y) of each changed edge {x, y} by binary
# search of the shorter list in the longer (network output 1, table entry 0) or by a partitioned
# merge (output 2, table entry 1); the fixed rule searches when
# 16 d_long > search_ratio_x16 * d_short (log2 d_long + 1). Cells are (log2 d_short, log2 d_long)
# of the endpoints' degrees. The timings come from tc_count_batch (the cuStinger-path count of a
# sorted batch) over a sample of the graph's own edges, which leaves the graph unchanged.

def stream_sample(g, k: int, rng):
    """A sorted symmetric batch of k existing undirected edges (device arrays for tc_count_batch)
    and its per-cell statistics [256, 4]."""
    import torch
    src_of = np.repeat(np.arange(g.n, dtype=np.int32), np.diff(g.off))
    und = np.nonzero(src_of < g.ind)[0]
    pick = und[rng.choice(und.size, size=min(k, und.size), replace=False)]
    u, v = src_of[pick], g.ind[pick]
    deg = np.diff(g.off)
    la = np.minimum(deg[u], deg[v]).astype(np.float64)
    lb = np.maximum(deg[u], deg[v]).astype(np.float64)
    cell = (np.minimum(np.floor(np.log2(np.maximum(la, 1))), 15) * 16 +
            np.minimum(np.floor(np.log2(np.maximum(lb, 1))), 15)).astype(np.int64)
    stats = np.zeros((256, 4))
    np.add.at(stats[:, 0], cell, 1.0)
    np.add.at(stats[:, 1], cell, np.log2(1 + la))
    np.add.at(stats[:, 2], cell, np.log2(1 + lb))
    np.add.at(stats[:, 3], cell, la / np.maximum(lb, 1))
    s = np.concatenate([u, v]).astype(np.int32)
    d = np.concatenate([v, u]).astype(np.int32)
    ds, dd = torch.from_numpy(s).cuda(), torch.from_numpy(d).cuda()
    off = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
    dup = torch.zeros(max(s.size, 1), dtype=torch.int32, device="cuda")
    N.check(N.lib().tc_batch_sort(g.n, ds.data_ptr(), dd.data_ptr(), s.size, off.data_ptr(), dup.data_ptr(), None))
    return (ds, dd, off, dup, s.size), stats


def count_batch_ms(graph, batch, sched, reps: int, pv) -> tuple[float, int]:
    """Best event-timed tc_count_batch (sign +1) over reps after a warm-up, and its count."""
    import torch
    ds, dd, off, dup, b = batch
    delta = torch.zeros(1, dtype=torch.int64, device="cuda")
    best = float("inf")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream()
    for r in range(reps + 1):
        delta.zero_()
        e0.record(stream)
        N.check(N.lib().tc_count_batch(graph.handle, ds.data_ptr(), dd.data_ptr(), off.data_ptr(), dup.data_ptr(),
                                       b, 1, pv.data_ptr(), delta.data_ptr(),
                                       ctypes.byref(sched) if sched is not None else None, stream.cuda_stream))
        e1.record(stream)
        e1.synchronize()
        if r:
            best = min(best, e0.elapsed_time(e1))
    return best, int(delta.item())


def stream_forced(table_entry: int, cell_filter: int = -1):
    return forced(table_entry, cell_filter)


def collect_stream_graph(spec, k: int = 200000, reps: int = 5, seed: int = 0):
    import torch
    g = make_graph(spec)
    graph = api.Graph.from_csr(g)
    pv = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
    batch, stats = stream_sample(g, k, np.random.default_rng(seed))
    feat = cell_features(stats)
    t_none, _ = count_batch_ms(graph, batch, stream_forced(0, -2), reps, pv)
    rows = []
    for c in range(256):
        cnt = stats[c, 0]
        if cnt < MIN_CELL_EDGES / 2:
            continue
        ts = [count_batch_ms(graph, batch, stream_forced(e, c), reps, pv)[0] - t_none for e in (0, 1)]
        if min(ts) < MIN_CELL_MS:
            continue
        for e in (0, 1):  # table entry 0 = search = network output 1, entry 1 = merge = output 2
            rows.append((feat[c], e + 1, math.log2(ts[e] * 1e6 / cnt), c, cnt))
    graph.close()
    return rows, dict(n=g.n, m=g.m, t_none_ms=t_none)


def learned_stream_sched(params: np.ndarray, feat=None, base=None):
    """Streaming scheduler from the trained network (nominal cell degrees when feat is None)."""
    import torch
    s = base if base is not None else N.default_sched()
    d_params = torch.from_numpy(np.ascontiguousarray(params, dtype=np.float32)).cuda()
    N.check(N.lib().tc_sched_learned(d_params.data_ptr(), 1, feat.ctypes.data if feat is not None else None,
                                     ctypes.byref(s), torch.cuda.current_stream().cuda_stream))
    return s


def evaluate_stream_graph(params, spec, k: int = 400000, reps: int = 5):
    """Fixed rule vs learned table for the delta count of a batch of k of the graph's edges."""
    import torch
    g = make_graph(spec)
    graph = api.Graph.from_csr(g)
    pv = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
    batch, stats = stream_sample(g, k, np.random.default_rng(99))
    ls = learned_stream_sched(params, cell_features(stats))
    t_fixed, c_fixed = count_batch_ms(graph, batch, None, reps, pv)
    t_learned, c_learned = count_batch_ms(graph, batch, ls, reps, pv)
    t_search, c_search = count_batch_ms(graph, batch, stream_forced(0), reps, pv)
    t_merge, c_merge = count_batch_ms(graph, batch, stream_forced(1), reps, pv)
    graph.close()
    return dict(graph=spec_name(spec), n=g.n, m=g.m, batch_edges=int(batch[4] // 2), fixed_ms=round(t_fixed, 4),
                learned_ms=round(t_learned, 4), gain=round(t_fixed / t_learned, 4),
                always_search_ms=round(t_search, 4), always_merge_ms=round(t_merge, 4),
                counts_equal=len({c_fixed, c_learned, c_search, c_merge}) == 1)


STREAM_HELD_OUT = [("rmat", dict(scale=22, a=0.57, seed=4)), ("ba", dict(n_log=21, m0=16, seed=21)),
                   ("er", dict(n_log=20, deg=32, seed=20))]


def stream_main(a, report):
    specs = [sp for i, sp in enumerate(training_specs(a.quick)) if i % 2 == 0]  # 32 graphs
    ds_path = os.path.join(a.out_dir, "sched_stream_dataset.npz")
    w_path = os.path.join(a.out_dir, "sched_mlp_stream.bin")
    X, S, Y, meta = [], [], [], []
    for i, spec in enumerate(specs):
        t0 = time.time()
        rows, info = collect_stream_graph(spec, reps=a.reps, seed=i)
        for f, st, y, c, cnt in rows:
            X.append(f)
            S.append(st)
            Y.append(y)
            meta.append((i, c, cnt))
        print(f"[stream collect] {i + 1}/{len(specs)} {spec_name(spec)} rows={len(rows)} {time.time() - t0:.1f}s",
              flush=True)
    X = np.asarray(X, np.float32).reshape(-1, 4)
    S = np.asarray(S, np.int32)
    Y = np.asarray(Y, np.float32)
    meta = np.asarray(meta, np.float64).reshape(-1, 3)
    np.savez(ds_path, X=X, S=S, Y=Y, meta=meta)
    val = (meta[:, 0].astype(int) % 8) == 7
    params, loss = train(X[~val], S[~val], Y[~val], epochs=a.epochs)
    save(params, w_path)
    report["stream_train"] = dict(graphs=len(specs), rows=int((~val).sum()), val_rows=int(val.sum()),
                                  train_mse=round(loss, 4),
                                  val_mse=round(mse(params, X[val], S[val], Y[val]), 4) if val.any() else None)
    print(json.dumps(report["stream_train"]), flush=True)
    report["stream_held_out"] = []
    for spec in STREAM_HELD_OUT[:1] if a.quick else STREAM_HELD_OUT:
        r = evaluate_stream_graph(params, spec)
        report["stream_held_out"].append(r)
        print(json.dumps(r), flush=True)

# ---- driver ---------------------------------------------------------------------------------

def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("cmd", choices=["collect", "train", "evaluate", "all", "stream"])
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
    if a.cmd == "stream":
        stream_main(a, report)
        with open(os.path.join(a.out_dir, "sched_stream_report.json"), "w") as f:
            json.dump(report, f, indent=1)
        return
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
