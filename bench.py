#!/usr/bin/env python
"""Benchmark: static triangle count, edges intersected per second, on R-MAT scale 20.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--scale S]

Workload: R-MAT scale 20, edge factor 16 (a=.57 b=.19 c=.19 d=.05, seed 2), symmetrized,
deduplicated, self-loops removed, sorted int32 adjacency, ~31.4 M directed edges. One step is
one full static count through the library's hot path (degree orientation + intersections) with
per-vertex 2 t(v) output, the callDeviceAllTriangles semantics, on the graph resident in HBM.
The unit of work is an edge intersected: an undirected edge {u,v} with deg(u), deg(v) >= 2.

Timing: W warm-up steps, then K steps, each bracketed by CUDA events on the launching stream;
L2 (126 MB) is flushed by writing a 512 MB buffer between steps, outside the events. With N
GPUs (torchrun), each rank counts the edges whose centre (the endpoint with the larger
out-degree) falls in its shard of the vertex ids, then the per-vertex counts and the total are
all-reduced over NCCL inside the timed
step; the time is the max over ranks (strong scaling: the graph is fixed).

`--impl reference` times the reference's own CPU counter (hostSingleIntersection from
tests/cct.cpp, built into oracle/_ref) on all host cores over bounded random samples of source
vertices, extrapolated to the whole graph, on rank 0 only.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edges intersected/s (static triangle count)"
UNIT = "edges/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU-baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-streaming", action="store_true")
    ap.add_argument("--stream-scale", type=int, default=22)
    ap.add_argument("--stream-batches", type=int, default=200)
    ap.add_argument("--stream-verify", type=int, default=1, help="recount after every k-th batch (0 = never)")
    ap.add_argument("--stream-path", choices=["pipeline", "apply"], default="pipeline",
                    help="captured pipeline (tc_pipeline) or tc_apply_batch per batch")
    ap.add_argument("--stream-sched", choices=["learned", "fixed"], default="learned",
                    help="delta-kernel strategy table: trained network or the fixed ratio rule")
    ap.add_argument("--static-sched", choices=["learned", "fixed"], default="learned",
                    help="static count strategy table: trained network (from the first count's degree "
                         "cells) or the fixed length thresholds")
    return ap.parse_args()


def workload_config(a, n, m, e_int):
    return {"workload": f"static triangle count, R-MAT scale {a.scale} ef {a.edge_factor} "
                        f"(a=.57 b=.19 c=.19, seed {a.seed}), symmetrized sorted int32 CSR",
            "n": int(n), "directed_edges": int(m), "edges_intersected_per_step": int(e_int),
            "per_vertex_output": "int32 2t(v) (callDeviceAllTriangles)",
            "l2": "flushed between timed steps (512 MB write)"}


def make_graph(a):
    from custingeralg_b200 import generators as G
    return G.rmat(a.scale, a.edge_factor, 0.57, 0.19, 0.19, seed=a.seed)


def edges_intersected_host(g):
    deg = np.diff(g.off)
    src = np.repeat(np.arange(g.n, dtype=np.int64), deg)
    dst = g.ind.astype(np.int64)
    keep = (src < dst) & (deg[src] >= 2) & (deg[dst] >= 2)
    return int(keep.sum())


# ---------------------------------------------------------------------------------------------
# CPU reference timing (oracle/_ref: the reference's own hostSingleIntersection)
# ---------------------------------------------------------------------------------------------

def cpu_reference_sample(g, e_int, budget_s, seed=0, nthreads=0):
    """Time the reference counter over random source-vertex samples for about budget_s seconds.
    Returns (edges/s extrapolated to the whole graph, threads, description, kind)."""
    from oracle import pyoracle as O
    nt = nthreads or os.cpu_count() or 1
    rng = np.random.default_rng(seed)
    off32 = g.off32()
    if O.ref_available():
        kind = "reference"
        fn = lambda verts: O.ref_host_count_triangles_omp_sample(g.n, off32, g.ind, verts, nt)  # noqa: E731
    else:
        kind = "port"
        fn = lambda verts: O.sample_count(g.n, g.off, g.ind, verts, nt)  # noqa: E731
    k = min(g.n, max(64, g.n // 2000))
    t_tot, v_tot = 0.0, 0
    while t_tot < budget_s and v_tot < g.n:
        verts = rng.choice(g.n, size=min(k, g.n), replace=False).astype(np.int32)
        t0 = time.perf_counter()
        fn(verts)
        dt = time.perf_counter() - t0
        t_tot += dt
        v_tot += verts.size
        if dt < budget_s / 8:
            k = min(g.n, k * 2)
    frac = v_tot / g.n
    value = e_int * frac / t_tot
    desc = (f"{v_tot} uniformly sampled source vertices ({100 * frac:.3f}% of {g.n}), all their directed edges "
            f"intersected by the reference's hostSingleIntersection on {nt} threads in {t_tot:.2f} s; "
            f"whole-graph time extrapolated by 1/fraction")
    return value, nt, desc, kind, t_tot, frac


# ---------------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)

    def summary(self, t0, t1):
        rows = []
        for ts, line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            rows.append((ts, parts))
        inside = [r for r in rows if t0 <= r[0] <= t1] or rows
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(p[1]) for _, p in inside if num(p[1]) is not None]
        smax = [num(p[2]) for _, p in inside if num(p[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for _, p in inside:
            for nm, val in zip(names, p[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(inside),
                "power_w_max": max((num(p[3]) or 0.0) for _, p in inside)}


# ---------------------------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------------------------

def traffic_from_profile(scale):
    """DRAM bytes per k_count launch from the committed ncu summary, scaled to this graph."""
    path = os.path.join(ROOT, "profiles", f"k_count_rmat{scale}.md")
    if not os.path.exists(path):
        return None
    vals = {}
    for line in open(path):
        line = line.strip()
        if line.startswith("traffic_bytes_per_launch_scale"):
            k, v = line.split(":", 1)
            try:
                vals[int(k.rsplit("scale", 1)[1])] = float(v)
            except ValueError:
                pass
    return vals.get(scale)


def run_ours(a, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from custingeralg_b200 import api, native as N

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream()

    g = make_graph(a)
    e_int = edges_intersected_host(g)
    graph = api.Graph.from_csr(g, validate=True)
    out = torch.zeros(g.n + 1, dtype=torch.int32, device=dev)
    tri = torch.zeros(1, dtype=torch.int64, device=dev)
    sched = N.default_sched()
    sched.shard, sched.nshards = rank, world
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)

    # One synchronous count for the structural check, the work figures and the answer.
    T_full, info = graph.count(N.TC_PV_HANDLE, out, tri, sched=N.default_sched())
    ref_T = None
    checks = {"triangles": "no known answer for this graph"}
    gold_path = os.path.join(ROOT, "tests", "golden", "bench_configs.json")
    if os.path.exists(gold_path):
        gold = json.load(open(gold_path)).get(f"rmat{a.scale}_ef{a.edge_factor}_s{a.seed}")
        if gold:
            ref_T = gold["triangles"]
            if ref_T != T_full:
                raise SystemExit(f"count mismatch: {T_full} vs known answer {ref_T}")
            pv = out[:g.n].cpu().numpy()
            pv_digest = hashlib.sha256(np.ascontiguousarray(pv).astype("<i4").tobytes()).hexdigest()[:32]
            if pv_digest != gold["per_vertex_handle_digest"]:
                raise SystemExit("per-vertex counts differ from the known answer's digest")
            checks = {"triangles": "equals the known answer", "per_vertex_2t": "digest equals the known answer"}
    assert info.edges_intersected == e_int, (info.edges_intersected, e_int)
    d = N.default_sched()
    static_sched_desc = f"fixed rule (lane walk up to {d.lane_max_deg}, packed up to {d.packed_max_deg})"
    if a.static_sched == "learned":
        from custingeralg_b200 import sched_learn as L
        if os.path.exists(L.WEIGHTS):
            sched = L.learned_sched(L.load(L.WEIGHTS), graph, base=sched)  # cells of the count above
            static_sched_desc = "learned (custingeralg_b200/data/sched_mlp.bin, this graph's degree cells)"

    def step():
        graph.count(N.TC_PV_HANDLE, out, tri, sched=sched, sync=False)
        if world > 1:
            dist.all_reduce(out, op=dist.ReduceOp.SUM)
            dist.all_reduce(tri, op=dist.ReduceOp.SUM)

    N.lib().tc_profile_enable(1)
    for _ in range(a.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    count_ms, orient_ms, launches = [], [], 0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t_wall0 = time.perf_counter()
    for i in range(a.steps):
        flush.zero_()
        evs[i][0].record(stream)
        step()
        evs[i][1].record(stream)
        pt = N.PhaseTimes()
        N.check(N.lib().tc_profile_last(pt))
        count_ms.append(pt.count_ms)
        orient_ms.append(pt.orient_ms)
        launches += pt.launches
    torch.cuda.synchronize()
    t_wall1 = time.perf_counter()
    if world > 1:
        dist.barrier()
    time.sleep(0.2)
    clocks.stop()
    N.lib().tc_profile_enable(0)
    step_ms = [s.elapsed_time(e) for s, e in evs]
    tot_ms = sum(step_ms)
    t_max = torch.tensor([tot_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    tot_ms = float(t_max.item())
    ms_per_step = tot_ms / a.steps
    value = e_int / (ms_per_step / 1e3)
    T_check = int(tri.item())
    if T_check != T_full:
        raise SystemExit(f"timed count mismatch: {T_check} vs {T_full}")

    # Roofline of the dominant kernel (k_count): algorithmic bytes per launch (both oriented lists
    # read once per oriented edge + its endpoints + the offsets) over its event-timed duration.
    e_plus = g.m // 2
    b_alg = 4 * info.oriented_work + 8 * e_plus + 4 * (g.n + 1)
    t_count = statistics.mean(count_ms) / 1e3
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    achieved = b_alg / t_count / 1e9
    traffic = traffic_from_profile(a.scale)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": f"{peak_src} hbm_gbs",
                "kernel": "k_count", "kernel_ms": round(t_count * 1e3, 4),
                "algorithmic_bytes_per_launch": int(b_alg),
                "compulsory_bytes_per_launch": int(4 * e_plus + 8 * (g.n + 1)),
                "note": "algorithmic bytes = sum over oriented edges of 4(d+u + d+v) + 8|E+| + 4(n+1) (both "
                        "oriented lists read once per edge); the L2 serves repeated list reads, so DRAM "
                        "traffic (the ncu figure in 'traffic') stays below them"}

    result = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
              "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
              "scaling": "strong", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
              "config": workload_config(a, g.n, g.m, e_int),
              "triangles": T_full, "checks": checks, "gpu_launches": launches, "roofline": roofline,
              "phase_ms": {"orient": round(statistics.mean(orient_ms), 4),
                           "count": round(statistics.mean(count_ms), 4)},
              "clocks": clocks.summary(t_wall0, t_wall1)}
    result["config"]["static_scheduler"] = static_sched_desc
    if world > 1:
        result["config"]["parallelism"] = f"vertex shards over {world} GPUs + NCCL all-reduce"

    # End to end through the C ABI with host buffers: H2D of the CSR from pinned memory, the count
    # (callDeviceAllTrianglesCSR path with per-vertex output), D2H of the per-vertex counts and T.
    if not a.no_e2e:
        # int32 offsets while they fit: the reference's raw-CSR boundary types them as length_t
        # (int32, tests/cct_csr.cu:279-285); int64 beyond 2^31 - 1 directed edges
        off_host = g.off.astype(np.int32) if g.m < 2**31 else g.off
        h_off = torch.from_numpy(off_host).pin_memory()
        h_ind = torch.from_numpy(g.ind).pin_memory()
        d_off = torch.empty_like(h_off, device=dev)
        d_ind = torch.empty_like(h_ind, device=dev)
        h_out = torch.empty(g.n + 1, dtype=torch.int32).pin_memory()
        h_tri = torch.empty(1, dtype=torch.int64).pin_memory()
        e2e_ms = []

        def e2e_step():
            d_off.copy_(h_off, non_blocking=True)
            d_ind.copy_(h_ind, non_blocking=True)
            api.count_all_triangles_csr(g.n, d_off, d_ind, out, pv_mode=N.TC_PV_HANDLE, sched=sched, sync=False,
                                        triangles_dev=tri)
            if world > 1:
                dist.all_reduce(out, op=dist.ReduceOp.SUM)
                dist.all_reduce(tri, op=dist.ReduceOp.SUM)
            h_out.copy_(out, non_blocking=True)
            h_tri.copy_(tri, non_blocking=True)

        for _ in range(max(1, a.warmup)):
            e2e_step()
        torch.cuda.synchronize()
        for i in range(a.steps):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            e2e_step()
            e.record(stream)
            e.synchronize()
            e2e_ms.append(s.elapsed_time(e))
        if int(h_tri.item()) != T_full:
            raise SystemExit(f"e2e count mismatch: {int(h_tri.item())} vs {T_full}")
        t = torch.tensor([sum(e2e_ms)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_step_s = float(t.item()) / a.steps / 1e3
        result["e2e"] = {"value": e_int / e2e_step_s, "unit": UNIT,
                         "h2d_bytes_per_step": int(h_off.numel() * h_off.element_size() + h_ind.numel() * 4),
                         "d2h_bytes_per_step": int(h_out.numel() * 4 + 8),
                         "ms_per_step": e2e_step_s * 1e3,
                         "path": ("tc_count_csr32" if h_off.dtype == torch.int32 else "tc_count_csr64")
                                 + " (callDeviceAllTrianglesCSR boundary), pinned host CSR in, per-vertex counts out"}

    if rank == 0 and world == 1 and not a.no_streaming:
        result["streaming"] = run_streaming(a, dev)

    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        v, nt, desc, kind, _, _ = cpu_reference_sample(g, e_int, a.cpu_seconds)
        result["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": nt, "kind": kind, "sample": desc}
    return result


def streaming_batches(scale, nbatch, base, seed=4):
    """Batch sizes log-uniform on [1, 2^20]; 70% insertions with R-MAT endpoints, 30% deletions
    sampled from the base graph's edges (an already-deleted pick is a no-op)."""
    from custingeralg_b200 import generators as G
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(0.0, np.log(2.0 ** 20), nbatch))).astype(np.int64)
    sizes = np.clip(sizes, 1, 1 << 20)
    src_of = np.repeat(np.arange(base.n, dtype=np.int32), np.diff(base.off))
    out = []
    for i, b in enumerate(sizes.tolist()):
        n_del = int(round(0.3 * b))
        n_ins = b - n_del
        s_ins, d_ins = G.rmat_pairs(scale, n_ins, seed=seed, stream=i + 1)
        pick = rng.integers(0, base.m, n_del)
        s = np.concatenate([s_ins, src_of[pick]]).astype(np.int32)
        d = np.concatenate([d_ins, base.ind[pick]]).astype(np.int32)
        dl = np.concatenate([np.zeros(n_ins, np.uint8), np.ones(n_del, np.uint8)])
        perm = rng.permutation(b)
        out.append((s[perm], d[perm], dl[perm]))
    return out


def run_streaming(a, dev):
    """Update edges per second on R-MAT scale 22 (seed 4) with 200 uneven batches; the running
    count is checked against a full static recount after every batch (outside the timing)."""
    import torch
    from custingeralg_b200 import api, generators as G, native as N
    base = G.rmat(a.stream_scale, 16, 0.57, 0.19, 0.19, seed=4)
    graph = api.Graph.from_csr(base, slack=0.25)
    pv = torch.zeros(base.n + 1, dtype=torch.int32, device=dev)
    delta = torch.zeros(1, dtype=torch.int64, device=dev)
    scratch = torch.zeros(base.n + 1, dtype=torch.int32, device=dev)
    T0, _ = graph.count(N.TC_PV_HANDLE, scratch)
    batches = streaming_batches(a.stream_scale, a.stream_batches, base)
    dbat = [(torch.from_numpy(s).to(dev), torch.from_numpy(d).to(dev), torch.from_numpy(x).to(dev))
            for s, d, x in batches]
    pipe = None
    sched, sched_desc = None, "fixed rule (search_ratio_x16 = 16)"
    if getattr(a, "stream_sched", "learned") == "learned":
        from custingeralg_b200 import sched_learn as L
        if os.path.exists(L.STREAM_WEIGHTS):
            sched = L.learned_stream_sched(L.load(L.STREAM_WEIGHTS))
            sched_desc = "learned (custingeralg_b200/data/sched_mlp_stream.bin, nominal cell degrees)"
    if getattr(a, "stream_path", "pipeline") == "pipeline":
        pipe = api.Pipeline(graph, max(s.numel() for s, _, _ in dbat), sched=sched)
        pipe.prepare(per_vertex=pv, delta_dev=delta)  # pool headroom and captures, before timing
        pipe.autotune(24)   # the first 24 timed batches also try the candidate delta grids
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    total_ms, updates, checked = 0.0, 0, 0
    for i, (s, d, x) in enumerate(dbat):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if pipe is not None:
            pipe.apply(s, d, x, per_vertex=pv, delta_dev=delta)
        else:
            graph.apply_batch(s, d, x, per_vertex=pv, delta_dev=delta, sched=sched, sync=False)
        e1.record(stream)
        e1.synchronize()
        if pipe is not None:
            pipe.sync()
        total_ms += e0.elapsed_time(e1)
        updates += s.numel()
        if a.stream_verify and (i % a.stream_verify == 0 or i == len(dbat) - 1):
            T, _ = graph.count(N.TC_PV_HANDLE, scratch)
            if T != T0 + int(delta.item()):
                raise SystemExit(f"streaming mismatch after batch {i}: recount {T} vs running {T0 + int(delta.item())}")
            if not torch.equal(scratch[: base.n], (pv[: base.n].to(torch.int64) +
                                                  _static_pv_cache(graph, base, T0, dev)).to(torch.int32)):
                raise SystemExit(f"per-vertex streaming mismatch after batch {i}")
            checked += 1
    path = "tc_pipeline (one captured CUDA graph per batch-size bin)" if pipe is not None else "tc_apply_batch"
    bins = pipe.info() if pipe is not None else None
    if pipe is not None:
        pipe.close()
    return {"value": updates / (total_ms / 1e3), "unit": "update edges/s", "batches": len(dbat),
            "updates": updates, "ms_total": total_ms, "recount_checks": checked, "path": path,
            "scheduler": sched_desc,
            "bins": [{"capacity": c, "delta_ctas_per_sm": b} for c, b in bins] if bins else None,
            "workload": f"R-MAT scale {a.stream_scale} ef 16 seed 4 base (slack 0.25), {len(dbat)} batches of "
                        "log-uniform size in [1, 2^20], 70% R-MAT insertions / 30% deletions of base edges; "
                        "timed per batch over sort + classify + structure update + delta count, batches resident "
                        "on the device",
            "final_triangles": T0 + int(delta.item())}


_PV0 = {}


def _static_pv_cache(graph, base, T0, dev):
    """Per-vertex 2t(v) of the base graph (computed once on a fresh handle)."""
    import torch
    from custingeralg_b200 import api, native as N
    key = id(base)
    if key not in _PV0:
        g0 = api.Graph.from_csr(base)
        out = torch.zeros(base.n + 1, dtype=torch.int32, device=dev)
        g0.count(N.TC_PV_HANDLE, out)
        _PV0[key] = out[: base.n].to(torch.int64)
        g0.close()
    return _PV0[key]


def run_reference(a, rank, world):
    if rank != 0:
        return None
    from oracle import pyoracle as O
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libref_cct.so (the reference CPU counter built "
                                                    "from tests/cct.cpp) was not built"}
    g = make_graph(a)
    e_int = edges_intersected_host(g)
    per_step = max(1.0, min(6.0, 120.0 / max(1, a.steps + a.warmup)))
    for i in range(a.warmup):
        cpu_reference_sample(g, e_int, per_step / 2, seed=1000 + i)
    vals, times, fracs, nt, desc = [], [], [], 0, ""
    for i in range(a.steps):
        v, nt, desc, kind, t, f = cpu_reference_sample(g, e_int, per_step, seed=i)
        vals.append(v)
        times.append(t)
        fracs.append(f)
    value = e_int * sum(fracs) / sum(times)
    ms_per_step = 1e3 * sum(times) / sum(fracs) / a.steps if sum(fracs) else None
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "int32", "data": "synthetic", "impl": "reference",
            "config": workload_config(a, g.n, g.m, e_int),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nt, "kind": "reference",
                             "sample": f"each step: {desc}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "gpu_launches": 0}


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and a.impl == "ours":
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    if a.impl == "reference":
        res = run_reference(a, rank, world)
    else:
        res = run_ours(a, rank, world, local_rank)
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)
    if world > 1 and a.impl == "ours":
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
