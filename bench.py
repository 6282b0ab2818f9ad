#!/usr/bin/env python
"""Benchmark: static triangle count (edges intersected per second) and streaming triangle count
(update edges per second) on R-MAT graphs, learned against fixed scheduling.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload (the JSON line's `value`): R-MAT scale 20, edge factor 16 (a=.57 b=.19 c=.19
d=.05, seed 2), symmetrized, deduplicated, self-loops removed, sorted int32 adjacency, ~31.4 M
directed edges. One step is one full static count through the library's hot path (degree
orientation + intersections) with per-vertex 2 t(v) output, the callDeviceAllTriangles
semantics, on the graph resident in HBM. The unit of work is an edge intersected: an undirected
edge {u,v} with deg(u), deg(v) >= 2 (the reference's avoidCalc filter).

The same line carries:
  fixed      the same count with the fixed degree-threshold rule instead of the learned table;
  e2e        the count through tc_count_csr32 (the callDeviceAllTrianglesCSR boundary) with the
             CSR copied from pinned host memory and the per-vertex counts copied back each step;
  c3         R-MAT scale 24 (seed 3, ~521 M directed edges): learned and fixed, its own roofline,
             its known-answer checks (total and per-vertex digest pinned to the reference);
  streaming  R-MAT scale 22 (seed 4) under 200 batches of log-uniform size in [1, 2^20] (70 %
             R-MAT insertions, 30 % deletions of present edges) through the captured pipeline,
             learned and fixed, with the delta kernels' roofline; the running count is checked
             against a full static recount after every batch;
  cpu_baseline, cpu_baseline_1core  the reference's own CPU counter (oracle/_ref).

Timing: W warm-up steps, then K steps, each bracketed by CUDA events on the launching stream;
L2 (126 MB) is flushed by writing a 512 MB buffer between steps, outside the events. With N
GPUs each rank counts a contiguous range of edge centres balanced by predicted work, then the
per-vertex counts and the total are all-reduced over NCCL inside the timed step; the time is the
max over ranks (strong scaling: the graph is fixed). `--gpus N` starts the N ranks itself when
it is not already running under torchrun.

`--impl reference` times the reference's own CPU counter (hostSingleIntersection from
tests/cct.cpp, built into oracle/_ref) on all host cores over bounded random samples of source
vertices, on rank 0 only. Its graph is generated by a child process and read back as raw
arrays, so the timed process maps no library of this repository.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import socket
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edges intersected/s (static triangle count)"
# Host threads of the graph generators per rank (0 = all cores): with N ranks on one node each
# rank takes its share, so N concurrent generators do not oversubscribe the host.
GEN_THREADS = 0
UNIT = "edges/s"
RMAT_ABC = (0.57, 0.19, 0.19)


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--c3-scale", type=int, default=24, help="second static workload (0 = skip)")
    ap.add_argument("--c3-seed", type=int, default=3)
    ap.add_argument("--c3-steps", type=int, default=10)
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU-baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fixed", action="store_true", help="skip the fixed-rule comparison runs")
    ap.add_argument("--no-split", action="store_true", help="skip the one-GPU measurement of the multi-GPU split")
    ap.add_argument("--no-streaming", action="store_true")
    ap.add_argument("--no-stream-tune", action="store_true",
                    help="run the streaming pipeline with its default plan (no untimed autotuning first)")
    ap.add_argument("--stream-plan", default=None,
                    help="run the streaming pipeline on the plan (bins and tile shapes) recorded in an "
                         "earlier bench line (a file holding that JSON line) instead of tuning one")
    ap.add_argument("--stream-hub-min", type=int, default=None,
                    help="changed edges an endpoint must hold to be counted as a hub (the scheduler's "
                         "stream_hub_min; default: the library's)")
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
    return ap.parse_args(argv)


def workload_config(scale, ef, seed, n, m, e_int):
    """The `config` object, identical in both arms for the same workload."""
    return {"workload": f"static triangle count, R-MAT scale {scale} ef {ef} "
                        f"(a=.57 b=.19 c=.19, seed {seed}), symmetrized sorted int32 CSR",
            "n": int(n), "directed_edges": int(m), "edges_intersected_per_step": int(e_int),
            "per_vertex_output": "int32 2t(v) (callDeviceAllTriangles)",
            "l2": "flushed between timed steps (512 MB write)"}


class HostCsr:
    """A CSR held as numpy arrays only (off int64[n+1], ind int32[m])."""

    def __init__(self, n, off, ind):
        self.n, self.off, self.ind = int(n), off, ind

    @property
    def m(self):
        return int(self.off[-1])

    def off32(self):
        return self.off.astype(np.int32)


def read_tccsr(path):
    """Read the library's binary CSR cache (.tccsr: 8-byte magic, int64 n, int64 m, int64
    offsets[n+1], int32 ids[m]) with numpy alone."""
    with open(path, "rb") as f:
        magic = f.read(8)
        if not magic.startswith(b"TCCSRv1"):
            raise ValueError(f"{path}: not a binary CSR cache")
        n, m = (int(x) for x in np.fromfile(f, dtype="<i8", count=2))
        off = np.fromfile(f, dtype="<i8", count=n + 1)
        ind = np.fromfile(f, dtype="<i4", count=m)
    return HostCsr(n, off, ind)


def rmat_graph(ctx, scale, ef, seed):
    """The R-MAT graph of a workload. With several ranks, rank 0 generates it once and the others
    read it back from a binary CSR file (the generator is a pure function of its parameters)."""
    from custingeralg_b200 import generators as G
    if ctx.world == 1:
        return G.rmat(scale, ef, *RMAT_ABC, seed=seed, nthreads=GEN_THREADS)
    path = os.path.join(tempfile.gettempdir(),
                        f"tc_bench_{os.environ.get('MASTER_PORT', '0')}_rmat{scale}_{ef}_{seed}.tccsr")
    if ctx.rank == 0:
        G.write_binary(G.rmat(scale, ef, *RMAT_ABC, seed=seed), path)
    ctx.barrier()
    g = read_tccsr(path)
    ctx.barrier()
    if ctx.rank == 0:
        os.remove(path)
    return g


def generate_in_child(family_args, path):
    """Write a generated graph to `path` from a separate process (python -m
    custingeralg_b200.generators), so the caller never maps the generator library."""
    r = subprocess.run([sys.executable, "-m", "custingeralg_b200.generators"] + family_args + ["--out", path],
                       cwd=ROOT, capture_output=True, text=True)
    if r.returncode != 0:
        raise SystemExit(f"graph generation failed: {r.stdout}{r.stderr}")


def edges_intersected_host(g):
    deg = np.diff(g.off)
    src = np.repeat(np.arange(g.n, dtype=np.int64), deg)
    dst = g.ind.astype(np.int64)
    keep = (src < dst) & (deg[src] >= 2) & (deg[dst] >= 2)
    return int(keep.sum())


def known_answer(scale, ef, seed):
    path = os.path.join(ROOT, "tests", "golden", "bench_configs.json")
    if not os.path.exists(path):
        return None
    return json.load(open(path)).get(f"rmat{scale}_ef{ef}_s{seed}")


def pv_digest(pv):
    return hashlib.sha256(np.ascontiguousarray(pv).astype("<i4").tobytes()).hexdigest()[:32]


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return float(json.load(open(path))["hbm_gbs"]), "measured hbm_gbs"
    return 6650.0, "fallback (no MEASURED_PEAKS.json)"


# ---------------------------------------------------------------------------------------------
# CPU reference timing (oracle/_ref: the reference's own hostSingleIntersection)
# ---------------------------------------------------------------------------------------------

def cpu_reference_sample(g, e_int, budget_s, seed=0, nthreads=0):
    """Time the reference counter over random source-vertex samples for about budget_s seconds.
    Returns (edges/s extrapolated to the whole graph, threads, description, kind, seconds, fraction)."""
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


def cpu_reference_1core(c1, e_int1):
    """hostCountTriangles as written (tests/cct.cpp:71-89), one thread, over the whole C1 graph
    (Erdos-Renyi n = 2^14, average degree 16, seed 1)."""
    from oracle import pyoracle as O
    if not O.ref_available():
        return None
    t0 = time.perf_counter()
    tot, _ = O.ref_host_count_triangles(c1.n, c1.off, c1.ind)
    dt = time.perf_counter() - t0
    return {"value": e_int1 / dt, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"whole graph: Erdos-Renyi n=2^14, average degree 16, seed 1 ({c1.m} directed edges, "
                      f"{e_int1} edges intersected, 6T = {tot}); hostCountTriangles as written, one thread, "
                      f"{dt * 1e3:.1f} ms"}


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

    def summary(self, windows):
        rows = []
        for ts, line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            rows.append((ts, parts))
        inside = [r for r in rows if any(t0 <= r[0] <= t1 for t0, t1 in windows)] or rows
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

class Ctx:
    """Per-rank state shared by the measurements."""

    def __init__(self, a, rank, world, local_rank):
        import torch
        self.a, self.rank, self.world, self.local_rank = a, rank, world, local_rank
        torch.cuda.set_device(local_rank)
        self.dev = torch.device("cuda", local_rank)
        self.stream = torch.cuda.current_stream()
        self.flush = torch.empty(512 << 20, dtype=torch.uint8, device=self.dev)
        self.windows = []   # wall-clock windows of the timed regions (for the clock record)

    def allreduce_(self, t, op="sum"):
        if self.world > 1:
            import torch.distributed as dist
            dist.all_reduce(t, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MAX)
        return t

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(self, values):
        """Elementwise max over ranks of a list of floats."""
        import torch
        t = torch.tensor(values, dtype=torch.float64, device=self.dev)
        self.allreduce_(t, "max")
        return t.cpu().tolist()


def shard_sched(base, ctx):
    """The scheduler of this rank's shard (contiguous centre range balanced by predicted work)."""
    base.shard, base.nshards = ctx.rank, ctx.world
    return base


def time_static(ctx, graph, out, tri, sched, steps, warmup):
    """W untimed and K timed full static counts; per step: event time, count and orientation
    kernel times, launches. The per-vertex counts and the total are all-reduced inside the step
    when there are several ranks."""
    import torch
    from custingeralg_b200 import native as N

    def step():
        graph.count(N.TC_PV_HANDLE, out, tri, sched=sched, sync=False)
        ctx.allreduce_(out)
        ctx.allreduce_(tri)

    N.lib().tc_profile_enable(1)
    for _ in range(warmup):
        ctx.flush.zero_()
        step()
    torch.cuda.synchronize()
    ctx.barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    count_ms, orient_ms, launches = [], [], 0
    torch.cuda.synchronize()
    ctx.barrier()
    t0 = time.perf_counter()
    for i in range(steps):
        ctx.flush.zero_()
        evs[i][0].record(ctx.stream)
        step()
        evs[i][1].record(ctx.stream)
        pt = N.PhaseTimes()
        N.check(N.lib().tc_profile_last(pt))
        count_ms.append(pt.count_ms)
        orient_ms.append(pt.orient_ms)
        launches += pt.launches
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    ctx.barrier()
    ctx.windows.append((t0, t1))
    N.lib().tc_profile_enable(0)
    step_ms = ctx.max_over_ranks([s.elapsed_time(e) for s, e in evs])
    count_ms = ctx.max_over_ranks(count_ms)
    return step_ms, count_ms, orient_ms, launches


def roofline_for(g, info, count_ms, kernel="k_count"):
    """Roofline of the count kernel: algorithmic bytes per launch (both oriented lists read once
    per oriented edge + its endpoints + the offsets) over its event-timed mean duration."""
    e_plus = g.m // 2
    b_alg = 4 * info.oriented_work + 8 * e_plus + 4 * (g.n + 1)
    t = statistics.mean(count_ms) / 1e3
    peak, src = measured_peak()
    achieved = b_alg / t / 1e9
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": None, "peak_source": src,
            "kernel": kernel, "kernel_ms": round(t * 1e3, 4),
            "algorithmic_bytes_per_launch": int(b_alg),
            "compulsory_bytes_per_launch": int(4 * e_plus + 8 * (g.n + 1)),
            "note": "algorithmic bytes = sum over oriented edges of 4(d+u + d+v) + 8|E+| + 4(n+1) (both oriented "
                    "lists read once per edge); traffic (ncu dram bytes per launch) is not measured inside the "
                    "timed run: the committed k_count summaries under profiles/ give it with their commands"}


def static_workload(ctx, g, scale, ef, seed, steps, warmup, fixed_too, e2e):
    """One static workload: learned (or fixed) timed counts, the known-answer checks, optionally
    the fixed rule and the end-to-end path. Returns (result dict, graph handle, info)."""
    import torch
    from custingeralg_b200 import api, native as N
    a = ctx.a
    e_int = edges_intersected_host(g)
    graph = api.Graph.from_csr(g, validate=True)
    out = torch.zeros(g.n + 1, dtype=torch.int32, device=ctx.dev)
    tri = torch.zeros(1, dtype=torch.int64, device=ctx.dev)

    # One synchronous whole-graph count (not sharded) for the structural check, the work figures
    # and the answer.
    T_full, info = graph.count(N.TC_PV_HANDLE, out, tri, sched=N.default_sched())
    gold = known_answer(scale, ef, seed)
    checks = {"triangles": "no known answer for this graph"}
    if gold:
        if gold["triangles"] != T_full:
            raise SystemExit(f"count mismatch: {T_full} vs known answer {gold['triangles']}")
        if pv_digest(out[:g.n].cpu().numpy()) != gold["per_vertex_handle_digest"]:
            raise SystemExit("per-vertex counts differ from the known answer's digest")
        checks = {"triangles": "equals the known answer", "per_vertex_2t": "int32 digest equals the known answer",
                  "known_answer_from": gold.get("checked_by", ""),
                  "max_2t": gold.get("max_2t"), "vertices_wrapping_int32": gold.get("wraps_int32")}
    assert info.edges_intersected == e_int, (info.edges_intersected, e_int)

    fixed = shard_sched(N.default_sched(), ctx)
    d = N.default_sched()
    fixed_desc = f"fixed rule (lane walk up to {d.lane_max_deg}, packed up to {d.packed_max_deg}, CTA above {d.warp_max_deg})"
    sched, desc = fixed, fixed_desc
    if a.static_sched == "learned":
        from custingeralg_b200 import sched_learn as L
        if os.path.exists(L.WEIGHTS):
            sched = shard_sched(L.learned_sched(L.load(L.WEIGHTS), graph, base=N.default_sched()), ctx)
            desc = "learned (custingeralg_b200/data/sched_mlp.bin, this graph's degree cells)"

    step_ms, count_ms, orient_ms, launches = time_static(ctx, graph, out, tri, sched, steps, warmup)
    if int(tri.item()) != T_full:
        raise SystemExit(f"timed count mismatch: {int(tri.item())} vs {T_full}")
    ms = sum(step_ms) / steps
    res = {"value": e_int / (ms / 1e3), "ms_per_step": ms, "steps": steps, "warmup": warmup,
           "config": workload_config(scale, ef, seed, g.n, g.m, e_int), "triangles": T_full, "checks": checks,
           "scheduler": desc, "gpu_launches": launches, "roofline": roofline_for(g, info, count_ms),
           "phase_ms": {"orient": round(statistics.mean(orient_ms), 4), "count": round(statistics.mean(count_ms), 4)}}
    if fixed_too and sched is not fixed:
        f_step, f_count, _, _ = time_static(ctx, graph, out, tri, fixed, steps, warmup)
        if int(tri.item()) != T_full:
            raise SystemExit(f"fixed-rule count mismatch: {int(tri.item())} vs {T_full}")
        f_ms = sum(f_step) / steps
        res["fixed"] = {"value": e_int / (f_ms / 1e3), "ms_per_step": f_ms, "scheduler": fixed_desc,
                        "kernel_ms": round(statistics.mean(f_count), 4),
                        "learned_over_fixed": round(f_ms / ms, 4),
                        "kernel_learned_over_fixed": round(statistics.mean(f_count) / statistics.mean(count_ms), 4)}
    if e2e:
        res["e2e"] = e2e_static(ctx, g, e_int, out, tri, sched, steps, warmup, T_full)
    if ctx.world == 1 and not ctx.a.no_split:
        res["multi_gpu_split"] = split_balance(graph, out, sched, T_full)
    return res, graph


def split_balance(graph, out, sched, T_full, counts=(2, 4, 8), reps=3):
    """The multi-GPU split measured on one GPU: for N ranks, each shard r counted alone (the count
    rank r would run), its centre range, predicted work and best count-kernel time; the shards'
    totals must add up to the whole count. Reports max/mean of work and of time per N."""
    import copy
    from custingeralg_b200 import native as N
    N.lib().tc_profile_enable(1)
    rows = {}
    for n_sh in counts:
        works, times, total = [], [], 0
        for r in range(n_sh):
            sc = copy.copy(sched)
            sc.shard, sc.nshards = r, n_sh
            best = float("inf")
            for _ in range(reps):
                T, info = graph.count(N.TC_PV_HANDLE, out, sched=sc)
                pt = N.PhaseTimes()
                N.check(N.lib().tc_profile_last(pt))
                best = min(best, pt.count_ms)
            total += T
            works.append(info.shard_work)
            times.append(best)
        if total != T_full:
            raise SystemExit(f"{n_sh} shards add up to {total}, not {T_full}")
        rows[str(n_sh)] = {"work_max_over_mean": round(max(works) / (sum(works) / n_sh), 4),
                           "kernel_ms_max_over_mean": round(max(times) / (sum(times) / n_sh), 4),
                           "kernel_ms_per_shard": [round(t, 3) for t in times]}
    N.lib().tc_profile_enable(0)
    return {"note": "each shard of N counted alone on one GPU (the work rank r of N would do); shard totals add "
                    "up to the whole count", "by_ranks": rows}


def e2e_static(ctx, g, e_int, out, tri, sched, steps, warmup, T_full):
    """End to end through the C ABI with host buffers, every step: H2D of the CSR from pinned
    memory, the count (callDeviceAllTrianglesCSR path with per-vertex output), D2H of the
    per-vertex counts and T. The inputs are double-buffered: step i+1's upload runs on its own
    copy stream while step i counts, as a caller counting a sequence of graphs would run it; a
    step's count waits for its own upload, and an upload waits until the count two steps back has
    released its buffer. The L2 flush (a 512 MB write) runs before each count, inside the timed
    region."""
    import torch
    from custingeralg_b200 import api, native as N
    # int32 offsets while they fit: the reference's raw-CSR boundary types them as length_t
    # (int32, tests/cct_csr.cu:279-285); int64 beyond 2^31 - 1 directed edges
    off_host = g.off.astype(np.int32) if g.m < 2**31 else g.off
    h_off = torch.from_numpy(off_host).pin_memory()
    h_ind = torch.from_numpy(g.ind).pin_memory()
    bufs = [(torch.empty_like(h_off, device=ctx.dev), torch.empty_like(h_ind, device=ctx.dev)) for _ in range(2)]
    h_out = torch.empty(g.n + 1, dtype=torch.int32).pin_memory()
    h_tri = torch.empty(1, dtype=torch.int64).pin_memory()
    comp = ctx.stream
    copy = torch.cuda.Stream(device=ctx.dev)
    uploaded = [torch.cuda.Event() for _ in range(2)]
    released = [torch.cuda.Event() for _ in range(2)]
    for ev in released:
        ev.record(comp)

    def run(n):
        for i in range(n):
            k = i % 2
            d_off, d_ind = bufs[k]
            copy.wait_event(released[k])
            with torch.cuda.stream(copy):
                d_off.copy_(h_off, non_blocking=True)
                d_ind.copy_(h_ind, non_blocking=True)
                uploaded[k].record(copy)
            comp.wait_event(uploaded[k])
            ctx.flush.zero_()
            api.count_all_triangles_csr(g.n, d_off, d_ind, out, pv_mode=N.TC_PV_HANDLE, sched=sched, sync=False,
                                        triangles_dev=tri)
            released[k].record(comp)
            ctx.allreduce_(out)
            ctx.allreduce_(tri)
            h_out.copy_(out, non_blocking=True)
            h_tri.copy_(tri, non_blocking=True)

    run(max(1, warmup))
    torch.cuda.synchronize()
    ctx.barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    start.record(comp)
    copy.wait_event(start)
    run(steps)
    end.record(comp)
    end.synchronize()
    ctx.windows.append((t0, time.perf_counter()))
    if int(h_tri.item()) != T_full:
        raise SystemExit(f"e2e count mismatch: {int(h_tri.item())} vs {T_full}")
    total_ms = ctx.max_over_ranks([start.elapsed_time(end)])[0]
    step_s = total_ms / steps / 1e3
    del bufs
    return {"value": e_int / step_s, "unit": UNIT,
            "h2d_bytes_per_step": int(h_off.numel() * h_off.element_size() + h_ind.numel() * 4),
            "d2h_bytes_per_step": int(h_out.numel() * 4 + 8), "ms_per_step": step_s * 1e3,
            "path": ("tc_count_csr32" if h_off.dtype == torch.int32 else "tc_count_csr64")
                    + " (callDeviceAllTrianglesCSR boundary), pinned host CSR in, per-vertex counts out",
            "pipelining": "inputs double-buffered: step i+1's host-to-device copy (own stream) overlaps step i's "
                          "count; every step copies its whole CSR in and its counts out inside the timed region, "
                          "timed from the first copy to the last read-back"}


def run_ours(a, rank, world, local_rank):
    from custingeralg_b200 import generators as G
    global GEN_THREADS
    if world > 1:
        GEN_THREADS = max(1, (os.cpu_count() or 1) // world)
    ctx = Ctx(a, rank, world, local_rank)
    clocks = ClockSampler(local_rank)
    clocks.start()

    g = rmat_graph(ctx, a.scale, a.edge_factor, a.seed)
    main, graph = static_workload(ctx, g, a.scale, a.edge_factor, a.seed, a.steps, a.warmup,
                                  fixed_too=not a.no_fixed, e2e=not a.no_e2e)
    graph.close()
    result = {"metric": METRIC, "value": main["value"], "unit": UNIT, "n_gpus": world, "steps": a.steps,
              "warmup": a.warmup, "ms_per_step": main["ms_per_step"], "higher_is_better": True,
              "scaling": "strong", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
              "config": main["config"], "scheduler": {"static": main["scheduler"]},
              "triangles": main["triangles"], "checks": main["checks"], "gpu_launches": main["gpu_launches"],
              "roofline": main["roofline"], "phase_ms": main["phase_ms"]}
    if world > 1:
        result["parallelism"] = (f"{world} ranks: contiguous edge-centre ranges balanced by predicted work, "
                                 "NCCL all-reduce of per-vertex counts and total inside the step")
    for k in ("fixed", "e2e", "multi_gpu_split"):
        if k in main:
            result[k] = main[k]
    del g

    if a.c3_scale:
        c3g = rmat_graph(ctx, a.c3_scale, a.edge_factor, a.c3_seed)
        c3, graph = static_workload(ctx, c3g, a.c3_scale, a.edge_factor, a.c3_seed, a.c3_steps, a.warmup,
                                    fixed_too=not a.no_fixed, e2e=not a.no_e2e)
        graph.close()
        del c3g
        result["c3"] = c3

    if not a.no_streaming:
        result["streaming"] = run_streaming(ctx, a.stream_sched)
        if not a.no_fixed and a.stream_sched != "fixed":
            fx = run_streaming(ctx, "fixed", verify_every=10)
            result["streaming"]["fixed"] = {k: fx[k] for k in ("value", "ms_total", "updates", "recount_checks",
                                                                  "scheduler", "delta_kernel_ms")}
            result["streaming"]["fixed"]["learned_over_fixed"] = round(result["streaming"]["value"] / fx["value"], 4)
            if fx.get("delta_kernel_ms") and result["streaming"].get("delta_kernel_ms"):
                # the kernels the learned table schedules: the two delta kernels of every batch
                result["streaming"]["fixed"]["delta_kernel_learned_over_fixed"] = round(
                    fx["delta_kernel_ms"] / result["streaming"]["delta_kernel_ms"], 4)
        result["scheduler"]["streaming"] = result["streaming"]["scheduler"]

    clocks.stop()
    result["clocks"] = clocks.summary(ctx.windows)

    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        g = G.rmat(a.scale, a.edge_factor, *RMAT_ABC, seed=a.seed)
        e_int = edges_intersected_host(g)
        v, nt, desc, kind, _, _ = cpu_reference_sample(g, e_int, a.cpu_seconds)
        result["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": nt, "kind": kind, "sample": desc}
        c1 = G.erdos_renyi(1 << 14, 16.0 / (1 << 14), seed=1)
        one = cpu_reference_1core(c1, edges_intersected_host(c1))
        if one:
            v1, _, desc1, _, _, _ = cpu_reference_sample(g, e_int, min(5.0, a.cpu_seconds), seed=7, nthreads=1)
            one["rmat20_sampled_1core"] = {"value": v1, "sample": desc1}
            result["cpu_baseline_1core"] = one
    return result


def streaming_batches(scale, nbatch, base, seed=4):
    """Batch sizes log-uniform on [1, 2^20]; 70 % insertions with R-MAT endpoints, 30 % deletions.
    The deletions are distinct base edges drawn without replacement over the whole run, so each
    one removes an edge that is present when its batch runs (insertions never remove one)."""
    from custingeralg_b200 import generators as G
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(0.0, np.log(2.0 ** 20), nbatch))).astype(np.int64)
    sizes = np.clip(sizes, 1, 1 << 20)
    n_dels = [int(round(0.3 * b)) for b in sizes.tolist()]
    src_of = np.repeat(np.arange(base.n, dtype=np.int32), np.diff(base.off))
    und = np.flatnonzero(src_of < base.ind)           # each undirected base edge once
    picks = und[rng.permutation(und.size)[:sum(n_dels)]]
    out, at = [], 0
    for i, b in enumerate(sizes.tolist()):
        n_del = n_dels[i]
        n_ins = b - n_del
        s_ins, d_ins = G.rmat_pairs(scale, n_ins, seed=seed, stream=i + 1, nthreads=GEN_THREADS)
        pick = picks[at:at + n_del]
        at += n_del
        s = np.concatenate([s_ins, src_of[pick]]).astype(np.int32)
        d = np.concatenate([d_ins, base.ind[pick]]).astype(np.int32)
        dl = np.concatenate([np.zeros(n_ins, np.uint8), np.ones(n_del, np.uint8)])
        perm = rng.permutation(b)
        out.append((s[perm], d[perm], dl[perm]))
    return out


def plan_from_bench(path):
    """The pipeline plan recorded in an earlier bench line's streaming block (its bins)."""
    from custingeralg_b200 import native as N
    with open(path) as f:
        bins = json.loads(f.read().strip().splitlines()[-1])["streaming"]["bins"]
    plan = N.PipelinePlan()
    plan.nbins = len(bins)
    caps = [b["capacity"] for b in bins]
    for i, b in enumerate(bins):
        plan.bin_cap[i] = b["capacity"]
        plan.serve[i] = caps.index(b["served_by_capacity"])
        plan.ctas_per_sm[i] = b.get("plan_ctas_per_sm", 0)
        plan.chunk[i] = b["chunk"]
        plan.split_min[i] = b["split_min"]
    return plan


def tune_pipeline(base, max_b, sched, scale, dev, per_arm=2, small_per_arm=6, small_cap=4096, seed=104):
    """Autotune a pipeline on a twin of the base graph (untimed) and return its plan: for every
    bin of the ladder, batches of sizes inside that bin, two per arm of the tuner (five tile
    shapes and the next bin's graph; six per arm in the bins up to 4096, whose batches differ
    most in size and cost little), in the 70/30 insertion/deletion mix of the workload. The tuner
    gives each batch to the arm with the fewest samples, so every size is drawn once and repeated
    for each arm in turn: the arms are compared on the same sizes."""
    import torch
    from custingeralg_b200 import api, generators as G
    twin = api.Graph.from_csr(base, slack=0.25)
    tp = api.Pipeline(twin, max_b, sched=sched)
    caps = [c for c, _ in tp.info()]
    rng = np.random.default_rng(seed)
    src_of = np.repeat(np.arange(base.n, dtype=np.int32), np.diff(base.off))
    sizes = []
    for i, c in enumerate(caps):
        lo = 1 if i == 0 else caps[i - 1] + 1
        k = small_per_arm if c <= small_cap else per_arm
        for _ in range(k):
            sizes += [int(np.exp(rng.uniform(np.log(lo), np.log(c + 1))))] * 6
    tp.autotune(len(sizes))
    for k, b in enumerate(sizes):
        b = max(1, min(b, max_b))
        n_del = int(round(0.3 * b))
        s_ins, d_ins = G.rmat_pairs(scale, b - n_del, seed=seed, stream=k + 1, nthreads=GEN_THREADS)
        pick = rng.integers(0, base.m, n_del)
        s = torch.from_numpy(np.concatenate([s_ins, src_of[pick]]).astype(np.int32)).to(dev)
        d = torch.from_numpy(np.concatenate([d_ins, base.ind[pick]]).astype(np.int32)).to(dev)
        x = torch.from_numpy(np.concatenate([np.zeros(b - n_del, np.uint8), np.ones(n_del, np.uint8)])).to(dev)
        tp.apply(s, d, x)
    tp.sync()
    plan = tp.plan()
    tp.close()
    twin.close()
    return plan


def run_streaming(ctx, sched_kind, verify_every=None):
    """Update edges per second on R-MAT scale 22 (seed 4) with 200 uneven batches; the running
    count is checked against a full static recount after every batch (outside the timing)."""
    import torch
    from custingeralg_b200 import api, generators as G, native as N
    a, dev = ctx.a, ctx.dev
    verify_every = a.stream_verify if verify_every is None else verify_every
    base = rmat_graph(ctx, a.stream_scale, 16, 4)
    graph = api.Graph.from_csr(base, slack=0.25)
    pv = torch.zeros(base.n + 1, dtype=torch.int32, device=dev)
    delta = torch.zeros(1, dtype=torch.int64, device=dev)
    scratch = torch.zeros(base.n + 1, dtype=torch.int32, device=dev)
    T0, _ = graph.count(N.TC_PV_HANDLE, scratch)
    pv0 = scratch[: base.n].to(torch.int64)
    batches = streaming_batches(a.stream_scale, a.stream_batches, base)
    dbat = [(torch.from_numpy(s).to(dev), torch.from_numpy(d).to(dev), torch.from_numpy(x).to(dev))
            for s, d, x in batches]
    sched = N.default_sched()
    sched_desc = "fixed rule (search when 16 d_long > 16 d_short (log2 d_long + 1))"
    if sched_kind == "learned":
        from custingeralg_b200 import sched_learn as L
        if os.path.exists(L.STREAM_WEIGHTS):
            sched = L.learned_stream_sched(L.load(L.STREAM_WEIGHTS))
            sched_desc = "learned (custingeralg_b200/data/sched_mlp_stream.bin, nominal cell degrees)"
    sched.shard, sched.nshards = ctx.rank, ctx.world
    if a.stream_hub_min is not None:
        sched.stream_hub_min = a.stream_hub_min
    pipe, plan, tune_s = None, None, 0.0
    if a.stream_path == "pipeline":
        max_b = max(s.numel() for s, _, _ in dbat)
        t_tune = time.perf_counter()
        if a.stream_plan:
            plan = plan_from_bench(a.stream_plan)
        elif not a.no_stream_tune:
            plan = tune_pipeline(base, max_b, sched, a.stream_scale, dev)
        tune_s = time.perf_counter() - t_tune
        pipe = api.Pipeline(graph, max_b, sched=sched)
        if plan is not None:
            pipe.set_plan(plan)
        else:
            plan = pipe.plan()
        pipe.profile(True)  # delta-kernel event times and algorithmic bytes per batch
        pipe.prepare(per_vertex=pv, delta_dev=delta)  # pool headroom and captures, before timing
    torch.cuda.synchronize()
    ctx.barrier()
    stream = ctx.stream
    batch_ms, updates, checked, eff = [], 0, 0, {"inserted": 0, "deleted": 0, "ignored": 0}
    t0 = time.perf_counter()
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
            bi = pipe.sync()
            eff["inserted"] += bi.inserted
            eff["deleted"] += bi.deleted
            eff["ignored"] += bi.ignored
        batch_ms.append(e0.elapsed_time(e1))
        updates += s.numel()
        if verify_every and (i % verify_every == 0 or i == len(dbat) - 1):
            tot = ctx.allreduce_(delta.clone())
            T, _ = graph.count(N.TC_PV_HANDLE, scratch)
            if T != T0 + int(tot.item()):
                raise SystemExit(f"streaming mismatch after batch {i}: recount {T} vs running {T0 + int(tot.item())}")
            pv_all = ctx.allreduce_(pv.clone())
            if not torch.equal(scratch[: base.n], (pv_all[: base.n].to(torch.int64) + pv0).to(torch.int32)):
                raise SystemExit(f"per-vertex streaming mismatch after batch {i}")
            checked += 1
    ctx.windows.append((t0, time.perf_counter()))
    batch_ms = ctx.max_over_ranks(batch_ms)
    total_ms = sum(batch_ms)
    final = int(ctx.allreduce_(delta.clone()).item()) + T0
    res = {"value": updates / (total_ms / 1e3), "unit": "update edges/s", "batches": len(dbat),
           "updates": updates, "effective": eff if pipe is not None else None, "ms_total": total_ms,
           "recount_checks": checked, "scheduler": sched_desc, "hub_min": int(sched.stream_hub_min),
           "workload": f"R-MAT scale {a.stream_scale} ef 16 seed 4 base (slack 0.25), {len(dbat)} batches of "
                       "log-uniform size in [1, 2^20], 70% R-MAT insertions / 30% deletions of distinct present "
                       "edges; timed per batch over sort + classify + structure update + delta count, batches "
                       "resident on the device",
           "final_triangles": final, "delta_kernel_ms": None}
    if pipe is not None:
        st = pipe.stats()
        peak, src = measured_peak()
        res["path"] = ("tc_pipeline (one captured CUDA graph per batch-size bin; the delta count of each phase one "
                       "persistent kernel)")
        res["bins"] = [{"capacity": int(plan.bin_cap[i]), "served_by_capacity": int(plan.bin_cap[plan.serve[i]]),
                        "delta_ctas_per_sm": bps, "plan_ctas_per_sm": int(plan.ctas_per_sm[i]),
                        "split_min": int(plan.split_min[i]), "chunk": int(plan.chunk[i])}
                       for i, (_, bps) in enumerate(pipe.info())]
        if a.stream_plan:
            res["autotune"] = f"off: the plan recorded in {os.path.basename(a.stream_plan)}"
        elif a.no_stream_tune:
            res["autotune"] = "off: the pipeline's default plan"
        else:
            res["autotune"] = (f"on a twin of the base graph before the timed run ({tune_s:.1f} s, untimed): per "
                               "bin, two batches per arm (tile shapes, and the next bin's graph)")
        res["delta_kernel_ms"] = round(st["delta_ms"], 3)
        if st["delta_ms"] > 0:
            ach = st["delta_bytes"] / (st["delta_ms"] / 1e3) / 1e9
            res["roofline"] = {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                               "frac": round(ach / peak, 4), "traffic": None, "peak_source": src,
                               "kernel": "delta kernels (deletions + insertions, per batch)",
                               "kernel_ms_total": round(st["delta_ms"], 3),
                               "algorithmic_bytes_total": int(st["delta_bytes"]),
                               "note": "algorithmic bytes = sum over the batch's changed edges {x,y} of "
                                       "4(deg x + deg y) + 8 (both full lists read once per edge, as the "
                                       "reference's K1-K3 intersect them), over the event-timed delta kernels"}
        pipe.close()
    else:
        res["path"] = "tc_apply_batch"
    graph.close()
    torch.cuda.synchronize()
    return res


# ---------------------------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------------------------

def run_reference(a, rank, world):
    if rank != 0:
        return None
    from oracle import pyoracle as O
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libref_cct.so (the reference CPU counter built "
                                                    "from tests/cct.cpp) was not built"}
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "graph.tccsr")
        generate_in_child(["rmat", "--scale", str(a.scale), "--edge-factor", str(a.edge_factor), "--abc",
                           *map(str, RMAT_ABC), "--seed", str(a.seed)], path)
        g = read_tccsr(path)
    e_int = edges_intersected_host(g)
    per_step = max(1.0, min(6.0, 120.0 / max(1, a.steps + a.warmup)))
    for i in range(a.warmup):
        cpu_reference_sample(g, e_int, per_step / 2, seed=1000 + i)
    times, fracs, nt, desc = [], [], 0, ""
    for i in range(a.steps):
        _, nt, desc, kind, t, f = cpu_reference_sample(g, e_int, per_step, seed=i)
        times.append(t)
        fracs.append(f)
    value = e_int * sum(fracs) / sum(times)
    ms_per_step = 1e3 * sum(times) / sum(fracs)   # one whole-graph count, extrapolated
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "int32", "data": "synthetic", "impl": "reference",
            "config": workload_config(a.scale, a.edge_factor, a.seed, g.n, g.m, e_int),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nt, "kind": "reference",
                             "sample": f"each step: {desc}; ms_per_step is one whole-graph count at that rate"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "gpu_launches": 0}


# ---------------------------------------------------------------------------------------------
# launch
# ---------------------------------------------------------------------------------------------

def rank_main(local_rank, a, world, port):
    """One rank of a --gpus N run started by this script (torch.multiprocessing)."""
    os.environ.update({"RANK": str(local_rank), "LOCAL_RANK": str(local_rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    run(a, local_rank, world, local_rank)


def run(a, rank, world, local_rank):
    if world > 1 and a.impl == "ours":
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        res = run_reference(a, rank, world) if a.impl == "reference" else run_ours(a, rank, world, local_rank)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        if world > 1 and a.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def main(argv=None):
    a = parse(argv)
    if a.gpus < 1:
        raise SystemExit("--gpus must be at least 1")
    env_world = os.environ.get("WORLD_SIZE")
    if env_world is not None:
        world = int(env_world)
        if world != a.gpus:
            raise SystemExit(f"--gpus {a.gpus} but the launcher started {world} ranks")
        run(a, int(os.environ.get("RANK", "0")), world, int(os.environ.get("LOCAL_RANK", "0")))
        return
    if a.gpus == 1 or a.impl == "reference":
        run(a, 0, a.gpus, 0)
        return
    import torch
    import torch.multiprocessing as mp
    if torch.cuda.device_count() < a.gpus:
        raise SystemExit(f"--gpus {a.gpus} but only {torch.cuda.device_count()} CUDA devices are visible")
    mp.spawn(rank_main, args=(a, a.gpus, free_port()), nprocs=a.gpus, join=True)


if __name__ == "__main__":
    main()
