#!/usr/bin/env python
"""Multi-source traversal benchmark (GTEPS on one B200 per rank).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl xbtrav|reference]
                    [--workload rmat22_k1024|er335k_k256|rmat16_k64] [--path batched|plain]

Workload (default): undirected R-MAT scale 22, edge factor 16, a/b/c/d =
.57/.19/.19/.05 (symmetrised, cleaned, sorted int32 CSR), 1024 seeded sources
drawn from vertices of non-zero degree; one step = traversal of all 1024
sources producing the int32 level and parent tables (1024 x n each) in HBM.
Both paths are timed on the same inputs in the same run: the batched path
(xb_traverse_batched, one CUDA-graph launch per step; the headline `value`)
and the plain per-call path (xb_traverse, `plain_gteps`).
GTEPS = sum over sources of sum over reached vertices of deg(v) / time (the
"Processed Edges" unit of the reference's BFS_Throughput).  Synthetic seeded
data stands in for the reference's real datasets (not shipped).

N > 1: one process per GPU; the graph is replicated and every rank traverses
its own 1024 sources (weak scaling, no collective on the data path; NCCL is
used only for the barrier and the max/sum of the timing scalars).

--impl reference: the reference's own CPU BFS (Ligra BFS_F + edgeMap from the
reference sources, prebuilt in oracle/_ref/) on the same graph and metric,
all host threads, a bounded sample of sources per step; falls back to the
C restatement in oracle/ when oracle/_ref/ was not built.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "xblossom-sigmetrics27-ae_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

WORKLOADS = {
    "rmat22_k1024": dict(kind="rmat", scale=22, ef=16, k=1024),
    "er335k_k256": dict(kind="er", n=335_000, pairs=1_850_000, k=256),
    "rmat16_k64": dict(kind="rmat", scale=16, ef=16, k=64),
    # 128 independent R-MAT graphs (scale U[10,20], edge factor in {4,8,16,32}), 1..512 sources each
    # (log-uniform), uploaded as one concatenated CSR; all queries in one batched launch
    "multi128": dict(kind="multi", instances=128, k=0),
    # serving: resident graph, Poisson arrivals (seeded rate), 1..4096 sources per query (log-uniform),
    # digests per source, continuous batching over slots; reports GTEPS and p50/p99 latency
    "serve_rmat25": dict(kind="serve", scale=25, ef=32, queries=48, rate=2.0, kmax=4096, slots=3, max_words=2,
                         express=1),
    "serve_rmat22": dict(kind="serve", scale=22, ef=16, queries=96, rate=12.0, kmax=4096, slots=4, max_words=4,
                         express=1),
    # the default graph with one word of sources: ncu DRAM-traffic captures (about 4 GB on the device)
    "rmat22_k64": dict(kind="rmat", scale=22, ef=16, k=64),
    # one pass of the two-word layout (2 words x 64 sources): DRAM-traffic captures
    "rmat22_k128": dict(kind="rmat", scale=22, ef=16, k=128),
    # smaller case for kernel profiles (graph > L2, a few hundred MB on the device)
    "rmat20_k64": dict(kind="rmat", scale=20, ef=16, k=64),
    # one pass of the default layout (4 words x 64 sources) on the default graph: DRAM-traffic captures
    "rmat22_k256": dict(kind="rmat", scale=22, ef=16, k=256),
    # one pass of the two-word layout (2 words x 64 sources) for kernel profiles
    "rmat20_k128": dict(kind="rmat", scale=20, ef=16, k=128),
    # one pass of the default layout (4 words x 64 sources): kernel profiles and DRAM-traffic captures
    "rmat20_k256": dict(kind="rmat", scale=20, ef=16, k=256),
    # weighted: multi-source SSSP distances (xb_multi_sssp), seeded symmetric int32 weights in [1, 100]
    "msssp_rmat22_k64": dict(kind="sssp", graph="rmat", scale=22, ef=16, k=64, wmin=1, wmax=100),
    "msssp_rmat20_k64": dict(kind="sssp", graph="rmat", scale=20, ef=16, k=64, wmin=1, wmax=100),
    # alternating mode: maximum matching from the empty matching (xb_max_match)
    "match_rmat22": dict(kind="match", graph="rmat", scale=22, ef=16, k=0),
    "match_rmat20": dict(kind="match", graph="rmat", scale=20, ef=16, k=0),
}
SEED = 0x5EED
METRIC = "multi-source GTEPS at 1 B200, batched vs plain; p50/p99 query latency"
SSSP_METRIC = "multi-source SSSP GTEPS (directed edges of the graph / time of one call)"
MATCH_METRIC = "maximum matching GTEPS (directed edges of the graph / time of one FindMaximumMatch)"


def make_graph(w: dict):
    import xbtrav

    if w["kind"] == "rmat" or w.get("graph") == "rmat":
        return xbtrav.HostCSR.rmat(w["scale"], w["ef"], 0.57, 0.19, 0.19, seed=SEED)
    return xbtrav.HostCSR.er(w["n"], w["pairs"], seed=SEED)


def make_graph_cpu(w: dict):
    """The workload's graph for the CPU arms, rebuilt without the product
    library (oracle/inputs.py gives the same CSR as make_graph)."""
    from oracle import inputs

    if w["kind"] == "rmat" or w.get("graph") == "rmat":
        return inputs.rmat_csr(w["scale"], w["ef"], 0.57, 0.19, 0.19, seed=SEED)
    return inputs.er_csr(w["n"], w["pairs"], seed=SEED)


def workload_config(name: str, w: dict, info: dict) -> dict:
    """The workload's identity (same keys and values on every arm)."""
    cfg = {"workload": name, "n": info["n"], "m_directed": info["m"], "sources": w["k"], "seed": SEED,
           "l2": "inputs larger than L2 (colIndices > 126 MB); no flush"}
    if w["kind"] == "rmat" or w.get("graph") == "rmat":
        cfg.update(graph=f"rmat scale {w['scale']} ef {w['ef']} a/b/c/d .57/.19/.19/.05")
    else:
        cfg.update(graph=f"uniform n {w['n']} pairs {w['pairs']}")
    return cfg


def measured_peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def traffic_from_profile(workload: str):
    """DRAM bytes per step of each kernel class ({"0": level steps, "1": table
    pass}) from the committed ncu summary profiles/traffic_<workload>.txt."""
    p = os.path.join(ROOT, "profiles", f"traffic_{workload}.txt")
    out = {}
    try:
        for line in open(p):
            line = line.split("#", 1)[0].strip()
            if "=" in line:
                key, val = (x.strip() for x in line.split("=", 1))
                if key.startswith("class"):
                    out[key[5]] = float(val)
    except OSError:
        return None
    return out or None


def cpu_baseline_port(ro, ci, sources, budget_s: float = 15.0) -> dict:
    """The C restatement (oracle/) on all host cores, a bounded sample of sources."""
    from oracle import oracle

    cores = os.cpu_count() or 1
    sample = list(sources[: max(1, min(len(sources), cores))])
    t0 = time.perf_counter()
    _, _, e, _ = oracle.msbfs(ro, ci, np.array(sample, np.int32), threads=cores)
    dt = time.perf_counter() - t0
    # grow the sample toward the budget
    per = dt / len(sample)
    extra = int(min(len(sources) - len(sample), max(0, (budget_s - dt) / max(per, 1e-9))))
    if extra > 0:
        more = sources[len(sample): len(sample) + extra]
        t1 = time.perf_counter()
        _, _, e2, _ = oracle.msbfs(ro, ci, np.array(more, np.int32), threads=cores)
        dt += time.perf_counter() - t1
        e += e2
        sample += list(more)
    return {"value": e / dt / 1e9, "unit": "GTEPS", "cores": cores, "kind": "port",
            "sample": f"{len(sample)} of the workload's sources, levels + min-id parents, {dt:.1f} s"}


def sssp_weights(ro, ci, w):
    import xbtrav

    return xbtrav.symmetric_weights(ro, ci, SEED, w["wmin"], w["wmax"])


def sssp_cpu(ro, ci, wts, sources, cores):
    """One multi-source SSSP call on the host: the reference's Ligra MultiSSSP
    (oracle/_ref) on all cores, else the C restatement (one core)."""
    from oracle import oracle

    t0 = time.perf_counter()
    if oracle.ligra_msssp_available():
        oracle.ligra_msssp(ro, ci, wts, sources, threads=cores)
        kind, used, what = "reference", cores, "Ligra MultiSSSP from the reference sources (oracle/_ref)"
    else:
        oracle.msssp(ro, ci, wts, sources)
        kind, used, what = "port", 1, "C restatement (oracle/)"
    return time.perf_counter() - t0, kind, used, what


def run_reference_sssp(args, w, name) -> None:
    from oracle import inputs

    ro, ci = make_graph_cpu(w)
    info = {"n": len(ro) - 1, "m": len(ci)}
    wts = inputs.symmetric_weights(ro, ci, SEED, w["wmin"], w["wmax"])
    sources = inputs.select_sources(ro, SEED + 1, w["k"])
    cores = os.cpu_count() or 1
    times = []
    for step in range(args.warmup + args.steps):
        secs, kind, used, what = sssp_cpu(ro, ci, wts, sources, cores)
        if step >= args.warmup:
            times.append(secs)
    value = info["m"] / (sum(times) / len(times)) / 1e9
    cfg = workload_config(name, w, info)
    cfg.update(weights=f"symmetric int32 in [{w['wmin']}, {w['wmax']}]")
    print(json.dumps({
        "impl": "reference", "metric": SSSP_METRIC, "path": "Ligra MultiSSSP (reference CPU code)", "value": value, "unit": "GTEPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator)", "config": cfg,
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": used, "kind": kind,
                         "sample": f"the whole workload ({w['k']} sources) per step, {what}"},
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_sssp(args, w, name) -> None:
    """Multi-source SSSP (xb_multi_sssp) on one weighted resident graph: one
    step = one call over the workload's sources producing the float distance
    array in HBM."""
    import torch

    import xbtrav

    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    csr = make_graph(w)
    ro, ci = csr.arrays()
    info = csr.info()
    wts = sssp_weights(ro, ci, w)
    ctx = xbtrav.Context(0)
    g = ctx.upload(csr)
    g.set_weights(wts)
    sources = g.select_sources(SEED + 1, w["k"])
    src_dev = torch.from_numpy(sources).to(dev)
    dist_dev = torch.empty(g.n, dtype=torch.float32, device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
    setup_s = time.perf_counter() - t0

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        stats = [fn() for _ in range(steps)]
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        return ev0.elapsed_time(ev1), stats

    clocks = ClockSampler(0)
    clocks.start()
    ms, stats = timed(lambda: ctx.multi_sssp(g, src_dev, out="device", dist=dist_dev)[1], args.steps)
    clk = clocks.stop()
    value = g.m * args.steps / (ms / 1e3) / 1e9
    relaxed = sum(st["edges_scanned"] for st in stats) / args.steps
    # the relax kernel alone (per-launch CUDA events on the engine's stream)
    ctx.set_tuning(timing=1)
    _, tstats = timed(lambda: ctx.multi_sssp(g, src_dev, out="device", dist=dist_dev)[1], args.steps)
    ctx.set_tuning(timing=0)
    relax_ms = sum(st["class_ms"][0] for st in tstats)
    relax_bytes = sum(st["class_bytes"][0] for st in tstats)
    relax_launches = sum(st["class_launches"][0] for st in tstats)
    peak, peak_src = measured_peaks()
    achieved = relax_bytes / (relax_ms / 1e3) / 1e9 if relax_ms > 0 else None
    launches = sum(sum(st["class_launches"]) for st in stats)
    # end to end through the host-buffer call: sources in, distances out
    host_dist = np.empty(g.n, np.float32)
    e2e_ms, _ = timed(lambda: ctx.multi_sssp(g, sources, out="host", dist=host_dist)[1], args.steps)
    cpu = None
    if not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        secs, kind, used, what = sssp_cpu(ro, ci, wts, sources, cores)
        cpu = {"value": g.m / secs / 1e9, "unit": "GTEPS", "cores": used, "kind": kind,
               "sample": f"one call over all {w['k']} sources ({secs:.2f} s), {what}"}
    cfg = workload_config(name, w, info)
    cfg.update(weights=f"symmetric int32 in [{w['wmin']}, {w['wmax']}]")
    line = {
        "metric": SSSP_METRIC, "parallelism": "replicas1",
        "path": "xb_multi_sssp (edge-balanced rounds, host loop over rounds)", "value": value, "unit": "GTEPS", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded R-MAT generator, seeded weights)",
        "config": cfg,
        "relaxations_per_step": relaxed, "grelax_per_s": relaxed * args.steps / (ms / 1e3) / 1e9,
        "rounds": stats[-1]["levels"],
        "roofline": {"bound": "hbm", "kernel": "k_sssp_relax", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak if achieved else None, "peak_source": peak_src,
                     "traffic": None, "bytes_model": "8 B per relaxation (column index + weight)",
                     "relax_ms_per_step": relax_ms / args.steps, "relax_launches_per_step": relax_launches / args.steps},
        "cpu_baseline": cpu,
        "e2e": {"value": g.m * args.steps / (e2e_ms / 1e3) / 1e9, "unit": "GTEPS",
                "h2d_bytes_per_step": 4 * len(sources), "d2h_bytes_per_step": 4 * g.n},
        "clocks": clk, "gpu_launches": launches, "setup_s": setup_s,
    }
    print(json.dumps(line), flush=True)
    g.close()
    ctx.close()


def match_cpu(ro, ci, cores):
    """One maximum matching on the host: the reference's own CPU engine
    (oracle/_ref) on all cores, else the Edmonds restatement (one core)."""
    from oracle import oracle

    t0 = time.perf_counter()
    if oracle.ref_match_available():
        size, _ = oracle.ref_max_match(ro, ci, threads=cores)
        kind, used, what = "reference", cores, "X-Blossom CPU engine par_pro_pernode from the reference sources (oracle/_ref)"
    else:
        size, _ = oracle.max_match(ro, ci)
        kind, used, what = "port", 1, "Edmonds restatement (oracle/)"
    return time.perf_counter() - t0, size, kind, used, what


def run_reference_match(args, w, name) -> None:
    ro, ci = make_graph_cpu(w)
    info = {"n": len(ro) - 1, "m": len(ci)}
    cores = os.cpu_count() or 1
    times = []
    for step in range(args.warmup + args.steps):
        secs, size, kind, used, what = match_cpu(ro, ci, cores)
        if step >= args.warmup:
            times.append(secs)
    value = info["m"] / (sum(times) / len(times)) / 1e9
    print(json.dumps({
        "impl": "reference", "metric": MATCH_METRIC, "value": value, "unit": "GTEPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generator)", "config": workload_config(name, w, info), "matching_size": size,
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": used, "kind": kind,
                         "sample": f"the whole workload (one maximum matching from the empty one) per step, {what}"},
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_match(args, w, name) -> None:
    """Alternating mode: one step = a maximum matching of the resident graph
    from the empty matching (xb_max_match), mate array in HBM."""
    import torch

    import xbtrav

    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    csr = make_graph(w)
    ro, ci = csr.arrays()
    info = csr.info()
    ctx = xbtrav.Context(0)
    g = ctx.upload(csr)
    empty = torch.full((g.n,), -1, dtype=torch.int32, device=dev)
    mate = torch.empty_like(empty)
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
    setup_s = time.perf_counter() - t0

    def step():
        mate.copy_(empty)
        return ctx.max_match(g, init=mate)[1]

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        stats = [fn() for _ in range(steps)]
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        return ev0.elapsed_time(ev1), stats

    clocks = ClockSampler(0)
    clocks.start()
    ms, stats = timed(step, args.steps)
    clk = clocks.stop()
    size = int((mate >= 0).sum().item()) // 2
    value = g.m * args.steps / (ms / 1e3) / 1e9
    ctx.set_tuning(timing=1)
    _, tstats = timed(step, args.steps)
    ctx.set_tuning(timing=0)
    exp_ms = sum(st["class_ms"][0] for st in tstats)
    exp_bytes = sum(st["class_bytes"][0] for st in tstats)
    peak, peak_src = measured_peaks()
    achieved = exp_bytes / (exp_ms / 1e3) / 1e9 if exp_ms > 0 else None
    launches = sum(sum(st["class_launches"]) for st in stats)
    host_mate = np.full(g.n, -1, np.int32)
    e2e_ms, _ = timed(lambda: ctx.max_match(g, init=host_mate)[1], args.steps)
    cpu = None
    if not args.no_cpu_baseline:
        secs, rsize, kind, used, what = match_cpu(ro, ci, os.cpu_count() or 1)
        cpu = {"value": g.m / secs / 1e9, "unit": "GTEPS", "cores": used, "kind": kind,
               "sample": f"one maximum matching ({secs:.2f} s, size {rsize}), {what}"}
    cfg = workload_config(name, w, info)
    last = stats[-1]
    print(json.dumps({
        "metric": MATCH_METRIC, "parallelism": "replicas1",
        "path": "xb_max_match from the empty matching (host loop over phases, each phase's levels in a "
                "captured CUDA-graph WHILE loop)", "value": value, "unit": "GTEPS", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded R-MAT generator)", "config": cfg,
        "matching_size": size, "phases": last["batches"], "levels": last["levels"],
        "blossom_levels": last["pull_levels"], "augmentations": last["vertices_scanned"],
        "entries_scanned": last["edges_scanned"],
        "roofline": {"bound": "hbm", "kernel": "k_mm_expand", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "peak_source": peak_src, "traffic": None,
                     "bytes_model": "8 B per scanned adjacency entry (column index + neighbour state)",
                     "expand_ms_per_step": exp_ms / args.steps},
        "cpu_baseline": cpu,
        "e2e": {"value": g.m * args.steps / (e2e_ms / 1e3) / 1e9, "unit": "GTEPS",
                "h2d_bytes_per_step": 4 * g.n, "d2h_bytes_per_step": 4 * g.n},
        "clocks": clk, "gpu_launches": launches, "setup_s": setup_s,
    }), flush=True)
    g.close()
    ctx.close()


def run_reference(args, w, name) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if w["kind"] == "sssp":
        run_reference_sssp(args, w, name)
        return
    if w["kind"] == "match":
        run_reference_match(args, w, name)
        return
    from oracle import inputs, oracle

    t_gen = time.perf_counter()
    ro, ci = make_graph_cpu(w)
    info = {"n": len(ro) - 1, "m": len(ci)}
    sources = inputs.select_sources(ro, SEED + 1, w["k"])
    cores = os.cpu_count() or 1
    use_ligra = oracle.ligra_available()
    # a bounded sample of the workload's sources per step (the whole run stays
    # within a few minutes); consecutive steps take consecutive slices
    per_step = min(w["k"], 64)
    times, edges = [], []
    for step in range(args.warmup + args.steps):
        sel = np.roll(sources, -step * per_step)[:per_step]
        if use_ligra:
            _, secs, e = oracle.ligra_bfs(ro, ci, sel, threads=cores, want_parents=False)
        else:
            t0 = time.perf_counter()
            _, _, e, _ = oracle.msbfs(ro, ci, sel, threads=cores, want_tables=False)
            secs = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(secs)
            edges.append(e)
    value = sum(edges) / sum(times) / 1e9
    kind = "reference" if use_ligra else "port"
    what = ("Ligra BFS_F/edgeMap from the reference sources (oracle/_ref), parents only"
            if use_ligra else "C restatement (oracle/), levels only")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GTEPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator)",
        "config": workload_config(name, w, info),
        "path": what,
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": cores, "kind": kind,
                         "sample": f"{per_step} of the workload's {w['k']} sources per step (consecutive slices), "
                                   f"{what}; inputs rebuilt in numpy (oracle/inputs.py)"},
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "setup_s": time.perf_counter() - t_gen,
    }
    print(json.dumps(line), flush=True)


def multi_instances(count: int, seed: int):
    """Seeded instance specs of the uneven workload: (scale, edge factor, k, graph seed)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        scale = int(rng.integers(10, 21))
        ef = int(rng.choice([4, 8, 16, 32]))
        k = int(np.floor(np.exp(rng.uniform(0.0, np.log(513.0)))))
        specs.append((scale, ef, max(1, min(512, k)), seed + 1000 + i))
    return specs


def run_multi(args, w, name) -> None:
    """Config of many uneven graphs: batched (one launch) vs plain (one call per query)."""
    import torch

    import xbtrav

    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    specs = multi_instances(w["instances"], SEED)
    hosts = [xbtrav.HostCSR.rmat(sc, ef, 0.57, 0.19, 0.19, seed=gs) for sc, ef, _, gs in specs]
    ctx = xbtrav.Context(0)
    # this workload's tuning (autotuner, batched path): many small queries fill
    # 64-source passes better than 128-source ones, and more chains overlap
    # the many short passes
    ctx.set_tuning(words=1, chains=args.chains or 8)
    graphs = ctx.upload_batch(hosts)
    queries = []
    for (sc, ef, k, gs), g in zip(specs, graphs):
        queries.append((g, torch.from_numpy(g.select_sources(gs + 1, k)).to(dev)))
    outs = [(torch.empty((int(q.numel()), g.n), dtype=torch.int32, device=dev),
             torch.empty((int(q.numel()), g.n), dtype=torch.int32, device=dev)) for g, q in queries]
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)

    def batched():
        return ctx.traverse_batched(queries, outputs=outs)[1]["edges_traversed"]

    def plain():
        e = 0
        for (g, q), (lv, pr) in zip(queries, outs):
            e += ctx.traverse(g, q, out="device", level=lv, parent=pr).stats["edges_traversed"]
        return e

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            ev0.record(stream)
        e = sum(fn() for _ in range(steps))
        with torch.cuda.stream(stream):
            ev1.record(stream)
        torch.cuda.synchronize(dev)
        return ev0.elapsed_time(ev1), e

    clocks = ClockSampler(0)
    clocks.start()
    b_ms, b_e = timed(batched, args.steps)
    clk = clocks.stop()
    p_ms, p_e = timed(plain, args.steps)
    value = b_e / (b_ms / 1e3) / 1e9
    plain_v = p_e / (p_ms / 1e3) / 1e9
    tun = ctx.tuning()
    line = {
        "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": b_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic (seeded R-MAT generator)",
        "config": {"workload": name, "instances": len(specs), "sources": int(sum(s[2] for s in specs)),
                   "vertices": int(sum(g.n for g in graphs)), "m_directed": int(sum(g.m for g in graphs)),
                   "seed": SEED, "layout": "one concatenated CSR, per-instance offsets (xb_graph_upload_batch)"},
        "path": f"xb_traverse_batched, {tun['chains']} chains",
        "batched_gteps": value, "plain_gteps": plain_v, "batched_over_plain": value / plain_v,
        "plain_ms_per_step": p_ms / args.steps, "clocks": clk, "setup_s": setup_s,
    }
    print(json.dumps(line), flush=True)
    for g in graphs:
        g.close()
    ctx.close()


def run_serve(args, w, name) -> None:
    """Serving: queries arrive (Poisson, seeded), are admitted and packed into
    slot passes on the fly; throughput over the whole trace and per-query
    latency from arrival to the last digest."""
    import torch

    import xbtrav
    from xbtrav import serve

    t0 = time.perf_counter()
    csr = xbtrav.HostCSR.rmat(w["scale"], w["ef"], 0.57, 0.19, 0.19, seed=SEED)
    info = csr.info()
    ctx = xbtrav.Context(0)
    # passes start at one word (64 sources: low latency); max_words lets large
    # queries open wider passes where per-slot memory allows (a two-word slot's
    # workspace is about 20 GB at scale 25, plus scratch rows only for passes
    # that mix tables and digests), so that graph runs three slots of at most
    # two words
    ctx.set_tuning(words=1)
    g = ctx.upload(csr)
    del csr
    slots = args.chains or w["slots"]
    srv = serve.Server(ctx, slots=slots, max_words=w.get("max_words", 1), express=w.get("express", 0))
    # warm-up: one full pass per slot and width (workspaces, scratch, captured pass graphs)
    srv.warmup(g, SEED + 99)
    setup_s = time.perf_counter() - t0
    # one trace per arrival rate on the same resident graph and server; the
    # same seed gives the same queries at every rate, their gaps scaled
    rates = [float(x) for x in args.rates.split(",") if x.strip()] or [w["rate"]]
    sweep = []
    for rate in rates:
        srv.completed.clear()
        srv.edges = 0
        srv.passes = 0
        trace = serve.poisson_trace([g], rate, w["queries"], SEED + 3, kmax=w["kmax"])
        clocks = ClockSampler(0)
        clocks.start()
        out = srv.run_trace(trace)
        clk = clocks.stop()
        sweep.append({"rate_per_s": rate, "gteps": out["gteps"], "p50_ms": out["p50_ms"], "p99_ms": out["p99_ms"],
                      "mean_ms": out["mean_ms"], "max_ms": out["max_ms"], "passes": out["passes"],
                      "trace_seconds": out["seconds"], "clocks": clk})
        print(json.dumps({"serve_rate": sweep[-1]}), file=sys.stderr, flush=True)
    sel = next((x for x in sweep if x["rate_per_s"] == w["rate"]), sweep[0])
    out = {"gteps": sel["gteps"], "seconds": sel["trace_seconds"], "p50_ms": sel["p50_ms"], "p99_ms": sel["p99_ms"],
           "mean_ms": sel["mean_ms"], "max_ms": sel["max_ms"], "passes": sel["passes"]}
    clk = sel["clocks"]
    ks = [len(t[2]) for t in trace]
    line = {
        "metric": METRIC, "value": out["gteps"], "unit": "GTEPS", "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": out["seconds"] * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic (seeded R-MAT generator, seeded Poisson arrivals)",
        "config": {"workload": name, "n": info["n"], "m_directed": info["m"], "seed": SEED,
                   "graph": f"rmat scale {w['scale']} ef {w['ef']} a/b/c/d .57/.19/.19/.05",
                   "queries": len(trace), "sources_total": int(sum(ks)), "k_range": [1, w["kmax"]],
                   "arrival_rate_per_s": sel["rate_per_s"], "slots": slots, "max_words": srv.max_words,
                   "express_slots": srv.express,
                   "result": "per-source digests"},
        "path": "xbtrav.serve.Server over xb_slot_launch (continuous batching)",
        "latency_ms": {"p50": out["p50_ms"], "p99": out["p99_ms"], "mean": out["mean_ms"], "max": out["max_ms"]},
        "passes": out["passes"], "trace_seconds": out["seconds"], "clocks": clk, "setup_s": setup_s,
    }
    if len(sweep) > 1:
        line["rate_sweep"] = [{k: v for k, v in x.items() if k != "clocks"} for x in sweep]
    print(json.dumps(line), flush=True)
    ctx.slots_release()
    g.close()
    ctx.close()


SERVE_LEG = dict(queries=48, rate=12.0, kmax=4096, slots=4, max_words=4, express=1)


def serve_leg(ctx, g, dev, rank, dist, max_over_ranks, sum_over_ranks, barrier) -> dict:
    """Serving on the headline's resident graph: seeded Poisson arrivals (rate
    12/s), 1..4096 sources per query (log-uniform), digests, continuous
    batching over 4 slots (one an express lane at high stream priority for
    small queries), shortest query first, passes 1, 2 or 4 words wide
    as the opening query needs (xbtrav.serve).  Latency
    = arrival to the query's last digest; p50/p99 are the largest over ranks,
    throughput the sum of the ranks' processed edges over the longest trace."""
    from xbtrav import replicas, serve

    ctx.set_tuning(words=1)
    srv = serve.Server(ctx, slots=SERVE_LEG["slots"], max_words=SERVE_LEG["max_words"],
                       express=SERVE_LEG["express"])
    srv.warmup(g, SEED + 99)  # every slot and width: workspaces, scratch rows, captured pass graphs
    srv.completed.clear()
    srv.edges = 0
    srv.passes = 0
    trace = serve.poisson_trace([g], SERVE_LEG["rate"], SERVE_LEG["queries"],
                                replicas.rank_seed(SEED + 3, rank), kmax=SERVE_LEG["kmax"])
    barrier()
    clocks = ClockSampler(dev.index)
    clocks.start()
    out = srv.run_trace(trace)
    clk = clocks.stop()
    barrier()
    ctx.slots_release()
    for s in range(SERVE_LEG["slots"]):
        ctx.slot_set_priority(s, 0)
    secs = max_over_ranks(out["seconds"])
    edges = sum_over_ranks(srv.edges)
    return {
        "latency_ms": {"p50": max_over_ranks(out["p50_ms"]), "p99": max_over_ranks(out["p99_ms"]),
                       "mean": max_over_ranks(out["mean_ms"]), "max": max_over_ranks(out["max_ms"])},
        "gteps": edges / secs / 1e9, "trace_seconds": secs, "queries": len(trace),
        "sources_total": int(sum(len(t[2]) for t in trace)), "arrival_rate_per_s": SERVE_LEG["rate"],
        "k_range": [1, SERVE_LEG["kmax"]], "slots": SERVE_LEG["slots"],
        "sources_per_pass": [srv.word_bits * srv.base_words, srv.word_bits * srv.max_words],
        "order": "shortest query first, queries waiting over 1 s first; 1 express slot (high priority, small queries)",
        "passes": out["passes"], "result": "per-source digests", "clocks": clk,
        "path": "xbtrav.serve.Server over xb_slot_launch (continuous batching, admission by free HBM)",
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="xbtrav", choices=["xbtrav", "reference"])
    ap.add_argument("--workload", default="rmat22_k1024", choices=sorted(WORKLOADS))
    ap.add_argument("--path", default="batched", choices=["batched", "plain"],
                    help="path the headline value measures (both are timed)")
    ap.add_argument("--chains", type=int, default=0, help="batched chains (0: tuned default)")
    ap.add_argument("--plain-only", action="store_true",
                    help="time the plain path only (short runs for kernel profiles)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving (latency) leg")
    ap.add_argument("--rates", default="",
                    help="serve workloads: comma-separated arrival rates per second, one trace each on the "
                         "same resident graph (default: the workload's rate)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        if w["kind"] in ("multi", "serve"):
            print(json.dumps({"impl": "reference", "unavailable": "the multi-graph and serving workloads are timed "
                              "on the GPU paths only; the reference arm runs the single-graph workloads"}))
            return
        run_reference(args, w, args.workload)
        return
    if w["kind"] == "multi":
        run_multi(args, w, args.workload)
        return
    if w["kind"] == "serve":
        run_serve(args, w, args.workload)
        return
    if w["kind"] == "sssp":
        run_sssp(args, w, args.workload)
        return
    if w["kind"] == "match":
        run_match(args, w, args.workload)
        return

    import torch

    import xbtrav
    from xbtrav import replicas

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    t_setup = time.perf_counter()
    csr = make_graph(w)
    info = csr.info()
    ro, ci = csr.arrays()
    ctx = xbtrav.Context(local)
    if args.chains:
        ctx.set_tuning(chains=args.chains)
    g = ctx.upload(csr)
    k = w["k"]
    sources = g.select_sources(replicas.rank_seed(SEED + 1, rank), k)
    src_dev = torch.from_numpy(sources).to(dev)
    level = torch.empty((k, g.n), dtype=torch.int32, device=dev)
    parent = torch.empty((k, g.n), dtype=torch.int32, device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
    setup_s = time.perf_counter() - t_setup

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(dist, x, dev)

    def sum_over_ranks(x: float) -> float:
        return replicas.sum_over_ranks(dist, x, dev)

    def plain_step():
        return ctx.traverse(g, src_dev, out="device", level=level, parent=parent).stats

    def batched_step():
        return ctx.traverse_batched([(g, src_dev)], outputs=[(level, parent)])[1]

    def timed(step, steps, label, sampler=None):
        """steps of `step` between CUDA events on the engine's stream; returns
        (ms, summed stats).  The steps run inside an NVTX range named `label`
        (a profiler can capture one leg's launches with --nvtx-include)."""
        barrier()
        if sampler is not None:
            sampler.start()
        torch.cuda.nvtx.range_push(label)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        agg = {"edges_traversed": 0, "class_ms": [0.0, 0.0, 0.0], "class_bytes": [0, 0, 0],
               "class_launches": [0, 0, 0], "levels": 0, "push_levels": 0, "pull_levels": 0, "algo_bytes": 0}
        with torch.cuda.stream(stream):
            ev0.record(stream)
        for _ in range(steps):
            s = step()
            agg["edges_traversed"] += s["edges_traversed"]
            agg["algo_bytes"] += s["algo_bytes"]
            for i in range(3):
                agg["class_ms"][i] += s["class_ms"][i]
                agg["class_bytes"][i] += s["class_bytes"][i]
                agg["class_launches"][i] += s["class_launches"][i]
            agg["levels"] = s["levels"]
            agg["push_levels"] += s["push_levels"]
            agg["pull_levels"] += s["pull_levels"]
        with torch.cuda.stream(stream):
            ev1.record(stream)
        torch.cuda.nvtx.range_pop()
        barrier()
        clk = sampler.stop() if sampler is not None else None
        return max_over_ranks(ev0.elapsed_time(ev1)), agg, clk

    # plain per-call path (the drop-in): one pass of the layout's words per launch
    # sequence, host level loop
    ctx.set_tuning(timing=0)
    for _ in range(args.warmup):
        plain_step()
    plain_ms, plain_agg, _ = timed(plain_step, args.steps, "plain")
    plain_gteps = sum_over_ranks(plain_agg["edges_traversed"]) / (plain_ms / 1e3) / 1e9

    # the plain path with one word (64 sources) per launch sequence
    tun0 = ctx.tuning()
    ctx.set_tuning(words=1)
    plain_step()
    pw_ms, pw_agg, _ = timed(plain_step, max(1, min(args.steps, 3)), "plain_one_word")
    plain_word_gteps = sum_over_ranks(pw_agg["edges_traversed"]) / (pw_ms / 1e3) / 1e9
    ctx.set_tuning(words=tun0["words"])

    # per-kernel-class device times of the same kernels (one step, event-timed per class)
    ctx.set_tuning(timing=1)
    _, cls_agg, _ = timed(plain_step, 1, "plain_classes")
    ctx.set_tuning(timing=0)

    # batched path: the whole step is one CUDA-graph launch
    clocks = ClockSampler(local)
    if args.plain_only:
        args.path = "plain"
        b_ms, b_agg, clk = plain_ms, plain_agg, {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["not sampled"]}
    else:
        # clocks sampled from the warm-up on: the timed region alone is shorter
        # than a few sampling periods
        clocks.start()
        for _ in range(args.warmup):
            batched_step()
        b_ms, b_agg, _ = timed(batched_step, args.steps, "batched")
        clk = clocks.stop()
    edges_total = sum_over_ranks(b_agg["edges_traversed"])
    value = edges_total / (b_ms / 1e3) / 1e9
    headline = value if args.path == "batched" else plain_gteps
    ms = b_ms if args.path == "batched" else plain_ms

    # roofline of the dominant kernel class (its kernels event-timed per class)
    peak, peak_kind = measured_peaks()
    dom = 0 if cls_agg["class_ms"][0] >= cls_agg["class_ms"][1] else 1
    dom_name = ["level steps (k_pull_lanes / k_pull_heavy / k_pull_hubs; k_push_*)",
                "table pass (k_tables)"][dom]
    achieved = (cls_agg["class_bytes"][dom] / (cls_agg["class_ms"][dom] / 1e3) / 1e9
                if cls_agg["class_ms"][dom] > 0 else None)
    tr = traffic_from_profile(args.workload)
    engine_gbs = b_agg["algo_bytes"] / (b_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                "traffic": tr.get(str(dom)) if isinstance(tr, dict) else None,
                "class_ms_per_step": cls_agg["class_ms"],
                "class_gbytes_per_step": [x / 1e9 for x in cls_agg["class_bytes"]],
                "batched_engine_gbs": engine_gbs, "batched_engine_frac": engine_gbs / peak}

    # end to end through the C ABI with host buffers (pinned), copies in the timed region
    def e2e_run(batched: bool, steps: int):
        # every rank takes the same branch: a rank whose page-locked tables
        # cannot be allocated makes all ranks skip the measurement together
        # (no rank waits in a collective the others never reach)
        try:
            hl = torch.empty((k, g.n), dtype=torch.int32, pin_memory=True)
            hp = torch.empty((k, g.n), dtype=torch.int32, pin_memory=True)
            ok = 1.0
        except Exception:  # noqa: BLE001
            hl = hp = None
            ok = 0.0
        if dist is not None:
            ok = -max_over_ranks(-ok)  # the minimum over ranks
        if ok < 1.0:
            raise RuntimeError("page-locked host tables could not be allocated on every rank")
        hs = torch.from_numpy(sources).pin_memory().numpy()
        ln, pn = hl.numpy(), hp.numpy()

        def one():
            if batched:
                return ctx.traverse_batched([(g, hs)], out="host", outputs=[(hl, hp)])[1]["edges_traversed"]
            return ctx.traverse(g, hs, level=ln, parent=pn).stats["edges_traversed"]

        one()
        barrier()
        t0 = time.perf_counter()
        et = 0
        for _ in range(steps):
            et += one()
        barrier()
        dt = max_over_ranks(time.perf_counter() - t0)
        et = sum_over_ranks(et)
        del hl, hp
        return et / dt / 1e9

    e2e = None
    if not args.no_e2e:
        try:
            e2e_steps = args.steps
            e2e = {"value": e2e_run(args.path == "batched", e2e_steps), "unit": "GTEPS",
                   "h2d_bytes_per_step": 4 * k, "d2h_bytes_per_step": 8 * k * g.n, "steps": e2e_steps,
                   "note": ("xb_traverse_batched" if args.path == "batched" else "xb_traverse") +
                           " with a host source list and page-locked host level/parent tables; graph resident"}
            e2e["plain_value"] = e2e_run(False, e2e_steps) if args.path == "batched" else e2e["value"]
        except Exception as ex:  # noqa: BLE001
            e2e = {"value": None, "unit": "GTEPS", "error": str(ex)[:200]}

    # the latency half of the metric: a seeded Poisson trace of queries served
    # on the same resident graph with continuous batching over slots
    tun = ctx.tuning()
    serving = None
    if not args.plain_only and not args.no_serve:
        del level, parent
        torch.cuda.empty_cache()
        serving = serve_leg(ctx, g, dev, rank, dist, max_over_ranks, sum_over_ranks, barrier)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_port(ro, ci, sources)

    if rank == 0:
        path_desc = (f"xb_traverse_batched (one CUDA-graph launch per step, device level loop, "
                     f"{tun['chains']} chains, {tun['word_bits']} sources per word x {tun['words']})"
                     if args.path == "batched" else "xb_traverse (host level loop, one pass per launch sequence)")
        agg = b_agg if args.path == "batched" else plain_agg
        line = {
            "metric": METRIC, "value": headline, "unit": "GTEPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded R-MAT / uniform generator)",
            "config": workload_config(args.workload, w, info),
            "parallelism": f"replicas{world}", "path": path_desc,
            "batched_gteps": value, "plain_gteps": plain_gteps, "batched_over_plain": value / plain_gteps,
            "plain_one_word_gteps": plain_word_gteps, "batched_over_plain_one_word": value / plain_word_gteps,
            "plain_ms_per_step": plain_ms / args.steps,
            "undirected_gteps": headline / 2,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "latency_ms": serving["latency_ms"] if serving else None, "serving": serving,
            "gpu_launches": sum(agg["class_launches"]),
            "levels": agg["levels"], "push_levels_per_step": agg["push_levels"] / args.steps,
            "pull_levels_per_step": agg["pull_levels"] / args.steps, "setup_s": setup_s,
        }
        print(json.dumps(line), flush=True)
    g.close()
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
