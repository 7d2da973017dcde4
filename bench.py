#!/usr/bin/env python3
"""Benchmark: ForceAtlas2 / Barnes-Hut node-ticks/s on B200.

A step is one FA2 tick over the whole graph (tree build, repulsion walk,
attraction, gravity, FP64 swing/traction, speed, update). The default workload
is the 1M-node power-law configuration-model graph laid out in 2D (theta 1.2);
every rank runs its own replica (weak scaling: the single graph has no exchange
step to shard).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One JSON line on rank 0. The roofline block is the repulsion walk's: its
algorithmic FLOPs (10 operations per far-cell or exact-pair interaction, the
interactions counted on a replay of the timed ticks) over its CUDA-event time,
against the nominal FP32 FMA rate, and its algorithmic bytes against the
measured HBM copy bandwidth. The CPU baseline is the FP64 restatement of the
reference's tick (the oracle) on this host's cores, over a bounded sample of ticks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 2 ** 20
FLUSH_BYTES = 256 * 2 ** 20
FLOPS_PER_INTERACTION = {2: 10, 3: 13}
REF_1M_NODE_TICKS = 1_000_000 * 100 / 123.03169  # perf-fa2bh.md:60-63, 1 thread, other host


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="graph_render_b200", choices=["graph_render_b200", "reference"])
    ap.add_argument("--workload", default="powerlaw-2d",
                    choices=["powerlaw-2d", "powerlaw-3d", "sbm1500", "ba100k"])
    ap.add_argument("--n", type=int, default=0, help="override the node count (profiling cases)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-ticks", type=int, default=100)
    ap.add_argument("--cpu-budget-s", type=float, default=20.0)
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-3d", action="store_true")
    ap.add_argument("--no-d3", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the other configs and the reference's benchmark")
    ap.add_argument("--walk-schedule", type=int, default=-1,
                    help="walk schedule for the main workload (default: the autotuner's choice)")
    ap.add_argument("--adjoint-ticks", type=int, default=200, help="ticks of the differentiated workload's run")
    ap.add_argument("--batched-graphs", type=int, default=4096, help="graphs per GPU")
    ap.add_argument("--batched-ticks", type=int, default=200)
    ap.add_argument("--batched-sample", type=int, default=48, help="graphs timed one launch sequence each")
    return ap.parse_args()


def walk_traffic_per_node():
    """DRAM bytes per node of one walk launch, from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "k_walk_traffic.txt")
    try:
        kv = dict(line.strip().split("=", 1) for line in open(path) if "=" in line and not line.startswith("#"))
        return float(kv["dram_read_bytes_per_node"]) + float(kv["dram_write_bytes_per_node"])
    except (OSError, KeyError, ValueError):
        return None


def measure_fp32_tflops(iters: int = 200_000):
    """This GPU's FP32 FMA rate (TFLOP/s, an FMA as two) from the engine's own
    FMA-chain kernel, timed with CUDA events; None if the call fails."""
    import ctypes as C

    from graph_render_b200 import _native as N

    v = C.c_double()
    try:
        N.check(N.lib().gr_measure_fp32_rate(iters, C.byref(v)))
    except N.EngineError:
        return None
    return v.value


def walk_hbm_view(n: int, n_cells: int, dim: int, walk_ms: float) -> dict:
    """The walk against the measured HBM copy bandwidth: its algorithmic bytes per
    launch (every cell record and sorted node read once, the per-node indices read,
    the repulsion written) over the walk phase's time."""
    cell_bytes = 32 if dim == 2 else 48
    algo = n_cells * cell_bytes + n * (16 + 12) + n * dim * 4
    peak = None
    try:
        peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        pass
    ach = algo / (walk_ms / 1e3) / 1e9
    return {"bytes_per_launch": algo, "achieved": ach, "peak": peak, "unit": "GB/s",
            "frac": (ach / peak) if peak else None,
            "note": "cells x record size + nodes x (16 B point + 12 B indices) + nodes x dim x 4 B written; "
                    "the walk is bound by instruction issue and load latency, not by this"}


def workload(name: str, n: int = 0):
    from graph_render_b200 import synth

    if name == "powerlaw-2d":
        return synth.powerlaw_1m(n=n or 1_000_000, dim=2)
    if name == "powerlaw-3d":
        return synth.powerlaw_1m(n=n or 1_000_000, dim=3)
    if name == "sbm1500":
        return synth.sbm_1500()
    if name == "ba100k":
        return synth.ba_100k(n=n or 100_000)
    raise ValueError(name)


# ----------------------------------------------------------------- clocks --

class ClockSampler:
    """nvidia-smi samples of this GPU's clocks and throttle reasons."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id: str):
        self.dev = device_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.dev, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, pw, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
                pw.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        loaded = [s for s in sm if s > 600] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ------------------------------------------------------------ distributed --

class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None

    def init(self, backend: str):
        import datetime

        import torch
        import torch.distributed as dist

        if self.world > 1:
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            if self.pg.get_backend() == "nccl":
                import torch

                self.pg.barrier(device_ids=[self.local])
            else:
                self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch

        dev = "cuda" if self.pg.get_backend() == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def done(self):
        if self.pg:
            self.pg.destroy_process_group()


# -------------------------------------------------------------- CPU arms --

def host_cpu() -> dict:
    """This host's CPU as lscpu names it, and the threads the CPU arms use."""
    info = {"threads_used": os.cpu_count() or 1}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        kv = {k.strip(): v.strip() for k, v in (ln.split(":", 1) for ln in out.splitlines() if ":" in ln)}
        for key, name in (("Model name", "model"), ("CPU(s)", "cpus"), ("Socket(s)", "sockets"),
                          ("Core(s) per socket", "cores_per_socket"), ("Thread(s) per core", "threads_per_core")):
            if key in kv:
                info[name] = kv[key]
    except (OSError, subprocess.SubprocessError):
        info["model"] = "lscpu unavailable"
    return info


def cpu_port_rate(wl, threads: int, budget_s: float, min_ticks: int = 1, max_ticks: int = 1000):
    """The oracle (FP64 restatement of graph-core's tick) on the host cores:
    (node-ticks/s, ticks timed, seconds)."""
    from oracle import oracle as O

    lo, hi, ws = O.simple_graph(wl.n, wl.src, wl.dst, wl.weight)
    p = wl.params
    st = O.State(wl.n, lo, hi, w=ws, pos0=wl.pos0.astype(np.float64), dim=p.get("dim", 2),
                 theta=p.get("theta", 0.8), lin_log=p.get("lin_log", 0),
                 strong_gravity=p.get("strong_gravity", 0), dissuade_hubs=p.get("dissuade_hubs", 0),
                 edge_weight_influence=p.get("edge_weight_influence", 0.0), seed=p.get("seed", 0),
                 threads=threads)
    t0 = time.perf_counter()
    ticks = 0
    while ticks < max_ticks:
        st.iterate()
        ticks += 1
        el = time.perf_counter() - t0
        if ticks >= min_ticks and el > budget_s * 0.5:
            break
    el = time.perf_counter() - t0
    return wl.n * ticks / el, ticks, el


def run_reference(args, dist: Dist):
    """--impl reference: the reference's algorithm (the oracle port, FP64, OpenMP
    walk) on this box's host cores, rank 0 only."""
    if dist.rank != 0:
        return
    from oracle import oracle as O
    from graph_render_b200 import synth

    O.build()
    synth.use_library(O.LIB_PATH)  # the same seeded graphs, drawn by the oracle's copy of the generators
    wl = workload(args.workload, args.n)
    threads = os.cpu_count() or 1

    lo, hi, ws = O.simple_graph(wl.n, wl.src, wl.dst, wl.weight)
    p = wl.params
    st = O.State(wl.n, lo, hi, w=ws, pos0=wl.pos0.astype(np.float64), dim=p.get("dim", 2),
                 theta=p.get("theta", 0.8), lin_log=p.get("lin_log", 0),
                 strong_gravity=p.get("strong_gravity", 0), dissuade_hubs=p.get("dissuade_hubs", 0),
                 edge_weight_influence=p.get("edge_weight_influence", 0.0), seed=p.get("seed", 0),
                 threads=threads)
    budget = 150.0
    warm = 0
    t0 = time.perf_counter()
    while warm < args.warmup and time.perf_counter() - t0 < budget * 0.2:
        st.iterate()
        warm += 1
    t0 = time.perf_counter()
    steps = 0
    while steps < args.steps:
        st.iterate()
        steps += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    v = wl.n * steps / el
    print(json.dumps({
        "impl": "reference", "metric": "FA2 node-ticks/s at 1M nodes", "value": v, "unit": "node-ticks/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": warm, "ms_per_step": 1e3 * el / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": wl.name, "n": wl.n, "m_raw": wl.m, "theta": p.get("theta"), "dim": p.get("dim")},
        "cpu_baseline": {"value": v, "unit": "node-ticks/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} full ticks of the {wl.name} workload after {warm} warm-up ticks",
                         "cpu": host_cpu()},
        "e2e": {"value": v, "unit": "node-ticks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "graph-core is Rust (no cargo here or on the GPU box); the reference arm is the FP64 C "
                "restatement of its FA2 tick (oracle/), OpenMP over per-node walks; vs_baseline is null: the "
                "published figure is for the reference's gate-model graph at theta 0.8, not this workload",
    }), flush=True)


# ---------------------------------------------------------- batched arm --

def run_batched(args, dist: Dist):
    """The mixed batch (SBM / BA / grid, n log-uniform in [50, 20000]), this rank's
    shard of graphs_per_gpu x world graphs, 200 ticks each in one persistent
    launch after autotuning; against the one-graph engine on a uniform sample of
    the same graphs, each run by itself (device-resident inputs both ways)."""
    import torch

    from graph_render_b200 import Fa2, batch

    total = args.batched_graphs * dist.world
    costs = [batch.graph_cost(4, i) for i in range(total)]
    mine = batch.shard(costs, dist.world)[dist.rank]
    graphs = [batch.mixed_graph(4, i, ticks=args.batched_ticks) for i in mine]
    nodes = int(sum(g.n for g in graphs))
    t0 = time.perf_counter()
    b = batch.Batch(graphs)
    create_s = time.perf_counter() - t0
    chosen, tune_ms = b.tune(2)
    warm = max(1, min(args.warmup, 3))
    b.run(warm)  # warm-up ticks, untimed
    dist.barrier()
    torch.cuda.synchronize()
    ms = b.run(args.batched_ticks)
    torch.cuda.synchronize()
    dist.barrier()
    st = b.stats()
    b.close()
    ms_max = dist.max(ms)
    rate = dist.world * len(graphs) / (ms_max / 1e3)
    # one-by-one: a uniform sample of this rank's graphs through the one-graph engine
    rng = np.random.default_rng(1234 + dist.rank)
    pick = sorted(rng.choice(len(graphs), size=min(args.batched_sample, len(graphs)), replace=False).tolist())
    one_s = 0.0
    for i in pick:
        g = graphs[i]
        with Fa2(g.n, g.src, g.dst, params=g.params, pos0=g.pos0) as e:
            e.tick(1)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            e.tick(args.batched_ticks)
            torch.cuda.synchronize()
            one_s += time.perf_counter() - t1
    one_rate = len(pick) / one_s if one_s > 0 else None
    one_rate = dist.max(-one_rate) * -1 if one_rate else None  # the slowest rank
    return {
        "metric": "batched graphs/s", "value": rate, "unit": "graphs/s",
        "graphs": dist.world * len(graphs), "nodes_per_gpu": nodes, "ticks": args.batched_ticks,
        "ms": ms_max, "cta_threads": chosen, "tune_ms": tune_ms, "create_s": create_s,
        "one_by_one": {"value": one_rate, "unit": "graphs/s", "sample": len(pick),
                       "how": "the one-graph engine (one captured tick graph) per graph, "
                              "inputs resident, timed over the same 200 ticks"},
        "speedup_vs_one_by_one": (rate / dist.world) / one_rate if one_rate else None,
        "converged_graphs": int((st["ticks"] < warm + args.batched_ticks).sum()),
        "device_errors": int((st["errors"] != 0).sum()),
        "scaling": "weak (graphs_per_gpu fixed, LPT shard of the global batch)",
    }


# ---------------------------------------------------------- adjoint arm --

def run_adjoint(args, dist: Dist):
    """The differentiated workload: SBM 50,000 nodes in 16 blocks, edge weights 1,
    200 ticks with positions checkpointed every 20, loss = sampled stress-1
    against hop distance over ~1M node pairs; gradients for start positions
    and edge weights through the adjoint ticks."""
    import torch

    from graph_render_b200 import Fa2, stress, synth

    wl = synth.sbm_50k()
    t0 = time.perf_counter()
    a, b, h = stress.sample_pairs(wl.n, wl.src, wl.dst, 1_000_000, 5)
    pairs_s = time.perf_counter() - t0
    with Fa2(wl.n, wl.src, wl.dst, wl.weight, params=wl.params, pos0=wl.pos0) as eng:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.adjoint_forward(args.adjoint_ticks, 20)
        torch.cuda.synchronize()
        fwd = time.perf_counter() - t0
        pT = eng.positions()
        L, g = stress.stress(pT, a, b, h)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gp, gw = eng.adjoint_backward(g)
        torch.cuda.synchronize()
        bwd = time.perf_counter() - t0
    return {"workload": "sbm50000-16blocks-2d", "ticks": args.adjoint_ticks, "checkpoint_every": 20,
            "pairs": int(len(a)), "stress": L, "forward_ms": 1e3 * fwd, "backward_ms": 1e3 * bwd,
            "backward_node_ticks_per_s": wl.n * args.adjoint_ticks / bwd, "pair_sampling_s": pairs_s,
            "grad_pos_norm": float(np.linalg.norm(gp)), "grad_w_norm": float(np.linalg.norm(gw)),
            "finite": bool(np.isfinite(gp).all() and np.isfinite(gw).all())}


def run_3d(args, dist: Dist):
    """The 1M-node configuration-model graph in 3D (octree), strong gravity, theta 1.2."""
    from graph_render_b200 import Fa2
    from graph_render_b200.fa2 import WALK_SCHEDULE_NAMES

    wl = workload("powerlaw-3d", 0)
    with Fa2(wl.n, wl.src, wl.dst, wl.weight, params=wl.params, pos0=wl.pos0) as eng:
        eng.set_interaction_counting(False)
        eng.tick(1)
        chosen, tuned = eng.tune(2)
        eng.tick(3)
        ms = eng.tick_timed(10, l2_flush_bytes=FLUSH_BYTES)
        inf = eng.info()
    t = float(ms[:, 3].sum())
    return {"workload": wl.name, "n": wl.n, "node_ticks_per_s": wl.n * len(ms) / (t / 1e3),
            "ms_per_tick": t / len(ms), "phase_ms": {"tree": float(ms[:, 0].mean()), "walk": float(ms[:, 1].mean()),
                                                    "finish": float(ms[:, 2].mean())},
            "n_cells": inf["n_cells"],
            "walk_schedule": {"chosen": WALK_SCHEDULE_NAMES[chosen],
                              "tuned_walk_ms": {WALK_SCHEDULE_NAMES[i]: v for i, v in tuned.items()}}}


def run_d3(args, dist: Dist):
    """The d3-force Barnes-Hut session (layout.force.barnes_hut.cuda) on the
    reference's benchmark model at 1M nodes (synthetic.rs, the graph of its
    `tick --n 1000000` bench): ms per tick after 3 warm-up ticks, then the whole
    frozen layout (112 ticks from the golden spiral) and its stress."""
    from graph_render_b200 import ForceSession, stress as S, synth

    n = 1_000_000
    src, dst, st = synth.gate(n)
    t0 = time.perf_counter()
    with ForceSession(n, src, dst, st) as s:
        create_s = time.perf_counter() - t0
        s.tick(3)
        T = 20
        tick_ms = s.tick_timed(T) / T  # CUDA events on the session's stream
        info = s.info()
    t0 = time.perf_counter()
    with ForceSession(n, src, dst, st) as s:
        t1 = time.perf_counter()
        s.tick(1)  # captures the tick graph
        t2 = time.perf_counter()
        s.tick(111)
        t3 = time.perf_counter()
        p = s.positions()
        t4 = time.perf_counter()
    frozen_s = t4 - t0
    frozen = {"create_s": t1 - t0, "first_tick_s": t2 - t1, "ticks_2_112_s": t3 - t2, "positions_s": t4 - t3}
    with ForceSession(n, src, dst, st) as s:  # the same session, many-body on the particle mesh
        s.use_mesh()
        s.tick(3)
        mesh_ms = s.tick_timed(T) / T
        s.tick(112 - 3 - T)
        pm = s.positions()
    mesh = {"ms_per_tick": mesh_ms, "kruskal_stress_after_112": S.kruskal_stress(pm[:, 0], pm[:, 1], src, dst, 16),
            "reference_published_ms_per_tick": {"8 workers": 107,
                                                "source": "docs/measurements/perf-bh-1m.md:98, other host"}}
    return {"workload": f"gate model, {n} nodes, {len(src)} raw edges (the reference's synthetic benchmark graph)",
            "particle_mesh": mesh,
            "ms_per_tick": tick_ms, "node_ticks_per_s": n / (tick_ms / 1e3), "graph_kernels": info["graph_kernels"],
            "create_s": create_s, "frozen_layout_s": frozen_s, "frozen_layout_parts": frozen,
            "kruskal_stress": S.kruskal_stress(p[:, 0], p[:, 1], src, dst, 16),
            "reference_published_ms_per_tick": {"1 worker": 1987.73, "16 workers": 664.12,
                                                "source": "docs/measurements/perf-bh-1m.md:36-43, other host"}}


# ------------------------------------------------------- the other configs --

REF_GATE_MS = {1_000: (1_541, 43.59, 0.4089), 5_000: (7_721, 263.41, 0.4205), 10_000: (15_474, 583.83, 0.4111),
               100_000: (154_978, 8_310.29, 0.4539), 1_000_000: (1_549_929, 123_031.69, 0.4486)}
REF_GATE_SOURCE = "docs/measurements/perf-fa2bh.md:54-60 (graph-cli bench, 100 iterations, 1 thread, other host)"


def one_shot(wl, ticks: int, calls: int) -> dict:
    """The public per-graph call from pinned host buffers: create from host
    edges, `ticks` ticks, positions back; wall clock, median of `calls`."""
    import torch

    from graph_render_b200 import Fa2

    dim = int(wl.params.get("dim", 2))
    src = torch.from_numpy(wl.src).pin_memory().numpy()
    dst = torch.from_numpy(wl.dst).pin_memory().numpy()
    pos0 = torch.from_numpy(np.ascontiguousarray(wl.pos0)).pin_memory().numpy()
    w = None if wl.weight is None else torch.from_numpy(wl.weight).pin_memory().numpy()
    out = torch.empty((wl.n, dim), dtype=torch.float32).pin_memory().numpy()
    prm = dict(wl.params, max_iter=ticks)
    times = []
    for _ in range(calls):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with Fa2(wl.n, src, dst, w, params=prm, pos0=pos0) as e:
            e.set_interaction_counting(False)
            ran = e.run()
            e.positions(out=out)
        times.append(time.perf_counter() - t0)
    el = float(np.median(times))
    return {"value": wl.n * ran / el, "unit": "node-ticks/s", "seconds": el, "ticks": ran,
            "h2d_bytes_per_call": wl.m * 8 + wl.n * dim * 4 + (0 if w is None else wl.m * 8),
            "d2h_bytes_per_call": wl.n * dim * 4, "of": f"median of {calls} calls"}


def device_run(wl, ticks: int) -> dict:
    """`ticks` ticks from the workload's start on a fresh handle (a warm-up
    handle ran first), each tick timed with CUDA events on the handle's stream,
    a 256 MiB buffer overwritten before each (outside the events)."""
    from graph_render_b200 import Fa2

    with Fa2(wl.n, wl.src, wl.dst, wl.weight, params=wl.params, pos0=wl.pos0) as e:
        e.set_interaction_counting(False)
        e.tick(3)
        e.tick_timed(2, l2_flush_bytes=FLUSH_BYTES)
    with Fa2(wl.n, wl.src, wl.dst, wl.weight, params=wl.params, pos0=wl.pos0) as e:
        e.set_interaction_counting(False)
        ms = e.tick_timed(ticks, l2_flush_bytes=FLUSH_BYTES)
        pos = e.positions()
    t = float(ms[:, 3].sum())
    return {"value": wl.n * len(ms) / (t / 1e3), "unit": "node-ticks/s", "ticks": int(len(ms)),
            "run_ms": t, "ms_per_tick": t / max(len(ms), 1),
            "phase_ms": {"tree": float(ms[:, 0].mean()), "walk": float(ms[:, 1].mean()),
                         "finish": float(ms[:, 2].mean())}}, pos


def run_config_legs(args, dist: Dist) -> dict:
    """The 1,500-node SBM for 100 ticks, the 100k-node BA graph (linlog,
    dissuade hubs, lognormal weights, theta 1.0) for 500 ticks and the 1M-node 3D
    octree graph (strong gravity, theta 1.2) for 300 ticks: device time of the
    whole run, the public call end to end, and the oracle on this host's cores on
    a bounded sample of the same run."""
    from graph_render_b200 import synth

    threads = os.cpu_count() or 1
    legs = {}
    for key, wl, ticks, calls in (("sbm1500_100_ticks", synth.sbm_1500(), 100, 5),
                                  ("ba100k_500_ticks", synth.ba_100k(), 500, 3),
                                  ("powerlaw1m_3d_300_ticks", synth.powerlaw_1m(n=1_000_000, dim=3), 300, 3)):
        dev, _ = device_run(wl, ticks)
        e2e = one_shot(wl, ticks, calls)
        v, t, el = cpu_port_rate(wl, threads, min(args.cpu_budget_s, 10.0), max_ticks=ticks)
        legs[key] = {"workload": wl.name, "n": wl.n, "m_raw": wl.m, "theta": wl.params.get("theta"),
                     "device": dev, "e2e": e2e,
                     "cpu_baseline": {"value": v, "unit": "node-ticks/s", "cores": threads, "kind": "port",
                                      "sample": f"the first {t} FP64 ticks of the same run, {el:.1f} s"}}
    return legs


def run_gate_legs(args, dist: Dist) -> dict:
    """The reference's own benchmark (graph-cli bench --layout
    layout.forceatlas2.barnes_hut): its gate-model graph at 1,000 .. 1,000,000
    nodes, the layout's defaults (theta 0.8, 100 iterations, Mulberry32(0)
    start), through the drop-in registry call (topology in, geometry out) with
    no positions given; wall clock of the call (median of 3), and the
    reference's Kruskal stress-1 of the result, beside its published time and
    stress for the same n."""
    import torch

    from graph_render_b200 import FA2_ID, Topology, find, stress as S, synth

    cap = find(FA2_ID)
    out = {}
    warm = synth.gate(1000)
    cap.run_params(Topology(1000, warm[0], warm[1], warm[2]), b"")
    for n, (m_ref, ms_ref, stress_ref) in REF_GATE_MS.items():
        src, dst, strength = synth.gate(n)
        topo = Topology(n, src, dst, strength)
        times = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            geom = cap.run_params(topo, b"")
            times.append(time.perf_counter() - t0)
        el = float(np.median(times))
        x, y = np.asarray(geom.x, np.float32), np.asarray(geom.y, np.float32)
        st = S.kruskal_stress(x, y, src, dst, 16)
        out[str(n)] = {"edges": int(len(src)), "ms": 1e3 * el, "node_ticks_per_s": n * 100 / el,
                       "kruskal_stress": st,
                       "reference": {"edges": m_ref, "ms": ms_ref, "kruskal_stress": stress_ref},
                       "speedup_vs_published": ms_ref / (1e3 * el)}
    # the oracle (the reference's algorithm, FP64, OpenMP walk) on this host's
    # cores, a bounded sample of the 1M-node run from the same start
    from oracle import oracle as O

    n = 1_000_000
    src, dst, strength = synth.gate(n)

    class Gate:
        pass

    g = Gate()
    g.n, g.src, g.dst, g.weight, g.m = n, src, dst, None, len(src)
    g.pos0 = O.initial_positions(n, 0, 2)
    g.params = dict(theta=0.8, dim=2, seed=0)
    threads = os.cpu_count() or 1
    v, t, el = cpu_port_rate(g, threads, min(args.cpu_budget_s, 12.0))
    out["cpu_baseline_1000000"] = {"value": v, "unit": "node-ticks/s", "cores": threads, "kind": "port",
                                   "sample": f"the first {t} FP64 ticks of the 1,000,000-node run, {el:.1f} s"}
    out["source"] = REF_GATE_SOURCE
    return out


# --------------------------------------------------------------- GPU arm --

def run_gpu(args, dist: Dist):
    import torch

    from graph_render_b200 import Fa2
    from graph_render_b200.fa2 import WALK_SCHEDULE_NAMES

    dev = dist.local if dist.world > 1 else 0
    torch.cuda.set_device(dev)
    wl = workload(args.workload, args.n)
    dim = int(wl.params.get("dim", 2))
    eng = Fa2(wl.n, wl.src, wl.dst, wl.weight, params=wl.params, pos0=wl.pos0)
    eng.set_interaction_counting(False)  # the walk without its diagnostic counters
    eng.tick(1)
    if args.walk_schedule >= 0:  # a fixed schedule (profiling), no autotuning
        schedule, schedule_ms = args.walk_schedule, {i: None for i in range(len(WALK_SCHEDULE_NAMES))}
        eng.set_walk_schedule(schedule)
    else:
        schedule, schedule_ms = eng.tune(3)  # walk schedule autotuner (state restored)
    eng.tick(max(args.warmup, 3))
    torch.cuda.synchronize()
    start_pos, start_ctl = eng.positions(), eng.controller()
    programmatic = eng.programmatic_launches()
    fp32_measured = measure_fp32_tflops()  # the walk roofline's denominator, at the clocks of the timed run
    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    sampler = ClockSampler(uuid if uuid.startswith("GPU-") else f"GPU-{uuid}")
    sampler.start()
    time.sleep(0.3)
    dist.barrier()
    torch.cuda.synchronize()
    ms = eng.tick_timed(args.steps, l2_flush_bytes=FLUSH_BYTES)
    torch.cuda.synchronize()
    dist.barrier()
    clocks = sampler.stop()
    end_pos = eng.positions()
    done = len(ms)
    total_ms = float(ms[:, 3].sum())
    max_ms = dist.max(total_ms)
    value = dist.world * wl.n * done / (max_ms / 1e3)
    walk_ms = float(ms[:, 1].mean())
    tree_ms = float(ms[:, 0].mean())
    fin_ms = float(ms[:, 2].mean())
    eng.close()
    # The timed ticks' interactions (the FLOP count): the same ticks from the same
    # state (positions and controller) on a second handle whose walk counts them.
    # Ticks are bit-reproducible, so its end positions equal the timed run's.
    with Fa2(wl.n, wl.src, wl.dst, wl.weight, params=wl.params, pos0=wl.pos0) as cnt:
        cnt.set_positions(start_pos)
        cnt.set_controller(**start_ctl)
        info0 = cnt.info()
        cnt.tick(done)
        info1 = cnt.info()
        replay_identical = bool(np.array_equal(cnt.positions(), end_pos))
    far = (info1["far_count"] - info0["far_count"]) / max(done, 1)
    pair = (info1["pair_count"] - info0["pair_count"]) / max(done, 1)
    flops = (far + pair) * FLOPS_PER_INTERACTION[dim]
    sm_max = clocks.get("sm_max_mhz") or 1965.0
    fp32_nominal = 148 * 128 * 2 * sm_max * 1e6
    fp32_peak = fp32_measured * 1e12 if fp32_measured else fp32_nominal
    achieved = flops / (walk_ms / 1e3)

    # e2e: the public one-shot path from pinned host buffers, create -> ticks -> positions
    e2e = None
    if not args.no_e2e:
        from graph_render_b200 import Fa2 as F

        src = torch.from_numpy(wl.src).pin_memory().numpy()
        dst = torch.from_numpy(wl.dst).pin_memory().numpy()
        pos0 = torch.from_numpy(np.ascontiguousarray(wl.pos0)).pin_memory().numpy()
        w = None if wl.weight is None else torch.from_numpy(wl.weight).pin_memory().numpy()
        out = torch.empty((wl.n, dim), dtype=torch.float32).pin_memory().numpy()
        T = args.e2e_ticks
        prm = dict(wl.params, max_iter=T)
        calls = []
        for _ in range(3):  # one call is ~50 ms of wall clock: the median of three
            dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            with F(wl.n, src, dst, w, params=prm, pos0=pos0) as e:
                e.set_interaction_counting(False)
                ran = e.run()
                e.positions(out=out)
            calls.append(dist.max(time.perf_counter() - t0))
        el = float(np.median(calls))
        h2d = wl.m * 8 + wl.n * dim * 4 + (0 if w is None else wl.m * 8)
        d2h = wl.n * dim * 4
        e2e = {"value": dist.world * wl.n * ran / el, "unit": "node-ticks/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "step": f"one layout call: create from host edges + {ran} ticks + positions back",
               "seconds": el, "calls_s": calls, "of": "median of 3 calls"}

    # the reference's quality measure of that layout (graph-cli bench.rs stress), on the device
    quality = None
    if e2e is not None and dist.rank == 0:
        from graph_render_b200 import stress as S

        t0 = time.perf_counter()
        s_end = S.kruskal_stress(out[:, 0], out[:, 1], wl.src, wl.dst, 16)
        t_s = time.perf_counter() - t0
        s_start = S.kruskal_stress(wl.pos0[:, 0], wl.pos0[:, 1], wl.src, wl.dst, 16)
        quality = {"kruskal_stress": s_end, "start_stress": s_start, "after_ticks": ran, "bfs_sources": 16,
                   "seconds": t_s, "how": "gr_stress: 16 evenly spaced BFS sources, every reachable target"}

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, ticks, el = cpu_port_rate(wl, threads, args.cpu_budget_s)
        cpu = {"value": v, "unit": "node-ticks/s", "cores": threads, "kind": "port",
               "sample": f"{ticks} full FP64 ticks of the same {wl.n}-node graph from the same start, "
                         f"{el:.1f} s (tree build serial, walks OpenMP)", "cpu": host_cpu()}

    batched = None
    if not args.no_batched:
        batched = run_batched(args, dist)
    adjoint = None
    if not args.no_adjoint and dist.rank == 0:
        adjoint = run_adjoint(args, dist)
    three_d = None
    if not args.no_3d and dist.rank == 0:
        three_d = run_3d(args, dist)
    d3 = None
    if not args.no_d3 and dist.rank == 0:
        d3 = run_d3(args, dist)
    legs = gate = None
    if not args.no_configs and dist.rank == 0:
        legs = run_config_legs(args, dist)
        gate = run_gate_legs(args, dist)
    # vs_baseline: the reference's published 1M-node run against the same
    # workload here (its gate model, theta 0.8, 100 iterations, its own start)
    vs = None
    if gate is not None:
        vs = gate["1000000"]["node_ticks_per_s"] / REF_1M_NODE_TICKS

    if dist.rank == 0:
        line = {
            "metric": "FA2 node-ticks/s at 1M nodes",
            "value": value,
            "unit": "node-ticks/s",
            "n_gpus": dist.world,
            "steps": done,
            "warmup": max(args.warmup, 3),
            "ms_per_step": max_ms / max(done, 1),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": vs,
            "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": wl.name, "n": wl.n, "m_raw": wl.m, "m_simple": int(info1["m"]),
                       "dim": dim, "theta": wl.params.get("theta"),
                       "l2": f"{FLUSH_BYTES >> 20} MiB buffer overwritten before every timed tick "
                             "(outside the events)",
                       "parallelism": f"{dist.world} independent replicas" if dist.world > 1 else "1 GPU",
                       "programmatic_launches": programmatic,
                       "phase_ms": {"tree": tree_ms, "walk": walk_ms, "finish": fin_ms},
                       "walk_schedule": {"chosen": WALK_SCHEDULE_NAMES[schedule],
                                         "tuned_walk_ms": {WALK_SCHEDULE_NAMES[i]: schedule_ms[i]
                                                           for i in range(len(WALK_SCHEDULE_NAMES))}}},
            "clocks": clocks,
            "e2e": e2e,
            "quality": quality,
            "gpu_launches": int(info1["graph_kernels"]) * done,
            "roofline": {"kernel": "k_walk_s", "bound": "fp32", "achieved": achieved / 1e12,
                         "peak": fp32_peak / 1e12, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                         "traffic": (walk_traffic_per_node() * wl.n if walk_traffic_per_node() and dim == 2
                                     else None),
                         "traffic_source": "ncu dram__bytes_read+write of k_walk_s at 2M nodes, scaled by nodes",
                         "peak_source": ("measured: gr_measure_fp32_rate, 8 independent FMA chains a thread, "
                                         "64 warps a SM, CUDA events, just before the timed ticks "
                                         "(MEASURED_PEAKS.json has no non-tensor FP32 figure)")
                                        if fp32_measured else "nominal FP32 FMA rate, 148 SM x 128 lanes x 2 x "
                                                              "sm_max_mhz",
                         "peak_nominal": fp32_nominal / 1e12,
                         "interactions_per_tick": {"far": far, "pair": pair},
                         "interactions_from": "the timed ticks replayed from their start state on a second handle "
                                              "whose walk counts them (the timed walk keeps no counters)",
                         "replay_identical": replay_identical,
                         "flops_per_interaction": FLOPS_PER_INTERACTION[dim],
                         "flops_convention": "operations per interaction, an FMA counted once (the peak counts it "
                                             "twice); with FMAs as 2 flops and the hi/lo centre subtractions, "
                                             "15 in 2D",
                         "hbm_view": walk_hbm_view(wl.n, int(info1["n_cells"]), dim, walk_ms)},
            "cpu_baseline": cpu,
            "batched": batched,
            "adjoint": adjoint,
            "powerlaw_1m_3d": three_d,
            "d3_force_1m": d3,
            "configs": legs,
            "reference_benchmark": gate,
            "vs_baseline_basis": "reference_benchmark['1000000'] (its gate-model graph at 1M nodes, theta 0.8, "
                                 "100 iterations from its Mulberry32 start, through the registry call) over the "
                                 "reference's published run of the same workload, 1 thread, other host "
                                 "(perf-fa2bh.md:60-63)",
        }
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    dist = Dist()
    if args.impl == "reference":
        run_reference(args, dist)  # rank 0 only; no collective involved
        return
    dist.init("nccl")
    try:
        run_gpu(args, dist)
    finally:
        dist.done()


if __name__ == "__main__":
    main()
