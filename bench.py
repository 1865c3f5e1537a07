#!/usr/bin/env python3
"""Benchmark of the force-and-step path on B200.

Workload (one GPU): the Barnes-Hut warp walk on 1,000,000 particles (two
exponential disks, seeded), theta 0.5, eps 0.05, dt 0.005, 30-bit Morton
keys, tree rebuilt every step.  A step is one full leapfrog step: opening kick
+ drift + bounding box, Morton keys, onesweep radix sort, Karras build,
centres of mass, warp walk with the closing kick fused.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One JSON line on rank 0.  `value` = steps/s over the K timed steps, each
step run as the library runs it by default (one captured CUDA graph per
step); sum of per-step CUDA-event windows around the graph on the
simulation's stream, L2 flushed by a 256 MB write before every step, max over
ranks; N ranks run N independent replicas.  `phases_ms_per_step` comes from a
second run of K steps launched kernel by kernel with events between the
phases (`eager_steps_per_s`).  `e2e` = the same metric through the C ABI with the state
(pos, vel) uploaded from pinned host memory before and downloaded after every
step (nb_step_host_state; a(x) stays on the device).  `roofline` = the warp walk, useful work 20 flop x per-thread-
criterion interactions, against the FP32 FMA peak measured on this GPU by a
calibration kernel.  `cpu_baseline` = the CPU oracle port (C + OpenMP) of the
same step on this host's cores, on a sample of targets.

--impl reference times that CPU port alone as the reference arm.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = ("steps/s at 1M (BH θ=0.5); served particle-steps/s + p99 vs "
          "plain, equal error")
N_DEFAULT = 1_000_000
FLOP_PER_PAIR = 20          # src/main.cu:203-207 convention
# algorithmic HBM bytes per particle of the step before the walk: kick, drift
# and box 112 (r pos, lo, vel, acc; w pos, lo, vel), Morton keys 20 (r pos,
# w key), four sort passes 60 (the first reads no values), sorted-position
# gather 32, first build level 68 (r keys, sorted positions; w two 24-byte
# child-pair halves per particle)
BUILD_BYTES_PER_PARTICLE = 292
HBM_FALLBACK_GBS = 6650.0   # copy bandwidth measured on this pool's B200s (no peaks file)
L2_FLUSH_BYTES = 256 << 20


def bh_kernels_per_step(n, key_bits=30):
    """Kernels of one Barnes-Hut step: prep, Morton keys, the sort passes,
    the first build level (1024-leaf groups), one launch per later build
    level (15 segments per CTA with 30-bit keys, 10 with 63-bit; the
    geometry of nbodyssey_b200/csrc/k_lbvh.cu) and the walk."""
    passes = 4 if key_bits == 30 else 8
    fan = 15 if key_bits == 30 else 10
    groups = (n + 1023) // 1024
    levels = 0
    while groups > 1:
        groups = (groups + fan - 1) // fan
        levels += 1
    return 1 + 1 + passes + 1 + levels + 1


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--theta", type=float, default=0.5)
    ap.add_argument("--traverse", choices=["thread", "warp"], default="warp")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--cpu-sample", type=int, default=16384)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--force", choices=["bh", "naive"], default="bh",
                    help="naive: time the all-pairs module instead (e.g. --n 262144)")
    ap.add_argument("--walk", choices=["pair", "list", "dfs"], default="pair",
                    help="tree-walk kernel: batched list walk or depth-first walk")
    ap.add_argument("--workload", choices=["single", "ensemble", "serve"],
                    default="single",
                    help="ensemble: batched encounters vs the plain path one at a "
                         "time; serve: request stream through the server vs FIFO")
    ap.add_argument("--nsims", type=int, default=512)
    ap.add_argument("--ens-force", choices=["auto", "bh", "naive"], default="auto")
    ap.add_argument("--no-served", action="store_true",
                    help="skip the served / batched sub-measurements of the default line")
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--serve-nmax", type=int, default=262144)
    ap.add_argument("--serve-smax", type=int, default=500)
    ap.add_argument("--hbm-budget-gb", type=float, default=24.0)
    ap.add_argument("--fifo-sample", type=float, default=1.0,
                    help="serve: plain capacity from this fraction of the requests")
    ap.add_argument("--fifo-prefix", type=int, default=0,
                    help="serve: plain latency over the first K arrivals (0: all)")
    ap.add_argument("--shard", action="store_true",
                    help="one simulation split over the --gpus ranks (strong "
                         "scaling) instead of one independent simulation per rank")
    return ap.parse_args()


def workload(args):
    common = {"n": args.n, "dt": 0.005, "eps": 0.05,
              "l2": "flushed before every timed step (256 MB write)",
              "parallelism": "replicas (one independent simulation per GPU)"}
    if args.force == "naive":
        return dict(common, workload="all-pairs, N=%d, eps 0.05, dt 0.005" % args.n,
                    force="naive")
    return dict(common, workload="Barnes-Hut %s walk, N=%d, theta %.2g, eps 0.05, "
                                 "dt 0.005, 30-bit Morton keys, tree rebuilt every "
                                 "step" % (args.traverse, args.n, args.theta),
                theta=args.theta, traverse=args.traverse, key_bits=30, force="bh",
                walk_kernel=args.walk)


# --------------------------------------------------------------------------
# distributed plumbing
# --------------------------------------------------------------------------
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


def dist_max(pg, value):
    if pg is None:
        return value
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(pg):
    if pg is not None:
        pg.barrier()


# --------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self, append=False):
        if not append or self.path is None:
            fd, self.path = tempfile.mkstemp(prefix="nb_clocks_", suffix=".csv")
            os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits",
                 "-lms", "50", "-i", str(self.index)],
                stdout=open(self.path, "a"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        if not rows:
            return None
        def num(x):
            try:
                return float(x)
            except ValueError:
                return float("nan")
        sm = [num(r[1]) for r in rows]
        mx = max(num(r[2]) for r in rows)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for r in rows:
            for k, name in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "samples": len(rows), "reasons": sorted(reasons),
                "power_w_max": max(num(r[3]) for r in rows)}


# --------------------------------------------------------------------------
# CPU port (the oracle), used for cpu_baseline and the reference arm
# --------------------------------------------------------------------------
def cpu_step_sample(pos, vel, theta, traverse, sample, rng):
    """One leapfrog step of the CPU port on all particles (kick, drift, LBVH
    build) with the tree walk on `sample` random targets; returns the
    extrapolated seconds for the full step."""
    from oracle import oracle as O
    n = pos.shape[0]
    acc0 = np.zeros_like(pos)
    t0 = time.perf_counter()
    vh = O.kick(vel, acc0, 0.0025)
    p1, _ = O.drift(pos, None, vh, 0.005, True)
    tree = O.Tree(p1, 30)
    t1 = time.perf_counter()
    if traverse == "warp":
        nw = (n + 31) // 32
        w = np.sort(rng.choice(nw, max(1, sample // 32), replace=False))
        tree.walk_warp(theta, 0.05, 1.0, w)
        frac = nw / w.shape[0]
    else:
        tg = np.sort(rng.choice(n, sample, replace=False))
        tree.walk_thread(theta, 0.05, 1.0, tg)
        frac = n / sample
    t2 = time.perf_counter()
    return (t1 - t0) + (t2 - t1) * frac, (t1 - t0), (t2 - t1)


def cpu_baseline(args, steps=2):
    from nbodyssey_b200 import ic
    from oracle import oracle as O
    pos, vel = ic.bh_config(args.n, seed=0)
    rng = np.random.default_rng(0)
    times = []
    for _ in range(steps):
        t, tb, tw = cpu_step_sample(pos, vel, args.theta, args.traverse,
                                    args.cpu_sample, rng)
        times.append(t)
    best = min(times)
    return {"value": 1.0 / best, "unit": "steps/s", "cores": O.num_threads(),
            "kind": "port",
            "sample": ("CPU oracle (C, OpenMP): kick + compensated drift + full LBVH "
                       "build of all %d particles, %s walk of %d sampled targets, "
                       "walk time scaled by N/sample; best of %d steps" %
                       (args.n, args.traverse, args.cpu_sample, steps))}


def run_reference(args, rank, world):
    if rank != 0:
        return
    steps = max(1, min(args.steps, 3))
    cb = cpu_baseline(args, steps=steps)
    v = cb["value"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s",
            "n_gpus": world, "steps": steps, "warmup": 0,
            "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload(args), "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# B200 arm
# --------------------------------------------------------------------------
def pinned_array(lib, shape, keep):
    from nbodyssey_b200 import _lib as L
    nbytes = int(np.prod(shape)) * 4
    p = ctypes.c_void_p()
    L.check(lib.nb_alloc_pinned(nbytes, ctypes.byref(p)))
    keep.append(p)
    buf = (ctypes.c_float * int(np.prod(shape))).from_address(p.value)
    return np.ctypeslib.as_array(buf).reshape(shape)


def interactions(sim, api, params):
    """Sum over particles of the per-thread-criterion interaction count
    (all-pairs: n^2, the self term included as the reference counts it)."""
    from dataclasses import replace
    if params.force == "naive":
        return sim.n * sim.n
    sim.set_params(replace(params, traverse="thread"))
    _, cnt = sim.debug_forces()
    sim.set_params(params)
    return int(cnt.astype(np.int64).sum())


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(path))
    except (OSError, ValueError):
        return {}


def profiled_traffic(kernel, traverse="warp", theta=0.5):
    """Per-launch DRAM bytes of the timed force kernel from its committed ncu
    summary (profiles/<kernel>_1m.md, the same 1M workload at theta 0.5), if
    present."""
    if theta != 0.5:
        return None
    name = {("k_walk_pair", "warp"): "walk_pair_1m.md",
            ("k_walk_pair", "thread"): "walk_pair_thread_1m.md",
            ("k_walk_list", "warp"): "walk_list_1m.md",
            ("k_walk_list", "thread"): "walk_list_thread_1m.md",
            ("k_walk_warp", "warp"): "walk_warp_dfs_1m.md"}.get((kernel, traverse))
    if name is None:
        return None
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


def run_b200(args, rank, world, local, pg):
    from nbodyssey_b200 import _lib as L
    from nbodyssey_b200 import api, ic
    lib = L.load()
    L.check(lib.nb_set_device(local))
    params = api.SimParams(dt=0.005, epsilon=0.05, theta=args.theta,
                           force=args.force, traverse=args.traverse, key_bits=30,
                           compensated=True, walk_kernel=args.walk)
    pos, vel = ic.bh_config(args.n, seed=rank)
    sim = api.Simulation(pos, vel, params)
    n = args.n

    # FP32 peak of this GPU (calibration kernel), before the sim's work
    ps, pp = ctypes.c_double(), ctypes.c_double()
    L.check(lib.nb_measure_fp32_peak(ctypes.byref(ps), ctypes.byref(pp)))
    fp32_peak = max(ps.value, pp.value)

    inter0 = interactions(sim, api, params)

    # warm-up: the step as the library runs it by default, one captured
    # CUDA graph per step
    sim.step(args.warmup)
    sim.sync()
    clocks = Clocks(local)
    # the disks move, and the walk's cost with them: every measurement below
    # starts from this state (pos, vel, a(x); the low position parts restart
    # at zero)
    snap = (sim.positions(), sim.velocities(), sim.accelerations())

    def restore():
        sim.set_state_acc(*snap)
        sim.sync()

    # timed steps (the headline): L2 flushed before every step, each step's
    # graph bracketed by two CUDA events on the simulation's stream
    dist_barrier(pg)
    clocks.start()
    total_ms = 0.0
    for _ in range(args.steps):
        L.check(lib.nb_flush_l2(sim._h, L2_FLUSH_BYTES))
        sim.record(2)
        sim.step(1)
        sim.record(3)
        total_ms += sim.elapsed_ms(2, 3)
    clk = clocks.stop()
    dist_barrier(pg)
    total_ms = dist_max(pg, total_ms)

    # the same steps launched kernel by kernel with an event between phases,
    # for the per-phase split (informational: the launches and events add
    # time between the kernels)
    restore()
    sim.reset_timing()
    sim.set_timing(True)
    clocks.start(append=True)
    for _ in range(args.steps):
        L.check(lib.nb_flush_l2(sim._h, L2_FLUSH_BYTES))
        sim.step(1)
    sim.sync()
    clk = clocks.stop() or clk
    phases, calls = sim.phase_times()
    eager_ms, fcalls = sim.force_timing()
    sim.set_timing(False)
    assert calls == args.steps and fcalls == args.steps, (calls, fcalls)
    dist_barrier(pg)
    eager_ms = dist_max(pg, eager_ms)
    inter1 = interactions(sim, api, params)
    inter = 0.5 * (inter0 + inter1)

    # steady state through the captured graph, no flush (informational)
    restore()
    sim.step(1)
    sim.sync()
    restore()
    clocks.start(append=True)
    sim.record(0)
    sim.step(args.steps)
    sim.record(1)
    graph_ms = sim.elapsed_ms(0, 1)
    clk = clocks.stop() or clk

    # end to end: pinned host state (positions, velocities) in, one step,
    # state out, every step (nb_step_host_state: a(x) stays on the device
    # while each step's inputs are the previous step's outputs, which the
    # library checks on the device every call), from the same starting state
    restore()
    keep = []
    bufs = [[pinned_array(lib, (n, 4), keep) for _ in range(2)] for _ in range(2)]
    L.check(lib.nb_get_positions(sim._h, L.ptr(bufs[0][0])))
    L.check(lib.nb_get_velocities(sim._h, L.ptr(bufs[0][1])))
    cur = 0
    for it in range(args.e2e_steps + 2):
        if it == 2:
            dist_barrier(pg)
            t0 = time.perf_counter()
        i, o = bufs[cur], bufs[cur ^ 1]
        L.check(lib.nb_step_host_state(sim._h, L.ptr(i[0]), L.ptr(i[1]),
                                       L.ptr(o[0]), L.ptr(o[1])))
        cur ^= 1
    e2e_s = dist_max(pg, time.perf_counter() - t0)
    for p in keep:
        lib.nb_free_pinned(p)
    sim.close()

    if rank != 0:
        return
    steps_total = args.steps * world
    value = steps_total / (total_ms * 1e-3)
    walk_ms = phases["walk"] / calls
    achieved = FLOP_PER_PAIR * inter / (walk_ms * 1e-3) / 1e12
    build_ms = sum(phases[k] for k in ("prep", "morton", "sort", "build", "com")) / calls
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    hbm_src = "MEASURED_PEAKS.json hbm_gbs (of measured)"
    if not hbm:   # the copy bandwidth measured earlier on this pool's B200s
        hbm, hbm_src = HBM_FALLBACK_GBS, "6,650 GB/s copy bandwidth (of fallback)"
    kernel = ({"pair": "k_walk_pair", "list": "k_walk_list"}.get(
        args.walk, "k_walk_%s" % args.traverse) if args.force == "bh" else "k_allpairs")
    traffic = (profiled_traffic(kernel, args.traverse, args.theta)
               if args.n == N_DEFAULT and args.force == "bh" else None)
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded two exponential disks (R_d 1 cut at 5, "
                "sigma_z 0.1, 0.05 v_c dispersion, centres (-+10,-+2,0), "
                "bulk -+0.25, B tilted 30 deg)",
        "config": workload(args),
        "particle_steps_per_s": value * n,
        "graph_steps_per_s_no_flush": world * args.steps / (graph_ms * 1e-3),
        "eager_steps_per_s": steps_total / (eager_ms * 1e-3),
        "phases_ms_per_step": {k: v / calls for k, v in phases.items() if v > 0},
        "phases_path": "kernel-by-kernel launches with an event between phases",
        "interactions_per_particle": inter / n,
        # the step's kernels plus the L2-flush kernel before each step
        "gpu_launches": ((bh_kernels_per_step(n) if args.force == "bh" else 2) + 1)
                        * args.steps,
        "e2e": {"value": world * args.e2e_steps / e2e_s, "unit": "steps/s",
                "h2d_bytes_per_step": 32 * n, "d2h_bytes_per_step": 32 * n,
                "path": "nb_step_host_state: pinned host pos / vel in, a device check "
                        "that the positions are the last ones returned (a(x) carries "
                        "on), one step, pos / vel out (positions return on a second "
                        "stream during the tree build and walk), wall clock"},
        "roofline": {"kernel": kernel, "bound": "fp32",
                     "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp32_peak, "traffic": traffic,
                     "work": ("20 flop x per-thread-criterion interactions "
                              "(%.4g per step)" % inter if args.force == "bh" else
                              "20 flop x N^2 pairs (%.4g per step)" % inter),
                     "peak_source": "measured on this GPU: FP32 FMA calibration "
                                    "kernel (scalar %.1f, packed f32x2 %.1f TFLOP/s)" %
                                    (ps.value, pp.value)},
        "roofline_build": {"bound": "hbm", "achieved":
                           BUILD_BYTES_PER_PARTICLE * n / (build_ms * 1e-3) / 1e9,
                           "peak": hbm, "unit": "GB/s",
                           "frac": (BUILD_BYTES_PER_PARTICLE * n / (build_ms * 1e-3) / 1e9
                                    / hbm),
                           "work": "292 B/particle (kick, drift and box 112, keys 20, "
                                   "4 sort passes 60, gather 32, child-pair records 68)",
                           "peak_source": hbm_src},
        "clocks": clk,
    }
    if args.force == "naive":
        line.pop("roofline_build")
        line.pop("interactions_per_particle")
    if world == 1 and not args.no_cpu_baseline and args.force == "bh":
        line["cpu_baseline"] = cpu_baseline(args)
    if world == 1 and not args.no_served and args.force == "bh":
        line["served"] = served_summary(args)
    print(json.dumps(line), flush=True)


def served_summary(args):
    """The second half of the headline metric at a size that fits beside the
    1M line: a 48-request served stream and a 128-encounter batched ensemble,
    each against the same work run one at a time through the plain drop-in
    path with the same parameters (force auto in both arms)."""
    srv = serve_measure(48, 131072, 300, 24.0, args.traverse, args.walk, seed=7, smin=50)
    ens = ensemble_measure(128, 100, 3, 0.5, args.traverse, args.walk, seed=3)
    return {"metric": "served particle-steps/s + p99 vs plain, equal accuracy",
            "value": srv["value"], "unit": "particle-steps/s",
            "config": {"workload": srv["workload"]},
            "plain_fifo_particle_steps_per_s": srv["plain_fifo_particle_steps_per_s"],
            "ratio_vs_plain": srv["ratio_vs_plain"],
            "latency_s": srv["latency_s"], "accuracy": srv["accuracy"],
            "ensemble": {"workload": "128 encounters, N log-uniform [2048, 131072], "
                                     "100 steps, force auto (all-pairs: %d batched below "
                                     "%d, %d plain below %d), theta 0.5" %
                                     (ens["allpairs_sims"]["batched"],
                                      ens["crossover"]["batch"],
                                      ens["allpairs_sims"]["plain"],
                                      ens["crossover"]["alone"]),
                         "same_module_batched": ens["same_module_batched"],
                         "value": ens["value"], "unit": "particle-steps/s",
                         "plain_fifo_particle_steps_per_s":
                             ens["plain_fifo_particle_steps_per_s"],
                         "ratio_vs_plain_device": ens["ratio_vs_plain_device"],
                         "wall_s": ens["wall_s"]}}


def run_shard(args, rank, world, local, pg):
    """One Barnes-Hut simulation split over the ranks (nbodyssey_b200/shard.py):
    every rank builds the whole tree, walks its Morton range of targets, and
    one NCCL all-gather of sorted accelerations completes each step.  Steps
    timed with CUDA events on the current stream, max over ranks; L2 flushed
    (256 MB write) before every timed step."""
    import torch
    from nbodyssey_b200 import _lib as L
    from nbodyssey_b200 import api, ic
    from nbodyssey_b200.shard import ShardedSimulation
    lib = L.load()
    L.check(lib.nb_set_device(local))
    torch.cuda.set_device(local)
    params = api.SimParams(dt=0.005, epsilon=0.05, theta=args.theta, force="bh",
                           traverse=args.traverse, key_bits=30, compensated=True,
                           walk_kernel=args.walk)
    n = args.n
    pos, vel = ic.bh_config(n, seed=0)   # the same simulation on every rank
    with api.Simulation(pos, vel, params) as one:
        inter = interactions(one, api, params)
    sim = ShardedSimulation(pos, vel, params)
    sim.step(args.warmup)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    torch.cuda.synchronize()
    clocks = Clocks(local)
    dist_barrier(pg)
    clocks.start()
    for e0, e1 in evs:
        flush.zero_()
        e0.record()
        sim.step(1)
        e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = dist_max(pg, sum(e0.elapsed_time(e1) for e0, e1 in evs))

    # end to end: this rank's whole state in from pinned host memory, one
    # step, state out
    eng = sim.engine
    hp = torch.empty((n, 4), dtype=torch.float32).pin_memory()
    hv, ha = torch.empty_like(hp).pin_memory(), torch.empty_like(hp).pin_memory()
    hp.copy_(eng.pos); hv.copy_(eng.vel); ha.copy_(eng.acc)
    for it in range(args.e2e_steps + 2):
        if it == 2:
            torch.cuda.synchronize()
            dist_barrier(pg)
            t0 = time.perf_counter()
        eng.pos.copy_(hp, non_blocking=True)
        eng.vel.copy_(hv, non_blocking=True)
        eng.acc.copy_(ha, non_blocking=True)
        sim.step(1)
        hp.copy_(eng.pos, non_blocking=True)
        hv.copy_(eng.vel, non_blocking=True)
        ha.copy_(eng.acc, non_blocking=True)
        torch.cuda.synchronize()
    e2e_s = dist_max(pg, time.perf_counter() - t0)
    sim.close()
    if rank != 0:
        return
    value = args.steps / (total_ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded two exponential disks (as the default run)",
        "config": dict(workload(args),
                       parallelism="one simulation split over %d GPUs: tree built "
                                   "on every GPU, walk split by Morton range, NCCL "
                                   "all-gather of sorted accelerations" % world),
        "particle_steps_per_s": value * n,
        "interactions_per_particle": inter / n,
        # per step: the step's kernels on each rank plus the gather kernel
        # (the flush and the all-gather are torch / NCCL kernels)
        "gpu_launches": world * (bh_kernels_per_step(n) + 1) * args.steps,
        "e2e": {"value": args.e2e_steps / e2e_s, "unit": "steps/s",
                "h2d_bytes_per_step": 48 * n * world, "d2h_bytes_per_step": 48 * n * world,
                "path": "each rank: pinned host state in, ShardedSimulation.step, "
                        "state out, wall clock"},
        "roofline": {"kernel": "whole step (split walk)", "bound": "fp32",
                     "achieved": FLOP_PER_PAIR * inter / (total_ms / args.steps * 1e-3) / 1e12,
                     "peak": None, "unit": "TFLOP/s", "frac": None, "traffic": None,
                     "work": "20 flop x per-thread-criterion interactions (%.4g per "
                             "step) over the whole step; the walk alone is in the "
                             "default (unsplit) line" % inter},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def ensemble_measure(nsims, steps, warmup, theta, traverse, walk, seed=0,
                     rank=0, world=1, pg=None, force="auto"):
    """Batched encounters against the same simulations one at a time through
    the plain handle path (create, steps, download, destroy), both with the
    same parameters (force "auto": all-pairs or Barnes-Hut per simulation by
    the tuned crossover, so both arms have the same method and accuracy per
    simulation).  Ranks shard the simulations with no collective."""
    from nbodyssey_b200 import api, ic
    from nbodyssey_b200.ensemble import Ensemble, shard
    specs = ic.ensemble_specs(nsims, seed=seed)
    mine = shard([s["n"] for s in specs], rank, world)
    states = [ic.from_spec(specs[i]) for i in mine]
    prm = api.SimParams(dt=0.005, epsilon=0.05, theta=theta, force=force,
                        traverse=traverse, walk_kernel=walk)
    parts = sum(p.shape[0] for p, _ in states)
    K, W = steps, warmup

    # batched: device time of K steps (graph), and wall time end to end
    dist_barrier(pg)
    t0 = time.perf_counter()
    ens = Ensemble(states, prm)
    ens.step(W)
    ens.sync()
    ens.record(0)
    ens.step(K)
    ens.record(1)
    dev_ms = ens.elapsed_ms(0, 1)
    for s in range(ens.nsims):
        ens.state(s)
    batch_forces = [ens.force(s) for s in range(ens.nsims)]
    kernels = ens.kernels_per_step()
    ens.close()
    wall_b = time.perf_counter() - t0
    dev_ms = dist_max(pg, dev_ms)
    wall_b = dist_max(pg, wall_b)

    # batched with the module each simulation gets alone (the plain path's
    # AUTO choice): the same arithmetic as the plain arm, bit for bit
    from dataclasses import replace
    tune = api.tune_get()
    x = tune["crossover"][1][1 if traverse == "warp" else 0]
    alone = [("naive" if force == "naive" or (force == "auto" and p.shape[0] < x) else "bh")
             for p, _ in states]
    ens = Ensemble(states, [replace(prm, force=f) for f in alone])
    ens.step(W)
    ens.sync()
    ens.record(0)
    ens.step(K)
    ens.record(1)
    same_ms = dist_max(pg, ens.elapsed_ms(0, 1))
    ens.close()

    # plain path, first in first out
    dist_barrier(pg)
    t0 = time.perf_counter()
    plain_ms = 0.0
    n_allpairs = 0
    for pos, vel in states:
        sim = api.Simulation(pos, vel, prm)
        sim.step(W)
        sim.sync()
        sim.record(0)
        sim.step(K)
        sim.record(1)
        plain_ms += sim.elapsed_ms(0, 1)
        sim.positions()
        sim.velocities()
        sim.close()
    wall_p = time.perf_counter() - t0
    plain_ms = dist_max(pg, plain_ms)
    wall_p = dist_max(pg, wall_p)
    total_parts = sum(sp["n"] for sp in specs)   # all ranks' shares together
    assert world > 1 or parts == total_parts
    value = total_parts * K / (dev_ms * 1e-3)
    plain = total_parts * K / (plain_ms * 1e-3)
    same = total_parts * K / (same_ms * 1e-3)
    return {"value": value, "unit": "particle-steps/s", "steps": K, "warmup": W,
            "ms_per_step": dev_ms / K, "particles": total_parts, "nsims": nsims,
            "plain_fifo_particle_steps_per_s": plain,
            "ratio_vs_plain_device": value / plain,
            "wall_s": {"batched": wall_b, "plain_fifo": wall_p,
                       "ratio": wall_p / wall_b},
            "force": force, "kernels_per_step": kernels,
            "allpairs_sims": {"batched": batch_forces.count("naive"),
                              "plain": alone.count("naive")},
            "crossover": {"alone": x,
                          "batch": tune["crossover_batch"][[0.3, 0.5, 0.7].index(
                              min((0.3, 0.5, 0.7), key=lambda c: abs(c - theta)))]},
            "same_module_batched": {
                "value": same, "ratio_vs_plain_device": same / plain,
                "note": "each simulation with the module it gets alone (results "
                        "bit-identical to the plain arm)"}}


def run_ensemble(args, rank, world, local, pg):
    """The batched ensemble workload alone (--workload ensemble)."""
    from nbodyssey_b200 import _lib as L
    lib = L.load()
    L.check(lib.nb_set_device(local))
    r = ensemble_measure(args.nsims, args.steps, args.warmup, args.theta, args.traverse,
                         args.walk, rank=rank, world=world, pg=pg, force=args.ens_force)
    if rank != 0:
        return
    line = {"metric": "particle-steps/s, batched ensemble of %d encounters" % args.nsims,
            "value": r["value"], "unit": "particle-steps/s", "n_gpus": world,
            "steps": r["steps"], "warmup": r["warmup"], "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic: seeded encounter recipe",
            "config": {"workload": "ensemble of %d %s theta %.2g %s encounters, N "
                                   "log-uniform [2048, 131072]" % (args.nsims, args.ens_force,
                                                                  args.theta, args.traverse),
                       "particles": r["particles"], "l2": "inputs larger than L2"},
            "plain_fifo_particle_steps_per_s": r["plain_fifo_particle_steps_per_s"],
            "ratio_vs_plain_device": r["ratio_vs_plain_device"],
            "wall_s": r["wall_s"], "allpairs_sims": r["allpairs_sims"],
            "crossover": r["crossover"], "same_module_batched": r["same_module_batched"],
            "accuracy": "batched AUTO takes Barnes-Hut theta %.2g (median force error "
                        "<= 1%% vs FP64) above the batch crossover where the plain "
                        "path takes all-pairs below its own crossover; "
                        "same_module_batched compares the same arithmetic" % args.theta,
            "gpu_launches": r["kernels_per_step"] * r["steps"]}
    print(json.dumps(line), flush=True)


def serve_requests(requests, nmax, smax, traverse, walk, rng, smin=100):
    """The request stream: N log-uniform in [4096, nmax], steps U[smin, smax],
    theta from {0.3, 0.5, 0.7}, encounter geometry as the ensemble recipe, a
    frame every 50 steps; force "auto" (all-pairs or Barnes-Hut per request
    by the tuned crossover, the same for the served and the plain arm)."""
    from nbodyssey_b200 import api, ic
    import math
    reqs = []
    for k in range(requests):
        n = int(round(math.exp(rng.uniform(math.log(4096), math.log(nmax)))))
        spec = dict(n=n, mass_ratio=float(rng.uniform(0.25, 1.0)),
                    impact=float(rng.uniform(2.0, 8.0)),
                    inclination_deg=float(rng.uniform(0.0, 90.0)),
                    approach=float(rng.uniform(0.3, 0.7)),
                    seed=int(rng.integers(0, 2 ** 31 - 1)))
        pos, vel = ic.from_spec(spec)
        prm = api.SimParams(dt=0.005, epsilon=0.05, force="auto",
                            theta=float(rng.choice([0.3, 0.5, 0.7])),
                            traverse=traverse, walk_kernel=walk)
        steps = int(rng.integers(smin, smax + 1))
        reqs.append((pos, vel, prm, steps))
    return reqs


def _pcts(lat):
    lat = np.asarray(lat)
    return {"p50": float(np.percentile(lat, 50)), "p95": float(np.percentile(lat, 95)),
            "p99": float(np.percentile(lat, 99))}


def serve_measure(requests, nmax, smax, budget_gb, traverse, walk, seed, smin=100,
                  fifo_sample=1.0, fifo_prefix=0):
    """Served request stream vs FIFO one at a time through the plain path.
    (1) capacity: every request submitted at t=0, particle-steps/s;
    (2) latency: Poisson arrivals at 80 % of the plain path's capacity, the
    same arrival times for both, p50/p95/p99 completion latency."""
    from nbodyssey_b200 import api
    from nbodyssey_b200.server import Server
    rng = np.random.default_rng(seed)
    reqs = serve_requests(requests, nmax, smax, traverse, walk, rng, smin=smin)
    work = float(sum(p.shape[0] * s for p, _, _, s in reqs))
    budget = int(budget_gb * (1 << 30))

    def plain_one(pos, vel, prm, steps):
        with api.Simulation(pos, vel, prm) as sim:
            done = 0
            while done < steps:   # frames every 50 steps, as the server's
                k = min(50 - done % 50, steps - done)
                sim.step(k)
                done += k
                sim.positions()
            sim.velocities()

    def serve_all(arrivals):
        lat = []
        with Server(hbm_budget_bytes=budget, max_sims=1023) as srv:
            t0 = time.perf_counter()
            ids = []
            for (pos, vel, prm, steps), ta in zip(reqs, arrivals):
                d = t0 + ta - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                ids.append((srv.submit(pos, vel, prm, steps, dump_every=50),
                            time.perf_counter()))
            for rid, ts in ids:
                srv.wait(rid, 3600)
                st, t_sub, t_adm, t_done = srv.poll(rid)
                lat.append(t_done - t_sub)
                srv.result(rid)
            wall = time.perf_counter() - t0
            stats = srv.stats()
        return wall, lat, stats

    def fifo_all(arrivals, which=None):
        which = range(len(reqs)) if which is None else which
        lat = []
        t0 = time.perf_counter()
        for k in which:
            pos, vel, prm, steps = reqs[k]
            d = t0 + arrivals[k] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            plain_one(pos, vel, prm, steps)
            lat.append(time.perf_counter() - (t0 + arrivals[k]))
        return time.perf_counter() - t0, lat

    plain_one(*reqs[0])                      # warm-up (pages in the library)
    zero = [0.0] * len(reqs)
    wall_s, _, st = serve_all(zero)
    cap_s = work / wall_s
    # plain capacity: every request, or a uniform random sample of them
    if fifo_sample < 1.0:
        srng = np.random.default_rng(seed + 1)
        sample = sorted(srng.choice(len(reqs), max(1, int(round(fifo_sample * len(reqs)))),
                                    replace=False).tolist())
        wall_f, _ = fifo_all(zero, sample)
        cap_f = sum(reqs[k][0].shape[0] * reqs[k][3] for k in sample) / wall_f
    else:
        wall_f, _ = fifo_all(zero)
        cap_f = work / wall_f
    lam = 0.8 * cap_f / (work / len(reqs))   # requests per second
    arrivals = np.cumsum(rng.exponential(1.0 / lam, size=len(reqs))).tolist()
    _, lat_s, st2 = serve_all(arrivals)
    # plain latency: FIFO over every arrival, or over the first fifo_prefix
    # arrivals (a FIFO request's latency depends only on the ones before it,
    # so the prefix's latencies are exact), against the served latencies of
    # the same requests
    prefix = len(reqs) if fifo_prefix <= 0 else min(fifo_prefix, len(reqs))
    _, lat_f = fifo_all(arrivals, range(prefix))
    lat_s_cmp = lat_s[:prefix]
    tune = api.tune_get()
    # all-pairs requests: served below the batch crossover, plain below the
    # crossover alone (the same theta class)
    def cls(prm):
        return [0.3, 0.5, 0.7].index(round(prm.theta, 1))
    n_ap = sum(1 for p, _, prm, _ in reqs if p.shape[0] < tune["crossover_batch"][cls(prm)])
    n_ap_plain = sum(1 for p, _, prm, _ in reqs
                     if p.shape[0] < tune["crossover"][cls(prm)][1 if traverse == "warp" else 0])
    return {"value": cap_s, "unit": "particle-steps/s",
            "workload": "%d requests, N log-uniform [4096, %d], steps U[%d, %d], theta "
                        "{0.3,0.5,0.7}, force auto (all-pairs: %d served, %d plain), "
                        "frame every 50 steps, HBM budget %.0f GB" %
                        (requests, nmax, smin, smax, n_ap, n_ap_plain, budget_gb),
            "particle_steps": work,
            "plain_fifo_particle_steps_per_s": cap_f,
            "ratio_vs_plain": cap_s / cap_f,
            "latency_s": {"served": _pcts(lat_s_cmp), "plain_fifo": _pcts(lat_f),
                          "served_all_requests": _pcts(lat_s),
                          "compared_requests": prefix,
                          "arrival_rate_per_s": lam,
                          "load": "80 % of the plain path's capacity"},
            "plain_capacity_from": ("all requests" if fifo_sample >= 1.0 else
                                    "a uniform random %.0f %% sample of the requests"
                                    % (100 * fifo_sample)),
            "server": {"peak_running": st["peak_running"],
                       "engine_steps": st["engine_steps"], "frames": st["frames"],
                       "frame_bytes": st["frame_bytes"]},
            "accuracy": "each request's result is bit-identical served and alone "
                        "with the same module (tests/test_gpu_server.py); AUTO takes "
                        "Barnes-Hut (median force error <= 1% vs FP64) from the batch "
                        "crossover served, from its own crossover plain"}


def run_serve(args, rank, world, local, pg):
    """The served request stream alone (--workload serve)."""
    from nbodyssey_b200 import _lib as L
    lib = L.load()
    L.check(lib.nb_set_device(local))
    r = serve_measure(args.requests, args.serve_nmax, args.serve_smax, args.hbm_budget_gb,
                      args.traverse, args.walk, seed=1000 + rank,
                      fifo_sample=args.fifo_sample, fifo_prefix=args.fifo_prefix)
    if rank != 0:
        return
    line = {"metric": "served particle-steps/s + p99 vs plain (request stream)",
            "value": r["value"], "unit": "particle-steps/s", "n_gpus": world,
            "steps": None, "warmup": 1, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic request stream",
            "config": {"workload": r["workload"], "particle_steps": r["particle_steps"]}}
    line.update({k: r[k] for k in ("plain_fifo_particle_steps_per_s", "ratio_vs_plain",
                                    "latency_s", "server", "accuracy",
                                    "plain_capacity_from")})
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    rank, world, local, pg = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.workload == "ensemble":
            run_ensemble(args, rank, world, local, pg)
        elif args.workload == "serve":
            run_serve(args, rank, world, local, pg)
        elif args.shard:
            run_shard(args, rank, world, local, pg)
        else:
            run_b200(args, rank, world, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
