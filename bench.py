"""Benchmark of the flip2_b200 fluid step (one JSON line on rank 0).

Workload (default): the 256^3 dam-break at scale -- block x,y in [0,0.5],
z in [0,1] of the unit box, 8 jittered particles per fluid voxel (seed 0),
33,554,432 particles, FP32 state, FLIP 0.95, dt = 1/480, Jacobi-PCG to 1e-6
relative residual with FP64 reductions.  A step is one pass of the whole path:
bin (keys, radix sort, gather, segment heads), P2G, gravity + divergence,
pressure solve, projection, G2P + RK2 advection.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: the step does not shard (one box per GPU), so N ranks run N
independent replicas of the workload; the time is the maximum over ranks.
"""
import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CELLS = 256
BLOCK = (0.5, 0.5, 1.0)
DT = 1.0 / 480.0
METRIC = "particle-steps/s"
WORKLOAD = ("dam-break 256^3 voxels (cell 1/256), block 0.5x0.5x1, 8 jittered particles per fluid voxel (seed 0), "
            "FP32 state, FLIP 0.95, RK2, dt=1/480, Jacobi-PCG to 1e-6 relative residual (FP64 dots)")
# algorithmic bytes of one PCG iteration per active voxel, fused minimum:
# matvec+pAp 9 B, x/r/z update with r.z 28 B, direction update 12 B
PCG_BYTES_PER_VOXEL = 49.0
# one learned multilevel FCG iteration on the fine level: direction+matvec and
# update 49 B, V-cycle down (code, r in; t, coarse r out) 9.5 B and up (code,
# r, t in; z out) 12.5 B, plus q in 4 B for the FCG dot products the up
# kernel takes as it writes z; coarse levels not counted
MG_BYTES_PER_VOXEL = 75
CLOCK_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,timestamp")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="flip2_b200", choices=["flip2_b200", "reference"])
    ap.add_argument("--cells", type=int, default=N_CELLS, help="voxels per axis (default 256)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-c4", action="store_true", help="skip the learned-vs-plain pressure comparison")
    ap.add_argument("--no-c3", action="store_true", help="skip the 64M-particle binning microbenchmark")
    ap.add_argument("--no-c5", action="store_true", help="skip the 200-step learned-solve block")
    ap.add_argument("--config", default="c2", choices=["c2", "c5"],
                    help="c2: the 256^3 dam-break (default); c5: dam-break + sphere with the learned pressure solve")
    return ap.parse_args()


C5_SPHERE = (0.5, 0.75, 0.5, 0.15)  # centre-top sphere of radius 0.15 above the block


def scene(cells, config="c2"):
    from flip2_b200 import scenes
    return scenes.dam_break(cells, block=BLOCK, seed=0, sphere=C5_SPHERE if config == "c5" else None)


# ---------------------------------------------- learned vs plain pressure
C4_CELLS = 128
C4_PROBLEMS = 4
C4_SEED0 = 900_000


def c4_pressure(F, device):
    """128^3 pressure problems (solid spheres of radius 4..16 voxels to 10% of
    the box, fluid surface at 50-85% height, Gaussian impulses plus gravity),
    solved to 1e-6 by Jacobi-PCG and by the learned multilevel FCG
    (pressure_method 2: V-cycle whose 16^3 coarsest level the committed
    network solves), by the same V-cycle without the network and with a
    one-CTA Jacobi-PCG on the coarsest level instead of the network, and by
    FCG with the network on the solver's grid (pressure_method 1, committed
    weights, Jacobi-PCG restart after 100 iterations).  Device ms from CUDA
    events inside the engine; the relative residuals are FP64 true
    residuals."""
    data = os.path.join(ROOT, "flip2_b200", "data")
    if not (os.path.exists(os.path.join(data, "mg_weights.npy")) and os.path.exists(os.path.join(data, "lprec_weights.npy"))):
        return None
    R = C4_CELLS // 4
    engines = {}
    for name, kw, wfile in (("learned", {}, "mg_weights.npy"), ("no_network", {"mg_coarse": 1}, "mg_weights.npy"),
                            ("coarse_cg", {"mg_coarse": 2}, "mg_weights.npy"),
                            ("fine_grid_network", {}, "lprec_weights.npy")):
        P = F.Particles(1, mode=F.MODE_NATIVE, params=F.default_params(F.MODE_NATIVE, device=device, **kw))
        P.setDomain(0.0, 0.0, 0.0, R, R, R, 1.0)
        P.lp_set_weights(np.load(os.path.join(data, wfile)))
        engines[name] = P
    method = {"learned": 2, "no_network": 2, "coarse_cg": 2, "fine_grid_network": 1}
    for name, P in engines.items():  # warm-up: graphs and buffers
        # the same iteration caps as the timed solves: a solve's loop graph is
        # built for its cap, and a new cap would rebuild it inside a timed solve
        P.poisson_generate(seed=C4_SEED0)
        P.poisson_solve(0, 1e-6, 20000)
        P.poisson_solve(method[name], 1e-6, 100)
    rows = []
    for k in range(C4_PROBLEMS):
        row = {}
        for name, P in engines.items():
            P.poisson_generate(seed=C4_SEED0 + k)
            if name == "learned":
                a = P.poisson_solve(0, 1e-6, 20000)
                row.update({"plain_ms": a.ms, "plain_iters": a.iters, "plain_rel_residual": a.rel_residual})
            b = P.poisson_solve(method[name], 1e-6, 100)
            row.update({name + "_ms": b.ms, name + "_iters": b.iters, name + "_fell_back": b.fell_back,
                        name + "_restart_iters": b.plain_iters, name + "_rel_residual": b.rel_residual})
        rows.append(row)
    for P in engines.values():
        P.close()
    mean = lambda key: sum(r[key] for r in rows) / len(rows)
    return {"workload": "128^3 generated pressure problems (seeds %d..%d), tol 1e-6" % (C4_SEED0, C4_SEED0 + C4_PROBLEMS - 1),
            "learned": "pressure_method 2: FCG, V-cycle (damped Jacobi, 4 levels) with the network solving the 16^3 level",
            "plain_ms_mean": mean("plain_ms"), "learned_ms_mean": mean("learned_ms"),
            "no_network_ms_mean": mean("no_network_ms"), "coarse_cg_ms_mean": mean("coarse_cg_ms"),
            "fine_grid_network_ms_mean": mean("fine_grid_network_ms"),
            "plain_iters_mean": mean("plain_iters"), "learned_iters_mean": mean("learned_iters"),
            "no_network_iters_mean": mean("no_network_iters"), "coarse_cg_iters_mean": mean("coarse_cg_iters"),
            "speedup_learned_over_plain": mean("plain_ms") / mean("learned_ms"),
            "speedup_learned_over_no_network": mean("no_network_ms") / mean("learned_ms"),
            "fallback_rate": mean("learned_fell_back"), "problems": rows}


# ------------------------------------------------ C5: full step, learned solve
C5_STEPS = 200


def c5_learned(F, torch, dev, cells, steps=C5_STEPS, warmup=3):
    """The full step with the learned preconditioner at scale: the 256^3
    dam-break plus a sphere of fluid (radius 0.15 at (0.5, 0.75, 0.5)), 8
    particles per fluid voxel, FP32 state, dt 1/480, pressure by the learned
    multilevel FCG (the network solving the 16^3 level of a V-cycle) with the
    Jacobi-PCG restart, 200 steps, each one CUDA graph launch.  Device time
    from CUDA events around the 200 steps; iterations and restarts from the
    engine's device-side counters (read once, after the steps)."""
    pos, vel = scene(cells, "c5")
    n = pos.shape[0]
    stream = torch.cuda.Stream(device=dev)
    P = F.Particles(n, mode=F.MODE_NATIVE, params=F.default_params(F.MODE_NATIVE, device=dev.index, pressure_method=2),
                    stream=stream.cuda_stream)
    R = cells // 4
    P.setDomain(0.0, 0.0, 0.0, R, R, R, 4.0 / cells)
    P.lp_set_weights(np.load(os.path.join(ROOT, "flip2_b200", "data", "mg_weights.npy")))
    P.upload(pos, vel)
    del pos, vel
    for _ in range(warmup):
        P.step(DT)
    i0 = P.info()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        P.step(DT)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    i1 = P.info()
    P.close()
    solves = i1.solves - i0.solves
    return {"workload": "256^3 dam-break + fluid sphere r=0.15 at (0.5,0.75,0.5), %d particles, dt=1/480, learned "
                        "multilevel FCG to 1e-6 with Jacobi-PCG restart, %d steps, one CUDA graph launch per step"
                        % (n, steps),
            "particles": n, "steps": steps, "ms_per_step": ms / steps,
            "particle_steps_per_s": n * steps / (ms / 1e3),
            "pressure_iters_mean": (i1.pressure_iters_total - i0.pressure_iters_total) / max(1, solves),
            "fallback_rate": (i1.fallbacks - i0.fallbacks) / max(1, solves), "solves": solves,
            "last_rel_residual": i1.residual, "converged": i1.converged, "error_flags": i1.error_flags,
            "kernel_launches_per_step": (i1.launches - i0.launches) / steps,
            "graph_launched_steps": i1.graph_steps - i0.graph_steps}


# ----------------------------------------------------- C3 binning microbenchmark
C3_KEY_BITS = 28  # keys of a 512^3 domain of unit root cells are below 2^28


def c3_binning(F, torch, dev, reps=3):
    """The 64M-particle binning microbenchmark: positions in a 512^3 domain,
    50% uniform and 50% from 16 Gaussian blobs (sigma 8 cells, seed 1), FP64
    as the reference stores them.  Times the reference's own three methods
    through the engine in reference mode -- alignParticlesToGrid (cell keys),
    sortParticles (radix sort of the 28-bit keys with the index payload, then
    the gather of the positions) and generateVoxels (segment heads, y-row
    table, voxel activation, the scan of per-node counts, voxel compaction)
    -- each rep from the unsorted input, and checks every output against the
    SHA-256 of the reference engine's own output on the same input
    (tests/golden/ref_c3_hashes.json, which also holds the reference's B200
    times of the same methods)."""
    import hashlib
    from flip2_b200 import scenes
    h = json.load(open(os.path.join(ROOT, "tests", "golden", "ref_c3_hashes.json")))
    n = h["n"]
    pos = scenes.binning_mix(n, domain=512, seed=h["seed"]).astype(np.float64)
    host = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
    del pos
    stream = torch.cuda.Stream(device=dev)
    P = F.Particles(n, mode=F.MODE_REFERENCE, params=F.default_params(F.MODE_REFERENCE, device=dev.index),
                    stream=stream.cuda_stream)
    P.setDomain(0.0, 0.0, 0.0, 512, 512, 512, 1.0)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    times = {"align": [], "sort": [], "voxels": []}
    checks = None
    for r in range(reps + 1):
        P.upload(tuple(host), None)
        P.sync()
        ev[0].record(stream)
        P.alignParticlesToGrid()
        ev[1].record(stream)
        P.sortParticles()
        ev[2].record(stream)
        P.generateVoxels()
        ev[3].record(stream)
        torch.cuda.synchronize(dev)
        if r == 0:  # the first pass also sizes the voxel buffers; check its outputs
            sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
            info = P.info()
            checks = {"nodes": info.nodes == h["nodes"], "voxels": info.voxels == h["voxels"],
                      "keys": sha(P.read(F.BUF_KEYS)) == h["sha256_keys"],
                      "perm": sha(P.read(F.BUF_PERM)) == h["sha256_perm"],
                      "flags": sha(P.read(F.BUF_FLAGS)) == h["sha256_flags"],
                      "starts": sha(P.read(F.BUF_STARTS)) == h["sha256_starts"],
                      "node_voxels": sha(P.read(F.BUF_NODE_VOXELS)) == h["sha256_node_voxels"],
                      "voxel_ids": sha(P.read(F.BUF_VOXEL_IDS)) == h["sha256_voxel_ids"],
                      "solids": sha(P.read(F.BUF_SOLIDS)) == h["sha256_solids"]}
            continue
        times["align"].append(ev[0].elapsed_time(ev[1]))
        times["sort"].append(ev[1].elapsed_time(ev[2]))
        times["voxels"].append(ev[2].elapsed_time(ev[3]))
    P.close()
    ms = {k: statistics.median(v) for k, v in times.items()}
    ref_ms = {k: 1e3 * v for k, v in h["seconds"].items()}
    # algorithmic bytes: keys 24 B (FP64 x, y, z) + 4 B out; sort 4 B histogram +
    # 4 passes x 16 B (28-bit keys, 8-bit digits) + the gather of x, y, z by the
    # permutation (4 + 24 + 24 B)
    key_bytes, sort_bytes = 28.0 * n, (4 + 4 * 16 + 52) * n
    return {"workload": "64M particles (%d) in a 512^3 domain, 50%% uniform + 50%% in 16 Gaussian blobs (sigma 8, "
                        "seed %d), FP64 positions, 28-bit keys + index payload" % (n, h["seed"]),
            "ms": ms, "reference_b200_ms": ref_ms,
            "speedup_vs_reference_b200": {k: ref_ms[k] / ms[k] for k in ms},
            "keys_gbs": key_bytes / (ms["align"] / 1e3) / 1e9,
            "sort_gbs": sort_bytes / (ms["sort"] / 1e3) / 1e9,
            "sort_algorithmic_bytes": "120 B per key: histogram 4 + 4 onesweep passes x 16 + gather of x,y,z 52",
            "hash_check": checks, "bit_exact": bool(checks) and all(checks.values()), "reps": reps}


# ------------------------------------------------------------ CPU baseline
def cpu_sample(cells, max_particles):
    """Bounded sample of the same workload: the particles of the dam-break
    scene inside the corner sub-box [0, s]^2 x [0, 2s] (same density, same dt),
    run with the reference's algorithm restated on the host."""
    pos, vel = scene(cells)
    s = 0.5
    while True:
        m = (pos[:, 0] < s) & (pos[:, 1] < s) & (pos[:, 2] < 2 * s)
        if m.sum() <= max_particles or s < 1e-3:
            break
        s *= 0.5 ** (1.0 / 3.0)
    return pos[m].astype(np.float64), vel[m].astype(np.float64), s


# Host cost of one reference sub-step, measured on the GPU box's 16 cores:
# 262,084 particles took 22 s a step once the fluid moves (the first step from
# rest is about 40x cheaper, so samples warm up before they are timed).
REF_PARTICLES_PER_STEP_SECOND = 12_000


def ref_cpu_run(cells, steps, warm, budget_s):
    """Time `steps` sub-steps of the reference's algorithm restated on the host
    (oracle/flip_oracle.c orc_ref_substep: bin, tent P2G, Courant dt + red-black
    SOR pressure loop, projection, G2P, Euler advect; FP64, OpenMP on every
    host core) after `warm` untimed ones, on a corner sample of the workload
    sized so that the steps take about budget_s.  Returns (particles per
    second of a timed step, particles, seconds timed, sample description)."""
    from oracle import oracle as O
    target = int(max(5_000, min(400_000, budget_s / max(1, steps + warm) * REF_PARTICLES_PER_STEP_SECOND)))
    pos, vel, s = cpu_sample(cells, target)
    n = pos.shape[0]
    g = O.grid(0.0, 0.0, 0.0, cells // 4, cells // 4, cells // 4, 4.0 / cells)
    arrs = [pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1], vel[:, 2]]
    for _ in range(warm):
        arrs, _ = O.ref_substep(*arrs, g, frame_dt=DT, elapsed=0.0)
    t0 = time.perf_counter()
    for _ in range(steps):
        arrs, _ = O.ref_substep(*arrs, g, frame_dt=DT, elapsed=0.0)
    sec = time.perf_counter() - t0
    sample = ("reference algorithm restated on the host (oracle/flip_oracle.c orc_ref_substep, FP64, OpenMP, %d "
              "threads): %d particles of the workload inside [0,%.3f]^2x[0,%.3f], %d untimed then %d timed "
              "sub-steps" % (os.cpu_count(), n, s, 2 * s, warm, steps))
    return n * steps / sec, n, sec, sample


def testing_h_checks(cells):
    """The reference's CPU verification path (engine/testing.h:25-53:
    storeGridCellMap on the cell keys before the sort, validateGridCellOrdering
    on the sorted keys; std::map on one host thread, as the reference's),
    restated in the oracle and timed on the whole workload: the reference-mode
    cell keys of every particle (the reference grid of 4-voxel cells) and the
    same keys sorted."""
    from oracle import oracle as O
    pos, _ = scene(cells)
    g = O.grid(0.0, 0.0, 0.0, cells // 4, cells // 4, cells // 4, 4.0 / cells)
    keys, _, _, _ = O.ref_keys(pos[:, 0], pos[:, 1], pos[:, 2], g)
    del pos
    sorted_keys, _ = O.sort_pairs(keys)
    t0 = time.perf_counter()
    status, ncells = O.ref_grid_cell_checks(keys, sorted_keys)
    sec = time.perf_counter() - t0
    return {"what": "storeGridCellMap + validateGridCellOrdering (engine/testing.h:25-53) restated with std::map "
                    "(oracle/ref_checks.cpp), one host thread", "particles": int(keys.size), "cells": ncells,
            "seconds": sec, "particles_per_s": keys.size / sec, "passed": status == 0, "cores": 1}


def cpu_baseline(cells, budget_s=25.0):
    value, n, sec, sample = ref_cpu_run(cells, 3, 3, budget_s)
    return {"value": value, "unit": METRIC, "cores": os.cpu_count(), "kind": "port", "sample": sample,
            "seconds": sec, "testing_h_checks": testing_h_checks(cells)}


# ------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi sampling every 50 ms, started before the warm-up (the tool
    takes a moment to start) and filtered to the timed window's host times;
    a window shorter than the sampling interval reports the samples nearest
    to it and says so."""

    def __init__(self, gpu_index):
        self.p = None
        self.t0 = self.t1 = None
        self.path = os.path.join(tempfile.gettempdir(), "flip2_b200_bench_clocks_%d_%d.csv" % (gpu_index, os.getpid()))
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), "--query-gpu=" + CLOCK_QUERY,
                                       "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.p = None

    def begin(self):
        self.t0 = time.time()

    def end(self):
        self.t1 = time.time()

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.close()
        with open(self.path) as f:
            lines = f.read().splitlines()
        try:
            os.remove(self.path)
        except OSError:
            pass
        return self.summarize(lines, self.t0, self.t1)

    @staticmethod
    def summarize(lines, t0, t1):
        """Median SM clock, max clock, power and the active throttle reasons
        of the CLOCK_QUERY csv lines sampled inside [t0, t1] (host times;
        the two samples nearest the window's middle when none falls in it)."""
        rows = []
        for line in lines:
            c = [x.strip() for x in line.split(",")]
            if len(c) >= 9 and c[1].replace(".", "").isdigit():
                rows.append(c)
        if not rows:
            return None
        window = "timed region"
        if t0 is not None and t1 is not None:
            def ts(r):
                try:
                    return datetime.datetime.strptime(r[9], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                except (IndexError, ValueError):
                    return None
            stamped = [(ts(r), r) for r in rows if ts(r) is not None]
            inside = [r for t, r in stamped if t0 <= t <= t1]
            if inside:
                rows = inside
            elif stamped:
                mid = 0.5 * (t0 + t1)
                stamped.sort(key=lambda tr: abs(tr[0] - mid))
                rows = [r for _, r in stamped[:2]]
                window = "nearest samples (timed region shorter than the 50 ms sampling interval)"
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(float(r[2]) for r in rows),
                "reasons": reasons, "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows),
                "window": window}


# ------------------------------------------------------------ reference arm
def run_reference(args, rank):
    if rank != 0:
        return
    steps, warm = max(1, args.steps), max(0, args.warmup)
    # the whole --steps/--warmup run on the host stays within about 2.5 minutes
    value, n, sec, sample = ref_cpu_run(args.cells, steps, warm, 150.0)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": 1e3 * sec / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "particles_sampled": n},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": os.cpu_count(), "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------ replicas and ranks
class Ranks:
    """One process per GPU under torchrun: the replicas share nothing but a
    barrier around the timed region and the maximum of the ranks' times.
    backend "nccl" on GPUs, "gloo" for the host-only tests."""

    def __init__(self, backend="nccl", device=None, timeout_s=120):
        import datetime
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.device = device
        self.dist = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if backend == "nccl":
                kw["device_id"] = device
            dist.init_process_group(backend, **kw)
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max_over_ranks(self, x):
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


# ------------------------------------------------------------ own arm
def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch
    import flip2_b200 as F
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ranks = Ranks("nccl", dev)

    pos, vel = scene(args.cells, args.config)
    n = pos.shape[0]
    stream = torch.cuda.Stream(device=dev)
    c5 = args.config == "c5"
    params = F.default_params(F.MODE_NATIVE, device=local, pressure_method=2 if c5 else 0)
    P = F.Particles(n, mode=F.MODE_NATIVE, params=params, stream=stream.cuda_stream)
    R = args.cells // 4
    P.setDomain(0.0, 0.0, 0.0, R, R, R, 4.0 / args.cells)
    if c5:
        P.lp_set_weights(np.load(os.path.join(ROOT, "flip2_b200", "data", "mg_weights.npy")))
    # pinned host state for the end-to-end leg
    host = [torch.from_numpy(np.ascontiguousarray(pos[:, k])).pin_memory() for k in range(3)]
    host += [torch.from_numpy(np.ascontiguousarray(vel[:, k])).pin_memory() for k in range(3)]
    ptrs = [t.data_ptr() for t in host]
    P.upload_ptrs(ptrs)
    del pos, vel

    barrier, max_over_ranks = ranks.barrier, ranks.max_over_ranks

    vis = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    phys = int(vis[local]) if local < len(vis) and vis[local].strip().isdigit() else local
    clocks = Clocks(phys)  # sampling from here; kept for the timed window only
    for _ in range(max(3, args.warmup)):
        P.step(DT)
    P.sync()
    l0 = P.info().launches

    # ---- device-resident timed region
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize(dev)
    clocks.begin()
    fb0 = P.info().fallbacks
    ev0.record(stream)
    for _ in range(args.steps):
        P.step(DT)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    clocks.end()
    barrier()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    info = P.info()
    launches = info.launches - l0
    fell_back = info.fallbacks - fb0
    ms_max = max_over_ranks(ms)
    value = n * world * args.steps / (ms_max / 1e3)

    # ---- end to end through the C ABI with host buffers
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for _ in range(args.steps):
        # upload the state from pinned host memory, step, download the new
        # state; each call's download overlaps the next call's upload
        P.step_streamed(ptrs, DT)
    P.sync()  # orders the engine stream after the last download
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1))
    e2e = {"value": n * world * args.steps / (ms_e2e / 1e3), "unit": METRIC, "h2d_bytes_per_step": 24 * n,
           "d2h_bytes_per_step": 24 * n, "ms_per_step": ms_e2e / args.steps}

    # ---- per-stage breakdown (separate, synchronised steps)
    P.set_timing(True)
    P.stage_ms(reset=True)
    nprof = 3
    pcg_iters = 0
    iters = []
    for _ in range(nprof):
        P.step(DT)
        iters.append(P.info().pressure_iters)
        pcg_iters += iters[-1]
    stages = {k: v / nprof for k, v in P.stage_ms(reset=True).items()}
    P.set_timing(False)
    fluid_tiles = P.info().nodes
    voxels = fluid_tiles * 512
    t_iter_ms = stages["pcg_iterations"] / max(1.0, pcg_iters / nprof)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    per_voxel = MG_BYTES_PER_VOXEL if c5 else PCG_BYTES_PER_VOXEL
    achieved = per_voxel * voxels / (t_iter_ms / 1e3) / 1e9
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        traffic = tr.get("pcg_iteration_bytes_per_voxel")
        if traffic is not None:
            traffic = traffic * voxels
    except (OSError, ValueError):
        pass
    if c5:
        traffic = None  # the ncu traffic figure covers the Jacobi-PCG iteration only
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic,
                "kernel": ("learned multilevel FCG iteration (direction+matvec, update, V-cycle with the FCG dot fused)" if c5 else
                           "pcg iteration (matvec+pAp, x/r update with r.r and r.z, direction)"),
                "algorithmic_bytes": "%d B per active voxel per iteration x %d voxels" % (per_voxel, voxels),
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s"}

    # the particle-stage metric: binning, P2G and G2P/advection only
    part_keys = ["keys", "sort", "gather", "segment_heads", "grid_clear", "p2g", "g2p_advect"]
    part_ms = sum(stages[k] for k in part_keys)
    particle_stages = {"value": n / (part_ms / 1e3), "unit": METRIC, "ms_per_step": part_ms, "stages": part_keys,
                       "note": "stage times from CUDA events of the profiled steps; excludes pressure and projection"}
    # algorithmic bytes per stage (per particle p, per active voxel v of the
    # fluid tiles) and the bandwidth they make of the stage's CUDA-event time.
    # The segment heads have none: the sort's last pass finds them, and their
    # stage only compacts the per-tile table (one CTA, latency bound).
    it_step = pcg_iters / nprof
    stage_bytes = {
        "sort": 36.0 * n,                     # histogram 4 B + 2 onesweep passes x 16 B (tile keys)
        "gather": 52.0 * n,                   # permutation 4 B + 24 B read + 24 B write
        "p2g": 24.0 * n + 24.0 * voxels,      # state read; momentum and weight per face written
        "g2p_advect": 52.0 * n + 24.0 * voxels,  # state read, state + next key written; new and old faces read
        "pcg_iterations": per_voxel * voxels * it_step,
        "projection": 29.0 * voxels,
    }
    stages_gbs = {}
    for k, b in stage_bytes.items():
        if stages.get(k, 0.0) > 0.0:
            g = b / (stages[k] / 1e3) / 1e9
            stages_gbs[k] = {"ms": stages[k], "bytes": b, "gbs": g, "frac": g / peak}
    # the particle stages' headline figure: P2G + G2P/advect at their minimum,
    # 72 B per particle + 40 B per active voxel
    pg_ms = stages["p2g"] + stages["g2p_advect"]
    pg_bytes = 72.0 * n + 40.0 * voxels
    particle_stages["p2g_g2p"] = {"ms": pg_ms, "algorithmic_bytes": pg_bytes, "gbs": pg_bytes / (pg_ms / 1e3) / 1e9,
                                  "frac": pg_bytes / (pg_ms / 1e3) / 1e9 / peak,
                                  "particle_steps_per_s": n / (pg_ms / 1e3)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not c5:
        cpu = cpu_baseline(args.cells)
    c4 = None
    if rank == 0 and world == 1 and not args.no_c4 and not c5:
        c4 = c4_pressure(F, local)
    c3 = None
    if rank == 0 and world == 1 and not args.no_c3 and not c5:
        c3 = c3_binning(F, torch, dev)
    c5_block = None
    if rank == 0 and world == 1 and not args.no_c5 and not c5:
        c5_block = c5_learned(F, torch, dev, args.cells)
    if rank == 0:
        workload = WORKLOAD
        if c5:
            workload = WORKLOAD.replace("block 0.5x0.5x1", "block 0.5x0.5x1 + sphere r=0.15 at (0.5,0.75,0.5)").replace(
                "Jacobi-PCG to 1e-6", "learned multilevel FCG (V-cycle, network on the 16^3 level; 100-iteration cap, "
                "Jacobi-PCG restart) to 1e-6")
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": max(3, args.warmup), "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": workload, "particles": n, "grid": "%d^3" % args.cells, "dt": DT,
                           "parallelism": "replicas x%d" % world,
                           "l2": "inputs larger than L2: %.0f MB particle state per replica" % (24 * n / 1e6)},
                "particle_stages": particle_stages, "c4_pressure": c4, "c3_binning": c3, "c5_learned": c5_block,
                "e2e": e2e, "gpu_launches": launches, "clocks": clk, "roofline": roofline, "cpu_baseline": cpu,
                "pcg_iters_per_step": iters, "pressure_solve_ms": stages["pcg_setup"] + stages["pcg_iterations"],
                "stages_ms": stages, "stages_gbs": stages_gbs, "fluid_tiles": fluid_tiles,
                "pcg_rel_residual": info.residual, "error_flags": info.error_flags,
                "graph_steps": info.graph_steps}
        if c5:
            line["fallback_rate"] = fell_back / args.steps
        print(json.dumps(line), flush=True)
    P.close()
    ranks.close()


if __name__ == "__main__":
    main()
