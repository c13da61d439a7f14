"""Run a few native steps of the dam-break scene and print per-stage times.

    python -m flip2_b200.profile_step [--cells 256] [--steps 2] [--dt 1/480]
        [--method 0|1|2] [--poisson K] [--lp-grad K] [--lp-cuda-cores 0|1]
        [--binning N]

The scene is the benchmark's (block 0.5 x 0.5 x 1 of the unit box, 8
jittered particles per voxel, seed 0).  Each step runs in full; stage times
come from CUDA events on the engine stream.  --method picks the pressure
solve (1 and 2 load the committed weights of the learned preconditioner);
--poisson K solves K generated pressure problems of the grid (seeds 900000
and up) with that method instead of stepping; --lp-grad K evaluates the
network's training loss and weight gradient K times; --binning N runs the
reference-mode binning of N particles of the binning microbenchmark.  Short enough to run under a
profiler with a kernel filter.
"""
import argparse
import json
import os

import numpy as np

from . import MODE_NATIVE, Particles, default_params, scenes

WEIGHTS = {1: "lprec_weights.npy", 2: "mg_weights.npy"}


def lp_grad(args, params, R):
    """--lp-grad K: K evaluations of the network's training loss and weight
    gradient on a cells^3 problem (fluid below 0.7 of the height, 8% random
    solid cells, seed 3; random weights and residuals), with the 16 -> 16
    layers on tcgen05 unless --lp-cuda-cores 1."""
    import time
    n = args.cells
    rng = np.random.default_rng(3)
    j = np.arange(n)[None, :, None] * np.ones((n, n, n))
    typ = np.where(j < 0.7 * n, 1, 0).astype(np.uint8)
    typ[rng.random(typ.shape) < 0.08] = 2
    typ = typ.ravel()
    r = (rng.standard_normal(typ.size) * (typ == 1)).astype(np.float32)
    ev = (r + 0.5 * rng.standard_normal(typ.size) * (typ == 1)).astype(np.float32)
    P = Particles(1, mode=MODE_NATIVE, params=params)
    P.setDomain(0.0, 0.0, 0.0, R, R, R, 1.0)
    P.poisson_set(typ, np.zeros(typ.size, np.float32))
    from . import lib
    P.lp_set_weights((rng.standard_normal(lib().flip_lp_num_weights()) * 0.15).astype(np.float32))
    for k in range(args.lp_grad):
        t0 = time.perf_counter()
        _, loss = P.lp_eval(r, ev, want_grad=True)
        print(json.dumps({"lp_grad": k, "cells": n, "loss": loss, "ms_with_transfers": round(1e3 * (time.perf_counter() - t0), 3),
                          "error_flags": P.info().error_flags}))
    P.close()


def binning(args):
    """--binning N: the reference-mode binning of N particles in a 512^3
    domain (50% uniform, 50% in 16 Gaussian blobs of sigma 8, seed 1; FP64
    positions): alignParticlesToGrid, sortParticles and generateVoxels,
    --steps times, each from the unsorted input, timed with CUDA events."""
    import torch
    from . import MODE_REFERENCE
    pos = scenes.binning_mix(args.binning, domain=512, seed=1).astype(np.float64)
    host = tuple(np.ascontiguousarray(pos[:, k]) for k in range(3))
    del pos
    stream = torch.cuda.Stream()
    P = Particles(args.binning, mode=MODE_REFERENCE, params=default_params(MODE_REFERENCE), stream=stream.cuda_stream)
    P.setDomain(0.0, 0.0, 0.0, 512, 512, 512, 1.0)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    for k in range(args.steps):
        P.upload(host, None)
        P.sync()
        ev[0].record(stream)
        P.alignParticlesToGrid()
        ev[1].record(stream)
        P.sortParticles()
        ev[2].record(stream)
        P.generateVoxels()
        ev[3].record(stream)
        torch.cuda.synchronize()
        print(json.dumps({"binning": k, "particles": args.binning, "align_ms": ev[0].elapsed_time(ev[1]),
                          "sort_ms": ev[1].elapsed_time(ev[2]), "voxels_ms": ev[2].elapsed_time(ev[3]),
                          "voxels": P.info().voxels}))
    P.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=256)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--dt", type=float, default=1.0 / 480.0)
    ap.add_argument("--block", type=float, nargs=3, default=(0.5, 0.5, 1.0))
    ap.add_argument("--method", type=int, default=0, choices=(0, 1, 2))
    ap.add_argument("--lp-cuda-cores", type=int, default=0)
    ap.add_argument("--poisson", type=int, default=0)
    ap.add_argument("--lp-grad", type=int, default=0)
    ap.add_argument("--binning", type=int, default=0)
    args = ap.parse_args()
    params = default_params(MODE_NATIVE, pressure_method=args.method, lp_cuda_cores=args.lp_cuda_cores)
    R = args.cells // 4
    if args.lp_grad:
        lp_grad(args, params, R)
        return
    if args.binning:
        binning(args)
        return
    if args.poisson:
        P = Particles(1, mode=MODE_NATIVE, params=params)
        P.setDomain(0.0, 0.0, 0.0, R, R, R, 1.0)
        if args.method:
            P.lp_set_weights(np.load(os.path.join(os.path.dirname(__file__), "data", WEIGHTS[args.method])))
        for k in range(args.poisson):
            P.poisson_generate(seed=900_000 + k)
            i = P.poisson_solve(args.method, 1e-6, 20000 if args.method == 0 else 100)
            print(json.dumps({"problem": 900_000 + k, "method": args.method, "iters": i.iters, "ms": round(i.ms, 3),
                              "fell_back": i.fell_back, "rel_residual": i.rel_residual}))
        P.close()
        return
    pos, vel = scenes.dam_break(args.cells, block=tuple(args.block), seed=0)
    P = Particles(pos.shape[0], mode=MODE_NATIVE, params=params)
    P.setDomain(0.0, 0.0, 0.0, R, R, R, 4.0 / args.cells)
    if args.method:
        P.lp_set_weights(np.load(os.path.join(os.path.dirname(__file__), "data", WEIGHTS[args.method])))
    P.upload(pos, vel)
    P.set_timing(True)
    for k in range(args.steps):
        P.step(args.dt)
        info = P.info()
        print(json.dumps({"step": k, "particles": pos.shape[0], "pcg_iters": info.pressure_iters,
                          "rel_residual": info.residual, "stages_ms": P.stage_ms(reset=True)}))
    P.close()


if __name__ == "__main__":
    main()
