"""Train the learned pressure preconditioner on the GPU and evaluate it.

    python -m flip2_b200.train_preconditioner --cells 128 --minutes 10 \
        --out flip2_b200/data/lprec_weights.npy

Training problems on a cells^3 grid: generated pressure problems (solid
spheres of radius 4..16 voxels to 10% of the box, a fluid surface at 50-85%
of the height, six Gaussian velocity impulses plus gravity) alternating with
the pressure problems of a dam-break simulation that runs in the same engine
(block 0.5 x 0.5 x 1 of the box, Jacobi-PCG, dt 1/480).  The solver applies
M(r) = N(r) + D^-1 r.  A sample is (r, e) with A e = r: 70% the residual and
error of x_k after k Jacobi-PCG iterations from x = 0 (k drawn from 0, 2, 5,
10, 20, 40, 80; e = x* - x_k against the problem's converged solution), 30%
white-noise errors e with r = A e.  The loss is the A-norm error of M(r) as
an estimate of e, relative to |e|_A; Adam.

With --mg the network is trained as the coarsest-level solve of the
multilevel preconditioner (pressure_method 2): a sample is the coarsest
right-hand side that one V-cycle makes of the residual after k Jacobi-PCG
iterations (k as above; its coarse solution from CG on the coarsest grid),
or a white-noise coarse error e with r = A e, and the loss is the same
A-norm error on the coarsest grid.

Evaluation: Jacobi-PCG against learned FPCG (tol 1e-6) on held-out generated
problems and on dam-break steps, iterations and device milliseconds, one
JSON line per problem kind; with --mg also the same V-cycle without the
network.
"""
import argparse
import json
import time

import numpy as np

from . import MODE_NATIVE, Particles, default_params, scenes

SAMPLE_ITERS = (0, 2, 5, 10, 20, 40, 80)


def make_engine(cells, pressure_method=0):
    pos, vel = scenes.dam_break(cells, block=(0.5, 0.5, 1.0), seed=0)
    P = Particles(pos.shape[0], mode=MODE_NATIVE, params=default_params(MODE_NATIVE, pressure_method=pressure_method))
    R = cells // 4
    P.setDomain(0.0, 0.0, 0.0, R, R, R, 4.0 / cells)
    P.upload(pos, vel)
    return P, pos, vel


def evaluate(P, cells, seeds, tol=1e-6, max_iter=100, method=1):
    rows = []
    for s in seeds:
        P.poisson_generate(seed=s)
        a = P.poisson_solve(0, tol, 20000)
        b = P.poisson_solve(method, tol, max_iter)
        rows.append((a.iters, a.ms, b.iters, b.ms, b.fell_back, b.rel_residual))
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=128)
    ap.add_argument("--minutes", type=float, default=10.0)
    ap.add_argument("--max-steps", type=int, default=1000000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--lr-final", type=float, default=2e-4)
    ap.add_argument("--steps-per-problem", type=int, default=4)
    ap.add_argument("--init", default=None, help="start from these weights (.npy)")
    ap.add_argument("--out", default="flip2_b200/data/lprec_weights.npy")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--eval-problems", type=int, default=8)
    ap.add_argument("--noise", type=float, default=0.3, help="fraction of white-noise error samples")
    ap.add_argument("--eval-max-iter", type=int, default=100, help="learned FCG cap in the evaluation")
    ap.add_argument("--eval-dam-steps", type=int, default=40, help="dam-break steps per method in the evaluation")
    ap.add_argument("--mg", action="store_true", help="train the coarsest solve of the multilevel preconditioner")
    args = ap.parse_args()
    method = 2 if args.mg else 1

    P, pos, vel = make_engine(args.cells)
    if args.init:
        P.lp_set_weights(np.load(args.init))
    else:
        P.lp_init(args.seed)
    rng = np.random.default_rng(args.seed)
    t0 = time.time()
    budget = 60.0 * args.minutes
    step, prob, losses = 0, 0, []
    sim_steps = 0
    while step < args.max_steps and time.time() - t0 < budget:
        # new problem: even ones generated, odd ones the next dam-break step
        if prob % 2 == 0:
            P.poisson_generate(seed=10_000 * (args.seed + 1) + prob)
        else:
            if sim_steps % 200 == 0:
                P.upload(pos, vel)  # restart the dam break
            P.step(1.0 / 480.0)
            sim_steps += 1
        prob += 1
        frac = min(1.0, (time.time() - t0) / budget)
        lr = args.lr * (args.lr_final / args.lr) ** frac
        for _ in range(args.steps_per_problem):
            k = int(SAMPLE_ITERS[rng.integers(len(SAMPLE_ITERS))]) if rng.random() >= args.noise else -1
            losses.append(P.mg_train_step(k, lr) if args.mg else P.lp_train_step(k, lr))
            step += 1
        if prob % 50 == 0:
            print(json.dumps({"step": step, "problems": prob, "loss": float(np.mean(losses[-50:])), "lr": lr,
                              "s": round(time.time() - t0, 1)}), flush=True)
    w = P.lp_weights()
    np.save(args.out, w)
    train_s = time.time() - t0
    print(json.dumps({"trained_steps": step, "problems": prob, "seconds": round(train_s, 1),
                      "final_loss": float(np.mean(losses[-100:])), "out": args.out}), flush=True)

    seeds = range(900_000, 900_000 + args.eval_problems)
    rows = evaluate(P, args.cells, seeds, max_iter=args.eval_max_iter, method=method)
    a = np.array(rows)
    print(json.dumps({"eval": "generated", "cells": args.cells, "method": method, "jacobi_iters": a[:, 0].tolist(),
                      "jacobi_ms": np.round(a[:, 1], 2).tolist(), "learned_iters": a[:, 2].tolist(),
                      "learned_ms": np.round(a[:, 3], 2).tolist(), "fell_back": int(a[:, 4].sum())}), flush=True)
    P.close()
    if args.mg:
        # the same V-cycle without the network
        Q = Particles(1, mode=MODE_NATIVE, params=default_params(MODE_NATIVE, mg_coarse=1))
        R = args.cells // 4
        Q.setDomain(0.0, 0.0, 0.0, R, R, R, 4.0 / args.cells)
        a = np.array(evaluate(Q, args.cells, seeds, max_iter=args.eval_max_iter, method=2))
        print(json.dumps({"eval": "generated", "cells": args.cells, "method": 2, "network": False,
                          "iters": a[:, 2].tolist(), "ms": np.round(a[:, 3], 2).tolist(),
                          "fell_back": int(a[:, 4].sum())}), flush=True)
        Q.close()
    # dam-break steps with each method
    for m in ((0, method) if args.eval_dam_steps > 0 else ()):
        Q, _, _ = make_engine(args.cells, pressure_method=m)
        if m:
            Q.lp_set_weights(w)
        Q.set_timing(True)
        its, ms, fb = [], [], 0
        for k in range(args.eval_dam_steps):
            Q.step(1.0 / 480.0)
            si = Q.solve_info()
            its.append(si.iters + si.plain_iters)
            ms.append(si.ms)
            fb += si.fell_back
        print(json.dumps({"eval": "dam_break", "cells": args.cells, "method": m, "iters": its,
                          "ms": np.round(ms, 2).tolist(), "fell_back": fb}), flush=True)
        Q.close()


if __name__ == "__main__":
    main()
