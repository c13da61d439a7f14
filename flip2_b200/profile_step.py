"""Run a few native steps of the dam-break scene and print per-stage times.

    python -m flip2_b200.profile_step [--cells 256] [--steps 2] [--dt 1/480]

The scene is the benchmark's (block 0.5 x 0.5 x 1 of the unit box, 8
jittered particles per voxel, seed 0).  Each step runs in full; stage times
come from CUDA events on the engine stream.  Short enough to run under a
profiler with a kernel filter.
"""
import argparse
import json

from . import MODE_NATIVE, Particles, default_params, scenes


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=256)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--dt", type=float, default=1.0 / 480.0)
    ap.add_argument("--block", type=float, nargs=3, default=(0.5, 0.5, 1.0))
    args = ap.parse_args()
    pos, vel = scenes.dam_break(args.cells, block=tuple(args.block), seed=0)
    P = Particles(pos.shape[0], mode=MODE_NATIVE, params=default_params(MODE_NATIVE))
    R = args.cells // 4
    P.setDomain(0.0, 0.0, 0.0, R, R, R, 4.0 / args.cells)
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
