"""Captured steps and frames.  With stage timing off, flip_step is one CUDA
graph launch and flip_solve_frame one graph launch per frame: the solve's
iteration loop, the Jacobi-PCG restart of a flexible solve that missed tol,
and the frame's Courant-limited sub-steps are conditional nodes, and the
host reads the solve's outcome back only when asked.  With stage timing on,
the same stages run launch by launch (the path the other tests exercise).
Each captured form must give what the launch-by-launch form gives."""
import os

import numpy as np
import pytest

import flip2_b200 as F
from flip2_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available()
    F.lib()
    return T


def engine(n, nc, **kw):
    P = F.Particles(n, mode=F.MODE_NATIVE, params=F.default_params(F.MODE_NATIVE, **kw))
    P.setDomain(0.0, 0.0, 0.0, nc // 4, nc // 4, nc // 4, 4.0 / nc)
    return P


def run(pos, vel, nc, steps, timing, dt=1.0 / 240, **kw):
    P = engine(pos.shape[0], nc, **kw)
    if kw.get("pressure_method") == 2:
        P.lp_set_weights(np.load(os.path.join(os.path.dirname(F.__file__), "data", "mg_weights.npy")))
    P.set_timing(timing)
    P.upload(pos, vel)
    iters = []
    for _ in range(steps):
        P.step(dt)
        i = P.info()
        assert i.converged == 1 and i.residual <= 1e-6 and i.error_flags == 0
        iters.append(i.pressure_iters)
    out = P.download()
    info = P.info()
    P.close()
    return out, iters, info


@pytest.mark.parametrize("method", [0, 2])
def test_captured_steps_match_stage_by_stage(torch, method):
    nc = 32
    pos, vel = scenes.dam_break(nc, seed=0)
    (pe, ve), ie, _ = run(pos, vel, nc, 6, True, pressure_method=method)
    (pg, vg), ig, info = run(pos, vel, nc, 6, False, pressure_method=method)
    assert info.solves == 6
    assert info.graph_steps == 6  # every step ran as one graph launch
    # the same kernels on the same data: iteration counts agree (float
    # atomics may reorder sums, so allow one chunk of slack) and the particles
    # agree far inside the parity tolerance against the FP64 oracle
    assert all(abs(a - b) <= 16 for a, b in zip(ie, ig)), (ie, ig)
    assert np.max(np.abs(pe - pg)) < 1e-4 / nc
    assert np.max(np.abs(ve - vg)) < 1e-4 * max(1.0, float(np.max(np.abs(ve))))


def test_captured_restart_branch(torch):
    """A flexible solve capped at two iterations misses tol every step: the
    graph's IF branch restarts Jacobi-PCG, which converges, and the device
    counts the fallbacks."""
    nc = 32
    pos, vel = scenes.dam_break(nc, seed=0)
    P = engine(pos.shape[0], nc, pressure_method=2, learned_max_iter=2)
    P.lp_set_weights(np.load(os.path.join(os.path.dirname(F.__file__), "data", "mg_weights.npy")))
    P.upload(pos, vel)
    for _ in range(3):
        P.step(1.0 / 240)
    s = P.solve_info()
    info = P.info()
    assert s.fell_back == 1 and s.plain_iters > 0 and s.converged == 1 and s.rel_residual <= 1e-6
    assert info.solves == 3 and info.fallbacks == 3 and info.graph_steps == 3
    P.close()


def test_captured_frame_matches_stage_by_stage(torch):
    """One frame at 24 fps: the device picks the sub-steps (Courant limit and
    max_substep_dt); the captured frame and the host-driven frame take the
    same number of sub-steps to the same end time and state.  The second
    frame starts from a moving fluid, so the Courant limit binds, and its
    nested solve loops must run on every sub-step (a loop inside another
    loop's body gets its condition set before it)."""
    nc = 32
    pos, vel = scenes.dam_break(nc, seed=0)
    res = {}
    for timing in (True, False):
        P = engine(pos.shape[0], nc)
        P.set_timing(timing)
        P.upload(pos, vel)
        for _ in range(2):
            P.solveFrame(24.0)
            i = P.info()
            assert i.converged == 1 and i.error_flags == 0
        res[timing] = (P.download(), P.info())
        P.close()
    (pe, ve), ie = res[True]
    (pg, vg), ig = res[False]
    assert abs(ie.elapsed_time - 2.0 / 24.0) < 1e-12 and abs(ig.elapsed_time - 2.0 / 24.0) < 1e-12
    assert ie.solves == ig.solves >= 20  # at least max_substep_dt's ten sub-steps per frame
    assert ie.graph_steps == 0 and ig.graph_steps == ig.solves  # the captured frames ran every sub-step
    assert np.max(np.abs(pe - pg)) < 1e-4 / nc
    assert pg[:, 1].mean() < pos[:, 1].mean()
