"""The multilevel learned preconditioner (pressure_method 2) on the GPU
through the C ABI: one V-cycle against the oracle's FP64 restatement (with
and without the network on the coarsest level, on cubic grids and on grids
whose coarse levels need padding), FCG solves against the oracle's FCG,
training of the network as the coarsest solve, and a native step with the
method.  Tolerances are written per check."""
import os

import numpy as np
import pytest

import flip2_b200 as F
from flip2_b200 import scenes
from oracle import oracle as O
from tests.test_gpu_lprec import engine, problem_arrays, solution_residual
from tests.util import rel_err, remove_pocket_constants, sealed_pockets, tiled_to_linear

pytestmark = pytest.mark.gpu
WEIGHTS = os.path.join(os.path.dirname(F.__file__), "data", "mg_weights.npy")


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available()
    F.lib()
    return T


def mg_engine(shape, mode, seed=3):
    P = engine(shape, mg_coarse=mode)
    P.poisson_generate(seed=seed, radius=(3.0, 8.0))
    P.lp_set_weights(np.load(WEIGHTS))
    return P


@pytest.mark.parametrize("shape", [(64, 64, 64), (48, 40, 56)])
@pytest.mark.parametrize("mode", [1, 0])
def test_vcycle_vs_oracle(torch, shape, mode):
    P = mg_engine(shape, mode)
    typ, b = problem_arrays(P, shape)
    rng = np.random.default_rng(5)
    r = np.where(typ == 1, rng.standard_normal(typ.size), 0.0).astype(np.float32)
    z = P.mg_apply(r)
    assert P.info().error_flags == 0
    zo = O.mg_apply(typ, r, np.load(WEIGHTS), shape, mode=mode)
    assert np.all(z[typ != 1] == 0.0)
    # FP32 against FP64: without the network the V-cycle agrees to FP32
    # rounding; with it, BF16 roundings of activations that sit at a rounding
    # tie in one and not the other move single outputs by a few BF16 ulps
    tol = 1e-5 if mode == 1 else 2e-2
    assert rel_err(z, zo) < tol
    assert np.linalg.norm(z - zo) <= (1e-5 if mode == 1 else 5e-3) * np.linalg.norm(zo)
    P.close()


@pytest.mark.parametrize("mode", [1, 0])
def test_fcg_vs_oracle(torch, mode):
    shape = (64, 64, 64)
    P = mg_engine(shape, mode, seed=11)
    info = P.poisson_solve(method=2, tol=1e-6, max_iter=400)
    assert info.converged == 1 and info.fell_back == 0
    assert info.rel_residual <= 1e-6
    typ, b = problem_arrays(P, shape)
    x = P.poisson_solution()
    assert solution_residual(typ, b, x, shape) <= 1.05e-6
    xo, ito, rro = O.mg_fcg(typ, b.astype(np.float64), np.load(WEIGHTS), shape, mode=mode, max_iter=400)
    assert rro <= 1e-6
    assert rel_err(x, xo) < 2e-3
    # the GPU's true-residual checks stop it at a chunk boundary at the latest
    assert abs(info.iters - ito) <= max(4, ito // 8) + 16
    plain = P.poisson_solve(method=0, tol=1e-6, max_iter=20000)
    assert info.iters * 4 < plain.iters
    P.close()


def test_training_reduces_coarse_loss(torch):
    shape = (64, 64, 64)
    P = engine(shape)
    P.lp_init(seed=0)
    losses = []
    ks = [0, 2, 5, 10, 20, -1]
    for step in range(180):
        if step % 6 == 0:
            P.poisson_generate(seed=2000 + step, radius=(3.0, 8.0))
        losses.append(P.mg_train_step(ks[step % len(ks)], 2e-3))
    assert np.all(np.isfinite(losses))
    assert np.mean(losses[-30:]) < 0.7 * np.mean(losses[:6])
    w = P.lp_weights()
    assert np.all(np.isfinite(w))
    P.close()


def test_native_step_with_method_2(torch):
    nc = 64
    pos, vel = scenes.dam_break(nc, block=(0.5, 0.5, 1.0), seed=0)
    out = {}
    for method in (0, 2):
        params = F.default_params(F.MODE_NATIVE, pressure_method=method)
        P = F.Particles(pos.shape[0], mode=F.MODE_NATIVE, params=params)
        P.setDomain(0.0, 0.0, 0.0, nc // 4, nc // 4, nc // 4, 4.0 / nc)
        if method:
            P.lp_set_weights(np.load(WEIGHTS))
        P.upload(pos, vel)
        its = []
        for _ in range(3):
            P.step(1.0 / 480)
            si = P.solve_info()
            assert si.converged == 1 and si.fell_back == 0 and si.rel_residual <= 1e-6
            its.append(si.iters)
        phi = tiled_to_linear(P.read(F.BUF_PRESSURE), nc, nc, nc)
        out[method] = (its, phi, P.download())
        P.close()
    its0, phi0, (p0, v0) = out[0]
    its2, phi2, (p2, v2) = out[2]
    assert max(its2) * 4 < min(its0)
    # both solves meet 1e-6; the pressures and the stepped state agree to
    # the solver tolerance amplified by the conditioning (positions compared
    # sorted per axis: the particle order follows the cell keys)
    assert rel_err(phi2, phi0) < 2e-3
    for k in range(3):
        assert np.max(np.abs(np.sort(p2[:, k]) - np.sort(p0[:, k]))) < 1e-3 * (4.0 / nc)


def test_coarse_cg_comparison_mode(torch):
    # mg_coarse = 2 (one-CTA Jacobi-PCG on the coarsest level, a comparison
    # without the network) is a valid preconditioner too: FCG meets tol
    shape = (64, 64, 64)
    P = mg_engine(shape, 2, seed=11)
    info = P.poisson_solve(method=2, tol=1e-6, max_iter=400)
    assert info.converged == 1 and info.fell_back == 0
    typ, b = problem_arrays(P, shape)
    assert solution_residual(typ, b, P.poisson_solution(), shape) <= 1.05e-6
    P.close()


def test_coarsest_network_tensor_cores_vs_cuda_cores(torch):
    # the coarsest level's 16 -> 16 layers on tcgen05 (default) against the
    # CUDA-core small-grid kernels: FP32 sums of the same BF16 products in a
    # different order, so a few activations round to the neighbouring BF16
    shape = (64, 64, 64)
    zs = []
    for cc in (0, 1):
        P = engine(shape, lp_cuda_cores=cc)
        P.poisson_generate(seed=3, radius=(3.0, 8.0))
        P.lp_set_weights(np.load(WEIGHTS))
        typ, _ = problem_arrays(P, shape)
        r = np.where(typ == 1, np.random.default_rng(5).standard_normal(typ.size), 0.0).astype(np.float32)
        zs.append(P.mg_apply(r))
        assert P.info().error_flags == 0
        P.close()
    assert np.linalg.norm(zs[0] - zs[1]) <= 1e-3 * np.linalg.norm(zs[1])


def test_trained_network_gain(torch):
    # what the trained network gains: the same V-cycle and FCG on the same
    # problems, with the committed weights, without the network, and with an
    # untrained (freshly initialised) network.  Iterations count the
    # Jacobi-PCG restart of a solve that falls back (the untrained network's
    # output is noise: FCG stalls and restarts)
    shape = (128, 128, 128)
    its, fell = {}, {}
    for name, mode, w in (("trained", 0, "committed"), ("no_network", 1, "committed"), ("untrained", 0, "init")):
        P = engine(shape, mg_coarse=mode)
        if w == "init":
            P.lp_init(seed=0)
        else:
            P.lp_set_weights(np.load(WEIGHTS))
        its[name], fell[name] = [], 0
        for s in range(900_000, 900_003):
            P.poisson_generate(seed=s)
            info = P.poisson_solve(method=2, tol=1e-6, max_iter=100)
            assert info.converged == 1 and info.rel_residual <= 1e-6
            its[name].append(info.iters + info.plain_iters)
            fell[name] += info.fell_back
        P.close()
    print(its, fell)
    assert fell["trained"] == 0 and fell["no_network"] == 0
    assert sum(its["trained"]) < 0.6 * sum(its["no_network"])
    assert sum(its["trained"]) < 0.6 * sum(its["untrained"])


@pytest.mark.parametrize("sample", [-1, 5])
def test_coarse_training_loss_and_gradient_vs_oracle(torch, sample):
    # the training step of the multilevel form on its coarsest level: the
    # small-grid forward (tcgen05 16 -> 16 layers) and the backward kernels
    # against the oracle's FP64 loss and gradient on the same coarse problem
    # (types, right-hand side and error read back from the engine)
    shape = (64, 64, 64)
    P = engine(shape)
    P.poisson_generate(seed=21, radius=(3.0, 8.0))
    w = np.load(WEIGHTS)
    P.lp_set_weights(w)
    loss = P.mg_train_step(sample, 0.0)
    g = P.lp_grad()
    cshape = O.mg_levels(shape)[-1]
    typ = tiled_to_linear(P.read(F.BUF_MG_COARSE_TYPE, np.uint8), *cshape)
    r = tiled_to_linear(P.read(F.BUF_MG_COARSE_R, np.float32), *cshape)
    ev = tiled_to_linear(P.read(F.BUF_MG_COARSE_E, np.float32), *cshape)
    assert P.info().error_flags == 0
    P.close()
    assert np.any(typ == 1) and np.any(r[typ == 1] != 0.0)
    lo, zo, go = O.lp_loss_grad(typ.reshape(cshape[::-1]), r, ev, w, cshape, round_bf16=True)
    # the loss to 2e-3 as in the network's own parity test.  The gradient: FP32
    # sums against FP64, and activations whose BF16 rounding flips between the
    # two; on the 4,096 voxels of the coarsest level fewer of those flips
    # average out than on the solver-grid tests (5e-3 there), so 1e-2 in L2
    # over all weights and 2e-2 per layer
    assert abs(loss - lo) <= 2e-3 * max(1.0, abs(lo))
    assert np.linalg.norm(g - go) <= 1e-2 * np.linalg.norm(go)
    offs = [0, 27 * 3 * 16, 27 * 3 * 16 + 27 * 256, 27 * 3 * 16 + 2 * 27 * 256, g.size]
    for l in range(4):
        a, b = offs[l], offs[l + 1]
        assert np.linalg.norm(g[a:b] - go[a:b]) <= 2e-2 * np.linalg.norm(go[a:b])


@pytest.mark.parametrize("mode", [0, 1])
def test_fcg_on_padded_levels(torch, mode):
    # a grid whose coarse levels need padding (48 x 40 x 56 -> 24 x 20 x 28
    # padded to 24 x 24 x 32 -> 12 x 10 x 14 padded to 16^3): FCG with the
    # V-cycle meets tol and its solution is the oracle's
    shape = (48, 40, 56)
    P = mg_engine(shape, mode, seed=13)
    info = P.poisson_solve(method=2, tol=1e-6, max_iter=400)
    assert info.converged == 1 and info.fell_back == 0 and info.rel_residual <= 1e-6
    typ, b = problem_arrays(P, shape)
    x = P.poisson_solution()
    assert solution_residual(typ, b, x, shape) <= 1.05e-6
    xo, ito, rro = O.mg_fcg(typ, b.astype(np.float64), np.load(WEIGHTS), shape, mode=mode, max_iter=400)
    assert rro <= 1e-6
    pocket, _ = sealed_pockets(typ, shape)
    assert rel_err(remove_pocket_constants(x, xo, pocket), xo) < 2e-3
    assert abs(info.iters - ito) <= max(4, ito // 8) + 16
    P.close()


@pytest.mark.parametrize("shape", [(16, 16, 16), (16, 8, 16)])
@pytest.mark.parametrize("mode", [0, 1])
def test_fcg_single_level(torch, shape, mode):
    # every axis at most 16 cells: the hierarchy is the solver's grid alone,
    # the network (or Jacobi) works on it directly, and FCG's dot products
    # run as their own kernel (there is no post-smoothing kernel above the
    # coarsest level to take them)
    P = engine(shape, mg_coarse=mode)
    P.poisson_generate(seed=17, radius=(2.0, 4.0))
    P.lp_set_weights(np.load(WEIGHTS))
    info = P.poisson_solve(method=2, tol=1e-6, max_iter=400)
    assert info.converged == 1 and info.fell_back == 0 and info.rel_residual <= 1e-6
    assert P.info().error_flags == 0
    typ, b = problem_arrays(P, shape)
    x = P.poisson_solution()
    assert solution_residual(typ, b, x, shape) <= 1.05e-6
    xo, ito, rro = O.mg_fcg(typ, b.astype(np.float64), np.load(WEIGHTS), shape, mode=mode, max_iter=400)
    assert rro <= 1e-6
    pocket, _ = sealed_pockets(typ, shape)
    assert rel_err(remove_pocket_constants(x, xo, pocket), xo) < 2e-3
    assert abs(info.iters - ito) <= max(4, ito // 8) + 16
    P.close()


def test_solve_frame_with_method_2(torch):
    # one frame of Courant sub-steps (solveFrame) with the learned multilevel
    # solve on a 32^3 grid (V-cycle 32^3 -> 16^3, the network on 16^3) against
    # the same frame with Jacobi-PCG: every solve meets 1e-6, so the sub-step
    # sequence and the particles agree to the solver tolerance (positions
    # compared sorted per axis: the particle order follows the cell keys)
    nc = 32
    pos, _ = scenes.dam_break(nc, seed=0)
    vel = scenes.random_velocities(pos.shape[0], seed=3, scale=2.0)
    out = {}
    for method in (0, 2):
        params = F.default_params(F.MODE_NATIVE, pressure_method=method)
        P = F.Particles(pos.shape[0], mode=F.MODE_NATIVE, params=params)
        P.setDomain(0.0, 0.0, 0.0, nc // 4, nc // 4, nc // 4, 4.0 / nc)
        if method:
            P.lp_set_weights(np.load(WEIGHTS))
        P.upload(pos, vel)
        P.solveFrame(24.0)
        info = P.info()
        assert info.converged == 1 and info.error_flags == 0
        si = P.solve_info()
        assert si.fell_back == 0 and si.rel_residual <= 1e-6
        out[method] = (P.download()[0], info.elapsed_time)
        P.close()
    (p0, t0), (p2, t2) = out[0], out[2]
    assert abs(t0 - t2) < 1e-12
    for k in range(3):
        assert np.max(np.abs(np.sort(p2[:, k]) - np.sort(p0[:, k]))) < 1e-3 * (4.0 / nc)
