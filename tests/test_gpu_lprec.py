"""The learned pressure preconditioner and the standalone pressure problems
on the GPU, through the C ABI: the network's forward pass, loss and weight
gradient against the oracle's FP64 restatement (with the same BF16
roundings), Jacobi-PCG and learned FPCG solves against the oracle's FP64
operator and solver, on-device training, and the native step with the
learned preconditioner.  Tolerances are written per check."""
import numpy as np
import pytest

import flip2_b200 as F
from flip2_b200 import scenes
from oracle import oracle as O
from tests.test_lprec_oracle import centre_chain_weights
from tests.util import rel_err, tiled_to_linear

pytestmark = pytest.mark.gpu
ERR_ARG, ERR_STATE = 1, 5


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available()
    F.lib()
    return T


def engine(shape, **kw):
    """An engine whose native grid is shape = (nx, ny, nz) voxels (multiples of 8)."""
    nx, ny, nz = shape
    P = F.Particles(1, mode=F.MODE_NATIVE, params=F.default_params(F.MODE_NATIVE, **kw))
    P.setDomain(0.0, 0.0, 0.0, nx // 4, ny // 4, nz // 4, 1.0)
    return P


def random_types(shape, seed):
    """fluid below a surface, air above, random solid cells (x fastest)"""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    typ = np.where(j < 0.7 * ny, 1, 0).astype(np.uint8)
    typ[rng.random(typ.shape) < 0.08] = 2
    return typ.ravel()


def problem_arrays(P, shape):
    nx, ny, nz = shape
    typ = tiled_to_linear(P.read(F.BUF_CELL_TYPE, np.uint8), nx, ny, nz)
    b = tiled_to_linear(P.read(F.BUF_DIVU, np.float32), nx, ny, nz)
    return typ, b


def solution_residual(typ, b, x, shape):
    Po = O.nat_params(*shape, 1.0)
    ax = O.nat_apply_A(typ, x, Po)
    fl = typ == 1
    bd = b.astype(np.float64)
    return float(np.linalg.norm((bd - ax)[fl]) / np.linalg.norm(bd[fl]))


# ------------------------------------------------------------- network
@pytest.mark.parametrize("a,expect", [(1 + 2.0 ** -9, 1.0), (1 + 3 * 2.0 ** -9, 1 + 2.0 ** -7),
                                      (1 + 2.0 ** -8, 1.0), (1 + 3 * 2.0 ** -8, 1 + 2.0 ** -6)])
def test_lp_centre_chain_exact(torch, a, expect):
    # one path through the centre taps: z = bf16(a) * r exactly, on fluid cells only
    shape = (16, 16, 8)
    P = engine(shape)
    typ = random_types(shape, 1)
    P.poisson_set(typ, np.zeros(typ.size, np.float32))
    P.lp_set_weights(centre_chain_weights(a))
    r = np.where(typ == 1, 1.0, 0.0).astype(np.float32)
    z, loss = P.lp_eval(r, r)
    assert np.all(z[typ == 1] == np.float32(expect))
    assert np.all(z[typ != 1] == 0.0)
    P.close()


@pytest.mark.parametrize("shape,seed", [((32, 24, 16), 0), ((16, 16, 40), 1)])
def test_lp_forward_loss_grad_vs_oracle(torch, shape, seed):
    P = engine(shape)
    typ = random_types(shape, seed)
    rng = np.random.default_rng(seed + 10)
    r = (rng.standard_normal(typ.size) * (typ == 1)).astype(np.float32)
    ev = (r + 0.5 * rng.standard_normal(typ.size) * (typ == 1)).astype(np.float32)
    w = (rng.standard_normal(F.lib().flip_lp_num_weights()) * 0.15).astype(np.float32)
    P.poisson_set(typ, np.zeros(typ.size, np.float32))
    P.lp_set_weights(w)
    z, loss = P.lp_eval(r, ev, want_grad=True)
    g = P.lp_grad()
    lo, zo, go = O.lp_loss_grad(typ.reshape(shape[::-1]), r, ev, w, shape, round_bf16=True)
    # FP32 sums on the GPU vs FP64 here, and the rare activation whose BF16
    # rounding flips with that: 2e-3 in L2 and 2e-2 of the largest value
    assert np.linalg.norm(z - zo) <= 2e-3 * np.linalg.norm(zo)
    assert rel_err(z, zo) <= 2e-2
    # the loss is (m.Am - 2 m.r)/e.r + 1: compare the A-norm terms, 2e-3 of their size
    assert abs(loss - lo) <= 2e-3 * max(1.0, abs(lo))
    # the gradient sums millions of products through FP32 atomics: 5e-3 in L2
    # over all weights and per layer
    assert np.linalg.norm(g - go) <= 5e-3 * np.linalg.norm(go)
    offs = [0, 27 * 3 * 16, 27 * 3 * 16 + 27 * 256, 27 * 3 * 16 + 2 * 27 * 256, g.size]
    for l in range(4):
        a, b = g[offs[l]:offs[l + 1]], go[offs[l]:offs[l + 1]]
        assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b), l
    P.close()


def test_lp_tensor_cores_match_cuda_cores(torch):
    # the tcgen05 implicit-GEMM layers against the CUDA-core kernels on the
    # same problem and weights: both accumulate BF16 products in FP32, in
    # different orders, so the BF16 activations differ by at most a rare
    # rounding step
    shape = (64, 48, 40)
    typ = random_types(shape, 5)
    rng = np.random.default_rng(6)
    r = (rng.standard_normal(typ.size) * (typ == 1)).astype(np.float32)
    w = (rng.standard_normal(F.lib().flip_lp_num_weights()) * 0.15).astype(np.float32)
    zs = []
    for cc in (0, 1):
        P = engine(shape, lp_cuda_cores=cc)
        P.poisson_set(typ, np.zeros(typ.size, np.float32))
        P.lp_set_weights(w)
        z, loss = P.lp_eval(r, r)
        assert P.info().error_flags == 0
        zs.append(z)
        P.close()
    assert np.linalg.norm(zs[0] - zs[1]) <= 1e-3 * np.linalg.norm(zs[1])
    assert rel_err(zs[0], zs[1]) <= 1e-2


@pytest.mark.parametrize("shape,seed", [((64, 48, 40), 7), ((24, 16, 40), 8)])
def test_lp_backward_tensor_cores_match_cuda_cores(torch, shape, seed):
    # the weight gradient with the 16 -> 16 layers' backward pass on tcgen05
    # (input gradients rounded to BF16 as MMA operands; the weight gradient
    # takes the output gradient as a BF16 pair, FP32 accumulation) against
    # the CUDA-core kernels (FP32 throughout), forward and backward of each
    # run on its own path
    typ = random_types(shape, seed)
    rng = np.random.default_rng(seed + 1)
    r = (rng.standard_normal(typ.size) * (typ == 1)).astype(np.float32)
    ev = (r + 0.5 * rng.standard_normal(typ.size) * (typ == 1)).astype(np.float32)
    w = (rng.standard_normal(F.lib().flip_lp_num_weights()) * 0.15).astype(np.float32)
    gs = []
    for cc in (0, 1):
        P = engine(shape, lp_cuda_cores=cc)
        P.poisson_set(typ, np.zeros(typ.size, np.float32))
        P.lp_set_weights(w)
        P.lp_eval(r, ev, want_grad=True)
        assert P.info().error_flags == 0
        gs.append(P.lp_grad())
        P.close()
    offs = [0, 27 * 3 * 16, 27 * 3 * 16 + 27 * 256, 27 * 3 * 16 + 2 * 27 * 256, gs[0].size]
    assert np.linalg.norm(gs[0] - gs[1]) <= 3e-3 * np.linalg.norm(gs[1])
    for l in range(4):
        a, b = gs[0][offs[l]:offs[l + 1]], gs[1][offs[l]:offs[l + 1]]
        assert np.linalg.norm(a - b) <= 5e-3 * np.linalg.norm(b), l


# ------------------------------------------------------ pressure problems
def test_generated_problem_pcg_vs_oracle(torch):
    shape = (64, 64, 64)
    P = engine(shape)
    P.poisson_generate(seed=4, radius=(3.0, 8.0))
    typ, b = problem_arrays(P, shape)
    nx, ny, nz = shape
    nsolid = float((typ == 2).mean())
    assert 0.03 < nsolid < 0.15  # ~10% of the box in spheres (overlaps and walls cut it)
    j = (np.arange(typ.size) // nx) % ny
    assert not np.any((typ == 1) & (j >= ny - 1))  # fluid stays below the surface
    assert np.all(b[typ != 1] == 0.0)
    info = P.poisson_solve(method=0, tol=1e-6, max_iter=4000)
    assert info.converged == 1 and info.fell_back == 0
    assert info.rel_residual <= 1e-6
    x = P.poisson_solution()
    assert solution_residual(typ, b, x, shape) <= 1.05e-6
    xo, it, rr = O.nat_pcg(typ, b.astype(np.float64), O.nat_params(*shape, 1.0, tol=1e-6))
    assert rel_err(x, xo) < 2e-3
    assert abs(info.iters - it) <= max(3, it // 10)
    P.close()


def test_fpcg_with_untrained_net_still_solves(torch):
    # an untrained network: FPCG either converges or hits its cap and the
    # Jacobi-PCG restart finishes the solve; either way the answer meets tol
    shape = (32, 32, 32)
    P = engine(shape)
    P.poisson_generate(seed=9, radius=(2.0, 5.0))
    P.lp_init(seed=1)
    info = P.poisson_solve(method=1, tol=1e-6, max_iter=25)
    assert info.converged == 1
    assert info.iters <= 25 + 16
    typ, b = problem_arrays(P, shape)
    assert solution_residual(typ, b, P.poisson_solution(), shape) <= 1.05e-6
    P.close()


@pytest.fixture(scope="module")
def trained(torch):
    """weights after 240 training steps on generated 32^3 problems"""
    shape = (32, 32, 32)
    P = engine(shape)
    P.lp_init(seed=0)
    losses = []
    iters = [0, 2, 5, 10, 20, 40, -1]
    for step in range(240):
        if step % 4 == 0:
            P.poisson_generate(seed=1000 + step, radius=(2.0, 5.0))
        losses.append(P.lp_train_step(iters[step % len(iters)], 2e-3))
    w = P.lp_weights()
    P.close()
    return w, losses


def test_training_reduces_loss(trained):
    w, losses = trained
    assert np.all(np.isfinite(losses)) and np.all(np.isfinite(w))
    assert np.mean(losses[-24:]) < 0.7 * np.mean(losses[:6])


def test_fpcg_vs_oracle_fpcg(trained):
    w, _ = trained
    shape = (32, 32, 32)
    P = engine(shape)
    P.poisson_generate(seed=77, radius=(2.0, 5.0))
    P.lp_set_weights(w)
    learned = P.poisson_solve(method=1, tol=1e-6, max_iter=400)
    plain = P.poisson_solve(method=0, tol=1e-6, max_iter=4000)
    typ, b = problem_arrays(P, shape)
    xo, ito, rro = O.lp_fpcg(typ, b.astype(np.float64), w, shape, tol=1e-6, max_iter=400)
    assert learned.converged == 1 and plain.converged == 1
    if ito <= 400 and rro <= 1e-6:
        # FCG with this network converges: the GPU run (FP32 vectors, BF16
        # network, FP64 dots) does too, without the fallback, in about as many
        # iterations, to the same solution
        assert learned.fell_back == 0
        assert abs(learned.iters - ito) <= max(4, ito // 4)
        P.poisson_solve(method=1, tol=1e-6, max_iter=400)
        x = P.poisson_solution()
        assert rel_err(x, xo) < 2e-3
    else:
        # it stalls in FP64 too: the GPU run stops (cap or stagnation) and Jacobi-PCG finishes
        assert learned.fell_back == 1 and learned.iters <= 400
        assert learned.plain_iters == plain.iters
        x = P.poisson_solution()
    assert solution_residual(typ, b, x, shape) <= 1.05e-6
    P.close()


def test_native_step_learned_matches_plain(trained):
    w, _ = trained
    nc, dt = 32, 1.0 / 240
    pos, vel = scenes.dam_break(nc, seed=0)
    out = {}
    for method in (0, 1):
        P = F.Particles(pos.shape[0], mode=F.MODE_NATIVE, params=F.default_params(F.MODE_NATIVE, pressure_method=method))
        P.setDomain(0.0, 0.0, 0.0, nc // 4, nc // 4, nc // 4, 4.0 / nc)
        if method:
            P.lp_set_weights(w)
        P.upload(pos, vel)
        P.step(dt)
        info = P.info()
        si = P.solve_info()
        assert info.converged == 1 and info.residual <= 1e-6
        out[method] = (tiled_to_linear(P.read(F.BUF_PRESSURE), nc, nc, nc), si, P.download())
        P.close()
    (p0, s0, (x0, v0)), (p1, s1, (x1, v1)) = out[0], out[1]
    # the learned solve either converges itself or restarts on Jacobi-PCG; the
    # pressure meets the same tolerance either way
    if s1.fell_back:
        assert s1.plain_iters == s0.iters
    assert rel_err(p1, p0) < 2e-3
    assert rel_err(v1, v0, floor=1e-3) < 2e-3


def test_lp_errors(torch):
    shape = (16, 16, 16)
    P = engine(shape)
    with pytest.raises(F.FlipError) as ei:
        P.poisson_solve(method=0)
    assert ei.value.status == ERR_STATE
    P.poisson_generate(seed=0, radius=(2.0, 4.0))
    with pytest.raises(F.FlipError) as ei:
        P.poisson_solve(method=1)  # no weights yet
    assert ei.value.status == ERR_STATE
    with pytest.raises(F.FlipError) as ei:
        P.lp_set_weights(np.zeros(10, np.float32))
    assert ei.value.status == ERR_ARG
    with pytest.raises(F.FlipError) as ei:
        P.poisson_solve(method=2)  # the multilevel form needs the weights too
    assert ei.value.status == ERR_STATE
    with pytest.raises(F.FlipError) as ei:
        P.poisson_solve(method=3)
    assert ei.value.status == ERR_ARG
    with pytest.raises(F.FlipError) as ei:
        P.poisson_generate(seed=0, surface=(0.9, 0.1))
    assert ei.value.status == ERR_ARG
    P.close()
    R = F.Particles(8, mode=F.MODE_REFERENCE)
    R.setDomain(0.0, 0.0, 0.0, 4, 4, 4, 1.0)
    with pytest.raises(F.FlipError) as ei:
        R.poisson_generate(seed=0)
    assert ei.value.status == ERR_STATE
    R.close()
