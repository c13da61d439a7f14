"""The native-mode step (FLIP_MODE_NATIVE, FP32 state) against the FP64 oracle
of the same step: trilinear MAC P2G, Jacobi-PCG pressure with FP64
reductions, projection, FLIP 0.95 blend and RK2 advection.  Tolerances are
written per quantity below: P2G faces 2e-6 and projected faces 1e-5 of the
largest face velocity, pressure 1e-5 of max |phi|, particle velocities 1e-5
of max |v|, positions 1e-4 h."""
import numpy as np
import pytest

import flip2_b200 as F
from flip2_b200 import scenes
from oracle import oracle as O
from tests.util import native_step_errors, rel_err, tiled_to_linear

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available()
    F.lib()
    return T


def native(n, nc, **kw):
    p = F.default_params(F.MODE_NATIVE, **kw)
    P = F.Particles(n, mode=F.MODE_NATIVE, params=p)
    P.setDomain(0.0, 0.0, 0.0, nc // 4, nc // 4, nc // 4, 4.0 / nc)
    return P


@pytest.mark.parametrize("vscale", [0.0, 1.0])
def test_native_step_vs_fp64_oracle(torch, vscale):
    nc, dt = 32, 1.0 / 240
    pos, _ = scenes.dam_break(nc, seed=0)
    vel = scenes.random_velocities(pos.shape[0], seed=7, scale=vscale)
    P = native(pos.shape[0], nc)
    P.upload(pos, vel)
    P.step(dt)
    info = P.info()
    perm = P.read(F.BUF_PERM)
    Po = O.nat_params(nc, nc, nc, 1.0 / nc, dt=dt)
    ref = O.nat_step(pos, vel, Po)
    # cell classification: bit-exact
    typ = tiled_to_linear(P.read(F.BUF_CELL_TYPE, np.uint8), nc, nc, nc)
    assert int((typ == 1).sum()) == ref["fluid_cells"]
    # pressure: converged to the relative residual target, measured by the
    # FP64 oracle operator on the FP64 right-hand side
    assert info.converged == 1
    assert info.residual <= 1e-6
    assert abs(info.pressure_iters - ref["iters"]) <= max(3, ref["iters"] // 10)
    # grids and particles (GPU particle order is sorted: particle j is input
    # particle perm[j]); P2G sums are FP32 against FP64
    err = native_step_errors(P, ref, nc, F)
    if vscale > 0:
        assert err["p2g_face_rel_err"] < 2e-6, err
    assert err["pressure_rel_err_max"] < 1e-5, err
    assert err["proj_face_rel_err"] < 1e-5, err
    assert err["velocity_rel_err_max"] < 1e-5, err
    assert err["position_err_max_in_h"] < 1e-4, err
    P.close()


def test_native_twenty_steps(torch):
    nc, dt = 32, 1.0 / 240
    pos, vel = scenes.dam_break(nc, seed=0)
    P = native(pos.shape[0], nc)
    P.upload(pos, vel)
    for _ in range(20):
        P.step(dt)
        info = P.info()
        assert info.converged == 1 and info.residual <= 1e-6
        assert info.error_flags == 0
    pg, vg = P.download()
    assert np.all(np.isfinite(pg)) and np.all(np.isfinite(vg))
    assert pg.min() > 0.0 and pg.max() < 1.0
    # the block falls and spreads: centre of mass goes down, mean vy < 0
    assert pg[:, 1].mean() < pos[:, 1].mean()
    assert vg[:, 1].mean() < 0.0
    P.close()


def test_native_warm_start(torch):
    # twenty steps from the previous step's pressure and twenty from zero:
    # every solve meets 1e-6 either way, the warm runs take fewer iterations,
    # and the particles end up where the cold run puts them
    nc, dt = 32, 1.0 / 240
    pos, vel = scenes.dam_break(nc, seed=0)
    out = {}
    for warm in (0, 1):
        P = native(pos.shape[0], nc, pcg_warm_start=warm)
        P.upload(pos, vel)
        iters = 0
        for _ in range(20):
            P.step(dt)
            info = P.info()
            assert info.converged == 1 and info.residual <= 1e-6
            iters += info.pressure_iters
        out[warm] = (iters, P.download())
        P.close()
    (ic, (pc, _)), (iw, (pw, _)) = out[0], out[1]
    assert iw < ic
    # the particle order differs between the runs (each step re-sorts), so
    # compare each coordinate's sorted values: the two fluids agree to 5% of a cell
    for k in range(3):
        assert np.max(np.abs(np.sort(pc[:, k]) - np.sort(pw[:, k]))) < 0.05 / nc


@pytest.mark.parametrize("usolid", [(0.0, 0.0, 0.0), (0.3, 0.5, -0.2)])
def test_native_solid_sphere(torch, usolid):
    """Interior solid cells (the learned-preconditioner problems carry solid
    spheres): faces between a solid and a non-solid cell carry the solid's
    velocity (0 for a still solid), the solve converges, and the result
    matches the oracle run with the same mask and velocity."""
    nc, dt = 32, 1.0 / 240
    pos, _ = scenes.dam_break(nc, block=(1.0, 0.5, 1.0), seed=3)
    vel = scenes.random_velocities(pos.shape[0], seed=4, scale=0.5)
    k, j, i = np.meshgrid(np.arange(nc), np.arange(nc), np.arange(nc), indexing="ij")
    c = (np.stack([i, j, k], -1) + 0.5) / nc
    solid = (np.sum((c - np.array([0.5, 0.25, 0.5])) ** 2, -1) < 0.15 ** 2).astype(np.uint8).ravel()
    P = native(pos.shape[0], nc)
    P.set_solid_mask(solid)
    P.set_solid_velocity(*usolid)
    P.upload(pos, vel)
    P.step(dt)
    info = P.info()
    assert info.converged == 1
    Po = O.nat_params(nc, nc, nc, 1.0 / nc, dt=dt, solid_velocity=usolid)
    ref = O.nat_step(pos, vel, Po, solid=solid)
    typ = tiled_to_linear(P.read(F.BUF_CELL_TYPE, np.uint8), nc, nc, nc)
    assert np.array_equal(typ == 2, solid == 1)
    phi = tiled_to_linear(P.read(F.BUF_PRESSURE), nc, nc, nc).astype(np.float64)
    assert rel_err(phi, ref["phi"]) < 1e-5
    u = tiled_to_linear(P.read(F.BUF_GRID_U, np.float32), nc, nc, nc)
    solid3 = solid.reshape(nc, nc, nc)
    s_b = solid3.ravel() == 1
    s_a = np.roll(solid3, 1, axis=2).ravel() == 1
    assert np.all(u[s_b & s_a] == 0.0)
    assert np.all(u[s_b ^ s_a] == np.float32(usolid[0]))  # the sphere is away from the walls
    err = native_step_errors(P, ref, nc, F)
    assert err["proj_face_rel_err"] < 1e-5, err
    assert err["velocity_rel_err_max"] < 1e-5, err
    assert err["position_err_max_in_h"] < 1e-4, err
    P.close()


def test_native_engine_errors(torch):
    P = F.Particles(64, mode=F.MODE_NATIVE)
    with pytest.raises(F.FlipError) as ei:
        P.step(0.01)
    assert ei.value.status == 5
    with pytest.raises(F.FlipError) as ei:
        P.setDomain(0, 0, 0, 3, 4, 4, 0.25)  # 12 voxels: not a multiple of 8
    assert ei.value.status == 1
    P.close()


def test_position_frames(torch, tmp_path):
    # writePositionsToFile's "x, y, z" text (particles.cu:817-828, read by
    # visualizeSavedPoints.py) and the binary variant hold the same frame
    nc = 16
    pos, vel = scenes.dam_break(nc, seed=1)
    P = native(pos.shape[0], nc)
    P.upload(pos, vel)
    P.step(1.0 / 240)
    pg, _ = P.download()
    P.writePositionsToFile(tmp_path / "frame.csv")
    P.write_positions_bin(tmp_path / "frame.bin")
    P.close()
    txt = np.loadtxt(tmp_path / "frame.csv", delimiter=",")
    binf = F.read_positions_bin(tmp_path / "frame.bin")
    assert binf.shape == pg.shape and np.array_equal(binf, pg)
    assert txt.shape == pg.shape and np.max(np.abs(txt - pg)) <= 5e-6 * np.max(np.abs(pg))
    with open(tmp_path / "frame.bin", "rb") as f:
        assert f.read(8) == b"FLIP2POS"


def test_native_solve_frame_courant(torch):
    # solveFrame sub-steps: min(max_substep_dt, 0.7 h / max |v component|, the
    # rest of the frame); the limit comes from a device-side max over particles
    nc = 32
    pos, _ = scenes.dam_break(nc, seed=0)
    vel = scenes.random_velocities(pos.shape[0], seed=3, scale=8.0)  # Courant limit below max_substep_dt
    P = native(pos.shape[0], nc)
    P.upload(pos, vel)
    h = 1.0 / nc
    expect = 0.7 * h / float(np.max(np.abs(vel.astype(np.float32))))
    got = P.getCourantDt()
    assert abs(got - expect) <= 1e-6 * expect
    t0 = P.info().elapsed_time
    P.solveFrame(24.0)
    info = P.info()
    assert abs(info.elapsed_time - t0 - 1.0 / 24.0) < 1e-12
    assert 0.0 < info.dt <= F.default_params(F.MODE_NATIVE).max_substep_dt + 1e-15
    assert info.converged == 1
    pg, vg = P.download()
    assert np.all(np.isfinite(pg)) and pg.min() > 0.0 and pg.max() < 1.0
    # at rest the limit is 0 (no Courant bound)
    Q = native(pos.shape[0], nc)
    Q.upload(pos, np.zeros_like(vel))
    assert Q.getCourantDt() == 0.0
    Q.close()
    P.close()


def test_step_streamed_matches_step(torch):
    # the streamed round trip (upload, step, download in overlapping ranges)
    # gives what upload + step + download give, step after step (to the
    # rounding of P2G's float atomics, whose order differs between runs)
    nc, dt = 32, 1.0 / 240
    pos, vel = scenes.dam_break(nc, seed=2)
    n = pos.shape[0]
    ref = []
    P = native(n, nc)
    hp, hv = pos.copy(), vel.copy()
    for _ in range(4):
        P.upload(hp, hv)
        P.step(dt)
        hp, hv = P.download()
        ref.append(hp.copy())
    P.close()
    host = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in
            (pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1], vel[:, 2])]
    ptrs = [t.data_ptr() for t in host]
    Q = native(n, nc)
    for k in range(4):
        Q.step_streamed(ptrs, dt)
        Q.sync()
        got = np.stack([host[0].numpy(), host[1].numpy(), host[2].numpy()], axis=1)
        assert got.shape == ref[k].shape
        assert np.max(np.abs(got - ref[k])) < 1e-4 / nc, k
    # several calls in flight before one sync
    for _ in range(3):
        Q.step_streamed(ptrs, dt)
    Q.sync()
    assert np.all(np.isfinite(host[1].numpy()))
    Q.close()


def test_native_particles_stay_out_of_solids(torch):
    """The native reseed (the counterpart of the reference's moveSolids,
    engine/particles.cu:674-740): a block of fluid falls onto a solid slab
    for 40 steps; no particle ever sits in a solid cell, and the slab holds
    the fluid up (nothing passes below it)."""
    nc, dt = 32, 1.0 / 120
    pos, _ = scenes.dam_break(nc, block=(1.0, 0.3, 1.0), seed=5)
    pos[:, 1] += 0.45  # the block starts above the slab
    k, j, i = np.meshgrid(np.arange(nc), np.arange(nc), np.arange(nc), indexing="ij")
    slab = ((j >= 8) & (j < 12)).astype(np.uint8).ravel()  # y in [0.25, 0.375)
    P = native(pos.shape[0], nc)
    P.set_solid_mask(slab)
    P.upload(pos, np.zeros_like(pos))
    for _ in range(40):
        P.step(dt)
        pg, _ = P.download()
        cell = np.clip(np.floor(pg * nc).astype(np.int64), 0, nc - 1)
        inside = slab.reshape(nc, nc, nc)[cell[:, 2], cell[:, 1], cell[:, 0]] == 1
        assert not inside.any(), int(inside.sum())
    assert pg[:, 1].min() >= 0.375 - 1e-6
    info = P.info()
    assert info.converged == 1 and info.error_flags == 0
    P.close()


def _tile_keys(px, py, pz, nc):
    """Tile key of each position as the binning computes it: grid coordinate
    p / h in FP32 (exact here: h is a power of two), cell floor(g) clamped
    into [0, nc), key = tx + (nc / 8) (ty + (nc / 8) tz) of the 8^3 tile."""
    t = nc // 8
    c = [np.clip(np.floor(np.asarray(a, np.float32) * np.float32(nc)), 0, nc - 1).astype(np.int64) >> 3
         for a in (px, py, pz)]
    return c[0] + t * (c[1] + t * c[2])


def test_native_binning_segments(torch):
    """The native binning's sort and segment heads (the tile list and each
    tile's first particle, found by the sort's last radix pass) against numpy:
    a stable argsort of the tile keys and the first index of every run, on two
    consecutive steps (the second step's keys come from G2P)."""
    nc, dt = 64, 1.0 / 120
    pos, _ = scenes.dam_break(nc, seed=1)
    vel = scenes.random_velocities(pos.shape[0], seed=5, scale=2.0)
    P = native(pos.shape[0], nc)
    P.upload(pos, vel)
    for _ in range(2):
        x0, _ = P.download()  # positions at the start of the step, in the engine's order
        P.step(dt)
        keys = _tile_keys(x0[:, 0], x0[:, 1], x0[:, 2], nc)
        perm = P.read(F.BUF_PERM).astype(np.int64)
        assert np.array_equal(perm, np.argsort(keys, kind="stable"))
        sk = keys[perm]
        heads = np.flatnonzero(np.r_[True, sk[1:] != sk[:-1]])
        assert np.array_equal(P.read(F.BUF_TILE_LIST).astype(np.int64), sk[heads])
        assert np.array_equal(P.read(F.BUF_STARTS).astype(np.int64), heads)
    P.close()
