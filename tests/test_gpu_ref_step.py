"""The reference's step math on the GPU (FLIP_MODE_REFERENCE), against the
oracle: tent-kernel P2G/G2P (particles.cu:370-662), gravity, divergence,
red-black SOR and projection (voxelSolveFunctions.cu), the pressureSolve host
loop with its Courant dt and dt halving (particles.cu:493-555), advection and
moveSolids (particles.cu:664-769).  FP64 on both sides."""
import numpy as np
import pytest

import flip2_b200 as F
from flip2_b200 import scenes
from oracle import oracle as O
from tests.util import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available()
    F.lib()
    return T


def dam(nc, seed=0, vscale=1.0):
    pos = scenes.dam_break(nc, seed=seed)[0].astype(np.float64)
    vel = scenes.random_velocities(pos.shape[0], seed=seed + 100, scale=vscale).astype(np.float64)
    g = (0.0, 0.0, 0.0, nc // 4, nc // 4, nc // 4, 4.0 / nc)
    return pos, vel, g


def test_ref_p2g_g2p_primitives(torch):
    pos, vel, g = dam(32)
    og = O.grid(*g)
    b = O.ref_bin(pos[:, 0], pos[:, 1], pos[:, 2], og)
    dev = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a).view(dt)).cuda()
    px, py, pz = dev(b["spx"], np.float64), dev(b["spy"], np.float64), dev(b["spz"], np.float64)
    # velocities keep the unsorted order: sortParticles gathers positions only (particles.cu:69-71)
    vx, vy, vz = (dev(vel[:, k].copy(), np.float64) for k in range(3))
    starts, sk = dev(b["starts"], np.int32), dev(b["sorted_keys"], np.int32)
    nv, ids, sol = dev(b["node_voxels"], np.int32), dev(b["voxel_ids"], np.int32), dev(b["solids"], np.int8)
    grid = F.make_grid(*g)
    U = F.ref_p2g(starts, sk, b["nodes"], px, py, pz, vx, vy, vz, nv, ids, sol, grid)
    for d in range(3):
        uo = O.ref_p2g(b, vel[:, d], og, d)
        assert rel_err(U[d].cpu().numpy(), uo) < 1e-12
    # G2P from the oracle's voxel velocities
    Uo = [O.ref_p2g(b, vel[:, d], og, d) for d in range(3)]
    Ud = [dev(u, np.float64) for u in Uo]
    V = F.ref_g2p(starts, sk, b["nodes"], px, py, pz, nv, ids, Ud[0], Ud[1], Ud[2], grid)
    for d in range(3):
        vo = O.ref_g2p(b, b["spx"], b["spy"], b["spz"], Uo[d], og, d)
        assert rel_err(V[d].cpu().numpy(), vo) < 1e-12


def _oracle_pressure(b, U, vel, og, frame_dt=1.0 / 24.0, elapsed=0.0):
    """Particles::pressureSolve (particles.cu:507-555) written over oracle calls."""
    vmax = max(abs(O.ref_getmax(vel[:, 0])), abs(O.ref_getmax(vel[:, 1])), abs(O.ref_getmax(vel[:, 2])))
    vs = float(np.float32(og.cellSize)) / 4.0
    dt = 0.7 * (vs / vmax)
    if frame_dt - elapsed < dt:
        dt = frame_dt - elapsed
    ux, uy, uz = U
    uy = O.ref_gravity(b, uy, dt)
    div = O.ref_divergence(b, ux, uy, uz, og)
    p = np.zeros(b["voxels"])
    prev = 100.0
    total = 0
    while True:
        term, it, p, res = O.ref_gs_solve(b, div, p, dt, og)
        total += it
        if not (prev - term > 0):
            break
        if term < 0.01:
            break
        uy = O.ref_gravity(b, uy, dt, remove=True)
        dt /= 2.0
        p = np.zeros(b["voxels"])
        uy = O.ref_gravity(b, uy, dt)
        prev = term
        div = O.ref_divergence(b, ux, uy, uz, og)
    return dict(dt=dt, p=p, res=res, div=div, ux=ux, uy=uy, uz=uz, term=term, iters=total)


@pytest.mark.parametrize("nc", [16, 32])
def test_ref_engine_substep_vs_oracle(torch, nc):
    pos, vel, g = dam(nc)
    og = O.grid(*g)
    P = F.Particles(pos.shape[0], mode=F.MODE_REFERENCE)
    P.setDomain(*g)
    P.upload(pos, vel)
    P.initialize()
    b = O.ref_bin(pos[:, 0], pos[:, 1], pos[:, 2], og)
    info = P.info()
    assert info.nodes == b["nodes"] and info.voxels == b["voxels"]
    assert np.array_equal(P.read(F.BUF_KEYS), b["sorted_keys"])
    assert np.array_equal(P.read(F.BUF_PERM), b["perm"])
    assert np.array_equal(P.read(F.BUF_FLAGS), b["flags"])
    assert np.array_equal(P.read(F.BUF_STARTS), b["starts"])
    assert np.array_equal(P.read(F.BUF_YTABLE), b["ytable"])
    assert np.array_equal(P.read(F.BUF_NODE_VOXELS), b["node_voxels"])
    assert np.array_equal(P.read(F.BUF_VOXEL_IDS), b["voxel_ids"])
    assert np.array_equal(P.read(F.BUF_SOLIDS), b["solids"])
    assert np.array_equal(P.read(F.BUF_PX), b["spx"])
    # P2G
    P.particleVelToVoxels()
    U = [O.ref_p2g(b, vel[:, d], og, d) for d in range(3)]
    for d, which in enumerate((F.BUF_UX, F.BUF_UY, F.BUF_UZ)):
        assert rel_err(P.read(which), U[d]) < 1e-12
    # pressure: the GPU's own P2G output feeds the oracle so both start equal
    Ug = [P.read(w) for w in (F.BUF_UX, F.BUF_UY, F.BUF_UZ)]
    ref = _oracle_pressure(b, Ug, vel, og)
    P.pressureSolve()
    info = P.info()
    assert info.dt == pytest.approx(ref["dt"], rel=1e-12)
    assert rel_err(P.read(F.BUF_DIVU), ref["div"]) < 1e-10
    assert rel_err(P.read(F.BUF_P), ref["p"], floor=1e-30) < 1e-8
    assert info.pressure_iters == ref["iters"]
    # projection
    P.updateVoxelVelocities()
    Uo = O.ref_velocity_update(b, ref["p"], ref["ux"], ref["uy"], ref["uz"], ref["dt"], og)
    Ug = [P.read(w) for w in (F.BUF_UX, F.BUF_UY, F.BUF_UZ)]
    for d in range(3):
        assert rel_err(Ug[d], Uo[d]) < 1e-8
    # G2P + advection
    P.voxelVelsToParticles()
    P.advectParticles()
    pg, vg = P.download()
    for d in range(3):
        vo = O.ref_g2p(b, b["spx"], b["spy"], b["spz"], Ug[d], og, d)
        assert rel_err(vg[:, d], vo) < 1e-12
        xo = np.array(b[("spx", "spy", "spz")[d]])
        O.lib().orc_ref_advect(xo.size, info.dt, xo, np.ascontiguousarray(vg[:, d]))
        assert np.array_equal(pg[:, d], xo)
    P.close()


def test_ref_move_solids_targets(torch):
    """moveSolids: which particles are re-seeded and into which voxel (the
    random offsets come from curand's device API and are only range-checked)."""
    pos, vel, g = dam(16, vscale=8.0)
    og = O.grid(*g)
    P = F.Particles(pos.shape[0], mode=F.MODE_REFERENCE)
    P.setDomain(*g)
    P.upload(pos, vel)
    P.initialize()
    b = O.ref_bin(pos[:, 0], pos[:, 1], pos[:, 2], og)
    # push particles outside their tiles / into solid voxels: advect with a big dt
    x = [b["spx"] + 0.06 * vel[:, 0], b["spy"] + 0.06 * vel[:, 1], b["spz"] + 0.06 * vel[:, 2]]
    P.upload(np.stack(x, 1), vel)  # uploads in the sorted order the keys refer to
    tgt = O.ref_move_targets(b, x[0], x[1], x[2], og)
    P.moveSolidParticles()
    pg, _ = P.download()
    moved = tgt != 0xFFFFFFFF
    assert moved.sum() > 0
    assert np.array_equal(pg[~moved, 0], x[0][~moved])
    scw = float(np.float32(og.cellSize) / np.float32(4.0))
    keys = b["sorted_keys"]
    X = og.sizeX
    gx = (keys % (X * og.sizeY)) % X
    gy = (keys % (X * og.sizeY)) // X
    gz = keys // (X * og.sizeY)
    for d, gidx in enumerate((gx, gy, gz)):
        v = tgt[moved]
        comp = (v % 8, (v % 64) // 8, v // 64)[d].astype(np.int64)
        lo = gidx[moved] * og.cellSize + (comp - 2) * scw
        got = pg[moved, d]
        assert np.all(got >= lo - 1e-12) and np.all(got <= lo + scw + 1e-12)
    P.close()


def test_ref_engine_errors(torch):
    P = F.Particles(100, mode=F.MODE_REFERENCE)
    with pytest.raises(F.FlipError) as ei:
        P.initialize()
    assert ei.value.status == 5
    P.setDomain(0, 0, 0, 4, 4, 4, 0.25)
    with pytest.raises(F.FlipError) as ei:
        P.particleVelToVoxels()
    assert ei.value.status == 5
    with pytest.raises(F.FlipError) as ei:
        P.upload(np.zeros((99, 3)))
    assert ei.value.status == 1
    P.close()
