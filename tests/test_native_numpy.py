"""An independent numpy restatement of the native step, which pins the FP64
oracle (oracle/flip_oracle.c orc_nat_step_ex) that the GPU parity tests trust.

The native step has no reference counterpart, so its oracle is checked here
against a second implementation written from the step's definition instead of
from the oracle's code: vectorised over particles, a direct sparse solve
instead of PCG, scatter through np.add.at.  It covers, on a 16^3 grid with a
few hundred particles (some within half a cell of the walls, a few inside the
clamp margin):
  * trilinear weights on the staggered MAC grid, with the wall faces of each
    component (own-axis index 0 and n) excluded from the sums;
  * the cell classification, gravity on the y faces that touch fluid, and the
    divergence right-hand side;
  * the pressure of the 7-point system (solid walls, air cells Dirichlet 0);
  * the projection of the faces next to fluid;
  * G2P: the FLIP 0.95 blend of the grid-velocity change, and RK2 (midpoint)
    advection through the projected grid, clamped 1e-3 h inside the box.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import oracle as O

NC = 16
H = 1.0 / NC
G = -9.8
FLIP = 0.95


def cell_of(p):
    """Cell of float32 positions in float32 arithmetic, clamped into [0, NC)."""
    t = np.floor((p.astype(np.float32) - np.float32(0.0)) / np.float32(H))
    c = np.where(t >= NC, NC - 1, t).astype(np.int64)
    return np.where(t > 0, c, 0)


def axis_stencil(s, m):
    """Base node and fraction of sample coordinate s on an axis of nodes
    0..m: s clamped into [0, m], base into [0, m - 1]."""
    s = np.clip(s, 0.0, float(m))
    b = np.clip(np.floor(s).astype(np.int64), 0, m - 1)
    return b, s - b


def corners(c, g):
    """The 8 (node index triple, weight) pairs of component c at grid
    coordinates g (n, 3), wall faces of component c flagged invalid."""
    sh = [0.0 if a == c else 0.5 for a in range(3)]
    ms = [NC if a == c else NC - 1 for a in range(3)]
    base, frac = zip(*(axis_stencil(g[:, a] - sh[a], ms[a]) for a in range(3)))
    out = []
    for dk in (0, 1):
        for dj in (0, 1):
            for di in (0, 1):
                d = (di, dj, dk)
                idx = [base[a] + d[a] for a in range(3)]
                w = np.ones(g.shape[0])
                for a in range(3):
                    w = w * (frac[a] if d[a] else 1.0 - frac[a])
                own = idx[c]
                valid = (own != 0) & (own != NC)
                out.append((idx, w, valid))
    return out


def p2g(pos, vel):
    g = pos.astype(np.float64) / H
    U = []
    for c in range(3):
        num = np.zeros((NC, NC, NC))
        den = np.zeros((NC, NC, NC))
        for (i, j, k), w, ok in corners(c, g):
            np.add.at(num, (k[ok], j[ok], i[ok]), (w * vel[:, c].astype(np.float64))[ok])
            np.add.at(den, (k[ok], j[ok], i[ok]), w[ok])
        U.append(np.divide(num, den, out=np.zeros_like(num), where=den > 0))
    return U


def sample(F, c, g):
    s = np.zeros(g.shape[0])
    for (i, j, k), w, ok in corners(c, g):
        ii, jj, kk = (np.where(ok, x, 0) for x in (i, j, k))
        s += np.where(ok, w * F[kk, jj, ii], 0.0)
    return s


def numpy_step(pos, vel, dt):
    U = p2g(pos, vel)
    Uold = [u.copy() for u in U]
    fluid = np.zeros((NC, NC, NC), bool)
    ci = [cell_of(pos[:, a]) for a in range(3)]
    fluid[ci[2], ci[1], ci[0]] = True
    # faces: index (k, j, i) is the negative face of cell (i, j, k); the
    # own-axis index 0 is a wall face (0), the positive wall is not stored
    for c in range(3):
        ax = 2 - c  # array axis of component c
        wall = np.zeros((NC, NC, NC), bool)
        sl = [slice(None)] * 3
        sl[ax] = 0
        wall[tuple(sl)] = True
        U[c][wall] = 0.0
        if c == 1:
            below = np.roll(fluid, 1, axis=ax)
            below[tuple(sl)] = False
            U[c][(fluid | below) & ~wall] += G * dt
    # b = -div U on fluid cells
    div = np.zeros((NC, NC, NC))
    for c in range(3):
        ax = 2 - c
        up = np.roll(U[c], -1, axis=ax)
        sl = [slice(None)] * 3
        sl[ax] = NC - 1
        up[tuple(sl)] = 0.0
        div += up - U[c]
    b = np.where(fluid, -div, 0.0)
    # 7-point system on the fluid cells: the diagonal counts the non-solid
    # neighbours (walls are solid), fluid neighbours couple with -1
    ids = -np.ones((NC, NC, NC), np.int64)
    fk = np.argwhere(fluid)
    ids[fluid] = np.arange(fk.shape[0])
    rows, cols, vals = [], [], []
    for r, (k, j, i) in enumerate(fk):
        d = 0
        for dk, dj, di in ((0, 0, -1), (0, 0, 1), (0, -1, 0), (0, 1, 0), (-1, 0, 0), (1, 0, 0)):
            kk, jj, ii = k + dk, j + dj, i + di
            if not (0 <= kk < NC and 0 <= jj < NC and 0 <= ii < NC):
                continue
            d += 1
            if fluid[kk, jj, ii]:
                rows.append(r); cols.append(ids[kk, jj, ii]); vals.append(-1.0)
        rows.append(r); cols.append(r); vals.append(float(d))
    A = sp.csr_matrix((vals, (rows, cols)), shape=(fk.shape[0],) * 2)
    x = spla.spsolve(A, b[fluid])
    phi = np.zeros((NC, NC, NC))
    phi[fluid] = x
    # projection of the faces with a fluid cell on either side (walls stay 0)
    for c in range(3):
        ax = 2 - c
        pa = np.roll(phi, 1, axis=ax)
        fa = np.roll(fluid, 1, axis=ax)
        sl = [slice(None)] * 3
        sl[ax] = 0
        inner = np.ones((NC, NC, NC), bool)
        inner[tuple(sl)] = False
        m = inner & (fluid | fa)
        U[c][m] -= (phi - pa)[m]
    # G2P: FLIP blend, then the RK2 midpoint through the projected grid
    g0 = pos.astype(np.float64) / H
    un = np.stack([sample(U[c], c, g0) for c in range(3)], 1)
    uo = np.stack([sample(Uold[c], c, g0) for c in range(3)], 1)
    v = FLIP * (vel.astype(np.float64) + (un - uo)) + (1.0 - FLIP) * un
    xm = pos.astype(np.float64) + 0.5 * dt * un
    gm = xm / H
    um = np.stack([sample(U[c], c, gm) for c in range(3)], 1)
    xn = np.clip(pos.astype(np.float64) + dt * um, 1e-3 * H, 1.0 - 1e-3 * H)
    return dict(u=Uold, u_proj=U, phi=phi, pos=xn.astype(np.float32), vel=v.astype(np.float32), fluid=fluid)


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_native_step_matches_numpy_restatement(seed):
    rng = np.random.default_rng(seed)
    n = 400
    pos = np.empty((n, 3), np.float32)
    pos[:300] = rng.uniform([0.05, 0.02, 0.1], [0.6, 0.55, 0.95], size=(300, 3))
    # particles within half a cell of the walls, where wall faces drop out
    walls = rng.uniform(0.0, 0.5 * H, size=(100, 3))
    hi = rng.random((100, 3)) < 0.5
    pos[300:] = np.where(hi, 1.0 - walls, walls)
    pos[300:, 1] = rng.uniform(0.0, 0.5, 100)
    # and a few closer to a wall than the clamp margin (1e-3 h)
    pos[390:, 0] = rng.uniform(0.0, 5e-4 * H, 10)
    pos = pos.astype(np.float32)
    vel = rng.normal(0.0, 1.0, size=(n, 3)).astype(np.float32)
    dt = 1.0 / 60.0  # fast: some particles hit the clamp
    mine = numpy_step(pos, vel, dt)
    ref = O.nat_step(pos, vel, O.nat_params(NC, NC, NC, H, dt=dt, tol=1e-14, max_iter=20000))
    lin = lambda a: a.reshape(NC, NC, NC)  # oracle arrays are x fastest: (k, j, i)
    assert int(mine["fluid"].sum()) == ref["fluid_cells"]
    for c, key in enumerate("uvw"):
        np.testing.assert_allclose(lin(ref[key]), mine["u"][c], rtol=0, atol=1e-12)
        scale = np.max(np.abs(mine["u_proj"][c]))
        np.testing.assert_allclose(lin(ref[key + "_proj"]), mine["u_proj"][c], rtol=0, atol=1e-9 * scale)
    np.testing.assert_allclose(lin(ref["phi"]), mine["phi"], rtol=0, atol=1e-9 * np.max(np.abs(mine["phi"])))
    # float32 outputs of FP64 arithmetic: equal to within one float32 rounding
    np.testing.assert_allclose(ref["vel"], mine["vel"], rtol=2e-7, atol=1e-7)
    np.testing.assert_allclose(ref["pos"], mine["pos"], rtol=2e-7, atol=1e-9)
    # the clamp engaged somewhere and some particles sat next to a wall face
    assert np.any(np.abs(mine["pos"] - np.float32(1e-3 * H)) < 1e-7) or np.any(
        np.abs(mine["pos"] - np.float32(1.0 - 1e-3 * H)) < 1e-7)
