"""The oracle's multilevel preconditioner (CPU): the level plan, one V-cycle
without the network against an independent numpy restatement, and FCG with
it against Jacobi-PCG on the same problem."""
import numpy as np

from oracle import oracle as O

AIR, FLUID, SOLID = 0, 1, 2


def problem(shape, seed):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    t = np.where(j < 0.7 * ny, FLUID, AIR).astype(np.uint8)
    for _ in range(6):
        c = rng.uniform(0, 1, 3) * np.array([nx, ny, nz])
        rad = rng.uniform(2.0, 5.0)
        t[(i - c[0]) ** 2 + (j - c[1]) ** 2 + (k - c[2]) ** 2 < rad * rad] = SOLID
    b = np.where(t == FLUID, rng.standard_normal(t.shape), 0.0)
    return t, b


def apply_A(t, x):
    """7-point operator on the fluid cells of t ([z][y][x]); outside the box is solid"""
    fl = t == FLUID
    y = np.zeros_like(x)
    for ax in range(3):
        for sgn in (1, -1):
            nb_t = np.full(t.shape, SOLID, np.uint8)
            nb_x = np.zeros_like(x)
            src = [slice(None)] * 3
            dst = [slice(None)] * 3
            if sgn == 1:
                dst[ax], src[ax] = slice(0, -1), slice(1, None)
            else:
                dst[ax], src[ax] = slice(1, None), slice(0, -1)
            nb_t[tuple(dst)] = t[tuple(src)]
            nb_x[tuple(dst)] = x[tuple(src)]
            y += np.where(nb_t != SOLID, x, 0.0) - np.where(nb_t == FLUID, nb_x, 0.0)
    return np.where(fl, y, 0.0)


def dinv(t):
    d = apply_A(t, np.ones(t.shape)) * 0.0
    cnt = np.zeros(t.shape)
    for ax in range(3):
        for sgn in (1, -1):
            nb = np.full(t.shape, SOLID, np.uint8)
            src = [slice(None)] * 3
            dst = [slice(None)] * 3
            if sgn == 1:
                dst[ax], src[ax] = slice(0, -1), slice(1, None)
            else:
                dst[ax], src[ax] = slice(1, None), slice(0, -1)
            nb[tuple(dst)] = t[tuple(src)]
            cnt += nb != SOLID
    return np.where((t == FLUID) & (cnt > 0), 1.0 / np.maximum(cnt, 1), d)


def coarsen(t):
    nz, ny, nx = t.shape
    c = t.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2).transpose(0, 2, 4, 1, 3, 5).reshape(nz // 2, ny // 2, nx // 2, 8)
    out = np.full(c.shape[:3], SOLID, np.uint8)
    out[(c == FLUID).any(-1)] = FLUID
    out[(c == AIR).any(-1)] = AIR
    return out


def vcycle(ts, l, r, w=2.0 / 3.0):
    t = ts[l]
    di = dinv(t)
    sweep = lambda x: np.where(t == FLUID, x + w * di * (r - apply_A(t, x)), 0.0)
    if l == len(ts) - 1:
        return sweep(sweep(w * di * r))
    x = sweep(w * di * r)
    res = r - apply_A(t, x)
    nz, ny, nx = t.shape
    rc = 0.5 * res.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2).sum(axis=(1, 3, 5))
    rc = np.where(ts[l + 1] == FLUID, rc, 0.0)
    ec = vcycle(ts, l + 1, rc, w)
    x = np.where(t == FLUID, x + ec.repeat(2, 0).repeat(2, 1).repeat(2, 2), 0.0)
    return sweep(sweep(x))


def test_level_plan():
    assert O.mg_levels((64, 64, 64)) == [(64, 64, 64), (32, 32, 32), (16, 16, 16)]
    assert O.mg_levels((256, 256, 256))[-1] == (16, 16, 16)
    assert len(O.mg_levels((256, 256, 256))) == 5
    # ceil halving, padded to whole 8^3 tiles
    assert O.mg_levels((48, 40, 56)) == [(48, 40, 56), (24, 24, 32), (16, 16, 16)]
    assert O.mg_levels((16, 16, 16)) == [(16, 16, 16)]


def test_vcycle_matches_numpy():
    shape = (32, 32, 32)
    t, _ = problem(shape, 0)
    r = np.where(t == FLUID, np.random.default_rng(1).standard_normal(t.shape), 0.0).astype(np.float32)
    z = O.mg_apply(t.ravel(), r.ravel(), np.zeros(O.lib().orc_lp_num_weights(), np.float32), shape, mode=1)
    ts = [t, coarsen(t)]
    zn = vcycle(ts, 0, r.astype(np.float64))
    assert np.max(np.abs(z - zn.ravel())) <= 1e-12 * np.max(np.abs(zn))


def test_vcycle_is_symmetric_without_network():
    # damped Jacobi before and after, R = P^T / 2 up to the coarse scaling:
    # u.M(v) = v.M(u)
    shape = (32, 32, 32)
    t, _ = problem(shape, 2)
    rng = np.random.default_rng(3)
    u = np.where(t == FLUID, rng.standard_normal(t.shape), 0.0).astype(np.float32).ravel()
    v = np.where(t == FLUID, rng.standard_normal(t.shape), 0.0).astype(np.float32).ravel()
    w0 = np.zeros(O.lib().orc_lp_num_weights(), np.float32)
    mu = O.mg_apply(t.ravel(), u, w0, shape, mode=1)
    mv = O.mg_apply(t.ravel(), v, w0, shape, mode=1)
    a, b = float(v @ mu), float(u @ mv)
    assert abs(a - b) <= 1e-10 * max(abs(a), 1.0)
    assert float(u @ mu) > 0.0


def test_fcg_beats_jacobi_pcg():
    shape = (64, 64, 64)
    t, b = problem(shape, 4)
    w0 = np.zeros(O.lib().orc_lp_num_weights(), np.float32)
    x, it, rr = O.mg_fcg(t.ravel(), b.ravel(), w0, shape, mode=1, max_iter=400)
    assert rr <= 1e-6
    _, itp, rrp = O.nat_pcg(t.ravel(), b.ravel(), O.nat_params(*shape, 1.0, tol=1e-6, max_iter=20000))
    assert rrp <= 1e-6
    assert it * 4 < itp


def test_fcg_on_padded_levels():
    # 48 x 40 x 56: the coarse levels are padded with solid cells to whole
    # 8^3 tiles (24 x 24 x 32, then 16^3); the V-cycle still preconditions FCG
    # to the tolerance, and its operator is still symmetric
    shape = (48, 40, 56)
    assert O.mg_levels(shape)[1:] == [(24, 24, 32), (16, 16, 16)]
    t, b = problem(shape, 6)
    w0 = np.zeros(O.lib().orc_lp_num_weights(), np.float32)
    x, it, rr = O.mg_fcg(t.ravel(), b.ravel(), w0, shape, mode=1, max_iter=400)
    assert rr <= 1e-6 and it < 200
    rng = np.random.default_rng(7)
    u = np.where(t == FLUID, rng.standard_normal(t.shape), 0.0).astype(np.float32).ravel()
    v = np.where(t == FLUID, rng.standard_normal(t.shape), 0.0).astype(np.float32).ravel()
    a = float(v @ O.mg_apply(t.ravel(), u, w0, shape, mode=1))
    c = float(u @ O.mg_apply(t.ravel(), v, w0, shape, mode=1))
    assert abs(a - c) <= 1e-10 * max(abs(a), 1.0)


def test_single_level():
    # every axis at most 16 cells: the hierarchy is the grid alone and the
    # V-cycle is the coarsest level's start and two sweeps; FCG with it
    # still meets the tolerance
    for shape in ((16, 16, 16), (16, 8, 16)):
        assert O.mg_levels(shape) == [shape]
        t, b = problem(shape, 8)
        r = np.where(t == FLUID, np.random.default_rng(9).standard_normal(t.shape), 0.0).astype(np.float32)
        w0 = np.zeros(O.lib().orc_lp_num_weights(), np.float32)
        z = O.mg_apply(t.ravel(), r.ravel(), w0, shape, mode=1)
        zn = vcycle([t], 0, r.astype(np.float64))
        assert np.max(np.abs(z - zn.ravel())) <= 1e-12 * np.max(np.abs(zn))
        x, it, rr = O.mg_fcg(t.ravel(), b.ravel(), w0, shape, mode=1, max_iter=400)
        assert rr <= 1e-6


def test_degenerate_problems():
    # b = 0 on a fluid region, and a grid without fluid cells: both solves
    # stop before their first iteration with x = 0 and a zero residual, and
    # the V-cycle of a zero residual is zero
    shape = (32, 32, 32)
    t, _ = problem(shape, 10)
    w0 = np.zeros(O.lib().orc_lp_num_weights(), np.float32)
    for typ in (t, np.zeros_like(t)):
        b = np.zeros(typ.size)
        x, it, rr = O.mg_fcg(typ.ravel(), b, w0, shape, mode=1, max_iter=50)
        assert it == 0 and rr == 0.0 and not np.any(x)
        x, it, rr = O.nat_pcg(typ.ravel(), b, O.nat_params(*shape, 1.0, tol=1e-6, max_iter=50))
        assert it == 0 and rr == 0.0 and not np.any(x)
        assert not np.any(O.mg_apply(typ.ravel(), np.zeros(typ.size, np.float32), w0, shape, mode=1))
