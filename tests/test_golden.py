"""The oracle against the reference itself.

tests/golden/*.npz and ref_c3_hashes.json were produced by running the
reference engine, built from its own sources, on a B200
(tests/golden/make_golden.py).  These CPU tests pin the oracle to them; the
GPU tests then hold the CUDA path to the oracle."""
import hashlib
import json
import os

import numpy as np
import pytest

from flip2_b200 import scenes
from oracle import oracle as O
from tests.util import zapron_race_voxels

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    d = np.load(os.path.join(HERE, name))
    dom = d["domain"]
    g = O.grid(float(dom[0]), float(dom[1]), float(dom[2]), int(dom[3]), int(dom[4]), int(dom[5]), float(dom[6]))
    return d, g


@pytest.fixture(scope="module")
def dam16():
    d, g = load("ref_dam16.npz")
    pos = d["pos"]
    b = O.ref_bin(pos[:, 0], pos[:, 1], pos[:, 2], g)
    return d, g, b


def test_fixture_inputs_are_the_seeded_scene():
    d, _ = load("ref_dam16.npz")
    pos, _ = scenes.dam_break(16, seed=int(d["seed"]))
    vel = scenes.random_velocities(pos.shape[0], seed=int(d["seed"]) + 100)
    assert np.array_equal(d["pos"], pos.astype(np.float64))
    assert np.array_equal(d["vel"], vel.astype(np.float64))


def test_keys_and_clamp(dam16):
    d, g, b = dam16
    assert np.array_equal(b["keys"], d["a_keys"])
    for a, k in ((b["px"], "a_px"), (b["py"], "a_py"), (b["pz"], "a_pz")):
        assert np.array_equal(a, d[k])


def test_sort_and_gather(dam16):
    d, g, b = dam16
    assert np.array_equal(b["sorted_keys"], d["s_keys"])
    assert np.array_equal(b["perm"], d["s_perm"])
    for a, k in ((b["spx"], "s_px"), (b["spy"], "s_py"), (b["spz"], "s_pz")):
        assert np.array_equal(a, d[k])


def test_cell_starts_rows_and_voxels(dam16):
    d, g, b = dam16
    assert b["nodes"] == int(d["nodes"]) and b["voxels"] == int(d["voxels"])
    for k in ("flags", "starts", "ytable", "node_voxels", "voxel_ids", "solids"):
        assert np.array_equal(b[k], d["v_" + k]), k


@pytest.mark.parametrize("name", ["ref_mix20k.npz"])
def test_binning_mix(name):
    d, g = load(name)
    pos = d["pos"]
    b = O.ref_bin(pos[:, 0], pos[:, 1], pos[:, 2], g)
    assert np.array_equal(b["keys"], d["a_keys"])
    assert np.array_equal(b["sorted_keys"], d["s_keys"])
    assert np.array_equal(b["perm"], d["s_perm"])
    assert b["nodes"] == int(d["nodes"]) and b["voxels"] == int(d["voxels"])
    for k in ("flags", "starts", "ytable", "node_voxels", "voxel_ids", "solids"):
        assert np.array_equal(b[k], d["v_" + k]), k


def test_p2g(dam16):
    """Reference P2G run with its shared memory cleared before each axis (it
    reads its weight sums before writing them, particles.cu:408-415): equal to
    the restatement up to FP64 summation order."""
    d, g, b = dam16
    for dim, k in enumerate(("p2g_ux", "p2g_uy", "p2g_uz")):
        u = O.ref_p2g(b, d["vel"][:, dim], g, dim)
        ref = d[k]
        assert np.max(np.abs(u - ref)) <= 1e-15 * np.max(np.abs(ref)), k


def test_gravity_and_divergence(dam16):
    d, g, b = dam16
    dt = float(d["dt_div"])
    uy = O.ref_gravity(b, d["p2g_uy"], dt)
    assert np.array_equal(uy, d["div_uy"])
    div = O.ref_divergence(b, d["p2g_ux"], uy, d["p2g_uz"], g)
    race = zapron_race_voxels(b, g)
    assert race.sum() < 0.2 * race.size
    assert np.array_equal(div[~race], d["div_divU"][~race])


def test_one_sor_iteration(dam16):
    d, g, b = dam16
    dt = float(d["dt_div"])
    p = np.zeros(int(d["voxels"]))
    p1, _ = O.ref_gs_pass(b, d["div_divU"], p, dt, True, g=g)
    p2, res = O.ref_gs_pass(b, d["div_divU"], p1, dt, False, g=g)
    scale = np.max(np.abs(d["gs_p"]))
    assert np.max(np.abs(p2 - d["gs_p"])) <= 1e-14 * scale
    assert np.max(np.abs(res - d["gs_res"])) <= 1e-14 * max(1.0, np.max(np.abs(d["gs_res"])))


def test_pressure_solve_dt_and_sor(dam16):
    """pressureSolve: Courant dt from the reference's getMax, then the SOR
    loop; fed the reference's divergence the SOR result agrees to rounding."""
    d, g, b = dam16
    vel = d["vel"]
    vmax = max(abs(O.ref_getmax(vel[:, k])) for k in range(3))
    dt = min(0.7 * (float(np.float32(g.cellSize)) / 4.0 / vmax), 1.0 / 24.0)
    assert dt == float(d["pr_dt"])
    term, it, p, res = O.ref_gs_solve(b, d["pr_divU"], np.zeros(int(d["voxels"])), dt, g)
    scale = np.max(np.abs(d["pr_p"]))
    assert np.max(np.abs(p - d["pr_p"])) <= 1e-12 * scale


def test_projection_g2p_advect(dam16):
    d, g, b = dam16
    dt = float(d["pr_dt"])
    U = O.ref_velocity_update(b, d["pr_p"], d["p2g_ux"], d["pr_uy"], d["p2g_uz"], dt, g)
    for u, k in zip(U, ("vu_ux", "vu_uy", "vu_uz")):
        assert np.array_equal(u, d[k]), k
    for dim, k in enumerate(("g2p_vx", "g2p_vy", "g2p_vz")):
        v = O.ref_g2p(b, b["spx"], b["spy"], b["spz"], d[("vu_ux", "vu_uy", "vu_uz")[dim]], g, dim)
        assert np.array_equal(v, d[k]), k
    for dim, k in enumerate(("adv_px", "adv_py", "adv_pz")):
        x = np.array(b[("spx", "spy", "spz")[dim]])
        O.lib().orc_ref_advect(x.size, dt, x, np.ascontiguousarray(d[("g2p_vx", "g2p_vy", "g2p_vz")[dim]]))
        assert np.array_equal(x, d[k]), k


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_c3_binning_hashes_full_size():
    """64M particles of the binning microbenchmark: keys, permutation, head
    flags and cell starts of the oracle hash to the reference's outputs."""
    h = json.load(open(os.path.join(HERE, "ref_c3_hashes.json")))
    pos = scenes.binning_mix(h["n"], domain=512, seed=h["seed"])
    g = O.grid(0.0, 0.0, 0.0, 512, 512, 512, 1.0)
    cols = [pos[:, k].astype(np.float64) for k in range(3)]
    del pos
    keys, *_ = O.ref_keys(cols[0], cols[1], cols[2], g)
    del cols
    sk, perm = O.sort_pairs(keys)
    assert sha(sk) == h["sha256_keys"]
    assert sha(perm) == h["sha256_perm"]
    flags = np.empty_like(sk)
    nodes = O.lib().orc_mark_unique_scan(sk.size, sk, flags)
    assert nodes == h["nodes"]
    assert sha(flags) == h["sha256_flags"]
    starts = np.empty(nodes, np.uint32)
    O.lib().orc_cell_starts(sk.size, flags, starts)
    assert sha(starts) == h["sha256_starts"]
