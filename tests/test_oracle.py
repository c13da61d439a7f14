"""The CPU oracle on its own (no GPU): restated reference semantics checked
against independent numpy formulations and hand-worked cases."""
import numpy as np
import pytest

from flip2_b200 import scenes
from oracle import oracle as O


def test_keys_match_numpy_restatement():
    rng = np.random.default_rng(0)
    pos = rng.uniform(-1.0, 9.0, size=(20000, 3))
    g = O.grid(0.0, 0.0, 0.0, 8, 8, 8, 1.0)
    keys, px, py, pz = O.ref_keys(pos[:, 0], pos[:, 1], pos[:, 2], g)
    c = np.clip(pos, 0.0, 8.0)
    k = np.floor(c.astype(np.float32)).astype(np.uint32)
    assert np.array_equal(keys, k[:, 0] + 8 * k[:, 1] + 64 * k[:, 2])
    assert np.array_equal(px, c[:, 0])


def test_sort_is_stable_and_matches_numpy():
    rng = np.random.default_rng(1)
    keys = rng.integers(0, 1000, size=100000).astype(np.uint32)
    ko, perm = O.sort_pairs(keys)
    ref = np.argsort(keys, kind="stable")
    assert np.array_equal(perm, ref)
    assert np.array_equal(ko, keys[ref])
    vals = rng.integers(0, 2 ** 32, size=keys.size, dtype=np.uint64).astype(np.uint32)
    _, vo = O.sort_pairs(keys, vals)
    assert np.array_equal(vo, vals[ref])


def test_sort_full_32bit_keys():
    rng = np.random.default_rng(2)
    keys = rng.integers(0, 2 ** 32, size=50000, dtype=np.uint64).astype(np.uint32)
    ko, perm = O.sort_pairs(keys)
    assert np.array_equal(perm, np.argsort(keys, kind="stable"))


def test_grid_cell_checks_of_testing_h():
    # the reference's CPU verification of its binning (engine/testing.h):
    # passes on the oracle's own sort, and catches a key out of order and a
    # sorted array whose per-cell counts differ (mistakes planted in the
    # input, on the CPU)
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 5000, 200_000).astype(np.uint32)
    ko, _ = O.sort_pairs(keys)
    assert O.ref_grid_cell_checks(keys, ko) == (0, np.unique(keys).size)
    m = ko.size // 2
    bad = ko.copy()
    bad[m] = bad[m - 1] - 1  # keys near the middle are far above 0
    assert O.ref_grid_cell_checks(keys, bad)[0] == m + 1  # 1 + the index of the first decrease
    shifted = ko.copy()
    j = int(np.searchsorted(shifted, shifted[shifted.size // 2], side="right"))
    shifted[j - 1] = shifted[j]  # one particle moves to the next cell: two counts differ
    assert O.ref_grid_cell_checks(keys, shifted)[0] == -2


def test_getmax_quirk():
    """CudaVec::getMax compares element t with t+256 only (cudaVec.cu:216-222):
    each 512-block yields the pick of its elements 0 and 256."""
    a = np.zeros(2000)
    a[5] = 100.0         # never inspected
    a[512] = -3.0        # block 1, element 0
    a[512 + 256] = 2.0   # block 1, element 256
    a[1024] = 1.0
    assert O.ref_getmax(a, True) == 0.0  # block 0 element 0 is 0; final level picks it
    b = np.zeros(600)
    b[0] = 1.5
    b[256] = -2.5
    assert O.ref_getmax(b, True) == -2.5
    assert O.ref_getmax(b, False) == 1.5


def test_binning_invariants_dam32():
    pos = scenes.dam_break(32)[0].astype(np.float64)
    g = O.grid(0.0, 0.0, 0.0, 8, 8, 8, 0.125)
    b = O.ref_bin(pos[:, 0], pos[:, 1], pos[:, 2], g)
    k = b["sorted_keys"]
    assert np.all(k[1:] >= k[:-1])
    assert b["nodes"] == np.unique(k).size
    assert np.array_equal(k[b["starts"]], np.unique(k))
    # every particle's own voxel and the 2-voxel apron stay inside the tile
    assert b["node_voxels"][-1] == b["voxels"]
    counts = np.diff(np.concatenate([[0], b["node_voxels"]]))
    assert counts.max() <= 512
    for node in range(0, b["nodes"], 17):
        s = 0 if node == 0 else b["node_voxels"][node - 1]
        ids = b["voxel_ids"][s:b["node_voxels"][node]]
        assert np.all(np.diff(ids.astype(np.int64)) > 0)


def test_ref_p2g_constant_velocity_is_reproduced():
    """With every particle moving at the same velocity, each non-solid voxel
    touched by particles reads that velocity (normalised tent weights)."""
    pos = scenes.dam_break(16)[0].astype(np.float64)
    g = O.grid(0.0, 0.0, 0.0, 4, 4, 4, 0.25)
    b = O.ref_bin(pos[:, 0], pos[:, 1], pos[:, 2], g)
    v = np.full(pos.shape[0], 0.75)
    u = O.ref_p2g(b, v, g, 0)
    touched = np.abs(u) > 1e-3
    assert np.allclose(u[touched], 0.75, rtol=1e-6)
    assert np.all(u[b["solids"] == 1] == 0.0)


def test_nat_pcg_reaches_tolerance():
    nc = 16
    P = O.nat_params(nc, nc, nc, 1.0 / nc, tol=1e-8)
    typ = np.zeros(nc ** 3, np.uint8)
    t3 = typ.reshape(nc, nc, nc)
    t3[:8, :, :] = 1  # lower half fluid (z < 8), upper half air
    rng = np.random.default_rng(0)
    b = rng.standard_normal(nc ** 3) * (typ == 1)
    x, it, rr = O.nat_pcg(typ, b, P)
    assert rr <= 1e-8
    r = b - O.nat_apply_A(typ, x, P)
    assert np.linalg.norm(r[typ == 1]) <= 1.01e-8 * np.linalg.norm(b)
    assert 5 < it < 400


def test_nat_step_projects_to_zero_divergence():
    nc = 16
    pos, vel = scenes.dam_break(nc, seed=0)
    vel = scenes.random_velocities(pos.shape[0], seed=1)
    P = O.nat_params(nc, nc, nc, 1.0 / nc, tol=1e-10, dt=1.0 / 240)
    r = O.nat_step(pos, vel, P)
    assert r["rel_residual"] <= 1e-10
    assert np.all(np.isfinite(r["pos"]))
    assert r["pos"].min() > 0 and r["pos"].max() < 1


def test_substep_runs_and_reports():
    pos = scenes.dam_break(16)[0].astype(np.float64)
    vel = scenes.random_velocities(pos.shape[0], seed=3).astype(np.float64)
    g = O.grid(0.0, 0.0, 0.0, 4, 4, 4, 0.25)
    arrs, info = O.ref_substep(pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1], vel[:, 2], g)
    assert info.nodes > 0 and info.voxels > 0 and info.dt > 0
    assert all(np.all(np.isfinite(a)) for a in arrs)
