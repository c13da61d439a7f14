"""Binning on the GPU, bit-exact against the oracle: root-cell keys, the
onesweep radix sort (keys + permutation), prefix sums, segment heads (the
reference's uniqueGridNodeIndices / gridNodeIndicesToFirstParticleIndex), the
y-row table and the sparse-voxel compaction (particleToGridFunctions.cu,
radixSortKernels.cu, parallelPrefixSumKernels.cu, particles.cu:88-368)."""
import numpy as np
import pytest

import flip2_b200 as F
from flip2_b200 import scenes
from oracle import oracle as O
from tests.util import u32

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available(), "GPU tests need a CUDA device"
    F.lib()
    return T


def to_dev(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a).view(dtype)).cuda()


# ------------------------------------------------------------------ keys
@pytest.mark.parametrize("case", ["dam32", "mix", "outside"])
def test_ref_keys_bitexact(torch, case):
    if case == "dam32":
        pos = scenes.dam_break(32)[0].astype(np.float64)
        g = (0.0, 0.0, 0.0, 8, 8, 8, 0.125)
    elif case == "mix":
        pos = scenes.binning_mix(200000, domain=512, seed=1).astype(np.float64)
        g = (0.0, 0.0, 0.0, 512, 512, 512, 1.0)
    else:  # clamp paths, a negative corner and a non power-of-two cell size
        rng = np.random.default_rng(5)
        pos = rng.uniform(-12.0, 18.0, size=(50000, 3))
        g = (-10.0, -10.0, -10.0, 100, 100, 100, 0.25)
    og = O.grid(*g)
    keys_o, cx, cy, cz = O.ref_keys(pos[:, 0], pos[:, 1], pos[:, 2], og)
    px, py, pz = (to_dev(torch, pos[:, k].copy(), np.float64) for k in range(3))
    keys, idx = F.ref_keys(px, py, pz, F.make_grid(*g), with_index=True)
    torch.cuda.synchronize()
    assert np.array_equal(u32(keys), keys_o)
    assert np.array_equal(idx.cpu().numpy(), np.arange(pos.shape[0], dtype=np.int32))
    for d, c in zip((px, py, pz), (cx, cy, cz)):
        assert np.array_equal(d.cpu().numpy(), c)


def test_ref_keys_upper_face_alias(torch):
    """A particle exactly on the upper face gets x == sizeX, which aliases into
    the next row (particleToGridFunctions.cu:25-27,40-43)."""
    g = (0.0, 0.0, 0.0, 4, 4, 4, 1.0)
    pos = np.array([[4.0, 0.5, 0.5], [0.5, 4.0, 0.5], [0.5, 0.5, 4.0], [5.0, 5.0, 5.0], [3.999, 0.0, 0.0]])
    keys_o, *_ = O.ref_keys(pos[:, 0], pos[:, 1], pos[:, 2], O.grid(*g))
    px, py, pz = (to_dev(torch, pos[:, k].copy(), np.float64) for k in range(3))
    keys = F.ref_keys(px, py, pz, F.make_grid(*g))
    assert np.array_equal(u32(keys), keys_o)
    assert keys_o[0] == 4 and keys_o[3] == 4 + 4 * 4 + 4 * 16


# ------------------------------------------------------------------ sort
def _sort_check(torch, keys_np, key_bits, with_vals=False, inplace=False):
    n = keys_np.size
    k_dev = to_dev(torch, keys_np.astype(np.uint32), np.int32)
    vals_np = None
    v_dev = None
    if with_vals:
        vals_np = np.random.default_rng(9).integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
        v_dev = to_dev(torch, vals_np, np.int32)
    if inplace:
        ok, ov, scr = F.sort_pairs(k_dev, v_dev, key_bits=key_bits, out_keys=k_dev, out_vals=v_dev,
                                   return_scratch=True)
    else:
        ok, ov, scr = F.sort_pairs(k_dev, v_dev, key_bits=key_bits, return_scratch=True)
    torch.cuda.synchronize()
    ko, vo = O.sort_pairs(keys_np.astype(np.uint32), vals_np)
    assert np.array_equal(u32(ok), ko)
    assert np.array_equal(u32(ov), vo)
    assert int(scr[:4].cpu().numpy().view(np.uint32)[0]) == 0, "device error word set"


@pytest.mark.parametrize("n", [1, 2, 31, 4095, 4096, 4097, 8192 + 5, 100003])
@pytest.mark.parametrize("key_bits", [1, 8, 9, 17, 24, 32])
def test_sort_sizes_and_bits(torch, n, key_bits):
    rng = np.random.default_rng(n * 131 + key_bits)
    hi = 2 ** key_bits
    keys = rng.integers(0, hi, size=n, dtype=np.uint64).astype(np.uint32)
    _sort_check(torch, keys, key_bits)


@pytest.mark.parametrize("pattern", ["equal", "descending", "few", "zipf"])
def test_sort_patterns(torch, pattern):
    n = 300000
    rng = np.random.default_rng(3)
    if pattern == "equal":
        keys = np.full(n, 12345, np.uint32)
    elif pattern == "descending":
        keys = np.arange(n, 0, -1).astype(np.uint32)
    elif pattern == "few":
        keys = rng.integers(0, 4, size=n).astype(np.uint32) * 0x01010101
    else:
        keys = np.minimum(rng.zipf(1.3, size=n), 2 ** 20).astype(np.uint32)
    _sort_check(torch, keys, 32, with_vals=(pattern == "few"))


@pytest.mark.parametrize("key_bits", [8, 16, 24, 32])
def test_sort_in_place(torch, key_bits):
    rng = np.random.default_rng(key_bits)
    keys = rng.integers(0, 2 ** key_bits, size=50001, dtype=np.uint64).astype(np.uint32)
    _sort_check(torch, keys, key_bits, with_vals=True, inplace=True)


def test_sort_c3_full_size(torch):
    """64M keys of the binning microbenchmark: size-independent properties
    (sorted, permutation, stable, gather-consistent)."""
    n = 1 << 26
    pos = scenes.binning_mix(n, domain=512, seed=1)
    g = F.make_grid(0.0, 0.0, 0.0, 512, 512, 512, 1.0)
    pd = [torch.from_numpy(pos[:, k].astype(np.float64)).cuda() for k in range(3)]
    del pos
    keys = F.ref_keys(pd[0], pd[1], pd[2], g)
    del pd
    ok, ov, scr = F.sort_pairs(keys, key_bits=28, return_scratch=True)
    torch.cuda.synchronize()
    assert int(scr[:4].cpu().numpy().view(np.uint32)[0]) == 0
    ku = ok.to(torch.int64) & 0xFFFFFFFF
    assert bool((ku[1:] >= ku[:-1]).all())
    pu = ov.to(torch.int64)
    assert bool((torch.sort(pu).values == torch.arange(n, device=pu.device)).all())
    same = ku[1:] == ku[:-1]
    assert bool((pu[1:][same] > pu[:-1][same]).all()), "not stable"
    assert bool((keys[pu] == ok).all())
    # multiset of keys unchanged (the reference's validateGridCellOrdering, testing.h:34-53)
    k_in = torch.sort(keys.to(torch.int64) & 0xFFFFFFFF).values
    assert bool((k_in == ku).all())


# ------------------------------------------------------------------ scans
@pytest.mark.parametrize("n", [1, 7, 4096, 4097, 1 << 20, (1 << 22) + 3])
def test_inclusive_scan(torch, n):
    rng = np.random.default_rng(n)
    x = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
    if n > 1000:
        x[::3] = rng.integers(0, 4, size=x[::3].size)
    d = to_dev(torch, x, np.int32)
    o, scr = F.inclusive_scan(d, return_scratch=True)
    torch.cuda.synchronize()
    ref = np.cumsum(x.astype(np.uint64)).astype(np.uint32)
    assert np.array_equal(u32(o), ref)
    # in place
    F.inclusive_scan(d, out=d)
    assert np.array_equal(u32(d), ref)


@pytest.mark.parametrize("n", [1, 5000, 300001])
def test_segment_heads(torch, n):
    rng = np.random.default_rng(n + 1)
    keys = np.sort(rng.integers(0, max(2, n // 7), size=n).astype(np.uint32))
    flags_o = np.empty(n, np.uint32)
    L = O.lib()
    cnt_o = L.orc_mark_unique_scan(n, keys, flags_o)
    starts_o = np.empty(cnt_o, np.uint32)
    L.orc_cell_starts(n, flags_o, starts_o)
    flags, starts, nk, cnt = F.segment_heads(to_dev(torch, keys, np.int32))
    assert cnt == cnt_o
    assert np.array_equal(u32(flags), flags_o)
    assert np.array_equal(u32(starts), starts_o)
    assert np.array_equal(u32(nk), keys[starts_o])


# ------------------------------------------------------- full binning
def _gpu_bin(torch, pos, g):
    px, py, pz = (to_dev(torch, pos[:, k].copy(), np.float64) for k in range(3))
    grid = F.make_grid(*g)
    keys = F.ref_keys(px, py, pz, grid)
    sk, perm = F.sort_pairs(keys, key_bits=32)
    pl = perm.long()
    spx, spy, spz = px[pl], py[pl], pz[pl]
    flags, starts, _, nodes = F.segment_heads(sk)
    ytab = F.ref_ydim_rows(starts, sk, nodes, grid)
    counts, nv, ids, sol = F.ref_voxels(starts, sk, nodes, spx, spy, spz, grid)
    torch.cuda.synchronize()
    return dict(keys=u32(keys), sorted_keys=u32(sk), perm=u32(perm), flags=u32(flags), starts=u32(starts),
                nodes=nodes, ytable=u32(ytab), counts=u32(counts), node_voxels=u32(nv), voxel_ids=u32(ids),
                solids=sol.cpu().numpy(), spx=spx, spy=spy, spz=spz)


@pytest.mark.parametrize("case", ["dam32", "dam16", "mix64"])
def test_ref_binning_pipeline_bitexact(torch, case):
    if case.startswith("dam"):
        nc = int(case[3:])
        pos = scenes.dam_break(nc, seed=0)[0].astype(np.float64)
        g = (0.0, 0.0, 0.0, nc // 4, nc // 4, nc // 4, 4.0 / nc)
    else:
        pos = scenes.binning_mix(20000, domain=64, seed=1).astype(np.float64)
        g = (0.0, 0.0, 0.0, 64, 64, 64, 1.0)
    b_o = O.ref_bin(pos[:, 0], pos[:, 1], pos[:, 2], O.grid(*g))
    b_g = _gpu_bin(torch, pos, g)
    for k in ("keys", "sorted_keys", "perm", "flags", "starts", "ytable", "counts", "node_voxels", "voxel_ids"):
        assert np.array_equal(b_g[k], b_o[k]), k
    assert b_g["nodes"] == b_o["nodes"]
    assert np.array_equal(b_g["solids"], b_o["solids"])


def test_c3_full_size_matches_reference_hashes(torch):
    """64M particles in 512^3: every binning output of the CUDA path hashes
    to the reference engine's own output (tests/golden/ref_c3_hashes.json)."""
    import hashlib
    import json
    import os
    h = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_c3_hashes.json")))
    sha = lambda t: hashlib.sha256(np.ascontiguousarray(t.cpu().numpy()).tobytes()).hexdigest()
    pos = scenes.binning_mix(h["n"], domain=512, seed=h["seed"])
    g = F.make_grid(0.0, 0.0, 0.0, 512, 512, 512, 1.0)
    pd = [torch.from_numpy(pos[:, k].astype(np.float64)).cuda() for k in range(3)]
    del pos
    keys = F.ref_keys(pd[0], pd[1], pd[2], g)
    sk, perm = F.sort_pairs(keys, key_bits=28)
    del keys
    assert sha(sk) == h["sha256_keys"]
    assert sha(perm) == h["sha256_perm"]
    pl = perm.long()
    sp = [p[pl] for p in pd]
    del pd, pl
    flags, starts, _, nodes = F.segment_heads(sk, want_keys=False)
    assert nodes == h["nodes"]
    assert sha(flags) == h["sha256_flags"]
    assert sha(starts) == h["sha256_starts"]
    del flags
    counts, nv, ids, sol = F.ref_voxels(starts, sk, nodes, sp[0], sp[1], sp[2], g)
    assert int(nv[-1].item()) == h["voxels"]
    assert sha(nv) == h["sha256_node_voxels"]
    assert sha(ids) == h["sha256_voxel_ids"]
    assert sha(sol) == h["sha256_solids"]
