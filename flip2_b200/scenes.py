"""Seeded synthetic scenes with the shapes of the benchmark configurations.

The reference seeds nothing (engine/testing.h:55-76 draws positions from
std::random_device), so every scene here is generated from a fixed numpy seed
and documented by its parameters.
"""
import numpy as np


def dam_break(n_cells, block=(0.4, 0.6, 1.0), ppc=8, seed=0, sphere=None):
    """Jittered stratified particles of a dam-break block in the unit box.

    n_cells: voxels per axis (cell size 1/n_cells).  Every fluid cell is split
    into 2x2x2 strata; one particle sits uniformly inside each stratum (the
    +-0.5 stratum jitter).  A stratum is fluid when its centre lies inside the
    block (or inside the optional sphere (cx, cy, cz, r)).  Returns (pos, vel)
    as float32 (n, 3) arrays, velocities zero.
    """
    if ppc != 8:
        raise ValueError("stratified placement uses 2x2x2 strata per cell (8 particles per cell)")
    m = 2 * n_cells
    h2 = 1.0 / m
    rng = np.random.default_rng(seed)
    parts = []
    nb = [int(np.floor(b * m - 0.5)) + 1 for b in block]
    nb = [max(0, min(m, v)) for v in nb]
    k, j, i = np.meshgrid(np.arange(nb[2]), np.arange(nb[1]), np.arange(nb[0]), indexing="ij")
    centers = np.stack([(i.ravel() + 0.5) * h2, (j.ravel() + 0.5) * h2, (k.ravel() + 0.5) * h2], axis=1)
    parts.append(centers)
    if sphere is not None:
        cx, cy, cz, r = sphere
        lo = [max(0, int(np.floor((c - r) * m))) for c in (cx, cy, cz)]
        hi = [min(m, int(np.ceil((c + r) * m)) + 1) for c in (cx, cy, cz)]
        k, j, i = np.meshgrid(np.arange(lo[2], hi[2]), np.arange(lo[1], hi[1]), np.arange(lo[0], hi[0]), indexing="ij")
        c = np.stack([(i.ravel() + 0.5) * h2, (j.ravel() + 0.5) * h2, (k.ravel() + 0.5) * h2], axis=1)
        inside = np.sum((c - np.array([cx, cy, cz])) ** 2, axis=1) < r * r
        inblock = np.all(c < np.array(block), axis=1)
        parts.append(c[inside & ~inblock])
    centers = np.concatenate(parts, axis=0)
    jitter = rng.uniform(-0.5, 0.5, size=centers.shape) * h2
    pos = (centers + jitter).astype(np.float32)
    # keep strictly inside the box in float32
    pos = np.clip(pos, np.float32(1e-7), np.float32(1.0) - np.float32(1e-7)).astype(np.float32)
    vel = np.zeros_like(pos)
    return pos, vel


def binning_mix(n, domain=512, blobs=16, sigma=8.0, seed=1):
    """Positions for the binning microbenchmark: 50% uniform in [0,domain)^3,
    50% from `blobs` isotropic Gaussians (centres uniform), clipped into
    [0, domain*(1-2^-24)].  float32 (n, 3)."""
    rng = np.random.default_rng(seed)
    nu = n // 2
    ng = n - nu
    out = np.empty((n, 3), np.float32)
    out[:nu] = rng.uniform(0.0, domain, size=(nu, 3)).astype(np.float32)
    centres = rng.uniform(0.0, domain, size=(blobs, 3))
    which = rng.integers(0, blobs, size=ng)
    g = centres[which] + rng.normal(0.0, sigma, size=(ng, 3))
    out[nu:] = g.astype(np.float32)
    hi = np.float32(domain * (1.0 - 2.0 ** -24))
    np.clip(out, np.float32(0.0), hi, out=out)
    perm = rng.permutation(n)
    return out[perm]


def random_velocities(n, seed=2, scale=1.0):
    rng = np.random.default_rng(seed)
    return (rng.uniform(-1.0, 1.0, size=(n, 3)) * scale).astype(np.float32)
