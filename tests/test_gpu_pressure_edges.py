"""Pressure problems at the edges of the 7-point operator, through the C ABI:
a fluid cell walled in by solids on all six sides (its row of A is empty: the
Jacobi scaling takes D^-1 = 0 there and its pressure stays 0), a sealed pocket
of fluid cells with no air neighbour (pure Neumann: its pressure is defined up
to a constant), and a right-hand side that is zero.  The plain and the
learned solves meet tol with finite values, and the plain solution agrees
with the FP64 oracle's where it is unique."""
import os

import numpy as np
import pytest

import flip2_b200 as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu
FLUID, SOLID = 1, 2


@pytest.fixture(scope="module")
def torch():
    import torch as T
    assert T.cuda.is_available()
    F.lib()
    return T


def engine(shape, **kw):
    nx, ny, nz = shape
    P = F.Particles(1, mode=F.MODE_NATIVE, params=F.default_params(F.MODE_NATIVE, **kw))
    P.setDomain(0.0, 0.0, 0.0, nx // 4, ny // 4, nz // 4, 1.0)
    return P


def edge_problem(shape, seed):
    """Fluid below 60% of the height, air above, a few solid cells; an isolated
    fluid cell boxed in by solids and a sealed 2 x 2 x 2 pocket inside a solid
    shell.  b: N(0, 1) on fluid cells, 0 on the isolated cell (its row of A is
    empty), mean 0 on the pocket (the Neumann problem's compatibility)."""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    typ = np.zeros((nz, ny, nx), np.uint8)
    typ[:, : int(0.6 * ny), :] = FLUID
    typ[rng.random(typ.shape) < 0.03] = SOLID
    typ[2:7, 2:7, 2:7] = SOLID            # shell of the isolated cell at (4, 4, 4)
    typ[4, 4, 4] = FLUID
    typ[9:13, 2:6, 9:13] = SOLID          # shell of the pocket at x, y, z = 10..11, 3..4, 10..11
    typ[10:12, 3:5, 10:12] = FLUID
    b = (rng.standard_normal(typ.shape) * (typ == FLUID)).astype(np.float64)
    b[4, 4, 4] = 0.0
    pocket = np.zeros(typ.shape, bool)
    pocket[10:12, 3:5, 10:12] = True
    b[pocket] -= b[pocket].mean()
    return typ.ravel(), b.astype(np.float32).ravel(), pocket.ravel()


@pytest.mark.parametrize("seed", [0, 1])
def test_plain_solve_with_walled_cells(torch, seed):
    shape = (24, 16, 16)
    typ, b, pocket = edge_problem(shape, seed)
    P = engine(shape)
    P.poisson_set(typ, b)
    s = P.poisson_solve(0, 1e-6, 5000)
    x = P.poisson_solution()
    assert s.converged == 1 and s.rel_residual <= 1e-6
    assert np.all(np.isfinite(x))
    nx, ny, nz = shape
    assert x[4 + nx * (4 + ny * 4)] == 0.0  # the walled-in cell keeps its start value
    xo, it, _ = O.nat_pcg(typ, b.astype(np.float64), O.nat_params(*shape, 1.0))
    fl = (typ == FLUID) & ~pocket
    # off the pocket the solution is unique: 1e-5 of its largest value
    assert np.max(np.abs(x[fl] - xo[fl])) <= 1e-5 * np.max(np.abs(xo[fl]))
    # on the pocket, up to a constant
    d = x[pocket] - xo[pocket]
    assert np.max(np.abs(d - d.mean())) <= 1e-5 * np.max(np.abs(xo[fl]))
    assert abs(s.iters - it) <= max(3, it // 10)
    P.close()


def test_zero_rhs_and_learned_solve(torch):
    shape = (24, 16, 16)
    typ, b, _ = edge_problem(shape, 2)
    P = engine(shape)
    # b = 0: converged at once with x = 0
    P.poisson_set(typ, np.zeros_like(b))
    s = P.poisson_solve(0, 1e-6, 5000)
    assert s.converged == 1 and s.iters == 0
    assert np.all(P.poisson_solution() == 0.0)
    # the learned multilevel solve on the same cells (its Jacobi-PCG restart
    # included): finite, converged
    P.close()
    P = engine(shape, pressure_method=2)
    P.lp_set_weights(np.load(os.path.join(os.path.dirname(F.__file__), "data", "mg_weights.npy")))
    P.poisson_set(typ, b)
    s = P.poisson_solve(2, 1e-6, 100)
    x = P.poisson_solution()
    assert s.converged == 1 and s.rel_residual <= 1e-6
    assert np.all(np.isfinite(x))
    P.close()
