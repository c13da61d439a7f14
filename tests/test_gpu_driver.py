"""The C++ facade (include/flip2/particles.hpp) driven the way the reference's
engine/main.cu drives libparticles.so: flip2_main (flip2_b200/driver/main.cpp,
built by flip2_b200/build.py) seeds particles, initialises, solves a frame at
24 fps and writes the frames.  Its frame must equal the same frame computed
through the Python binding from the same initial state, its CSV must be the
reference's "x, y, z" format of those positions, and CudaVec<double>::getMax
must return what the reference's reduction returns (the oracle's restatement
of cudaVec.cu:173-233, bit for bit)."""
import os
import subprocess

import numpy as np
import pytest

import flip2_b200 as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DRIVER = os.path.join(os.path.dirname(F.LIB_PATH), "flip2_main")


def test_facade_driver_frame_matches_python_binding(tmp_path):
    n = 65536
    r = subprocess.run([DRIVER, str(n), "1", "native", str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "frame 1:" in r.stdout
    p0 = F.read_positions_bin(str(tmp_path / "0.bin"))
    p1 = F.read_positions_bin(str(tmp_path / "1.bin"))
    assert p0.shape == (n, 3) and p1.shape == (n, 3)
    # the same frame from the same initial state through the Python binding
    P = F.Particles(n, mode=F.MODE_NATIVE)
    P.setDomain(-10.0, -10.0, -10.0, 64, 64, 64, 0.25)
    P.upload(p0, np.zeros_like(p0))
    P.initialize()
    P.solveFrame(24.0)
    q1, _ = P.download()
    info = P.info()
    P.close()
    assert info.converged == 1 and info.error_flags == 0
    h = 0.25 / 4
    # identical kernels on identical inputs; float atomics may order sums differently
    assert np.max(np.abs(q1 - p1)) < 1e-4 * h
    # the fluid fell under gravity during the frame
    assert p1[:, 1].mean() < p0[:, 1].mean()
    # the CSV is the binary frame printed with 6 significant digits
    csv = np.loadtxt(str(tmp_path / "1"), delimiter=",")
    assert csv.shape == (n, 3)
    assert np.all(np.abs(csv - p1) <= 5e-6 * np.maximum(np.abs(p1), 1e-30) + 1e-12)


def test_facade_cudavec_getmax_is_the_reference_reduction(tmp_path):
    n = 5000
    r = subprocess.run([DRIVER, str(n), "0", "native", str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    px0 = np.fromfile(str(tmp_path / "px0.f64"), dtype=np.float64)
    assert px0.size == n
    got = float(open(str(tmp_path / "getmax.txt")).read())
    assert got == O.ref_getmax(px0, absolute=True)
