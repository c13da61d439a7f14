"""Generate the golden fixtures of tests/golden/ by running the reference
engine itself (Aidan-F-Ryan/flip2, built from its own sources by
`make -C oracle ref` into oracle/_ref/libflip2ref.so) on a B200.

The reference publishes no test vectors, so these fixtures are the pin of the
CPU oracle (oracle/flip_oracle.c): tests/test_golden.py checks the oracle
against them on CPU, and the GPU tests check the CUDA path against the oracle.

Usage (on a GPU box):  python tests/golden/make_golden.py --out DIR [--c3]
  writes DIR/ref_dam16.npz, DIR/ref_mix20k.npz, DIR/ref_timing.json and, with
  --c3, DIR/ref_c3_hashes.json (sha256 of the 64M-particle binning outputs).
Inputs are seeded (numpy default_rng); the seeds and sizes are stored in the
fixtures.
"""
import argparse
import ctypes as C
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from flip2_b200 import scenes  # noqa: E402

LIB = os.path.join(ROOT, "oracle", "_ref", "libflip2ref.so")
BUF = dict(px=0, py=1, pz=2, vx=3, vy=4, vz=5, keys=6, perm=7, flags=8, starts=9, ytable=10, node_voxels=11,
           voxel_ids=12, solids=13, ux=14, uy=15, uz=16, divU=17, p=18, res=19)
DT = dict(px=np.float64, py=np.float64, pz=np.float64, vx=np.float64, vy=np.float64, vz=np.float64,
          keys=np.uint32, perm=np.uint32, flags=np.uint32, starts=np.uint32, ytable=np.uint32, node_voxels=np.uint32,
          voxel_ids=np.uint32, solids=np.int8, ux=np.float64, uy=np.float64, uz=np.float64, divU=np.float64,
          p=np.float64, res=np.float64)


class Ref:
    def __init__(self, lib, n, domain):
        self.L = lib
        self.h = C.c_void_p()
        nx, ny, nz, X, Y, Z, cell = domain
        rc = lib.ref_create(n, nx, ny, nz, X, Y, Z, cell, C.byref(self.h))
        assert rc == 0, rc
        self.n = n

    def upload(self, pos, vel):
        cols = [np.ascontiguousarray(pos[:, k], np.float64) for k in range(3)]
        cols += [np.ascontiguousarray(vel[:, k], np.float64) for k in range(3)]
        rc = self.L.ref_upload(self.h, *[c.ctypes.data_as(C.c_void_p) for c in cols])
        assert rc == 0, rc

    def stage(self, s, dt=0.0):
        t = time.perf_counter()
        rc = self.L.ref_stage(self.h, s, C.c_double(dt))
        assert rc == 0, (s, rc)
        return time.perf_counter() - t

    def info(self):
        a, b, d = C.c_uint32(), C.c_uint32(), C.c_double()
        self.L.ref_info(self.h, C.byref(a), C.byref(b), C.byref(d))
        return a.value, b.value, d.value

    def get(self, name):
        nb = C.c_size_t()
        rc = self.L.ref_download(self.h, BUF[name], None, 0, C.byref(nb))
        assert rc == 0
        out = np.empty(nb.value // np.dtype(DT[name]).itemsize, DT[name])
        if out.size:
            rc = self.L.ref_download(self.h, BUF[name], out.ctypes.data_as(C.c_void_p), out.nbytes, C.byref(nb))
            assert rc == 0
        return out

    def put(self, name, arr):
        arr = np.ascontiguousarray(arr, DT[name])
        rc = self.L.ref_upload_buf(self.h, BUF[name], arr.ctypes.data_as(C.c_void_p), arr.nbytes)
        assert rc == 0, rc

    def set_time(self, frame_dt, elapsed):
        self.L.ref_set_time(self.h, C.c_double(frame_dt), C.c_double(elapsed))

    def close(self):
        self.L.ref_destroy(self.h)


def load():
    L = C.CDLL(LIB)
    L.ref_create.argtypes = [C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint32, C.c_uint32, C.c_uint32,
                             C.c_double, C.POINTER(C.c_void_p)]
    L.ref_upload.argtypes = [C.c_void_p] + [C.c_void_p] * 6
    L.ref_stage.argtypes = [C.c_void_p, C.c_int, C.c_double]
    L.ref_info.argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_double)]
    L.ref_download.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]
    L.ref_upload_buf.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
    L.ref_set_time.argtypes = [C.c_void_p, C.c_double, C.c_double]
    L.ref_destroy.argtypes = [C.c_void_p]
    return L


def dam_case(L, n_cells, seed, dt_div):
    """Every stage of one reference sub-step on a seeded dam-break."""
    pos, _ = scenes.dam_break(n_cells, seed=seed)
    vel = scenes.random_velocities(pos.shape[0], seed=seed + 100).astype(np.float64)
    pos = pos.astype(np.float64)
    R = n_cells // 4
    domain = (0.0, 0.0, 0.0, R, R, R, 4.0 / n_cells)
    out = dict(pos=pos, vel=vel, domain=np.array(domain, np.float64), seed=seed, dt_div=dt_div)
    tm = {}
    # chain A: binning, P2G, gravity + divergence, one SOR iteration
    a = Ref(L, pos.shape[0], domain)
    a.upload(pos, vel)
    tm["align"] = a.stage(0)
    out["a_keys"] = a.get("keys")
    out["a_px"], out["a_py"], out["a_pz"] = a.get("px"), a.get("py"), a.get("pz")
    tm["sort"] = a.stage(1)
    out["s_keys"], out["s_perm"] = a.get("keys"), a.get("perm")
    out["s_px"], out["s_py"], out["s_pz"] = a.get("px"), a.get("py"), a.get("pz")
    tm["voxels"] = a.stage(2)
    nodes, voxels, _ = a.info()
    out["nodes"], out["voxels"] = nodes, voxels
    for k in ("flags", "starts", "ytable", "node_voxels", "voxel_ids", "solids"):
        out["v_" + k] = a.get(k)
    tm["p2g"] = a.stage(3)
    out["p2g_ux"], out["p2g_uy"], out["p2g_uz"] = a.get("ux"), a.get("uy"), a.get("uz")
    tm["gravity_div"] = a.stage(5, dt_div)
    out["div_uy"], out["div_divU"] = a.get("uy"), a.get("divU")
    tm["gs1"] = a.stage(10, dt_div)
    out["gs_p"], out["gs_res"] = a.get("p"), a.get("res")
    a.close()
    # chain B: the shipped P2G (weight sums not cleared) for the record
    b = Ref(L, pos.shape[0], domain)
    b.upload(pos, vel)
    for s in (0, 1, 2):
        b.stage(s)
    b.stage(4)
    out["p2g4_ux"], out["p2g4_uy"], out["p2g4_uz"] = b.get("ux"), b.get("uy"), b.get("uz")
    b.close()
    # chain C: pressureSolve (Courant dt, dt halving), projection, G2P, advect
    c = Ref(L, pos.shape[0], domain)
    c.upload(pos, vel)
    for s in (0, 1, 2, 3):
        c.stage(s)
    c.set_time(1.0 / 24.0, 0.0)
    tm["pressure"] = c.stage(6)
    _, _, dtc = c.info()
    out["pr_dt"] = dtc
    out["pr_p"], out["pr_res"], out["pr_divU"], out["pr_uy"] = c.get("p"), c.get("res"), c.get("divU"), c.get("uy")
    tm["velupdate"] = c.stage(7)
    out["vu_ux"], out["vu_uy"], out["vu_uz"] = c.get("ux"), c.get("uy"), c.get("uz")
    tm["g2p"] = c.stage(8)
    out["g2p_vx"], out["g2p_vy"], out["g2p_vz"] = c.get("vx"), c.get("vy"), c.get("vz")
    tm["advect"] = c.stage(9)
    out["adv_px"], out["adv_py"], out["adv_pz"] = c.get("px"), c.get("py"), c.get("pz")
    c.close()
    return out, tm


def mix_case(L, n, domain_cells, seed):
    pos = scenes.binning_mix(n, domain=domain_cells, seed=seed).astype(np.float64)
    vel = np.zeros_like(pos)
    R = domain_cells
    domain = (0.0, 0.0, 0.0, R, R, R, 1.0)
    out = dict(pos=pos, domain=np.array(domain, np.float64), seed=seed)
    a = Ref(L, n, domain)
    a.upload(pos, vel)
    a.stage(0)
    out["a_keys"] = a.get("keys")
    a.stage(1)
    out["s_keys"], out["s_perm"] = a.get("keys"), a.get("perm")
    a.stage(2)
    nodes, voxels, _ = a.info()
    out["nodes"], out["voxels"] = nodes, voxels
    for k in ("flags", "starts", "ytable", "node_voxels", "voxel_ids", "solids"):
        out["v_" + k] = a.get(k)
    a.close()
    return out


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def c3_case(L, n=1 << 26, seed=1):
    pos = scenes.binning_mix(n, domain=512, seed=seed).astype(np.float64)
    domain = (0.0, 0.0, 0.0, 512, 512, 512, 1.0)
    a = Ref(L, n, domain)
    a.upload(pos, np.zeros_like(pos))
    del pos
    tm = {"align": a.stage(0), "sort": a.stage(1), "voxels": a.stage(2)}
    nodes, voxels, _ = a.info()
    res = dict(n=n, seed=seed, nodes=nodes, voxels=voxels, seconds=tm)
    for k in ("keys", "perm", "flags", "starts", "node_voxels", "voxel_ids", "solids"):
        res["sha256_" + k] = sha(a.get(k))
    a.close()
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--c3", action="store_true")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    L = load()
    timing = {}
    d16, tm16 = dam_case(L, 16, seed=0, dt_div=0.001)
    np.savez_compressed(os.path.join(args.out, "ref_dam16.npz"), **d16)
    timing["dam16"] = tm16
    d32, tm32 = dam_case(L, 32, seed=0, dt_div=1.0 / 240)
    timing["dam32"] = tm32
    timing["dam32_sizes"] = dict(n=int(d32["pos"].shape[0]), nodes=int(d32["nodes"]), voxels=int(d32["voxels"]))
    np.savez_compressed(os.path.join(args.out, "ref_dam32_full.npz"), **d32)
    mx = mix_case(L, 20000, 64, seed=1)
    np.savez_compressed(os.path.join(args.out, "ref_mix20k.npz"), **mx)
    if args.c3:
        c3 = c3_case(L)
        with open(os.path.join(args.out, "ref_c3_hashes.json"), "w") as f:
            json.dump(c3, f, indent=1)
        timing["c3"] = c3["seconds"]
    with open(os.path.join(args.out, "ref_timing.json"), "w") as f:
        json.dump(timing, f, indent=1)
    print(json.dumps(timing, indent=1))


if __name__ == "__main__":
    main()
