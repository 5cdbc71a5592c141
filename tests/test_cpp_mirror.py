"""The C++ mirror of the reference interface (lbm_solver.hpp): a scenario
main written against LBMSolver compiles with g++, runs on the GPU and writes
the reference's probe files, which match the FP64 oracle."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from nlos_lbm import abi

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
PKG = os.path.join(REPO, "city-scale-nlos-acoustic-engine-code_b200")
LIBDIR = os.path.join(PKG, "nlos_lbm")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def build_driver(tmp):
    exe = os.path.join(tmp, "drive")
    cmd = [CXX, "-std=c++17", "-O2", "-I" + os.path.join(REPO, "include"), "-I" + PKG,
           os.path.join(HERE, "cpp", "drive_lbmsolver.cpp"), "-L" + LIBDIR, "-l:liblbm_b200.so",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


@pytest.mark.parametrize("fp16", [False, True])
def test_cpp_mirror_run_matches_oracle(fp16, gpu, tmp_path):
    tris = oracle.box_triangles([(10, 8, 0, 22, 20, 12), (30, 5, 0, 41, 14, 7), (26, 20, 0, 38, 30, 16)])
    stl = str(tmp_path / "city.stl")
    oracle.write_stl(stl, tris)
    exe = build_driver(str(tmp_path))
    r = subprocess.run([exe, stl] + (["fp16"] if fp16 else []), cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "WARNING: Probe A is trapped inside SOLID building!" in r.stdout   # 06:434
    got = {n: np.loadtxt(tmp_path / f"probe_{n}.txt") for n in "ABCD"}
    assert all(len(v) == 80 for v in got.values())
    # total_steps = 79, Frames = 2 -> out_interval = 39: frames at s = 0, 39, 78 (06:1068, 06:1094)
    vtk = sorted(os.listdir(tmp_path / "output_mpi"))
    assert vtk == ["flight_00000.vtk", "flight_00001.vtk", "flight_00002.vtk"]
    head = open(tmp_path / "output_mpi" / "flight_00001.vtk", "rb").read(400)
    assert b"DIMENSIONS 48 32 30" in head and b"BINARY" in head

    cfg = abi.reference_config(x_min=0, x_max=48, y_min=0, y_max=32, z_min=0, z_max=30, dx=1.0, tau=0.55)
    src = abi.reference_source(sx=24.3, sy=16.2, sz=12.7, ex=24.3, ey=16.2, ez=12.7, amp=10.0)
    probes = np.array([[20.5, 16.5, 10.5], [30.5, 16.5, 20.5], [5.2, 3.3, 2.1], [44.0, 28.0, 25.0]])
    o = oracle.OracleSolver(cfg, [src], probes, stl=stl)
    o.step(80)
    ref = o.get_probes()
    mine = np.stack([got[n] for n in "ABCD"], 1)
    tol = 1e-3 if fp16 else 1e-5
    err = np.linalg.norm(mine - ref) / np.linalg.norm(ref)
    assert err <= tol, err
