"""The C++ host classes of include/icempm_b200.hpp (HostSideSOA,
GPU_Implementation6, Model3D with the reference's method names): a C++
program drives Model3D::Step for a few frames. On CPU the program is
compiled with warnings as errors; on a B200 its final state and frame forces
are compared with the oracle."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from icempm_3dm_b200 import PRECISION_FP64_SVD64, PRECISION_MIXED
from icempm_3dm_b200._lib import LIB_PATH, POSX, VELX, FE00
from tests.helpers import perturbed_block

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "model3d_frames.cpp")


def build(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path / "model3d_frames"
    libdir = os.path.dirname(LIB_PATH)
    r = subprocess.run([cxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                        SRC, "-L", libdir, "-licempm_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_host_program_compiles(tmp_path):
    assert build(tmp_path).exists()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [PRECISION_FP64_SVD64, PRECISION_MIXED])
def test_cpp_model3d_frames_match_the_oracle(tmp_path, precision):
    """FP64 with the FP64 SVD: with the reference's FP32 SVD a 1e-16 difference
    in F_tr can cross a float rounding boundary and grow over substeps (the
    block250k case shows this), which would test that, not the host path."""
    from oracle import pyoracle as po
    exe = build(tmp_path)
    prms, soa = perturbed_block(n=3000, seed=41, ind_velocity=0.5)
    prms.UpdateEveryNthStep = 20
    n, frames = soa.shape[1], 3
    (tmp_path / "params.bin").write_bytes(ctypes.string_at(ctypes.addressof(prms), ctypes.sizeof(prms)))
    np.ascontiguousarray(soa).tofile(tmp_path / "soa.bin")
    r = subprocess.run([str(exe), str(tmp_path / "params.bin"), str(tmp_path / "soa.bin"), str(n), str(frames),
                        str(precision), str(tmp_path / "out.bin"), str(tmp_path / "forces.bin")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert f"SimulationStep {frames * 20}" in r.stdout
    out = np.fromfile(tmp_path / "out.bin").reshape(28, n)
    forces = np.fromfile(tmp_path / "forces.bin").reshape(frames, 3)
    sim = po.OracleSim(prms, soa, n, svd_mode=1)
    hist, err = sim.step(frames * 20)
    assert err == 0
    ref_forces = hist.reshape(frames, 20, 3).mean(axis=1)
    scale = np.abs(ref_forces).max()
    assert scale > 0
    if precision == PRECISION_FP64_SVD64:
        assert np.abs(forces - ref_forces).max() <= 1e-7 * scale
        for rows in (slice(POSX, POSX + 3), slice(VELX, VELX + 3), slice(FE00, FE00 + 9)):
            assert np.abs(out[rows] - sim.soa[rows]).max() <= 1e-7 * max(np.abs(sim.soa[rows]).max(), 1e-12)
    else:
        assert np.linalg.norm(forces - ref_forces) <= 1e-3 * np.linalg.norm(ref_forces)
        assert np.abs(out[POSX:POSX + 3] - sim.soa[POSX:POSX + 3]).max() < 1e-6
