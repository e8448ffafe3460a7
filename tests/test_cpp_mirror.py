"""The C++ mirror of the reference interface (include/glamer_b200.hpp): it
compiles with the reference's own struct shapes and links against the
library (CPU), and a program driving it through Lens / LensHalo* /
TreeQuadParticles / GridMap agrees with direct C-ABI calls and with the
oracle (GPU)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from slsimlib_b200 import synth
from tests import harness as H
from tests.conftest import rel_err

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "mirror_test.cpp")
LIBDIR = os.path.join(ROOT, "slsimlib_b200")


def build(tmp_path) -> str:
    if not os.path.exists(os.path.join(LIBDIR, "libglamer_b200.so")):
        pytest.skip("libglamer_b200.so is not built")
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    exe = str(tmp_path / "mirror_test")
    cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-o", exe, "-L", LIBDIR, "-lglamer_b200", f"-Wl,-rpath,{LIBDIR}", "-Wl,--allow-shlib-undefined"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return exe


def test_mirror_compiles_and_links(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_mirror_program_matches_capi_and_oracle(tmp_path):
    exe = build(tmp_path)
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([exe, str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("OK"), r.stdout + r.stderr
    p1 = np.fromfile(out / "plane1.bin", dtype=synth.PARTICLE_DTYPE)
    p2 = np.fromfile(out / "plane2.bin", dtype=synth.PARTICLE_DTYPE)
    y = np.fromfile(out / "grid_y.bin").reshape(-1, 2)
    A = np.fromfile(out / "grid_A.bin").reshape(-1, 4)
    arc = synth.ARCSEC
    spec = synth.LensSpec(zsource=2.0, halos=[
        synth.ParticlePlane(p1, 0.3), synth.ParticlePlane(p2, 0.6),
        synth.NFWHalo(5e13, 0.5, 0.45, 6.0, theta=(3 * arc, -2 * arc)),
        synth.NSIEHalo(1e13, 0.3, 220.0, 3e-4, 0.75, 0.4)])
    x = synth.grid_positions(24, range_rad=40 * arc)
    yo, Ao = H.OracleLens(spec).rayshoot(x)
    assert np.max(rel_err(y, yo)) < 1e-9
    assert np.max(np.abs(A - Ao)) < 1e-9
    s_in = np.fromfile(out / "smooth_in.bin", dtype=synth.PARTICLE_DTYPE)
    s_out = np.fromfile(out / "smooth_out.bin", dtype=synth.PARTICLE_DTYPE)
    assert np.array_equal(s_out["Size"], H.oracle_smoothing(s_in, 16))
