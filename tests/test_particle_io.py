"""Particle files (glmb, sizes cache, csv, ascii) read and written by
slsimlib_b200.particle_io against the reference's own readers and writers
(compiled in place) on the same files.  The csv cases that need smoothing
run the GPU."""
import os
import shutil

import numpy as np
import pytest

from slsimlib_b200 import particle_io as pio
from slsimlib_b200 import synth
from tests import harness as H

needs_ref = pytest.mark.skipif(not H.ref_available(), reason="reference not compiled here")


def particles(n, seed, sizes=True, types=False):
    r = np.random.default_rng(seed)
    p = synth.nfw_particles(r, n, 1e14, 5.0, 0.5, 0.0)
    p["x"] += np.float32(3.0)  # a bounding box away from the origin
    p["Mass"] = r.uniform(0.5, 2.0, n).astype(np.float32)
    if sizes:
        p["Size"] = r.uniform(1e-3, 1e-2, n).astype(np.float32)
    if types:
        p["type"] = r.integers(0, 3, n).astype(np.int32)
    return p


def write_csv(path, p, columns, comment=True):
    """Values printed with 9 significant digits, so both parsers recover the
    float exactly."""
    with open(path, "w") as f:
        if comment:
            f.write("# x,y,z,mass,size,type\n")
        for q in p:
            v = [f"{float(q['x'][0]):.9g}", f"{float(q['x'][1]):.9g}", f"{float(q['x'][2]):.9g}",
                 f"{float(q['Mass']):.9g}", f"{float(q['Size']):.9g}", str(int(q["type"]))]
            f.write(",".join(v[:columns]) + "\n")


def test_glmb_round_trip(tmp_path):
    p = particles(500, 1, types=True)
    f = str(tmp_path / "a.glmb")
    pio.write_glmb(f, p, 32, [300, 200, 0, 0, 0, 0], 0.75)
    d, ns, nbt, z = pio.read_glmb(f)
    assert np.array_equal(d.view(np.uint8), p.view(np.uint8)) and ns == 32 and nbt == [300, 200, 0, 0, 0, 0]
    assert z == 0.75 and os.path.getsize(f) == 68 + 24 * 500
    assert pio.read_glmb(str(tmp_path / "missing.glmb")) is None


def test_sizes_file_round_trip_and_errors(tmp_path):
    s = np.random.default_rng(2).uniform(1e-4, 1.0, 300).astype(np.float32)
    f = str(tmp_path / "p.64sizes")
    pio.write_sizes(f, 64, s)
    got = pio.read_sizes_file(f, 300, 64, 0.0)
    assert np.allclose(got, s, rtol=1e-5)
    assert np.all(pio.read_sizes_file(f, 300, 64, 0.5) >= np.float32(0.5))
    assert pio.read_sizes_file(f, 300, 32, 0.0) is None
    assert pio.read_sizes_file(str(tmp_path / "none"), 300, 64, 0.0) is None
    with pytest.raises(RuntimeError):
        pio.read_sizes_file(f, 299, 64, 0.0)


def test_ascii_positions(tmp_path):
    p = particles(50, 3)
    f = tmp_path / "pos.txt"
    with open(f, "w") as fh:
        fh.write("# nparticles 50\n# mass 2.5\n")
        for q in p:
            fh.write(" ".join(f"{float(v):.9g}" for v in q["x"]) + f" {float(q['Mass']):.9g}\n")
    got, m = pio.read_positions_ascii(str(f), multimass=False)
    assert m == 2.5 and np.array_equal(got["x"], p["x"]) and np.all(got["Mass"] == 0)
    with open(f, "w") as fh:
        fh.write("# nparticles 50\n")
        for q in p:
            fh.write(" ".join(f"{float(v):.9g}" for v in q["x"]) + f" {float(q['Mass']):.9g}\n")
    got, _ = pio.read_positions_ascii(str(f), multimass=True)
    assert np.array_equal(got["x"], p["x"]) and np.array_equal(got["Mass"], p["Mass"])
    with pytest.raises(RuntimeError):
        pio.read_positions_ascii(str(tmp_path / "none.txt"), True)


@needs_ref
def test_sizes_file_matches_reference(tmp_path):
    p = particles(400, 4)
    ref_f, our_f = str(tmp_path / "ref.sizes"), str(tmp_path / "our.sizes")
    R = H.RefDriver()
    R.write_sizes(p, 64, ref_f)
    pio.write_sizes(our_f, 64, p["Size"])
    assert open(ref_f, "rb").read() == open(our_f, "rb").read()
    for ns, n, mn in ((64, 400, 0.0), (64, 400, 5e-3), (32, 400, 0.0), (64, 399, 0.0)):
        ref = R.read_sizes(ref_f, n, ns, mn)
        try:
            ours = pio.read_sizes_file(ref_f, n, ns, mn)
        except RuntimeError:
            ours = "throw"
        if isinstance(ref, str) or ref is None:
            assert ours is ref or ours == ref, (ns, n, mn)
        else:
            assert np.array_equal(ours, ref), (ns, n, mn)


@needs_ref
@pytest.mark.parametrize("recenter", [False, True])
def test_csv5_and_glmb_match_reference(tmp_path, recenter):
    """csv5 (sizes in the file, no smoothing): records, centre of mass,
    bounding box, counts and the glmb cache file, then the glmb constructor."""
    p = particles(700, 5)
    for who in ("ref", "our"):
        os.makedirs(tmp_path / who)
        write_csv(tmp_path / who / "sim.csv", p, 5)
    R = H.RefDriver()
    ref, meta = R.make_particles(str(tmp_path / "ref" / "sim.csv"), 5, 16, recenter)
    m = pio.MakeParticleLenses(str(tmp_path / "our" / "sim.csv"), "csv5", 16, recenter)
    assert np.array_equal(m.data.view(np.uint8), ref.view(np.uint8))
    lo, hi = m.getBoundingBox()
    assert np.array_equal(np.concatenate([m.getCenterOfMass(), lo, hi]), meta[:9])
    assert m.getZoriginal() == meta[9] and m.getnp() == [int(v) for v in meta[10:16]]
    assert np.array_equal(m.densest_particle(), meta[16:19])
    g_ref, g_our = tmp_path / "ref" / "sim.csv_S16.glmb", tmp_path / "our" / "sim.csv_S16.glmb"
    assert open(g_ref, "rb").read() == open(g_our, "rb").read()
    # the glmb constructor on the reference's file
    ref2, meta2 = R.make_particles(str(g_ref), 0, 0, recenter)
    m2 = pio.MakeParticleLenses(str(g_ref), None, 0, recenter)
    assert np.array_equal(m2.data.view(np.uint8), ref2.view(np.uint8))
    lo, hi = m2.getBoundingBox()
    assert np.array_equal(np.concatenate([m2.getCenterOfMass(), lo, hi]), meta2[:9])
    # a second construction reads the cache, not the csv
    os.remove(tmp_path / "our" / "sim.csv")
    m3 = pio.MakeParticleLenses(str(tmp_path / "our" / "sim.csv"), "csv5", 16, recenter)
    assert np.array_equal(m3.data.view(np.uint8), ref.view(np.uint8))


@needs_ref
def test_csv6_refused_as_in_reference(tmp_path):
    p = particles(100, 6, types=True)
    write_csv(tmp_path / "s.csv", p, 6)
    ref, _ = H.RefDriver().make_particles(str(tmp_path / "s.csv"), 6, 8)
    assert ref is None
    with pytest.raises(ValueError):
        pio.MakeParticleLenses(str(tmp_path / "s.csv"), "csv6", 8)


def test_csv_too_few_columns(tmp_path):
    write_csv(tmp_path / "s.csv", particles(10, 7), 3)
    with pytest.raises(ValueError):
        pio.read_csv(str(tmp_path / "s.csv"), 4, 8)


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("columns", [3, 4])
def test_csv_with_smoothing_matches_reference(tmp_path, columns):
    """csv3 / csv4: sizes from the adaptive smoothing (GPU) -- records and the
    glmb cache byte for byte."""
    p = particles(3000, 8 + columns, sizes=False)
    for who in ("ref", "our"):
        os.makedirs(tmp_path / who)
        write_csv(tmp_path / who / "sim.csv", p, columns, comment=False)
    ref, meta = H.RefDriver().make_particles(str(tmp_path / "ref" / "sim.csv"), columns, 32)
    m = pio.MakeParticleLenses(str(tmp_path / "our" / "sim.csv"), f"csv{columns}", 32)
    assert np.array_equal(m.data.view(np.uint8), ref.view(np.uint8))
    assert (open(tmp_path / "ref" / "sim.csv_S32.glmb", "rb").read()
            == open(tmp_path / "our" / "sim.csv_S32.glmb", "rb").read())
    halos = m.CreateHalos(0.7, 0.4, 0.0)
    assert len(halos) == 1


@needs_ref
@pytest.mark.parametrize("recenter", [False, True])
def test_cpp_mirror_particle_files_match_reference(tmp_path, recenter):
    """The C++ mirror's MakeParticleLenses (csv5) and sizes-file helpers
    against the reference on the same csv file."""
    import subprocess
    gxx = shutil.which("g++")
    lib = os.path.join(H.ROOT, "slsimlib_b200")
    if gxx is None or not os.path.exists(os.path.join(lib, "libglamer_b200.so")):
        pytest.skip("no g++ or library")
    exe = str(tmp_path / "pio")
    r = subprocess.run([gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I",
                        os.path.join(H.ROOT, "include"), os.path.join(H.ROOT, "tests", "cpp", "particle_io_test.cpp"),
                        "-o", exe, "-L", lib, "-lglamer_b200", f"-Wl,-rpath,{lib}", "-Wl,--allow-shlib-undefined"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    p = particles(600, 9)
    for who in ("ref", "cpp"):
        os.makedirs(tmp_path / who)
        write_csv(tmp_path / who / "sim.csv", p, 5)
    ref, meta = H.RefDriver().make_particles(str(tmp_path / "ref" / "sim.csv"), 5, 16, recenter)
    out = str(tmp_path / "cpp" / "o")
    r = subprocess.run([exe, str(tmp_path / "cpp" / "sim.csv"), "16", str(int(recenter)), out],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "OK", r.stdout + r.stderr
    got = np.fromfile(out + ".bin", dtype=synth.PARTICLE_DTYPE)
    assert np.array_equal(got.view(np.uint8), ref.view(np.uint8))
    assert np.array_equal(np.fromfile(out + ".meta"), meta)
    assert (open(tmp_path / "ref" / "sim.csv_S16.glmb", "rb").read()
            == open(tmp_path / "cpp" / "sim.csv_S16.glmb", "rb").read())
    R = H.RefDriver()
    R.write_sizes(ref, 64, str(tmp_path / "ref.sizes"))
    assert open(tmp_path / "ref.sizes", "rb").read() == open(out + ".sizes", "rb").read()
    if not recenter:
        cx, cy, cz, rad = np.fromfile(out + ".cut.meta")
        cut_ref, _ = R.make_particles(str(tmp_path / "ref" / "sim.csv"), 5, 16, False, 1, (cx, cy, cz), rad)
        got_cut = np.fromfile(out + ".cut.bin", dtype=synth.PARTICLE_DTYPE)
        assert 0 < len(got_cut) < len(p)
        assert np.array_equal(got_cut.view(np.uint8), cut_ref.view(np.uint8))


def write_ascii(path, p, multimass=True):
    with open(path, "w") as f:
        f.write(f"# nparticles {len(p)}\n")
        if not multimass:
            f.write("# mass 1e9\n")
        for q in p:
            v = [f"{float(c):.9g}" for c in q["x"]]
            if multimass:
                v.append(f"{float(q['Mass']):.9g}")
            f.write(" ".join(v) + "\n")


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("recenter,rot,mscale,minp", [(False, (0.0, 0.0), 1.0, 0.0), (True, (0.3, -0.2), 2.5, 2e-3)])
def test_particle_lens_from_ascii_file_matches_reference(tmp_path, recenter, rot, mscale, minp):
    """LensHaloParticles from an ascii position file: the sizes cache written
    (smoothing on the GPU) and the lens's force against the reference's."""
    from tests.test_gpu_parity import RTOL64, force_err, pack
    r = np.random.default_rng(21)
    p = synth.nfw_particles(r, 20000, 2e14, 5.0, 0.4, 0.0)
    p["Mass"] = r.uniform(5e9, 2e10, len(p)).astype(np.float32)
    for who in ("ref", "our"):
        os.makedirs(tmp_path / who)
        write_ascii(tmp_path / who / "sim.txt", p)
    xx = r.uniform(-0.4, 0.4, (300, 2))
    R = H.RefDriver()
    xf = R._file(np.ascontiguousarray(xx))
    of = R._file()
    R.run([f"particlefile {tmp_path / 'ref' / 'sim.txt'} 0.4 32 1 0.0 {minp!r} {mscale!r} {int(recenter)} "
           f"{rot[0]!r} {rot[1]!r} {xf} {len(xx)} {of}"])
    ref = np.fromfile(of).reshape(-1, 7)
    halo, _ = pio.lens_halo_particles_from_file(str(tmp_path / "our" / "sim.txt"), 0.4, 32, rot, recenter, True,
                                                0.0, minp, mscale)
    f = pack(*halo.force_halo(xx))
    m, cols = force_err(f, ref)
    assert m < RTOL64, cols
    assert (open(tmp_path / "ref" / "sim.txt.32sizes", "rb").read()
            == open(tmp_path / "our" / "sim.txt.32sizes", "rb").read())
    # a second construction reads the sizes back from the cache (6 digits), on both sides
    of2 = R._file()
    R.run([f"particlefile {tmp_path / 'ref' / 'sim.txt'} 0.4 32 1 0.0 {minp!r} {mscale!r} {int(recenter)} "
           f"{rot[0]!r} {rot[1]!r} {xf} {len(xx)} {of2}"])
    ref2 = np.fromfile(of2).reshape(-1, 7)
    halo2, _ = pio.lens_halo_particles_from_file(str(tmp_path / "our" / "sim.txt"), 0.4, 32, rot, recenter, True,
                                                 0.0, minp, mscale)
    m2, cols2 = force_err(pack(*halo2.force_halo(xx)), ref2)
    assert m2 < RTOL64, cols2


@needs_ref
@pytest.mark.parametrize("cut", [1, 2])
def test_cuts_match_reference(tmp_path, cut):
    """radialCut / cylindricalCut: the records kept, in the reference's order."""
    p = particles(900, 10)
    centre = (float(np.median(p["x"][:, 0])), float(np.median(p["x"][:, 1])), float(np.median(p["x"][:, 2])))
    for who in ("ref", "our"):
        os.makedirs(tmp_path / who)
        write_csv(tmp_path / who / "sim.csv", p, 5)
    ref, meta = H.RefDriver().make_particles(str(tmp_path / "ref" / "sim.csv"), 5, 16, False, cut, centre, 0.05)
    m = pio.MakeParticleLenses(str(tmp_path / "our" / "sim.csv"), "csv5", 16, False)
    (m.radialCut if cut == 1 else m.cylindricalCut)(centre if cut == 1 else centre[:2], 0.05)
    assert 0 < len(m.data) < len(p)
    assert np.array_equal(m.data.view(np.uint8), ref.view(np.uint8))
    assert m.getnp() == [int(v) for v in meta[10:16]]
    assert np.array_equal(m.densest_particle(), meta[16:19])
