"""Generates tests/golden/*.npz from the reference itself.

The reference ships no test vectors, so the golden outputs come from the
reference's own sources compiled in place (oracle/_ref/glamer_ref, built by
oracle/Makefile from the SLsimLib tree).  Each fixture stores its inputs and
the reference's outputs, so tests need neither the reference tree nor the
generator at run time.

    make -C oracle REF=<SLsimLib> && python tests/golden/make_golden.py [tree halos lens field sources adaptive smoothing uniform]
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from slsimlib_b200 import synth  # noqa: E402
from tests import harness as H  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def tree_fixture():
    rng = np.random.default_rng(11)
    p = synth.nfw_particles(rng, 3000, 1e14, 5.0, 0.3, 1e-3)
    # a few particles with large softening to populate internal big-particle lists
    p["Size"][:40] = np.float32(0.05)
    rays = np.concatenate([rng.uniform(-0.05, 0.05, size=(48, 2)), rng.uniform(-0.6, 0.6, size=(16, 2))])
    R = H.RefDriver()
    out, exp = R.tree_force(p, rays, bucket=20, theta=0.1, inv_screening=1.0, export=True)
    np.savez_compressed(os.path.join(OUT, "tree_small.npz"), particles=p, rays=rays, force=out, export=exp,
                        bucket=20, theta=0.1, inv_screening=1.0)


def halo_fixture():
    rng = np.random.default_rng(12)
    x = rng.uniform(-1.0, 1.0, size=(64, 2)) * np.logspace(-4, 0.2, 64)[:, None]
    R = H.RefDriver()
    halos = {
        "nfw": synth.NFWHalo(1e14, 0.864, 0.3, 5.0),
        "nsie_cored": synth.NSIEHalo(1e13, 0.5, 250.0, 3.05e-4, 0.7, 0.0),
        "nsie_sis": synth.NSIEHalo(1e13, 0.5, 250.0, 0.0, 1.0, 0.0),
        "nsie_rot": synth.NSIEHalo(1e12, 0.5, 200.0, 1e-4, 0.5, 0.3),
    }
    data = {"x": x}
    for k, h in halos.items():
        f, prm = R.halo_force(h, x)
        data[k] = f
        data[k + "_params"] = np.array(prm)
    np.savez_compressed(os.path.join(OUT, "halos.npz"), **data)


def halo_subtract_fixture():
    """force_halo(..., subtract_point = true, screening) of the reference
    (MultiPlane/lens_halos.cpp:1528-1640) for NFW and NSIE haloes, positions
    inside and beyond Rmax."""
    rng = np.random.default_rng(15)
    x = rng.uniform(-1.0, 1.0, size=(64, 2)) * np.logspace(-4, 0.4, 64)[:, None]
    R = H.RefDriver()
    halos = {"nfw": synth.NFWHalo(1e14, 0.864, 0.3, 5.0), "nsie_sis": synth.NSIEHalo(1e13, 0.5, 250.0, 0.0, 1.0, 0.0),
             "nsie_rot": synth.NSIEHalo(1e12, 0.5, 200.0, 0.0, 0.6, 0.3)}
    data = {"x": x}
    for k, h in halos.items():
        for s in (1.0, 0.25):
            data[f"{k}_{s}"] = R.halo_force(h, x, screening=s)[0]
    np.savez_compressed(os.path.join(OUT, "halos_subtract.npz"), **data)


def lens_fixture():
    spec = synth.light_cone(seed=13, n_total=6000, n_planes=3, halos_per_plane=3)
    spec.halos.append(synth.NFWHalo(3e13, 0.4, 0.7, 6.0, theta=(2e-5, -1e-5)))
    R = H.RefDriver()
    rng_range = 60 * synth.ARCSEC
    y, A, _ = R.grid(spec, 16, range_rad=rng_range)
    rng = np.random.default_rng(14)
    x = rng.uniform(-30, 30, size=(64, 2)) * synth.ARCSEC
    zs = rng.uniform(0.2, 3.0, size=64)
    y2, A2, _ = R.rays(spec, x, zs)
    arrays = {"grid_y": y, "grid_A": A, "grid_n": 16, "grid_range": rng_range, "rays_x": x, "rays_zs": zs,
              "rays_y": y2, "rays_A": A2, "zsource": spec.zsource}
    for i, h in enumerate(spec.halos):
        if isinstance(h, synth.ParticlePlane):
            arrays[f"plane{i}_particles"] = h.particles
            arrays[f"plane{i}_z"] = h.z
    nsie = [h for h in spec.halos if isinstance(h, synth.NSIEHalo)][0]
    arrays["nsie"] = np.array([nsie.mass, nsie.z, nsie.sigma, nsie.rcore, nsie.fratio, nsie.pa])
    nfw = [h for h in spec.halos if isinstance(h, synth.NFWHalo)][0]
    arrays["nfw"] = np.array([nfw.mass, nfw.rsize, nfw.z, nfw.conc, nfw.theta[0], nfw.theta[1]])
    np.savez_compressed(os.path.join(OUT, "lens_small.npz"), **arrays)


FIELD_CASES = ((0.0, 0.0), (5.0, 0.0), (0.0, 2.0), (2.0, 1.0))  # (sigma_back, inv_screening)


def field_rows(halos):
    """8 doubles per field halo, as the reference driver's fieldplane command reads them."""
    rows = []
    for h in halos:
        if isinstance(h, synth.NFWHalo):
            rows.append([0, h.mass, h.rsize, h.conc, 0, 0, h.theta[0], h.theta[1]])
        else:
            rows.append([1, h.mass, h.sigma, h.rcore, h.fratio, h.pa, h.theta[0], h.theta[1]])
    return np.asarray(rows, dtype=np.float64)


def field_halos_from_rows(rows, z):
    out = []
    for r in rows:
        if r[0] == 0:
            out.append(synth.NFWHalo(r[1], r[2], z, r[3], theta=(r[6], r[7])))
        else:
            out.append(synth.NSIEHalo(r[1], z, r[2], r[3], r[4], r[5], theta=(r[6], r[7])))
    return out


def field_fixture():
    """LensPlaneTree::force of two field planes (NFW only; NFW + NSIE) for the
    four (sigma_back, inv_screening) cases at 300 plane positions."""
    z = 0.4
    cos = synth.Cosmology()
    half = 30 * synth.ARCSEC * cos.angdist(z)
    xx = np.random.default_rng(15).uniform(-half, half, (300, 2))
    R = H.RefDriver()
    arrays = {"z": z, "xx": xx, "cases": np.asarray(FIELD_CASES)}
    for name, halos in (("nfw", synth.field_halos(16, 300, z)),
                        ("mixed", synth.field_halos(17, 150, z, n_nsie=12))):
        arrays[name + "_rows"] = field_rows(halos)
        for c, (sb, iscr) in enumerate(FIELD_CASES):
            arrays[f"{name}_{c}"] = R.field_plane(synth.FieldPlane(z, halos, sb, iscr), xx)
    np.savez_compressed(os.path.join(OUT, "field_plane.npz"), **arrays)


# (kind, the reference driver's seven numbers, glb / oracle params)
SOURCE_CASES = (
    (0, (1e-5, -2e-5, 2e-5, 0, 0, 0, 0), (1e-5, -2e-5, 2e-5)),
    (1, (1e-5, -2e-5, 1.5e-5, 0, 0, 0, 0), (1e-5, -2e-5, 1.5e-5)),
    (2, (1e-5, -2e-5, 22.0, 0.8, 0.4, 2.5, 0.7), None),  # params get the reference's total flux
    (2, (-3e-6, 4e-6, 23.5, 0.3, -0.7, 1.0, 1.4), None),
)


def source_fixture():
    """Source::SurfaceBrightness of uniform, Gaussian and two Sersic sources."""
    y = np.random.default_rng(18).normal(0, 3e-5, (400, 2))
    y[:3] = [[1e-5, -2e-5], [-3e-6, 4e-6], [1e-5 + 1e-9, -2e-5]]  # centres: the r clamp
    R = H.RefDriver()
    arrays = {"y": y}
    for c, (kind, p7, _) in enumerate(SOURCE_CASES):
        sb, flux = R.source_sb(kind, p7, y)
        arrays[f"sb_{c}"] = sb
        arrays[f"flux_{c}"] = flux
    np.savez_compressed(os.path.join(OUT, "sources.npz"), **arrays)


def source_params(c, flux):
    kind, p7, prm = SOURCE_CASES[c]
    if prm is not None:
        return kind, prm
    return kind, (p7[0], p7[1], flux, p7[3], p7[4], p7[5], p7[6], -1.0)  # sb_limit -1: no cut


ADAPTIVE_N1D, ADAPTIVE_RANGE = 9, 30 * synth.ARCSEC


def adaptive_spec():
    return synth.LensSpec(zsource=2.0, halos=[synth.NFWHalo(3e14, 1.0, 0.4, 6.0),
                                              synth.NSIEHalo(2e12, 0.4, 200.0, 1e-4, 0.8, 0.3, theta=(2e-6, -1e-6))])


def adaptive_sources(ysrc):
    """(kind, the reference driver's seven numbers, glb / oracle params) for a
    Gaussian and an exponential Sersic source centred on a lensed grid point;
    both are smooth on the pixel scale, so the refinement converges in a few
    levels (the reference shoots its sub-rays one call each)."""
    x, y = float(ysrc[0]), float(ysrc[1])
    flux = 10 ** (-0.4 * 21.0)
    return ((1, (x, y, 1e-4, 0, 0, 0, 0), (x, y, 1e-4)),
            (2, (x, y, 21.0, 30.0, 0.5, 0.6, 0.8), (x, y, flux, 30.0, 0.5, 0.6, 0.8, -1.0)))


def adaptive_fixture():
    """GridMap::AdaptiveRefreshSurfaceBrightnesses totals from the reference."""
    spec = adaptive_spec()
    x = synth.grid_positions(ADAPTIVE_N1D, range_rad=ADAPTIVE_RANGE)
    y, _ = H.OracleLens(spec).rayshoot(x)
    ysrc = y[5 * ADAPTIVE_N1D + 4]
    R = H.RefDriver()
    totals = [R.adaptive(spec, ADAPTIVE_N1D, (0.0, 0.0), ADAPTIVE_RANGE, kind, p7)
              for kind, p7, _ in adaptive_sources(ysrc)]
    np.savez_compressed(os.path.join(OUT, "adaptive.npz"), ysrc=ysrc, totals=np.asarray(totals))


def smoothing_cases():
    """(name, particles, Nsmooth) of the kNN smoothing fixture: clustered and
    uniform sets, coincident particles, and N = 2*Nsmooth+1 (the reference's
    walk counts some particles twice there)."""
    rng = np.random.default_rng(41)
    cases = []
    cases.append(("nfw_500_8", synth.nfw_particles(rng, 500, 1e14, 5.0, 0.5, 0.0), 8))
    cube = np.zeros(3000, dtype=synth.PARTICLE_DTYPE)
    cube["x"] = rng.uniform(-1.0, 1.0, (3000, 3)).astype(np.float32)
    cube["Mass"] = 1.0
    cases.append(("cube_3000_16", cube, 16))
    cases.append(("nfw_3000_64", synth.nfw_particles(rng, 3000, 1e14, 5.0, 0.5, 0.0), 64))
    cases.append(("top_129_64", synth.nfw_particles(rng, 129, 1e14, 5.0, 0.5, 0.0), 64))
    cases.append(("top_17_8", synth.nfw_particles(rng, 17, 1e14, 5.0, 0.5, 0.0), 8))
    cases.append(("small_11_3", synth.nfw_particles(rng, 11, 1e14, 5.0, 0.5, 0.0), 3))
    dup = synth.nfw_particles(rng, 200, 1e14, 5.0, 0.5, 0.0)
    dup["x"][100:] = dup["x"][:100]
    cases.append(("dup_200_4", dup, 4))
    return cases


def smoothing_fixture():
    arrays = {}
    for name, p, ns in smoothing_cases():
        sizes, _ = H.RefDriver().smoothing(p, ns)
        arrays[f"{name}_particles"] = p
        arrays[f"{name}_sizes"] = sizes
        arrays[f"{name}_nsmooth"] = np.int32(ns)
    np.savez_compressed(os.path.join(OUT, "smoothing.npz"), **arrays)


UNIFORM_MAPS = (  # (map centre in arcsec, Nx, Ny, LensingVariable) on a 24^2 GridMap over 20 arcsec
    ((0.0, 0.0), 24, 24, 4),      # one pixel per grid point, KAPPA
    ((1.0, -0.5), 37, 31, 9),     # finer, offset, rectangular: INVMAG
    ((-2.0, 1.5), 41, 29, 2),     # ALPHA1
    ((0.5, 0.5), 33, 33, 5),      # GAMMA
)


def uniform_fixture():
    """GridMap::writePixelMapUniform (include/gridmap.h:506-690) on the lens of
    lens_small.npz; maps with at least as many pixels per side as the grid, so
    that no two grid points share a pixel (the reference's threads leave the
    value of a shared pixel unspecified)."""
    spec = lens_spec_from_fixture(np.load(os.path.join(OUT, "lens_small.npz")))
    R = H.RefDriver()
    rng_range = 20 * synth.ARCSEC
    arrays = {"grid_n": 24, "grid_range": rng_range}
    for k, ((cx, cy), nx, ny, var) in enumerate(UNIFORM_MAPS):
        of = R._file()
        R.run(R.lens_lines(spec) + [f"uniform 24 0 0 {rng_range!r} {cx * synth.ARCSEC!r} {cy * synth.ARCSEC!r} "
                                    f"{nx} {ny} {var} {of}"])
        arrays[f"map{k}"] = np.fromfile(of).reshape(ny, nx)
        arrays[f"map{k}_args"] = np.array([cx * synth.ARCSEC, cy * synth.ARCSEC, nx, ny, var])
    np.savez_compressed(os.path.join(OUT, "uniform_maps.npz"), **arrays)


def lens_spec_from_fixture(d) -> synth.LensSpec:
    """Rebuilds the LensSpec of lens_small.npz (insertion order as generated)."""
    halos = []
    i = 0
    while f"plane{i}_particles" in d:
        halos.append(synth.ParticlePlane(d[f"plane{i}_particles"], float(d[f"plane{i}_z"])))
        i += 1
    m, z, s, rc, f, pa = (float(v) for v in d["nsie"])
    halos.append(synth.NSIEHalo(m, z, s, rc, f, pa))
    m, r, z, c, tx, ty = (float(v) for v in d["nfw"])
    halos.append(synth.NFWHalo(m, r, z, c, theta=(tx, ty)))
    return synth.LensSpec(zsource=float(d["zsource"]), halos=halos)


if __name__ == "__main__":
    if not H.ref_available():
        sys.exit("oracle/_ref/glamer_ref missing: run `make -C oracle` where the reference tree exists")
    fixtures = {"tree": tree_fixture, "halos": halo_fixture, "lens": lens_fixture, "field": field_fixture,
                "sources": source_fixture, "adaptive": adaptive_fixture, "smoothing": smoothing_fixture,
                "uniform": uniform_fixture, "subtract": halo_subtract_fixture}
    for name in (sys.argv[1:] or fixtures):
        fixtures[name]()
    print("golden fixtures written to", OUT)
