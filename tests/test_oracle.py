"""The oracle (C restatement) against the reference's own outputs.

Golden fixtures come from the reference compiled in place
(tests/golden/make_golden.py); when oracle/_ref/glamer_ref is present the
oracle is also compared live on fresh seeded inputs.  CPU only."""
import numpy as np
import pytest

from slsimlib_b200 import synth
from tests import harness as H
from tests.golden.make_golden import lens_spec_from_fixture

EXACT = 1e-13  # the restatement performs the reference's operations in order


def test_tree_matches_golden(golden):
    d = golden("tree_small.npz")
    t = H.OracleTree(d["particles"], bucket=int(d["bucket"]), theta=float(d["theta"]),
                     inv_screening=float(d["inv_screening"]))
    np.testing.assert_allclose(t.export(), d["export"], rtol=EXACT, atol=0)
    np.testing.assert_allclose(t.force(d["rays"]), d["force"], rtol=EXACT, atol=0)


def test_halos_match_golden(golden):
    d = golden("halos.npz")
    halos = {
        "nfw": synth.NFWHalo(1e14, 0.864, 0.3, 5.0),
        "nsie_cored": synth.NSIEHalo(1e13, 0.5, 250.0, 3.05e-4, 0.7, 0.0),
        "nsie_sis": synth.NSIEHalo(1e13, 0.5, 250.0, 0.0, 1.0, 0.0),
        "nsie_rot": synth.NSIEHalo(1e12, 0.5, 200.0, 1e-4, 0.5, 0.3),
    }
    for k, h in halos.items():
        f, prm = H.oracle_halo_force(h, d["x"])
        np.testing.assert_allclose(f, d[k], rtol=1e-12, atol=0, err_msg=k)
        np.testing.assert_allclose(prm, d[k + "_params"], rtol=1e-6, err_msg=k)


def test_lens_matches_golden(golden):
    d = golden("lens_small.npz")
    spec = lens_spec_from_fixture(d)
    O = H.OracleLens(spec)
    x = synth.grid_positions(int(d["grid_n"]), range_rad=float(d["grid_range"]))
    y, A = O.rayshoot(x)
    np.testing.assert_allclose(y, d["grid_y"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(A, d["grid_A"], rtol=1e-10, atol=1e-12)
    y2, A2 = O.rayshoot(d["rays_x"], d["rays_zs"])
    np.testing.assert_allclose(y2, d["rays_y"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(A2, d["rays_A"], rtol=1e-10, atol=1e-12)


def test_tree_big_particles_and_edge_shapes():
    # ragged inputs: a handful of particles, a line-like cloud, sizes spanning the tree
    rng = np.random.default_rng(3)
    for n in (1, 2, 21, 500):
        p = np.zeros(n, dtype=synth.PARTICLE_DTYPE)
        p["x"][:, 0] = rng.uniform(-1, 1, n)
        p["x"][:, 1] = rng.uniform(-1, 1, n) * 1e-3
        p["Mass"] = 1.0
        p["Size"] = rng.uniform(1e-4, 0.5, n).astype(np.float32)
        if n == 1:
            t = H.OracleTree(p, bucket=5)
            f = t.force(np.array([[0.3, 0.2]]))
            assert np.all(np.isfinite(f))
            continue
        t = H.OracleTree(p, bucket=5)
        e = t.export()
        assert e[0, 5] == n
        # every particle is in exactly one leaf
        assert e[e[:, 14] == 1, 5].sum() == n


def test_same_place_raises():
    p = np.zeros(4, dtype=synth.PARTICLE_DTYPE)
    p["Mass"] = 1
    with pytest.raises(ValueError):
        H.OracleTree(p)


def test_direct_sum_is_close_to_tree():
    d = np.load(__import__("os").path.join(H.ROOT, "tests", "golden", "tree_small.npz"))
    p = d["particles"]
    rays = d["rays"][:16]
    t = H.OracleTree(p, bucket=20, theta=0.1)
    ft = t.force(rays)
    fd = H.direct_sum(p, rays)
    a_t = np.hypot(ft[:, 0], ft[:, 1])
    a_d = np.hypot(fd[:, 0], fd[:, 1])
    # quadTree.h:37-38: theta = 0.1 gives better than 1% on alpha
    assert np.max(np.abs(a_t - a_d) / a_d) < 1e-2


@pytest.mark.skipif(not H.ref_available(), reason="reference build (oracle/_ref) not present")
def test_oracle_matches_reference_live():
    spec = synth.light_cone(seed=21, n_total=8000, n_planes=2, halos_per_plane=2)
    R = H.RefDriver()
    y_r, A_r, _ = R.grid(spec, 12, range_rad=60 * synth.ARCSEC)
    O = H.OracleLens(spec)
    y_o, A_o = O.rayshoot(synth.grid_positions(12, range_rad=60 * synth.ARCSEC))
    np.testing.assert_allclose(y_o, y_r, rtol=1e-12, atol=0)
    np.testing.assert_allclose(A_o, A_r, rtol=1e-10, atol=1e-12)


def test_cosmology_shim_matches_product_restatement():
    # the oracle's adaptive-Simpson distances against the library's (and the
    # synthetic generator's) Gauss-Legendre ones
    L = H.oracle_lib()
    c = synth.Cosmology()
    for z in (0.1, 0.3, 0.5, 1.0, 2.5, 5.0):
        assert abs(L.orc_coordist(z) - c.coordist(z)) < 1e-9 * c.coordist(z)


def test_field_plane_matches_golden(golden):
    """TreeQuadHalos / LensPlaneTree restatement against the reference.  NFW
    fields agree to rounding; with NSIE haloes the cored NSIE's mass (a
    numerical integral whose upstream integrator is not available,
    lens_halos.cpp:1073-1075, 2469-2473) can differ by one FP32 ulp, which
    reaches the far-field cells' masses and the blend beyond Rsize."""
    from tests.golden.make_golden import field_halos_from_rows
    d = golden("field_plane.npz")
    z = float(d["z"])
    for name, tol in (("nfw", 1e-9), ("mixed", 2e-6)):
        halos = field_halos_from_rows(d[name + "_rows"], z)
        for c, (sb, iscr) in enumerate(d["cases"]):
            f, _ = H.oracle_halo_force(synth.FieldPlane(z, halos, float(sb), float(iscr)), d["xx"])
            ref = d[f"{name}_{c}"]
            scale = np.abs(ref).max(axis=0)
            err = np.abs(f - ref).max(axis=0) / np.where(scale > 0, scale, 1)
            assert err.max() < tol, (name, c, err)


def test_source_surface_brightness_matches_golden(golden):
    """Uniform, Gaussian and Sersic surface brightness against the reference's
    Source::SurfaceBrightness (the Sersic's total flux from its magnitude)."""
    from tests.golden.make_golden import SOURCE_CASES, source_params
    d = golden("sources.npz")
    for c in range(len(SOURCE_CASES)):
        kind, prm = source_params(c, float(d[f"flux_{c}"]))
        sb = H.oracle_source_sb(kind, prm, d["y"])
        np.testing.assert_allclose(sb, d[f"sb_{c}"], rtol=1e-13, atol=0, err_msg=str(c))


def test_adaptive_refresh_matches_golden(golden):
    """GridMap::AdaptiveRefreshSurfaceBrightnesses (the one-ray-per-call
    refinement client) restated: the total flux against the reference's."""
    from tests.golden.make_golden import (ADAPTIVE_N1D, ADAPTIVE_RANGE, adaptive_sources, adaptive_spec)
    d = golden("adaptive.npz")
    O = H.OracleLens(adaptive_spec())
    for (kind, _, prm), tref in zip(adaptive_sources(d["ysrc"]), d["totals"]):
        sb, tot = O.adaptive_sb(ADAPTIVE_N1D, (0.0, 0.0), ADAPTIVE_RANGE, kind, prm)
        assert abs(tot - tref) <= 1e-8 * abs(tref), (kind, tot, tref)
        # refinement happened: the refined map differs from the plain one
        x = synth.grid_positions(ADAPTIVE_N1D, range_rad=ADAPTIVE_RANGE)
        y, _ = O.rayshoot(x)
        assert np.any(sb != H.oracle_source_sb(kind, prm, y))


def smoothing_golden_cases(golden):
    d = golden("smoothing.npz")
    names = sorted({k[: -len("_particles")] for k in d.files if k.endswith("_particles")})
    return [(nm, d[f"{nm}_particles"], int(d[f"{nm}_nsmooth"]), d[f"{nm}_sizes"]) for nm in names]


def brute_kth(p, k):
    """Distance to the k-th nearest particle (1-based, the particle itself
    counted) with NNDistance's arithmetic: float differences, double sum."""
    x = p["x"]
    d2 = np.zeros((len(p), len(p)))
    for j in range(3):
        dx = (x[None, :, j] - x[:, None, j]).astype(np.float32).astype(np.float64)
        d2 += dx * dx
    return np.sqrt(np.sort(d2, axis=1)[:, k - 1]).astype(np.float32)


def test_smoothing_matches_golden(golden):
    """orc_calculate_smoothing reproduces calculate_smoothing bit for bit."""
    for name, p, ns, sizes in smoothing_golden_cases(golden):
        got = H.oracle_smoothing(p, ns)
        assert np.array_equal(got, sizes), name


def test_smoothing_golden_is_exact_knn_except_top_walk(golden):
    """The reference's answer is the exact (Nsmooth+1)-th nearest distance,
    except for N = 2*Nsmooth+1, where queries in the top node's first child
    (x below the median) see some particles twice and get a smaller value."""
    for name, p, ns, sizes in smoothing_golden_cases(golden):
        exact = brute_kth(p, ns + 1)
        if len(p) == 2 * ns + 1:
            xs = np.sort(p["x"][:, 0])
            first = p["x"][:, 0] < xs[len(p) // 2]
            assert np.array_equal(sizes[~first], exact[~first]), name
            assert np.all(sizes[first] <= exact[first]) and np.any(sizes[first] < exact[first]), name
        else:
            assert np.array_equal(sizes, exact), name


def test_smoothing_oracle_errors():
    p = synth.nfw_particles(np.random.default_rng(3), 10, 1e14, 5.0, 0.5, 0.0)
    with pytest.raises(ValueError):
        H.oracle_smoothing(p, 0)
    with pytest.raises(ValueError):
        H.oracle_smoothing(p, 9)  # N <= Nsmooth+1


@pytest.mark.skipif(not H.ref_available(), reason="reference not compiled here")
def test_smoothing_oracle_matches_reference_live():
    rng = np.random.default_rng(77)
    for n, ns in ((6000, 32), (65, 32), (2500, 1), (3, 1), (4, 1), (5, 2), (7, 3), (8, 3)):
        p = synth.nfw_particles(rng, n, 3e14, 4.0, 0.3, 0.0)
        ref, _ = H.RefDriver().smoothing(p, ns)
        assert np.array_equal(H.oracle_smoothing(p, ns), ref), (n, ns)


def test_uniform_pixelmap_restatement_matches_reference(golden):
    """The restatement of GridMap::writePixelMapUniform (harness.uniform_map_restated)
    over the oracle's rays reproduces the reference's maps (golden uniform_maps.npz)."""
    from tests.golden.make_golden import lens_spec_from_fixture
    d = golden("uniform_maps.npz")
    spec = lens_spec_from_fixture(golden("lens_small.npz"))
    n1d, rng = int(d["grid_n"]), float(d["grid_range"])
    x = synth.grid_positions(n1d, range_rad=rng)
    y, A = H.OracleLens(spec).rayshoot(x)
    a = x - y
    g1, g2 = (A[:, 0] - A[:, 3]) / 2, (A[:, 1] + A[:, 2]) / 2
    vals = {4: 1 - (A[:, 0] + A[:, 3]) / 2, 9: A[:, 0] * A[:, 3] - A[:, 1] * A[:, 2], 2: a[:, 0],
            5: np.hypot(g1, g2)}
    for k in range(4):
        cx, cy, nx, ny, var = d[f"map{k}_args"]
        m = H.uniform_map_restated(x, vals[int(var)], (cx, cy), int(nx), int(ny), rng)
        ref = d[f"map{k}"]
        np.testing.assert_array_equal(m == 0, ref == 0)
        assert np.max(np.abs(m - ref) / np.maximum(np.abs(ref), 1e-6 * np.abs(ref).max())) < 1e-9, k
