"""Parity of the sm_100a library with the reference (golden fixtures) and the
oracle (live, seeded inputs), through the C ABI.

FP64 tolerance: the GPU performs the reference's operations with fused
multiply-adds and a different (depth-first, bottom-up) summation order, so
results agree to ~1e-13 relative; the tests allow 1e-9 relative to
max(|ref|, 1e-6 x median |ref| of the column)."""
import numpy as np
import pytest

import slsimlib_b200 as glb
from slsimlib_b200 import synth
from tests import harness as H
from tests.conftest import rel_err
from tests.golden.make_golden import lens_spec_from_fixture

pytestmark = pytest.mark.gpu

RTOL64 = 1e-9


def pack(a, k, g, ph):
    return np.concatenate([a, k[:, None], g, ph[:, None]], axis=1)


def vec_err(a, b, floor_frac=1e-6):
    """|a-b| / max(|b|, floor_frac * median |b|) for 2-vectors (alpha, gamma)."""
    nb = np.hypot(b[:, 0], b[:, 1])
    floor = max(floor_frac * np.median(nb), 1e-300)
    return np.hypot(*(a - b).T) / np.maximum(nb, floor)


def scal_err(a, b, floor_frac):
    floor = max(floor_frac * np.max(np.abs(b)), 1e-300)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def force_err(f, ref):
    """Largest relative error of alpha (vector), kappa, gamma (vector) and the
    potential.  kappa and phi pass through zero (the potential is a sum of
    logarithms), so their floors are 1e-6 and 1e-3 of the column's largest
    magnitude."""
    cols = np.array([vec_err(f[:, 0:2], ref[:, 0:2]).max(), scal_err(f[:, 2], ref[:, 2], 1e-6).max(),
                     vec_err(f[:, 3:5], ref[:, 3:5]).max(), scal_err(f[:, 6], ref[:, 6], 1e-3).max()])
    return cols.max(), cols


def make_lens(spec: synth.LensSpec) -> glb.Lens:
    return glb.lens_from_spec(spec)


# ------------------------------------------------------------------ trees
def test_tree_build_matches_reference_branch_by_branch(golden):
    d = golden("tree_small.npz")
    t = glb.TreeQuadParticles(d["particles"], bucket=int(d["bucket"]), theta_force=float(d["theta"]),
                              inv_screening_scale=float(d["inv_screening"]), keep_export=True)
    e, r = t.export(), d["export"]
    assert e.shape == r.shape
    # geometry, membership counts, big-particle counts and leaf flags: exact
    for c in (0, 1, 2, 3, 4, 5, 6, 14, 15):
        np.testing.assert_array_equal(e[:, c], r[:, c], err_msg=f"column {c}")
    # mass and centre of mass: summation order only
    np.testing.assert_allclose(e[:, 7], r[:, 7], rtol=1e-12)
    w = r[:, 3] - r[:, 1]
    for c in (8, 9):
        assert np.all(np.abs(e[:, c] - r[:, c]) <= 1e-12 * (np.abs(r[:, c]) + w))
    scale = np.abs(r[:, 7]) * w * w + 1e-300
    for c in (10, 11, 12):
        assert np.all(np.abs(e[:, c] - r[:, c]) <= 1e-9 * scale), c
    np.testing.assert_allclose(e[:, 13], r[:, 13], rtol=1e-10)


def test_tree_force_matches_reference(golden):
    d = golden("tree_small.npz")
    t = glb.TreeQuadParticles(d["particles"], bucket=int(d["bucket"]), theta_force=float(d["theta"]),
                              inv_screening_scale=float(d["inv_screening"]))
    f = pack(*t.force2D_recur(d["rays"]))
    m, cols = force_err(f, d["force"])
    assert m < RTOL64, cols


@pytest.mark.parametrize("inv_area,screen,periodic,bucket,theta", [
    (0.0, 0.0, False, 20, 0.1),
    (0.5, 0.0, False, 5, 0.3),
    (0.0, 2.0, False, 1, 0.05),
    (0.1, 0.0, True, 8, 0.2),
])
def test_tree_force_matches_oracle(inv_area, screen, periodic, bucket, theta):
    rng = np.random.default_rng(5)
    p = synth.nfw_particles(rng, 20000, 1e14, 5.0, 0.3, 1e-3)
    p["Size"][:200] = np.float32(0.03)  # big particles on internal branches
    rays = np.concatenate([rng.uniform(-0.05, 0.05, (200, 2)), rng.uniform(-1, 1, (56, 2))])
    ref = H.OracleTree(p, bucket=bucket, theta=theta, inv_area=inv_area, periodic=periodic,
                       inv_screening=screen).force(rays)
    t = glb.TreeQuadParticles(p, inv_area=inv_area, bucket=bucket, theta_force=theta,
                              periodic_buffer=periodic, inv_screening_scale=screen)
    f = pack(*t.force2D_recur(rays))
    m, cols = force_err(f, ref)
    assert m < RTOL64, cols


def test_tree_same_place_error():
    p = np.zeros(30, dtype=synth.PARTICLE_DTYPE)
    p["Mass"] = 1
    with pytest.raises(glb.GlamerError) as e:
        glb.TreeQuadParticles(p)
    assert e.value.code == glb.GLB_ERR_SAME_PLACE


def test_tree_tiny_and_empty_inputs():
    rng = np.random.default_rng(9)
    for n in (1, 2, 3, 25):
        p = np.zeros(n, dtype=synth.PARTICLE_DTYPE)
        p["x"][:, :2] = rng.uniform(-1, 1, (n, 2))
        p["Mass"] = 2.0
        p["Size"] = 0.1
        rays = rng.uniform(-1, 1, (7, 2))
        ref = H.OracleTree(p, bucket=5).force(rays)
        f = pack(*glb.TreeQuadParticles(p, bucket=5).force2D_recur(rays))
        m, cols = force_err(f, ref)
        assert m < RTOL64, (n, cols)
    t = glb.TreeQuadParticles(np.zeros(0, dtype=synth.PARTICLE_DTYPE))
    a, k, g, ph = t.force2D_recur(rng.uniform(-1, 1, (4, 2)))
    assert not a.any() and not k.any()
    a, k, g, ph = glb.TreeQuadParticles(p).force2D_recur(np.zeros((0, 2)))
    assert a.shape == (0, 2)


# ------------------------------------------------------------------ halos
def test_analytic_halos_match_reference(golden):
    d = golden("halos.npz")
    halos = {
        "nfw": glb.LensHaloNFW(1e14, 0.864, 0.3, 5.0),
        "nsie_cored": glb.LensHaloRealNSIE(1e13, 0.5, 250.0, 3.05e-4, 0.7, 0.0),
        "nsie_sis": glb.LensHaloRealNSIE(1e13, 0.5, 250.0, 0.0, 1.0, 0.0),
        "nsie_rot": glb.LensHaloRealNSIE(1e12, 0.5, 200.0, 1e-4, 0.5, 0.3),
    }
    for k, h in halos.items():
        f = pack(*h.force_halo(d["x"]))
        m, cols = force_err(f, d[k])
        # the NFW shear's analytic bin-0 formula (g2function, nfw_lens.cpp:111-121)
        # cancels ~1e7-fold as x -> 0, so CUDA's and glibc's last-ulp libm
        # differences appear at ~2e-9 there
        tol = 1e-8 if k == "nfw" else RTOL64
        assert m < tol, (k, cols)
        np.testing.assert_allclose(h.params(), d[k + "_params"], rtol=1e-6, err_msg=k)


def test_analytic_halos_subtract_point_match_reference(golden):
    """force_halo(..., subtract_point = true, screening) against the
    reference's own output (golden halos_subtract.npz): the screened point
    mass of force_point inside Rmax plus, for NFW, force_halo_sym's unscreened
    one; nothing beyond Rmax."""
    d = golden("halos_subtract.npz")
    halos = {"nfw": glb.LensHaloNFW(1e14, 0.864, 0.3, 5.0),
             "nsie_sis": glb.LensHaloRealNSIE(1e13, 0.5, 250.0, 0.0, 1.0, 0.0),
             "nsie_rot": glb.LensHaloRealNSIE(1e12, 0.5, 200.0, 0.0, 0.6, 0.3)}
    for k, h in halos.items():
        for s in (1.0, 0.25):
            f = pack(*h.force_halo(d["x"], subtract_point=True, screening=s))
            m, cols = force_err(f, d[f"{k}_{s}"])
            assert m < (1e-8 if k == "nfw" else RTOL64), (k, s, cols)


def test_particle_halo_force_matches_oracle():
    rng = np.random.default_rng(6)
    p = synth.nfw_particles(rng, 5000, 1e13, 6.0, 0.5, 5e-4)
    x = rng.uniform(-0.2, 0.2, (128, 2))
    ref, _ = H.oracle_halo_force(synth.ParticlePlane(p, 0.5), x)
    f = pack(*glb.LensHaloParticles(p, 0.5).force_halo(x))
    m, cols = force_err(f, ref)
    assert m < RTOL64, cols


# ------------------------------------------------------------------- lens
def test_gridmap_and_rays_match_reference(golden):
    d = golden("lens_small.npz")
    spec = lens_spec_from_fixture(d)
    L = make_lens(spec)
    z, Dl, dDl = L.planes()
    zo, Dlo, dDlo = H.OracleLens(spec).planes()
    np.testing.assert_allclose(z, zo, rtol=0)
    np.testing.assert_allclose(Dl, Dlo, rtol=1e-12)
    gm = glb.GridMap(L, int(d["grid_n"]), (0.0, 0.0), float(d["grid_range"]))
    assert np.max(rel_err(gm.y, d["grid_y"])) < RTOL64
    assert np.max(np.abs(gm.A - d["grid_A"])) < 1e-9
    y, A = L.rayshooterInternal(d["rays_x"], d["rays_zs"])
    assert np.max(rel_err(y, d["rays_y"])) < RTOL64
    assert np.max(np.abs(A - d["rays_A"])) < 1e-9


def test_light_cone_matches_oracle_and_reset_source():
    spec = synth.light_cone(seed=31, n_total=60000, n_planes=5, halos_per_plane=6)
    L = make_lens(spec)
    O = H.OracleLens(spec)
    x = synth.grid_positions(48, range_rad=60 * synth.ARCSEC)
    y, A = L.rayshooterInternal(x)
    yo, Ao = O.rayshoot(x)
    assert np.max(rel_err(y, yo)) < RTOL64
    assert np.max(np.abs(A - Ao)) < 1e-9
    # a lower source plane (Lens::ResetSourcePlane)
    assert L.ResetSourcePlane(0.6, False) == O.reset_source(0.6, False)
    y, A = L.rayshooterInternal(x)
    yo, Ao = O.rayshoot(x)
    assert np.max(rel_err(y, yo)) < RTOL64
    assert np.max(np.abs(A - Ao)) < 1e-9


def test_single_plane_full_grid_matches_reference():
    """The single-plane workload at full size -- 2^18 NFW particles (1e14 Msun,
    c = 5, z = 0.3, 1 kpc softening), a 512^2 GridMap over 30 arcsec, z_s = 2 --
    in the FP64 form: against the reference's own GridMap (oracle/_ref) on
    every ray when it is built here, else against the oracle on 4096 seeded
    rays of the grid."""
    spec = synth.single_plane_nfw(seed=1)
    L = make_lens(spec)
    rng_rad = 30 * synth.ARCSEC
    gm = glb.GridMap(L, 512, (0.0, 0.0), rng_rad)
    if H.ref_available():
        yr, Ar, _ = H.RefDriver().grid(spec, 512, range_rad=rng_rad)
        y, A = gm.y, gm.A
    else:
        idx = np.sort(np.random.default_rng(8).choice(512 * 512, size=4096, replace=False))
        yr, Ar = H.OracleLens(spec).rayshoot(synth.grid_positions(512, range_rad=rng_rad)[idx])
        y, A = gm.y[idx], gm.A[idx]
    assert np.max(rel_err(y, yr)) < RTOL64
    assert np.max(np.abs(A - Ar)) < 1e-9


def test_light_cone_full_size_matches_reference():
    """The headline light cone at full size -- 10 particle planes holding
    4,194,304 particles and the NSIE, the 2048^2 grid over 60 arcsec -- in the
    FP64 form on the whole grid, checked on 2,048 seeded rays against the
    reference's own rayshooterInternal when oracle/_ref is built here, else
    against the oracle."""
    spec = synth.light_cone(seed=2)
    L = make_lens(spec)
    gm = glb.GridMap(L, 2048, (0.0, 0.0), 60 * synth.ARCSEC)
    idx = np.sort(np.random.default_rng(19).choice(2048 * 2048, size=2048, replace=False))
    x = synth.grid_positions(2048, range_rad=60 * synth.ARCSEC)[idx]
    if H.ref_available():
        yr, Ar, _ = H.RefDriver().rays(spec, x)
    else:
        yr, Ar = H.OracleLens(spec).rayshoot(x)
    assert np.max(rel_err(gm.y[idx], yr)) < RTOL64
    assert np.max(np.abs(gm.A[idx] - Ar)) < 1e-9


def test_lens_edge_cases():
    # no lens plane: identity (internal_rayshooter_multi.cpp:62-76)
    L = glb.Lens(2.0)
    x = np.random.default_rng(1).uniform(-1e-4, 1e-4, (5, 2))
    y, A = L.rayshooterInternal(x)
    np.testing.assert_array_equal(y, x)
    np.testing.assert_array_equal(A, np.tile([1.0, 0, 0, 1.0], (5, 1)))
    spec = synth.single_plane_nfw(seed=2, n=4096)
    L = make_lens(spec)
    y, A = L.rayshooterInternal(np.zeros((0, 2)))
    assert y.shape == (0, 2)
    with pytest.raises(ValueError):
        L.rayshooterInternal(x, source_zs=[1.0, 2.0])
    # a single ray, and sources in front of / behind the plane
    O = H.OracleLens(spec)
    x1 = np.array([[1e-5, -2e-5]])
    for zs in (None, np.array([0.1]), np.array([3.0])):
        y, A = L.rayshooterInternal(x1, zs)
        yo, Ao = O.rayshoot(x1, zs)
        assert np.max(rel_err(y, yo)) < RTOL64
        assert np.max(np.abs(A - Ao)) < 1e-9


# ------------------------------------------------------- split precision
def within(st, name, med=1e-6, p999=1e-5):
    return st[name]["median"] <= med and st[name]["p999"] <= p999


@pytest.mark.parametrize("n_total,n_planes", [(200000, 1), (200000, 4), (400000, 10)])
def test_split_precision_tolerance(n_total, n_planes):
    """The split form against the plain FP64 form (median <= 1e-6, 99.9th
    percentile <= 1e-5; kappa and gamma relative to max(|ref|, 1e-3), invmag
    where |invmag_ref| > 0.05).

    The deflection is within the bounds end to end, and on one plane so are
    kappa, gamma and invmag.  Through several planes of particle lenses whose
    particles have Einstein radii of about their softening length, the
    recursion amplifies any per-plane difference: a deflection difference of
    FP32 size moves the ray enough to change the shear at later planes, and a
    shear difference of FP32 size is carried through the products of later
    planes' Jacobians.  tests.harness.PlaneRecursion separates the two: the
    end-to-end kappa/gamma/invmag error is the propagated deflection
    difference (split deflection with FP64 kappa/gamma gives the same error),
    and the split kappa/gamma evaluated at the FP64 form's positions is within
    1e-6 at the median.  The 99.9th-percentile bound is not met through
    several planes (test_split_multi_plane_p999_bound)."""
    spec = synth.light_cone(seed=41, n_total=n_total, n_planes=n_planes, halos_per_plane=8)
    L = make_lens(spec)
    x = synth.grid_positions(96, range_rad=60 * synth.ARCSEC)
    y64, A64 = L.rayshooterInternal(x, precision=glb.PREC_FP64)
    y32, A32 = L.rayshooterInternal(x, precision=glb.PREC_SPLIT)
    st = H.error_stats(x, y32, A32, y64, A64)
    assert within(st, "alpha"), st
    if n_planes == 1:
        for name in ("kappa", "gamma", "invmag"):
            assert within(st, name), (name, st)
        return
    R = H.PlaneRecursion(spec, L)
    F, S = glb.PREC_FP64, glb.PREC_SPLIT
    y0, A0 = R.shoot(x, F, F)
    assert np.max(rel_err(y0, y64)) < 1e-10 and np.max(np.abs(A0 - A64)) < 1e-7  # the recursion is the library's
    ev = H.error_stats(x, *R.shoot(x, F, S), y0, A0)
    pr = H.error_stats(x, *R.shoot(x, S, F), y0, A0)
    for name in ("kappa", "gamma", "invmag"):
        assert ev[name]["median"] <= 1e-6, ("evaluation", name, ev)
        # the end-to-end error is the propagated one
        assert 0.5 * st[name]["median"] <= pr[name]["median"] <= 2 * st[name]["median"] + 1e-12, (name, st, pr)


@pytest.mark.xfail(strict=True, reason="through several planes of particles with Einstein radii about their "
                   "softening length, FP32-size per-plane deflection and shear differences are amplified beyond "
                   "1e-5 at the 99.9th percentile of kappa/gamma/invmag; the FP64 form with 1e-8 relative "
                   "deflection noise misses the bound too (bench line: kappa_gamma_attribution)")
def test_split_multi_plane_p999_bound():
    """The north-star 99.9th-percentile bound (1e-5) on kappa, gamma and
    invmag of the split form, end to end through four particle planes:
    recorded as not met (strict: an unexpected pass fails)."""
    spec = synth.light_cone(seed=41, n_total=200000, n_planes=4, halos_per_plane=8)
    L = make_lens(spec)
    x = synth.grid_positions(96, range_rad=60 * synth.ARCSEC)
    y64, A64 = L.rayshooterInternal(x, precision=glb.PREC_FP64)
    y32, A32 = L.rayshooterInternal(x, precision=glb.PREC_SPLIT)
    st = H.error_stats(x, y32, A32, y64, A64)
    for name in ("kappa", "gamma", "invmag"):
        assert st[name]["p999"] <= 1e-5, (name, st)


# --------------------------------------------- tree-force forms, direct sum
def test_tree_force_device_forms_and_direct_sum():
    import torch
    rng = np.random.default_rng(12)
    p = synth.nfw_particles(rng, 30000, 1e14, 5.0, 0.3, 1e-3)
    rays = rng.uniform(-0.1, 0.1, (1000, 2))
    t = glb.TreeQuadParticles(p, bucket=20, theta_force=0.1, inv_screening_scale=1.0)
    a, k, g, _ = t.force2D_recur(rays)
    ref = np.concatenate([a, k[:, None], g[:, :2]], axis=1)
    dr = torch.from_numpy(rays).cuda()
    outs = {}
    for prec in (glb.PREC_FP64, glb.PREC_SPLIT, glb.PREC_FP32):
        o = torch.zeros((len(rays), 5), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        t.force_device(len(rays), dr.data_ptr(), o.data_ptr(), prec, None)
        torch.cuda.synchronize()
        outs[prec] = o.cpu().numpy()
    assert np.max(vec_err(outs[glb.PREC_FP64][:, :2], ref[:, :2])) < 1e-12
    e_split = vec_err(outs[glb.PREC_SPLIT][:, :2], ref[:, :2])
    assert np.median(e_split) < 1e-6 and e_split.max() < 1e-5
    e32 = vec_err(outs[glb.PREC_FP32][:, :2], ref[:, :2])
    assert np.median(e32) < 1e-4  # the plain FP32 form: reported, loosely bounded
    # FP64 direct sum on the GPU against the oracle's
    pd = torch.from_numpy(p.view(np.uint8)).cuda()
    o = torch.zeros((64, 5), dtype=torch.float64, device="cuda")
    dr64 = dr[:64].contiguous()
    torch.cuda.synchronize()
    glb.direct_sum_device(len(p), pd.data_ptr(), 0.0, 64, dr64.data_ptr(), o.data_ptr(), None)
    torch.cuda.synchronize()
    ds = H.direct_sum(p, rays[:64])
    assert np.max(vec_err(o.cpu().numpy()[:, :2], ds[:, :2])) < 1e-10


def test_split_tree_force_two_rays_per_thread():
    """From 2^20 rays on (opening angle under 0.2) the split tree force walks
    two rays per thread: each ray's result is bit-identical to the one-ray
    kernel's (calls under 2^20 rays), in any ray order, including an odd
    count that leaves the last thread one ray; the split tolerance against
    the FP64 form holds."""
    import torch
    rng = np.random.default_rng(31)
    p = synth.nfw_particles(rng, 200000, 1e14, 5.0, 0.3, 1e-3)
    t = glb.TreeQuadParticles(p, bucket=5, theta_force=0.1)
    n = (1 << 20) + 1
    rays = np.concatenate([rng.normal(0, 0.02, (n // 2, 2)), rng.uniform(-0.3, 0.3, (n - n // 2, 2))])
    rays = rays[rng.permutation(n)]  # arbitrary order: pairs of rays far apart
    dr = torch.from_numpy(rays).cuda()

    def force(lo, hi, prec):
        o = torch.zeros((hi - lo, 5), dtype=torch.float64, device="cuda")
        d = dr[lo:hi].contiguous()
        torch.cuda.synchronize()
        t.force_device(hi - lo, d.data_ptr(), o.data_ptr(), prec, None)
        torch.cuda.synchronize()
        return o.cpu().numpy()

    two = force(0, n, glb.PREC_SPLIT)
    h = 1 << 19
    one = np.concatenate([force(0, h, glb.PREC_SPLIT), force(h, n, glb.PREC_SPLIT)])
    np.testing.assert_array_equal(two, one)
    ref = np.concatenate([force(0, h, glb.PREC_FP64), force(h, n, glb.PREC_FP64)])
    for name, e in (("alpha", vec_err(two[:, :2], ref[:, :2])), ("kappa", scal_err(two[:, 2], ref[:, 2], 1e-6)),
                    ("gamma", vec_err(two[:, 3:5], ref[:, 3:5]))):
        assert np.median(e) <= 1e-6 and np.percentile(e, 99.9) <= 1e-5, (name, np.median(e), e.max())


@pytest.mark.parametrize("inv_area,screen,negative", [(0.0, 0.0, False), (4.0, 0.0, False), (0.0, 1.0, False),
                                                     (4.0, 30.0, False), (4.0, 1.0, True)])
def test_split_tree_force_softened_regime(inv_area, screen, negative):
    """Split form against the FP64 form where most leaf particles lie within two
    softening lengths of the rays (softening larger than the core's leaves, so
    B-spline corrections are applied both at leaves and at ancestors), with and
    without the inv_area sheet (closed form for masses of one sign, term by
    term for mixed signs) and screening: alpha, kappa and gamma within 1e-6
    median / 1e-5 99.9th percentile; the plain FP32 form loosely."""
    import torch
    rng = np.random.default_rng(21)
    p = synth.nfw_particles(rng, 60000, 1e14, 5.0, 0.3, 4e-3)
    p["Size"][:500] = np.float32(2e-2)  # a few much larger softenings
    if negative:
        p["Mass"][::10] *= np.float32(-0.5)
    rays = np.concatenate([rng.normal(0, 0.01, (3000, 2)), rng.uniform(-0.2, 0.2, (1000, 2))])
    t = glb.TreeQuadParticles(p, inv_area=inv_area, bucket=20, theta_force=0.1, inv_screening_scale=screen)
    dr = torch.from_numpy(rays).cuda()
    outs = {}
    for prec in (glb.PREC_FP64, glb.PREC_SPLIT, glb.PREC_FP32):
        o = torch.zeros((len(rays), 5), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        t.force_device(len(rays), dr.data_ptr(), o.data_ptr(), prec, None)
        torch.cuda.synchronize()
        outs[prec] = o.cpu().numpy()
    ref = outs[glb.PREC_FP64]
    orc = H.OracleTree(p, bucket=20, theta=0.1, inv_area=inv_area, inv_screening=screen).force(rays[:100])
    assert np.max(vec_err(ref[:100, :2], orc[:, :2])) < RTOL64  # the FP64 form is the reference's walk
    s = outs[glb.PREC_SPLIT]
    for name, e in (("alpha", vec_err(s[:, :2], ref[:, :2])), ("kappa", scal_err(s[:, 2], ref[:, 2], 1e-6)),
                    ("gamma", vec_err(s[:, 3:5], ref[:, 3:5]))):
        assert np.median(e) <= 1e-6 and np.percentile(e, 99.9) <= 1e-5, (name, np.median(e), e.max())
    assert np.median(vec_err(outs[glb.PREC_FP32][:, :2], ref[:, :2])) < 1e-4
