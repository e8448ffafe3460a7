"""Field planes (LensPlaneTree over NFW / NSIE haloes, TreeQuadHalos walk) on
the GPU: the plane force against the oracle and the reference's golden
outputs, and lenses mixing field and particle planes through every entry
point (per-plane kernels, the batched launch, the allocation-free entry
point) against the oracle and the FP64 form."""
import ctypes as C

import numpy as np
import pytest

import slsimlib_b200 as glb
from slsimlib_b200 import synth
from tests import harness as H
from tests.golden.make_golden import lens_spec_from_fixture
from tests.conftest import rel_err
from tests.golden.make_golden import field_halos_from_rows
from tests.test_gpu_parity import RTOL64, force_err, pack

pytestmark = pytest.mark.gpu

Z = 0.4
CASES = ((0.0, 0.0), (5.0, 0.0), (0.0, 2.0), (2.0, 1.0))  # (sigma_background, inv_screening_scale)


def plane_positions(n=400, seed=1):
    half = 30 * synth.ARCSEC * synth.Cosmology().angdist(Z)
    return np.random.default_rng(seed).uniform(-half, half, (n, 2))


@pytest.mark.parametrize("sb,iscr", CASES)
def test_field_plane_force_matches_oracle(sb, iscr):
    fp = synth.FieldPlane(Z, synth.field_halos(21, 250, Z, n_nsie=10), sb, iscr)
    xx = plane_positions()
    f = pack(*glb.halo_from_spec(fp).force_halo(xx))
    ref = H.oracle_halo_force(fp, xx)[0]
    m, cols = force_err(f, ref)
    assert m < RTOL64, cols


def test_field_plane_matches_reference_golden(golden):
    d = golden("field_plane.npz")
    z = float(d["z"])
    for name, tol in (("nfw", 1e-9), ("mixed", 2e-6)):
        halos = field_halos_from_rows(d[name + "_rows"], z)
        for c, (sb, iscr) in enumerate(d["cases"]):
            fp = synth.FieldPlane(z, halos, float(sb), float(iscr))
            f = pack(*glb.halo_from_spec(fp).force_halo(d["xx"]))
            ref = d[f"{name}_{c}"]
            scale = np.abs(ref).max(axis=0)
            err = np.abs(f - ref).max(axis=0) / np.where(scale > 0, scale, 1)
            assert err.max() < tol, (name, c, err)


def mixed_spec(seed=5):
    spec = synth.light_cone(seed=seed, n_total=80000, n_planes=3, halos_per_plane=5, zs=2.0)
    spec.halos.append(synth.FieldPlane(0.2, synth.field_halos(seed + 1, 120, 0.2, n_nsie=4), 0.0, 0.0))
    spec.halos.append(synth.FieldPlane(0.8, synth.field_halos(seed + 2, 200, 0.8), 2.0, 1.0))
    return spec


def test_lens_with_field_planes_matches_oracle():
    spec = mixed_spec()
    L = glb.lens_from_spec(spec)
    O = H.OracleLens(spec)
    z, Dl, _ = L.planes()
    zo, Dlo, _ = O.planes()
    np.testing.assert_allclose(z, zo, rtol=0)
    np.testing.assert_allclose(Dl, Dlo, rtol=1e-12)
    assert L.getNplanes() == len(zo) - 1
    x = synth.grid_positions(40, range_rad=60 * synth.ARCSEC)
    y64, A64 = L.rayshooterInternal(x)
    yo, Ao = O.rayshoot(x)
    assert np.max(rel_err(y64, yo)) < RTOL64
    assert np.max(np.abs(A64 - Ao)) < 1e-9
    zs = np.random.default_rng(3).uniform(0.1, 2.5, len(x))
    y, A = L.rayshooterInternal(x, zs)
    yo, Ao = O.rayshoot(x, zs)
    assert np.max(rel_err(y, yo)) < RTOL64
    assert np.max(np.abs(A - Ao)) < 1e-9
    # the split form walks the particle planes in FP32: deflection within bounds
    ys, _ = L.rayshooterInternal(x, precision=glb.PREC_SPLIT)
    a, ar = x - ys, x - y64
    e = np.hypot(*(a - ar).T) / np.hypot(*ar.T)
    assert np.median(e) <= 1e-6 and np.percentile(e, 99.9) <= 1e-5


def test_batch_and_noalloc_with_field_planes():
    import torch
    spec = mixed_spec(seed=9)
    L = glb.lens_from_spec(spec)
    rng = 40 * synth.ARCSEC
    gm = glb.GridMap(L, 33, (0.0, 0.0), rng, glb.PREC_FP64)
    b = glb.GridBatch([L], [33], [(0.0, 0.0)], [rng], glb.PREC_FP64)
    b.run(True)
    y, A = b.result(0)
    # two FP64 kernels (per plane / all planes per launch) with different
    # multiply-add contraction; the grainy lens amplifies 1e-16 rounding (the
    # suite's FP64 tolerance)
    assert np.max(rel_err(y, gm.y)) < 1e-9
    assert np.max(np.abs(A - gm.A)) < 1e-9
    x = torch.from_numpy(gm.positions()).cuda()
    n = len(x)
    out = [torch.empty((n, 2), dtype=torch.float64, device="cuda"), torch.empty((n, 4), dtype=torch.float64,
                                                                                  device="cuda")]
    torch.cuda.synchronize()
    lib = glb.load_library()
    glb._check(lib.glb_lens_rayshoot_noalloc(L._h, n, x.data_ptr(), None, out[0].data_ptr(), out[1].data_ptr(),
                                             glb.PREC_FP64, None))
    torch.cuda.synchronize()
    assert np.max(rel_err(out[0].cpu().numpy(), gm.y)) < 1e-12
    assert np.max(np.abs(out[1].cpu().numpy() - gm.A)) < 1e-12


def test_field_plane_errors_and_edges():
    # members must be NFW / NSIE
    p = synth.nfw_particles(np.random.default_rng(1), 500, 1e13, 5.0, Z, 1e-3)
    with pytest.raises(glb.GlamerError) as e:
        glb.LensPlaneTree(Z, [glb.LensHaloParticles(p, Z)])._make()
    assert e.value.code == glb.GLB_ERR_UNSUPPORTED
    # haloes on one line span no area
    same = [synth.NFWHalo(1e13, 0.2, Z, 5.0, theta=(1e-5 * i, 0.0)) for i in range(3)]
    with pytest.raises(glb.GlamerError) as e:
        glb.halo_from_spec(synth.FieldPlane(Z, same))._make()
    assert e.value.code == glb.GLB_ERR_SAME_PLACE
    # an empty plane and a one-halo plane
    xx = plane_positions(50)
    a, k, g, ph = glb.LensPlaneTree(Z, []).force_halo(xx)
    assert not a.any() and not k.any()
    one = synth.FieldPlane(Z, [synth.NFWHalo(1e13, 0.2, Z, 5.0, theta=(1e-5, 2e-5))])
    f = pack(*glb.halo_from_spec(one).force_halo(xx))
    m, cols = force_err(f, H.oracle_halo_force(one, xx)[0])
    assert m < RTOL64, cols


def test_pixelmap_matches_gridmap_and_oracle():
    """writePixelMap on the device: every LensingVariable equals the value
    derived from the GridMap's y and A, which equal the oracle's."""
    spec = mixed_spec(seed=13)
    L = glb.lens_from_spec(spec)
    n1d, c, rng = 31, (1e-6, -2e-6), 50 * synth.ARCSEC
    gm = glb.GridMap(L, n1d, c, rng)
    x = gm.positions()
    yo, Ao = H.OracleLens(spec).rayshoot(x)
    assert np.max(rel_err(gm.y, yo)) < RTOL64
    a = x - gm.y
    g1, g2 = gm.gamma1(), gm.gamma2()
    expect = {glb.DELAYT: np.zeros(len(x)), glb.ALPHA: np.hypot(a[:, 0], a[:, 1]), glb.ALPHA1: a[:, 0],
              glb.ALPHA2: a[:, 1], glb.KAPPA: gm.kappa(), glb.GAMMA: np.hypot(g1, g2), glb.GAMMA1: g1,
              glb.GAMMA2: g2, glb.GAMMA3: gm.gamma3(), glb.INVMAG: gm.invmag()}
    for var, e in expect.items():
        m = glb.writePixelMap(L, n1d, c, rng, var).ravel()
        np.testing.assert_allclose(m, e, rtol=1e-12, atol=1e-15 * np.abs(e).max(), err_msg=str(var))
    for var in (glb.PHI, glb.SURF_BRIGHTNESS):
        with pytest.raises(glb.GlamerError) as ex:
            glb.writePixelMap(L, n1d, c, rng, var)
        assert ex.value.code == glb.GLB_ERR_UNSUPPORTED


def test_uniform_pixelmap_matches_reference(golden):
    """writePixelMapUniform on the device against the reference's own maps
    (golden uniform_maps.npz: one pixel per grid point, finer offset and
    rectangular maps; KAPPA, INVMAG, ALPHA1, GAMMA)."""
    d = golden("uniform_maps.npz")
    spec = lens_spec_from_fixture(golden("lens_small.npz"))
    L = glb.lens_from_spec(spec)
    n1d, rng = int(d["grid_n"]), float(d["grid_range"])
    for k in range(4):
        cx, cy, nx, ny, var = d[f"map{k}_args"]
        m = glb.writePixelMapUniform(L, n1d, (0.0, 0.0), rng, (cx, cy), int(nx), int(ny), int(var))
        ref = d[f"map{k}"]
        np.testing.assert_array_equal(m == 0, ref == 0)  # the same pixels written
        assert np.max(rel_err(m.ravel(), ref.ravel())) < 1e-9, k


def test_uniform_pixelmap_shared_pixels_and_errors():
    """A coarser map than the grid (several grid points per pixel: the last one
    in grid order is kept) and a map partly off the grid, against the
    restatement; argument errors."""
    spec = mixed_spec(seed=17)
    L = glb.lens_from_spec(spec)
    n1d, c, rng = 40, (0.0, 0.0), 30 * synth.ARCSEC
    gm = glb.GridMap(L, n1d, c, rng)
    x = gm.positions()
    for mc, nx, ny, var, vals in (((0.0, 0.0), 9, 7, glb.KAPPA, gm.kappa()),
                                  ((8 * synth.ARCSEC, -5 * synth.ARCSEC), 25, 30, glb.INVMAG, gm.invmag())):
        m = glb.writePixelMapUniform(L, n1d, c, rng, mc, nx, ny, var)
        e = H.uniform_map_restated(x, vals, mc, nx, ny, rng)
        np.testing.assert_allclose(m, e, rtol=1e-12, atol=1e-15 * np.abs(e).max())
    with pytest.raises(glb.GlamerError) as ex:
        glb.writePixelMapUniform(L, n1d, c, rng, c, 1, 5, glb.KAPPA)
    assert ex.value.code == glb.GLB_ERR_ARG
    with pytest.raises(glb.GlamerError) as ex:
        glb.writePixelMapUniform(L, n1d, c, rng, c, 8, 8, glb.PHI)
    assert ex.value.code == glb.GLB_ERR_UNSUPPORTED


def test_surface_brightness_matches_oracle(golden):
    """RefreshSurfaceBrightnesses on the device: each source's surface
    brightness at the GridMap's source positions equals the oracle's (itself
    pinned to the reference's Source::SurfaceBrightness), and the total is the
    reference's sum of sb x resolution^2."""
    from tests.golden.make_golden import SOURCE_CASES, source_params
    d = golden("sources.npz")
    spec = mixed_spec(seed=17)
    L = glb.lens_from_spec(spec)
    n1d, c, rng = 41, (0.0, 0.0), 50 * synth.ARCSEC
    gm = glb.GridMap(L, n1d, c, rng)
    for k in range(len(SOURCE_CASES)):
        kind, prm = source_params(k, float(d[f"flux_{k}"]))
        # put each source where the lens maps a grid point, so that it lights up
        prm = (gm.y[n1d * n1d // 2, 0], gm.y[n1d * n1d // 2, 1]) + tuple(prm[2:])
        sb, total = glb.refreshSurfaceBrightnesses(L, n1d, c, rng, kind, prm)
        ref = H.oracle_source_sb(kind, prm, gm.y)
        assert ref.max() > 0
        np.testing.assert_allclose(sb.ravel(), ref, rtol=1e-12, atol=1e-15 * ref.max(), err_msg=str(k))
        res2 = (rng / (n1d - 1)) ** 2
        expect = 0.0
        for v in sb.ravel():
            expect += v * res2
        assert total == expect
    with pytest.raises(glb.GlamerError) as ex:
        glb.refreshSurfaceBrightnesses(L, n1d, c, rng, 7, (0.0, 0.0, 1.0))
    assert ex.value.code == glb.GLB_ERR_UNSUPPORTED


def test_adaptive_refresh_matches_oracle(golden):
    """AdaptiveRefreshSurfaceBrightnesses with the refinement rays batched on
    the GPU: per-pixel refined surface brightness and total against the
    oracle's one-pixel-at-a-time restatement, on the reference-pinned case."""
    from tests.golden.make_golden import (ADAPTIVE_N1D, ADAPTIVE_RANGE, adaptive_sources, adaptive_spec)
    d = golden("adaptive.npz")
    cases = [(adaptive_spec(), ADAPTIVE_N1D, ADAPTIVE_RANGE, adaptive_sources(d["ysrc"]))]
    for spec, n1d, rng, sources in cases:
        L = glb.lens_from_spec(spec)
        O = H.OracleLens(spec)
        for kind, _, prm in sources:
            sb, tot = glb.adaptiveRefreshSurfaceBrightnesses(L, n1d, (0.0, 0.0), rng, kind, prm)
            sbo, toto = O.adaptive_sb(n1d, (0.0, 0.0), rng, kind, prm)
            np.testing.assert_allclose(sb.ravel(), sbo, rtol=1e-9, atol=1e-12 * np.abs(sbo).max())
            assert abs(tot - toto) <= 1e-9 * abs(toto)
