"""The link-level drop-in (slsimlib_b200/dropin/glamer_b200_dropin.cpp): the
reference's own sources -- GridMap, Grid and its refinement
(TreeCode_link/grid_maintenance.cpp), ImageFinding::find_crit
(TreeCode_link/find_crit.cpp), find_magnification_contour -- compiled in place
and linked with the drop-in instead of FullRange/internal_rayshooter_multi.cpp
(oracle/_ref/glamer_gpu), against the same sources linked with the reference's
CPU rayshooter (oracle/_ref/glamer_ref), on one lens: 65,536 NFW particles
(1e14 Msun, z = 0.3), an elliptical NSIE (z = 0.5) and an offset NFW halo
(z = 0.7).  The refinement decisions (which points, how many curves) must be
identical and the shot quantities agree to the FP64 tolerance (1e-9)."""
import os

import numpy as np
import pytest

from slsimlib_b200 import synth
from tests import harness as H
from tests.conftest import rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (os.path.exists(H.REF_BIN) and os.path.exists(H.DROPIN_BIN)),
                                 reason="oracle/_ref binaries not built (make -C oracle REF=<reference>)")]

RANGE = 12 * synth.ARCSEC


def lens_spec():
    spec = synth.single_plane_nfw(seed=5, n=65536)
    spec.halos.append(synth.NSIEHalo(1e13, 0.5, 250.0, 0.0, 0.7, 0.3))
    spec.halos.append(synth.NFWHalo(5e12, 0.3, 0.7, 6.0, theta=(3 * synth.ARCSEC, -2 * synth.ARCSEC)))
    return spec


def run_both(cmd_of, spec=None):
    """The same command through both binaries -> (cpu output, gpu output)."""
    spec = spec or lens_spec()
    out = []
    for binary in (H.REF_BIN, H.DROPIN_BIN):
        R = H.RefDriver(binary)
        of = R._file()
        R.run(R.lens_lines(spec) + [cmd_of(R, of)], timeout=900)
        out.append(np.fromfile(of))
    return out


def curves(o):
    """dump_curves -> list of (header[9], points (n, 8))."""
    n, k, res = int(o[0]), 1, []
    for _ in range(n):
        h = o[k:k + 9]
        m = int(h[2])
        res.append((h, o[k + 9:k + 9 + 8 * m].reshape(m, 8)))
        k += 9 + 8 * m
    assert k == len(o)
    return res


def check_rays(p_cpu, p_gpu):
    """x identical; y relative 1e-9; A absolute 1e-9 (p: (n, 8) x, y, A)."""
    np.testing.assert_array_equal(p_gpu[:, :2], p_cpu[:, :2])
    assert np.max(rel_err(p_gpu[:, 2:4], p_cpu[:, 2:4])) < 1e-9
    assert np.max(np.abs(p_gpu[:, 4:] - p_cpu[:, 4:])) < 1e-9


def test_dropin_ray_overloads():
    """Point*, LinkedPoint* + source_zs, RAY* (per-ray z; the default z = -1
    ray is not deflected) and rayshooter(RAY&)."""
    rng = np.random.default_rng(2)
    x = rng.uniform(-6, 6, (500, 2)) * synth.ARCSEC
    z = rng.uniform(0.2, 3.0, 500)
    z[:5] = -1.0
    c, g = run_both(lambda R, of: f"points {R._file(x)} {len(x)} {of} -")
    assert np.max(rel_err(g.reshape(-1, 6)[:, :2], c.reshape(-1, 6)[:, :2])) < 1e-9
    assert np.max(np.abs(g.reshape(-1, 6)[:, 2:] - c.reshape(-1, 6)[:, 2:])) < 1e-9
    c, g = run_both(lambda R, of: f"rays {R._file(x)} {len(x)} {R._file(z)} {of} -")
    c, g = c.reshape(-1, 6), g.reshape(-1, 6)
    np.testing.assert_array_equal(c[:5, :2], x[:5])  # z = -1: in front of every plane
    assert np.max(rel_err(g[:, :2], c[:, :2])) < 1e-9 and np.max(np.abs(g[:, 2:] - c[:, 2:])) < 1e-9
    c, g = run_both(lambda R, of: f"lpoints {R._file(x)} {len(x)} {R._file(np.abs(z))} {of}")
    c, g = c.reshape(-1, 6), g.reshape(-1, 6)
    assert np.max(rel_err(g[:, :2], c[:, :2])) < 1e-9 and np.max(np.abs(g[:, 2:] - c[:, 2:])) < 1e-9
    c, g = run_both(lambda R, of: f"rayshooter {R._file(x[:50])} 50 {of}")
    c, g = c.reshape(-1, 6), g.reshape(-1, 6)
    assert np.max(rel_err(g[:, :2], c[:, :2])) < 1e-9 and np.max(np.abs(g[:, 2:] - c[:, 2:])) < 1e-9


def test_dropin_find_crit_gridmap():
    """ImageFinding::find_crit(lens, GridMap, curves): the same critical curves
    (count, type, points) and the same caustics."""
    c, g = run_both(lambda R, of: f"findcritmap 96 0 0 {RANGE!r} {of}")
    cc, gc = curves(c), curves(g)
    assert len(cc) == len(gc) and len(cc) > 0
    for (hc, pc), (hg, pg) in zip(cc, gc):
        np.testing.assert_array_equal(hg[:6], hc[:6])  # type, edge, n, critical area and centre
        check_rays(pc, pg)
        assert np.all(np.abs(hg[6:] - hc[6:]) <= 1e-9 * (np.abs(hc[6:]) + 1e-12))


def test_dropin_magnification_contours():
    c, g = run_both(lambda R, of: f"magcontour 96 0 0 {RANGE!r} 0.3 {of}")
    assert len(c) == len(g) and c[0] == g[0] and c[0] > 0
    k = 1
    for _ in range(int(c[0])):
        m = int(c[k])
        assert g[k] == c[k] and g[k + 1] == c[k + 1]
        check_rays(c[k + 2:k + 2 + 8 * m].reshape(m, 8), g[k + 2:k + 2 + 8 * m].reshape(m, 8))
        k += 2 + 8 * m


def test_dropin_grid_refinement():
    """Grid ctor + Grid::RefineLeaves on every 5th point: the same points, the
    same source positions and Jacobians."""
    c, g = run_both(lambda R, of: f"gridrefine 32 0 0 {RANGE!r} 5 {of}")
    assert c[0] == g[0] and c[0] > 32 * 32
    check_rays(c[1:].reshape(-1, 8), g[1:].reshape(-1, 8))


def test_dropin_find_crit_grid_refinement_rounds():
    """ImageFinding::find_crit(lens, grid, ...): the kist refinement rounds
    (repeated small rayshooterInternal calls) give the same critical curves."""
    c, g = run_both(lambda R, of: f"gridcrit 32 0 0 {RANGE!r} {0.3 * synth.ARCSEC!r} {of}")
    cc, gc = curves(c), curves(g)
    assert len(cc) == len(gc) and len(cc) > 0
    for (hc, pc), (hg, pg) in zip(cc, gc):
        np.testing.assert_array_equal(hg[:6], hc[:6])
        check_rays(pc, pg)


def test_dropin_split_precision():
    """glamer_b200_dropin::set_precision(GLB_PREC_SPLIT): the reference's
    rayshooterInternal(N, Point*) through the split form stays within the
    deflection tolerance of the reference's FP64 result (median 1e-6,
    99.9th percentile 1e-5)."""
    rng = np.random.default_rng(4)
    x = rng.uniform(-6, 6, (4000, 2)) * synth.ARCSEC
    spec = lens_spec()
    out = []
    for binary, pre in ((H.REF_BIN, []), (H.DROPIN_BIN, ["dropin 1"])):
        R = H.RefDriver(binary)
        of = R._file()
        R.run(R.lens_lines(spec) + pre + [f"points {R._file(x)} {len(x)} {of} -"], timeout=900)
        out.append(np.fromfile(of).reshape(-1, 6))
    c, g = out
    ar, a = x - c[:, :2], x - g[:, :2]
    e = np.hypot(*(a - ar).T) / np.hypot(*ar.T)
    assert np.median(e) <= 1e-6 and np.percentile(e, 99.9) <= 1e-5, (np.median(e), e.max())
