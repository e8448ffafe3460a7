"""Concurrent use of one lens from several host threads, and the per-ray
status output (skip flags for the reference's in_image == MAYBE points,
non-finite results), and large calls cut into slabs, through the C ABI."""
import threading

import numpy as np
import pytest

import slsimlib_b200 as glb
from slsimlib_b200 import synth
from tests import harness as H

pytestmark = pytest.mark.gpu


def test_threads_share_one_lens():
    """Four host threads shoot different ray sets through one lens at the same
    time (ctypes releases the GIL during the calls) in both precisions; every
    result equals the same call made alone, bit for bit."""
    spec = synth.light_cone(seed=51, n_total=120000, n_planes=4, halos_per_plane=6)
    L = glb.lens_from_spec(spec)
    rng = np.random.default_rng(3)
    xs = [rng.uniform(-30, 30, (20000 + 1000 * i, 2)) * synth.ARCSEC for i in range(4)]
    precs = [glb.PREC_FP64, glb.PREC_SPLIT, glb.PREC_SPLIT, glb.PREC_FP64]
    alone = [L.rayshooterInternal(x, precision=p) for x, p in zip(xs, precs)]
    out = [None] * 4
    err = []

    def work(i):
        try:
            for _ in range(3):
                out[i] = L.rayshooterInternal(xs[i], precision=precs[i])
        except Exception as e:  # pragma: no cover - reported below
            err.append(e)

    th = [threading.Thread(target=work, args=(i,)) for i in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not err, err
    for i in range(4):
        np.testing.assert_array_equal(out[i][0], alone[i][0])
        np.testing.assert_array_equal(out[i][1], alone[i][1])
    # a GridMap from another thread while this one shoots rays
    gm_alone = glb.GridMap(L, 64, (0.0, 0.0), 60 * synth.ARCSEC)
    res = {}
    t = threading.Thread(target=lambda: res.setdefault("gm", glb.GridMap(L, 64, (0.0, 0.0), 60 * synth.ARCSEC)))
    t.start()
    y, A = L.rayshooterInternal(xs[0], precision=glb.PREC_FP64)
    t.join()
    np.testing.assert_array_equal(res["gm"].y, gm_alone.y)
    np.testing.assert_array_equal(y, alone[0][0])


def test_per_ray_status_and_skip():
    spec = synth.single_plane_nfw(seed=4, n=20000)
    L = glb.lens_from_spec(spec)
    rng = np.random.default_rng(7)
    x = rng.uniform(-15, 15, (1000, 2)) * synth.ARCSEC
    x[17] = np.nan  # a non-finite input ray
    skip = np.zeros(len(x), dtype=bool)
    skip[::7] = True
    y0 = np.full((len(x), 2), 5.0)
    A0 = np.full((len(x), 4), 7.0)
    for prec in (glb.PREC_FP64, glb.PREC_SPLIT):
        y, A, st = L.rayshooterInternal_status(x, skip=skip, y=y0, A=A0, precision=prec)
        yr, Ar = L.rayshooterInternal(x, precision=prec)
        assert np.all(st[skip] == glb.RAY_SKIPPED)
        np.testing.assert_array_equal(y[skip], y0[skip])  # skipped rays keep the caller's values
        np.testing.assert_array_equal(A[skip], A0[skip])
        keep = ~skip
        keep[17] = False
        np.testing.assert_array_equal(y[keep], yr[keep])
        np.testing.assert_array_equal(A[keep], Ar[keep])
        assert np.all(st[keep] == glb.RAY_OK)
        assert st[17] == glb.RAY_NONFINITE
    # per-ray source redshifts and no skip array
    zs = rng.uniform(1.0, 3.0, len(x))
    y, A, st = L.rayshooterInternal_status(x, source_zs=zs)
    yr, Ar = L.rayshooterInternal(x, source_zs=zs)
    ok = np.arange(len(x)) != 17
    np.testing.assert_array_equal(y[ok], yr[ok])
    assert np.all(st[ok] == glb.RAY_OK) and st[17] == glb.RAY_NONFINITE
    # a lens without planes: identity, with the same flags
    E = glb.Lens(2.0)
    y, A, st = E.rayshooterInternal_status(x, skip=skip, y=y0, A=A0)
    np.testing.assert_array_equal(y[skip], y0[skip])
    assert np.all(st[skip] == glb.RAY_SKIPPED) and st[17] == glb.RAY_NONFINITE
    np.testing.assert_array_equal(y[keep], x[keep])


def test_large_call_in_slabs_matches_small_calls():
    """Calls of 2^21 rays or more run as two slabs of sorted rays on two
    streams.  The FP64 form gives each ray the same bits as the same rays
    shot in calls small enough to run in one piece, with per-ray source
    redshifts, skip flags and status bytes across the slab boundary; the
    split form keeps the deflection tolerance."""
    spec = synth.light_cone(seed=5, n_total=12000, n_planes=3, halos_per_plane=2, zs=2.2)
    L = glb.lens_from_spec(spec)
    rng = np.random.default_rng(17)
    n = (1 << 21) + 4097
    x = rng.uniform(-20, 20, (n, 2)) * synth.ARCSEC
    zs = rng.uniform(1.0, 3.0, n)
    skip = np.zeros(n, dtype=bool)
    skip[::11] = True
    y0 = np.full((n, 2), 5.0)
    A0 = np.full((n, 4), 7.0)
    y, A, st = L.rayshooterInternal_status(x, source_zs=zs, skip=skip, y=y0, A=A0)
    np.testing.assert_array_equal(y[skip], y0[skip])
    np.testing.assert_array_equal(A[skip], A0[skip])
    assert np.all(st[skip] == glb.RAY_SKIPPED) and np.all(st[~skip] == glb.RAY_OK)
    for idx in np.array_split(np.arange(n), 5):  # about 420,000 rays a call: one piece
        ys, As = L.rayshooterInternal(x[idx], source_zs=zs[idx])
        k = ~skip[idx]
        np.testing.assert_array_equal(y[idx][k], ys[k])
        np.testing.assert_array_equal(A[idx][k], As[k])
    y64, A64 = L.rayshooterInternal(x, source_zs=zs)
    y32, A32 = L.rayshooterInternal(x, source_zs=zs, precision=glb.PREC_SPLIT)
    e = H.error_stats(x, y32, A32, y64, A64)["alpha"]
    assert e["median"] <= 1e-6 and e["p999"] <= 1e-5, e
