"""Batched lenses in one persistent launch (CUDA graph) and the served request
loop with continuous batching: parity with the per-lens path and the oracle,
and each request's result the same alone and in a mix."""
import threading

import numpy as np
import pytest

import slsimlib_b200 as glb
from slsimlib_b200 import synth
from tests import harness as H
from tests.test_gpu_parity import make_lens, rel_err


def defl_err(x, y, yref):
    a, ar = x - y, x - yref
    na = np.hypot(ar[:, 0], ar[:, 1])
    keep = na > 1e-6 * np.median(na)
    return np.hypot(*(a - ar).T)[keep] / na[keep]

pytestmark = pytest.mark.gpu


def _specs():
    rng = np.random.default_rng(3)
    out = [synth.single_plane_nfw(seed=4, n=8000, zs=1.5)]
    out.append(synth.light_cone(seed=5, n_total=12000, n_planes=3, halos_per_plane=2, zs=2.2))
    s = synth.single_plane_nfw(seed=6, n=3000, m200=5e13, zl=0.6, zs=2.8)
    s.halos.append(synth.NSIEHalo(2e12, 0.6, 180.0, 1e-4, 0.8, 0.4))
    out.append(s)
    out.append(synth.LensSpec(zsource=1.2, halos=[synth.NFWHalo(2e14, 1.2, 0.4, 4.0, theta=(3e-6, 0))]))
    return out


@pytest.mark.parametrize("precision", [glb.PREC_FP64, glb.PREC_SPLIT])
def test_batch_matches_per_lens_gridmaps(precision):
    specs = _specs()
    lenses = [make_lens(s) for s in specs]
    n1d = [17, 64, 33, 1]
    rng = 30 * synth.ARCSEC
    centers = [(0.0, 0.0), (1e-6, -2e-6), (0.0, 0.0), (5e-6, 5e-6)]
    ranges = [rng, 2 * rng, rng, rng]
    b = glb.GridBatch(lenses, n1d, centers, ranges, precision)

    def check():
        for i, L in enumerate(lenses):
            y, A = b.result(i)
            if precision == glb.PREC_FP64:  # the per-lens FP64 path, up to contraction order
                gm = glb.GridMap(L, n1d[i], centers[i], ranges[i], precision)
                assert np.max(rel_err(y, gm.y)) < 1e-9, i
                assert np.max(np.abs(A - gm.A)) < 1e-9, i
            else:  # the split form against FP64: the deflection tolerance
                gm = glb.GridMap(L, n1d[i], centers[i], ranges[i], glb.PREC_FP64)
                e = defl_err(gm.positions(), y, gm.y)
                assert np.median(e) <= 1e-6 and np.percentile(e, 99) <= 1e-5, (i, np.median(e), e.max())
    for use_graph in (True, True, False):
        b.run(use_graph)
        check()
    blk, ms = b.autotune()
    assert blk in (64, 128, 256) and ms > 0 and b.tile() in (8, 16, 32)
    b.run(True)
    check()
    for width in (16, 32, 8):  # every warp tile shape gives the same grids
        b.set_tile(width)
        b.run(True)
        check()
    with pytest.raises(glb.GlamerError):
        b.set_tile(12)


def test_server_results_match_oracle():
    specs = _specs()[:3]
    models = [make_lens(s) for s in specs]
    srv = glb.Server(models, max_rays_per_batch=20000, precision=glb.PREC_FP64, nslots=2)
    rng = np.random.default_rng(8)
    reqs = []
    for k in range(9):
        m = k % 3
        x = rng.normal(0, 5 * synth.ARCSEC, size=(int(rng.integers(1, 3000)), 2))
        zs = float(rng.uniform(1.0, 3.0)) if k % 2 else -1.0
        reqs.append((m, x, zs, srv.submit(m, x, zs)))
    for m, x, zs, t in reqs:
        y, A, times = srv.wait(t, timeout=120)
        assert times[0] <= times[1] <= times[2]
        O = H.OracleLens(specs[m])
        yo, Ao = O.rayshoot(x, None if zs < 0 else np.full(len(x), zs))
        assert np.max(rel_err(y, yo)) < 1e-9
        assert np.max(np.abs(A - Ao)) < 1e-9
    st = srv.stats()
    assert st["requests"] == 9 and st["batches"] >= 1
    srv.close()


@pytest.mark.parametrize("precision", [glb.PREC_FP64, glb.PREC_SPLIT])
def test_server_request_same_alone_and_in_the_mix(precision):
    specs = _specs()[:3]
    models = [make_lens(s) for s in specs]
    rng = np.random.default_rng(9)
    probe_x = rng.normal(0, 3 * synth.ARCSEC, size=(2500, 2))
    # alone
    srv = glb.Server(models, max_rays_per_batch=40000, precision=precision, nslots=3)
    y_alone, A_alone, _ = srv.wait(srv.submit(1, probe_x, 2.0), timeout=120)
    # in a mix: other requests submitted from several threads around it
    tickets = []

    def client(seed):
        r = np.random.default_rng(seed)
        for _ in range(6):
            x = r.normal(0, 8 * synth.ARCSEC, size=(int(r.integers(100, 4000)), 2))
            tickets.append(srv.submit(int(r.integers(0, 3)), x, float(r.uniform(1, 3))))

    th = [threading.Thread(target=client, args=(s,)) for s in range(3)]
    for t in th:
        t.start()
    probe = srv.submit(1, probe_x, 2.0)
    for t in th:
        t.join()
    y_mix, A_mix, _ = srv.wait(probe, timeout=120)
    for t in tickets:
        srv.wait(t, timeout=120)
    assert srv.stats()["batches"] >= 2
    np.testing.assert_array_equal(y_mix, y_alone)
    np.testing.assert_array_equal(A_mix, A_alone)
    srv.close()


@pytest.mark.parametrize("precision", [glb.PREC_FP64, glb.PREC_SPLIT])
def test_server_large_requests_take_the_lens_path(precision):
    """Requests of at least 2^20 rays run through the lens path's per-plane
    kernels inside the server: their results are the lens path's (the same
    kernels on the same rays), alone and mixed with small requests."""
    specs = _specs()[:3]
    models = [make_lens(s) for s in specs]
    rng = np.random.default_rng(11)
    srv = glb.Server(models, max_rays_per_batch=3_000_000, precision=precision, nslots=2)
    big = [(m, rng.normal(0, 6 * synth.ARCSEC, size=(n, 2)), zs)
           for m, n, zs in ((0, 1 << 20, -1.0), (1, (1 << 20) + 4001, 2.0), (2, (1 << 20) + 1, 1.1))]
    small = [(int(rng.integers(0, 3)), rng.normal(0, 6 * synth.ARCSEC, size=(int(rng.integers(1, 3000)), 2)),
              float(rng.uniform(1, 3))) for _ in range(6)]
    tickets = [srv.submit(m, x, zs) for m, x, zs in big + small]
    out = [srv.wait(t, timeout=240) for t in tickets]
    for (m, x, zs), (y, A, _) in zip(big, out[:3]):
        yl, Al = models[m].rayshooterInternal(x, None if zs < 0 else np.full(len(x), zs), precision)
        if precision == glb.PREC_FP64:
            assert np.max(rel_err(y, yl)) < 1e-12 and np.max(np.abs(A - Al)) < 1e-12
        else:
            e = defl_err(x, y, yl)
            assert np.median(e) <= 1e-6 and np.percentile(e, 99) <= 1e-5
    if precision == glb.PREC_FP64:  # every request against the oracle (its first 2,000 rays)
        for (m, x, zs), (y, A, _) in zip(big + small, out):
            k = min(len(x), 2000)
            yo, Ao = H.OracleLens(specs[m]).rayshoot(x[:k], None if zs < 0 else np.full(k, zs))
            assert np.max(rel_err(y[:k], yo)) < 1e-9 and np.max(np.abs(A[:k] - Ao)) < 1e-9
    # the same large request alone gives the same bits
    m, x, zs = big[1]
    y1, A1, _ = srv.wait(srv.submit(m, x, zs), timeout=240)
    np.testing.assert_array_equal(y1, out[1][0])
    np.testing.assert_array_equal(A1, out[1][1])
    srv.close()


def test_server_rejects_oversized_and_unknown():
    models = [make_lens(_specs()[0])]
    srv = glb.Server(models, max_rays_per_batch=1000, precision=glb.PREC_FP64, nslots=1)
    with pytest.raises(glb.GlamerError):
        srv.submit(0, np.zeros((1001, 2)))
    with pytest.raises(glb.GlamerError):
        srv.submit(3, np.zeros((10, 2)))
    y, A, _ = srv.wait(srv.submit(0, np.zeros((0, 2))), timeout=10)
    assert y.shape == (0, 2)
    srv.close()
