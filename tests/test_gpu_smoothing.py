"""Adaptive kNN smoothing (LensHaloParticles::calculate_smoothing) on the GPU:
bit-exact against the reference's golden sizes, against the oracle on seeded
clustered, uniform, coincident and outlier-heavy sets, and at four million
particles against the brute-force definition on sampled particles."""
import numpy as np
import pytest

import slsimlib_b200 as glb
from slsimlib_b200 import synth
from tests import harness as H
from tests.test_oracle import smoothing_golden_cases

pytestmark = pytest.mark.gpu


def gpu_sizes(p, ns):
    q = np.array(p, dtype=synth.PARTICLE_DTYPE, copy=True)
    glb.calculate_smoothing(ns, q)
    return q["Size"].copy()


def test_smoothing_matches_reference_golden(golden):
    for name, p, ns, sizes in smoothing_golden_cases(golden):
        assert np.array_equal(gpu_sizes(p, ns), sizes), name


def two_haloes(rng, n):
    a = synth.nfw_particles(rng, n // 2, 2e14, 4.0, 0.4, 0.0)
    b = synth.nfw_particles(rng, n - n // 2, 5e13, 8.0, 0.4, 0.0, center=(0.3, -0.1))
    return np.concatenate([a, b])


def cube(rng, n):
    p = np.zeros(n, dtype=synth.PARTICLE_DTYPE)
    p["x"] = rng.uniform(-2.0, 2.0, (n, 3)).astype(np.float32)
    p["Mass"] = 1.0
    return p


def outliers(rng, n):
    """A tight cluster plus 0.1 % of particles spread over a volume 10^4 times
    wider: the outliers' buckets see more candidate buckets than one CTA lists,
    so the per-query tree walk runs for them."""
    p = synth.nfw_particles(rng, n, 1e14, 10.0, 0.5, 0.0)
    k = max(n // 1000, 40)
    p["x"][:k] = rng.uniform(-300.0, 300.0, (k, 3)).astype(np.float32)
    return p


@pytest.mark.parametrize("maker,n,ns", [
    (two_haloes, 60000, 32),
    (cube, 100000, 64),
    (two_haloes, 50000, 1),
    (cube, 20000, 200),
    (outliers, 200000, 32),
])
def test_smoothing_matches_oracle(maker, n, ns):
    p = maker(np.random.default_rng(n + ns), n)
    assert np.array_equal(gpu_sizes(p, ns), H.oracle_smoothing(p, ns))


def test_smoothing_coincident_particles():
    """Groups of identical positions: distances of exactly 0 tie at the bound."""
    rng = np.random.default_rng(5)
    base = synth.nfw_particles(rng, 3000, 1e14, 5.0, 0.5, 0.0)
    p = np.concatenate([base] * 4)
    for ns in (2, 3, 8, 40):
        assert np.array_equal(gpu_sizes(p, ns), H.oracle_smoothing(p, ns)), ns


@pytest.mark.parametrize("ns", [1, 4, 64])
def test_smoothing_top_walk(ns):
    """N = 2*Nsmooth+1: the reference's walk counts particles twice for half
    of the queries; the device reproduces those values."""
    p = synth.nfw_particles(np.random.default_rng(ns), 2 * ns + 1, 1e14, 5.0, 0.5, 0.0)
    assert np.array_equal(gpu_sizes(p, ns), H.oracle_smoothing(p, ns))


def test_smoothing_npoints_prefix_and_errors():
    rng = np.random.default_rng(9)
    p = synth.nfw_particles(rng, 5000, 1e14, 5.0, 0.5, 0.0)
    p["Size"] = 7.0
    q = p.copy()
    glb.calculate_smoothing(16, q, 3000)
    assert np.array_equal(q["Size"][:3000], H.oracle_smoothing(p[:3000], 16))
    assert np.all(q["Size"][3000:] == 7.0)
    assert np.array_equal(q["x"], p["x"]) and np.array_equal(q["Mass"], p["Mass"])
    for ns, n in ((0, 100), (-3, 100), (10, 11), (10, 10)):
        with pytest.raises(glb.GlamerError) as e:
            glb.calculate_smoothing(ns, p[:n].copy())
        assert e.value.code == -1
    with pytest.raises(glb.GlamerError) as e:
        glb.calculate_smoothing(5000, synth.nfw_particles(rng, 20000, 1e14, 5.0, 0.5, 0.0))
    assert e.value.code == -6


def test_smoothing_device_entry_point():
    torch = pytest.importorskip("torch")
    p = two_haloes(np.random.default_rng(12), 40000)
    dev = torch.from_numpy(p.view(np.uint8).copy()).cuda()
    out = torch.empty(len(p), dtype=torch.float32, device="cuda")
    ms = glb.calculate_smoothing_device(32, len(p), dev.data_ptr(), out.data_ptr(),
                                        torch.cuda.current_stream().cuda_stream)
    assert ms[0] > 0 and ms[1] > 0
    assert np.array_equal(out.cpu().numpy(), H.oracle_smoothing(p, 32))


def test_smoothing_four_million_particles_against_definition():
    """Full size (a 4M-particle lens plane): sampled particles against the
    definition -- the (Nsmooth+1)-th smallest of ((dx^2 + dy^2) + dz^2) in
    double from float differences, over all particles."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2024)
    n, ns = 4_194_304, 64
    p = two_haloes(rng, n)
    sizes = gpu_sizes(p, ns)
    assert np.all(np.isfinite(sizes)) and np.all(sizes > 0)
    x = torch.from_numpy(p["x"].copy()).cuda()
    pick = rng.choice(n, 512, replace=False)
    want = []
    for c in range(0, len(pick), 16):
        q = x[torch.from_numpy(pick[c:c + 16]).cuda()]
        d2 = None
        for j in range(3):
            dj = (x[None, :, j] - q[:, None, j]).double()
            d2 = dj * dj if d2 is None else d2 + dj * dj
        want.append(torch.kthvalue(d2, ns + 1, dim=1).values.sqrt().float().cpu().numpy())
    assert np.array_equal(sizes[pick], np.concatenate(want))
