"""Seeded synthetic lens inputs for the benchmark and the parity tests.

The reference ships no datasets; its documented use is particle lenses built
from simulation snapshots (``LensHaloParticles``, include/particle_halo.h) plus
analytic main halos.  This module draws the equivalent inputs from a seed:

* NFW haloes sampled as equal-mass particles (3D radius by inverting the
  enclosed-mass profile m(x) = ln(1+x) - x/(1+x) on [0, c], isotropic
  direction, physical Mpc, stored as float32 ``ParticleType<float>`` records);
* the particle record layout of include/particle_types.h:46-58
  (x[3], Mass, Size, type: 24 bytes);
* lens descriptions (``LensSpec``) naming particle planes and NSIE / NFW
  analytic haloes, consumed by the CUDA library, the oracle and the reference
  driver alike, so every side sees identical inputs.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

PARTICLE_DTYPE = np.dtype(
    [("x", "<f4", (3,)), ("Mass", "<f4"), ("Size", "<f4"), ("type", "<i4")]
)
assert PARTICLE_DTYPE.itemsize == 24

ARCSEC = 0.000004848136811  # include/standard.h:51 (arcsecTOradians)
LIGHTSPEED = 2.99792458e5  # km/s
GRAV = 4.7788e-20  # include/standard.h:43, G/c^2 in Mpc/Msun


@dataclasses.dataclass
class Cosmology:
    """Flat LambdaCDM, Omega_r = 0 (the configuration every workload uses)."""

    omega_m: float = 0.3
    omega_l: float = 0.7
    h: float = 0.7

    def E(self, z):
        a = 1.0 + np.asarray(z, dtype=np.float64)
        return np.sqrt(self.omega_m * a**3 + self.omega_l + (1 - self.omega_m - self.omega_l) * a**2)

    def coordist(self, z: float) -> float:
        # 64-point Gauss-Legendre on [0, z]: ample for a smooth integrand.
        x, w = np.polynomial.legendre.leggauss(64)
        zz = 0.5 * z * (x + 1.0)
        return float(LIGHTSPEED / (100 * self.h) * 0.5 * z * np.sum(w / self.E(zz)))

    def angdist(self, z: float) -> float:
        return self.coordist(z) / (1 + z)

    def rho_crit(self, z: float) -> float:
        """Critical density in Msun/Mpc^3 (G in Mpc km^2 s^-2 Msun^-1)."""
        G = 4.30091727e-9
        H = 100 * self.h * float(self.E(z))
        return 3 * H * H / (8 * math.pi * G)

    def r200(self, m200: float, z: float) -> float:
        return (3 * m200 / (4 * math.pi * 200 * self.rho_crit(z))) ** (1.0 / 3.0)


def _nfw_m(x):
    return np.log1p(x) - x / (1 + x)


def sample_nfw_radii(rng: np.random.Generator, n: int, c: float) -> np.ndarray:
    """Radii in units of r_s, distributed as the NFW mass within x <= c."""
    target = rng.random(n) * _nfw_m(c)
    lo = np.zeros(n)
    hi = np.full(n, float(c))
    for _ in range(60):  # bisection to ~c * 2^-60
        mid = 0.5 * (lo + hi)
        below = _nfw_m(mid) < target
        lo = np.where(below, mid, lo)
        hi = np.where(below, hi, mid)
    return 0.5 * (lo + hi)


def nfw_particles(
    rng: np.random.Generator,
    n: int,
    m200: float,
    c: float,
    z: float,
    size: float,
    center=(0.0, 0.0),
    cosmo: Optional[Cosmology] = None,
    axis_ratios=(1.0, 1.0),
) -> np.ndarray:
    """n equal-mass particles of an NFW halo truncated at r200 (physical Mpc).

    ``axis_ratios`` (b/a, c/a) squashes y and z and rescales all three axes to
    keep the volume, giving a triaxial halo."""
    cosmo = cosmo or Cosmology()
    r200 = cosmo.r200(m200, z)
    rs = r200 / c
    r = sample_nfw_radii(rng, n, c) * rs
    mu = rng.uniform(-1.0, 1.0, n)
    ph = rng.uniform(0.0, 2 * math.pi, n)
    s = np.sqrt(1 - mu * mu)
    xyz = np.stack([r * s * np.cos(ph), r * s * np.sin(ph), r * mu], axis=1)
    qb, qc = axis_ratios
    if (qb, qc) != (1.0, 1.0):
        scale = (qb * qc) ** (-1.0 / 3.0)
        xyz *= np.array([1.0, qb, qc]) * scale
    xyz[:, 0] += center[0]
    xyz[:, 1] += center[1]
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    p["x"] = xyz.astype(np.float32)
    p["Mass"] = np.float32(m200 / n)
    p["Size"] = np.float32(size)
    return p


@dataclasses.dataclass
class ParticlePlane:
    particles: np.ndarray
    z: float
    inv_area: float = 0.0
    max_range: float = -1.0
    theta: tuple = (0.0, 0.0)


@dataclasses.dataclass
class NSIEHalo:
    mass: float
    z: float
    sigma: float
    rcore: float
    fratio: float
    pa: float
    theta: tuple = (0.0, 0.0)


@dataclasses.dataclass
class NFWHalo:
    mass: float
    rsize: float
    z: float
    conc: float
    theta: tuple = (0.0, 0.0)


@dataclasses.dataclass
class FieldPlane:
    """A plane of field haloes (LensPlaneTree, MultiPlane/planes.cpp:13-18):
    NFW / NSIE haloes at angular positions ``theta`` (their own redshifts are
    replaced by the plane's), the background density ``sigma_back`` and the
    screening scale ``inv_screening`` (0: none)."""

    z: float
    halos: List[object]
    sigma_back: float = 0.0
    inv_screening: float = 0.0


@dataclasses.dataclass
class LensSpec:
    """Haloes in insertion order (Lens::moveinMainHalo / insertMainHalo with
    addplanes = true) and the source redshift."""

    zsource: float
    halos: List[object]

    def n_particles(self) -> int:
        return sum(len(h.particles) for h in self.halos if isinstance(h, ParticlePlane))


def single_plane_nfw(seed: int = 1, n: int = 2**18, m200: float = 1e14, c: float = 5.0,
                     zl: float = 0.3, zs: float = 2.0, size: float = 1e-3) -> LensSpec:
    """One NFW particle halo on one plane: 2^18 particles of a 1e14 Msun,
    c = 5 halo at z = 0.3 softened by 1 kpc, source at z = 2."""
    rng = np.random.default_rng(seed)
    p = nfw_particles(rng, n, m200, c, zl, size)
    return LensSpec(zsource=zs, halos=[ParticlePlane(p, zl)])


def light_cone(seed: int = 2, n_total: int = 4_194_304, n_planes: int = 10,
               halos_per_plane: int = 32, field_arcsec: float = 60.0, size: float = 5e-4,
               zs: float = 2.5, nsie: bool = True) -> LensSpec:
    """Multi-plane light cone: planes at z = 0.1, 0.3, ..., each with
    ``halos_per_plane`` NFW haloes (M log-uniform in [1e12, 1e14] Msun, c = 5,
    centres uniform in the field), sampled at one common particle mass so
    particle counts follow halo mass; a main NSIE (sigma 250 km/s, q 0.7,
    core 0.05 arcsec, mass 1e13 Msun) at z = 0.5."""
    rng = np.random.default_rng(seed)
    cosmo = Cosmology()
    zplanes = [0.1 + 0.2 * i for i in range(n_planes)]
    masses = 10 ** rng.uniform(12, 14, size=(n_planes, halos_per_plane))
    counts = np.floor(n_total * masses / masses.sum()).astype(np.int64)
    short = n_total - counts.sum()
    order = np.argsort(-(n_total * masses / masses.sum() - counts), axis=None)
    counts.flat[order[:short]] += 1
    halos = []
    for j, z in enumerate(zplanes):
        da = cosmo.angdist(z)
        half = 0.5 * field_arcsec * ARCSEC * da
        parts = []
        for k in range(halos_per_plane):
            cxy = rng.uniform(-half, half, size=2)
            parts.append(nfw_particles(rng, int(counts[j, k]), masses[j, k],
                                       5.0, z, size, center=cxy, cosmo=cosmo))
        p = np.concatenate(parts)
        # equal particle mass across every halo of the cone
        p["Mass"] = np.float32(masses.sum() / n_total)
        halos.append(ParticlePlane(p, z))
    if nsie:
        zl = 0.5
        rcore = 0.05 * ARCSEC * cosmo.angdist(zl)
        halos.append(NSIEHalo(mass=1e13, z=zl, sigma=250.0, rcore=rcore, fratio=0.7, pa=0.0))
    return LensSpec(zsource=zs, halos=halos)


def grid_positions(n1d: int, center=(0.0, 0.0), range_rad: float = 30 * ARCSEC) -> np.ndarray:
    """GridMap ray positions, x fastest (TreeCode_link/utilities.cpp:149-158)."""
    i = np.arange(n1d * n1d)
    if n1d == 1:
        return np.array([[center[0], center[1]]], dtype=np.float64)
    x = center[0] + range_rad * (1.0 * (i % n1d) / (n1d - 1) - 0.5)
    y = center[1] + range_rad * (1.0 * (i // n1d) / (n1d - 1) - 0.5)
    return np.stack([x, y], axis=1)


def field_halos(seed: int, n: int, z: float, field_arcsec: float = 60.0, mmin: float = 1e10,
                mmax: float = 1e13, n_nsie: int = 0, cosmo: "Cosmology" = None) -> List[object]:
    """n NFW haloes (mass log-uniform in [mmin, mmax], c = 5 (M/1e14)^-0.1,
    truncated at r200) uniform in a square field, plus n_nsie NSIE haloes
    (sigma 150-250 km/s, q 0.6-0.9): the field haloes of one plane."""
    rng = np.random.default_rng(seed)
    cosmo = cosmo or Cosmology()
    out = []
    half = 0.5 * field_arcsec * ARCSEC
    for m in 10 ** rng.uniform(np.log10(mmin), np.log10(mmax), n):
        th = tuple(float(v) for v in rng.uniform(-half, half, 2))
        out.append(NFWHalo(float(m), float(cosmo.r200(m, z)), z, float(5.0 * (m / 1e14) ** -0.1), theta=th))
    for _ in range(n_nsie):
        th = tuple(float(v) for v in rng.uniform(-half, half, 2))
        sig = float(rng.uniform(150, 250))
        out.append(NSIEHalo(float(10 ** rng.uniform(12, 13)), z, sig, float(rng.uniform(5e-5, 2e-4)),
                            float(rng.uniform(0.6, 0.9)), float(rng.uniform(0, np.pi)), theta=th))
    return out
