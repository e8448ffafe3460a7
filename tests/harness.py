"""Test-side access to the oracle (oracle/liboracle.so) and to the reference
driver (oracle/_ref/glamer_ref).  Test infrastructure only: the product
library never imports this module."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from typing import Optional

import numpy as np

from slsimlib_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")
REF_BIN = os.path.join(ORACLE_DIR, "_ref", "glamer_ref")
# the reference's sources linked with the GPU drop-in (slsimlib_b200/dropin) in
# place of FullRange/internal_rayshooter_multi.cpp
DROPIN_BIN = os.path.join(ORACLE_DIR, "_ref", "glamer_gpu")

_dp = C.POINTER(C.c_double)
_vp = C.c_void_p


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


_lib = None


def oracle_lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(ORACLE_SO):
        subprocess.check_call(["make", "-s", "-C", ORACLE_DIR, "liboracle.so"])
    L = C.CDLL(ORACLE_SO)
    L.orc_coordist.restype = C.c_double
    L.orc_coordist.argtypes = [C.c_double]
    L.orc_angdist.restype = C.c_double
    L.orc_angdist.argtypes = [C.c_double]
    L.orc_tree_build.restype = _vp
    L.orc_tree_build.argtypes = [_vp, C.c_size_t, C.c_float, C.c_float, C.c_double, C.c_int,
                                 C.c_double, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_int)]
    L.orc_tree_free.argtypes = [_vp]
    L.orc_tree_force2D_recur.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp]
    L.orc_direct_sum.argtypes = [_vp, C.c_size_t, C.c_double, _vp, _vp, _vp, _vp, _vp]
    L.orc_tree_nbranches.restype = C.c_size_t
    L.orc_tree_nbranches.argtypes = [_vp]
    L.orc_tree_export.argtypes = [_vp, _vp]
    L.orc_tree_membership.argtypes = [_vp, _vp]
    L.orc_halo_nfw.restype = _vp
    L.orc_halo_nfw.argtypes = [C.c_float, C.c_float, C.c_double, C.c_float, C.c_float, C.c_float]
    L.orc_halo_nsie.restype = _vp
    L.orc_halo_nsie.argtypes = [C.c_float, C.c_double, C.c_float, C.c_float, C.c_float, C.c_float]
    L.orc_halo_particles.restype = _vp
    L.orc_halo_particles.argtypes = [_vp, C.c_size_t, C.c_double, C.c_double, C.c_double]
    L.orc_halo_set_theta.argtypes = [_vp, C.c_double, C.c_double]
    L.orc_halo_free.argtypes = [_vp]
    for f in ("orc_halo_mass", "orc_halo_rsize", "orc_halo_rmax"):
        getattr(L, f).restype = C.c_float
        getattr(L, f).argtypes = [_vp]
    L.orc_halo_force.argtypes = [_vp, C.c_size_t, _vp, _vp, _vp, _vp, _vp]
    L.orc_lens_create.restype = _vp
    L.orc_lens_create.argtypes = [C.c_double]
    L.orc_lens_free.argtypes = [_vp]
    L.orc_lens_add_halo.argtypes = [_vp, _vp, C.c_int]
    L.orc_lens_nplanes.restype = C.c_int
    L.orc_lens_nplanes.argtypes = [_vp]
    L.orc_lens_planes.argtypes = [_vp, _vp, _vp, _vp]
    L.orc_lens_reset_source.restype = C.c_int
    L.orc_lens_reset_source.argtypes = [_vp, C.c_double, C.c_int]
    L.orc_lens_rayshoot.argtypes = [_vp, C.c_size_t, _vp, _vp, _vp, _vp, C.c_int]
    L.orc_lens_plane_force.argtypes = [_vp, C.c_int, C.c_size_t, _vp, _vp, _vp, _vp, _vp]
    L.orc_grid_positions.argtypes = [C.c_size_t, _vp, C.c_double, _vp]
    L.orc_halo_field_plane.restype = _vp
    L.orc_halo_field_plane.argtypes = [_vp, C.c_int, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_int)]
    L.orc_lens_add_field_plane.argtypes = [_vp, _vp]
    L.orc_source_sb.argtypes = [C.c_int, _vp, C.c_size_t, _vp, _vp]
    L.orc_gridmap_adaptive_sb.restype = C.c_double
    L.orc_gridmap_adaptive_sb.argtypes = [_vp, C.c_size_t, _vp, C.c_double, C.c_int, _vp, _vp]
    L.orc_calculate_smoothing.restype = C.c_int
    L.orc_calculate_smoothing.argtypes = [_vp, C.c_size_t, C.c_int]
    _lib = L
    return L


# ----------------------------------------------------------------- trees
class OracleTree:
    def __init__(self, particles: np.ndarray, bucket=5, theta=0.1, inv_area=0.0,
                 periodic=False, inv_screening=0.0, max_range=-1.0):
        L = oracle_lib()
        self.p = np.ascontiguousarray(particles)
        err = C.c_int(0)
        self.h = L.orc_tree_build(_ptr(self.p), len(self.p), -1.0, -1.0, inv_area, bucket, theta,
                                  int(periodic), inv_screening, max_range, C.byref(err))
        if not self.h:
            raise ValueError("particles in same place.")

    def force(self, rays: np.ndarray) -> np.ndarray:
        """(n,7): alpha[2], kappa, gamma[3], phi from force2D_recur."""
        L = oracle_lib()
        rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 2)
        out = np.zeros((len(rays), 7))
        a = np.zeros(2); k = np.zeros(1); g = np.zeros(3); ph = np.zeros(1)
        for i in range(len(rays)):
            r = np.ascontiguousarray(rays[i])
            L.orc_tree_force2D_recur(self.h, _ptr(r), _ptr(a), _ptr(k), _ptr(g), _ptr(ph))
            out[i, :2] = a; out[i, 2] = k[0]; out[i, 3:6] = g; out[i, 6] = ph[0]
        return out

    def export(self) -> np.ndarray:
        L = oracle_lib()
        n = L.orc_tree_nbranches(self.h)
        out = np.zeros((n, 16))
        L.orc_tree_export(self.h, _ptr(out))
        return out

    def membership(self) -> np.ndarray:
        L = oracle_lib()
        n = L.orc_tree_nbranches(self.h)
        out = np.zeros((n, 2))
        L.orc_tree_membership(self.h, _ptr(out))
        return out

    def __del__(self):
        try:
            oracle_lib().orc_tree_free(self.h)
        except Exception:
            pass


def direct_sum(particles: np.ndarray, rays: np.ndarray, inv_area=0.0) -> np.ndarray:
    L = oracle_lib()
    p = np.ascontiguousarray(particles)
    rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 2)
    out = np.zeros((len(rays), 7))
    a = np.zeros(2); k = np.zeros(1); g = np.zeros(3); ph = np.zeros(1)
    for i in range(len(rays)):
        r = np.ascontiguousarray(rays[i])
        L.orc_direct_sum(_ptr(p), len(p), inv_area, _ptr(r), _ptr(a), _ptr(k), _ptr(g), _ptr(ph))
        out[i, :2] = a; out[i, 2] = k[0]; out[i, 3:6] = g; out[i, 6] = ph[0]
    return out


# ----------------------------------------------------------------- halos
def _make_halo(h):
    L = oracle_lib()
    if isinstance(h, synth.ParticlePlane):
        p = np.ascontiguousarray(h.particles)
        ptr = L.orc_halo_particles(_ptr(p), len(p), h.z, h.inv_area, h.max_range)
    elif isinstance(h, synth.NSIEHalo):
        ptr = L.orc_halo_nsie(h.mass, h.z, h.sigma, h.rcore, h.fratio, h.pa)
    elif isinstance(h, synth.NFWHalo):
        ptr = L.orc_halo_nfw(h.mass, h.rsize, h.z, h.conc, 1.0, 0.0)
    elif isinstance(h, synth.FieldPlane):
        members = (_vp * max(1, len(h.halos)))(*[_make_halo(m) for m in h.halos])
        err = C.c_int(0)
        ptr = L.orc_halo_field_plane(members, len(h.halos), h.z, h.sigma_back, h.inv_screening, C.byref(err))
        if err.value:
            raise ValueError("particles in same place.")
        return ptr
    else:
        raise TypeError(h)
    L.orc_halo_set_theta(ptr, h.theta[0], h.theta[1])
    return ptr


def oracle_halo_force(h, xcm: np.ndarray) -> np.ndarray:
    """(n,7) force_halo outputs for one halo at positions xcm (physical Mpc)."""
    L = oracle_lib()
    ptr = _make_halo(h)
    xcm = np.ascontiguousarray(xcm, dtype=np.float64).reshape(-1, 2)
    n = len(xcm)
    a = np.zeros((n, 2)); k = np.zeros(n); g = np.zeros((n, 3)); ph = np.zeros(n)
    L.orc_halo_force(ptr, n, _ptr(xcm), _ptr(a), _ptr(k), _ptr(g), _ptr(ph))
    params = (L.orc_halo_mass(ptr), L.orc_halo_rsize(ptr), L.orc_halo_rmax(ptr))
    L.orc_halo_free(ptr)
    return np.concatenate([a, k[:, None], g, ph[:, None]], axis=1), params


class OracleLens:
    def __init__(self, spec: synth.LensSpec):
        L = oracle_lib()
        self.h = L.orc_lens_create(spec.zsource)
        for halo in spec.halos:
            if isinstance(halo, synth.FieldPlane):
                L.orc_lens_add_field_plane(self.h, _make_halo(halo))
            else:
                L.orc_lens_add_halo(self.h, _make_halo(halo), 1)

    def planes(self):
        L = oracle_lib()
        n = L.orc_lens_nplanes(self.h)
        z = np.zeros(n + 1); Dl = np.zeros(n + 1); dDl = np.zeros(n + 1)
        L.orc_lens_planes(self.h, _ptr(z), _ptr(Dl), _ptr(dDl))
        return z, Dl, dDl

    def reset_source(self, z, nearest=False):
        return oracle_lib().orc_lens_reset_source(self.h, z, int(nearest))

    def rayshoot(self, x: np.ndarray, zs: Optional[np.ndarray] = None, threads=0):
        """y (n,2), A (n,4) from Lens::rayshooterInternal."""
        L = oracle_lib()
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 2)
        n = len(x)
        y = np.zeros((n, 2)); A = np.zeros((n, 4))
        zsp = None
        if zs is not None:
            zs = np.ascontiguousarray(zs, dtype=np.float64)
            zsp = _ptr(zs)
        L.orc_lens_rayshoot(self.h, n, _ptr(x), zsp, _ptr(y), _ptr(A), threads)
        return y, A

    def adaptive_sb(self, n1d, center, range_rad, kind, params):
        """GridMap::AdaptiveRefreshSurfaceBrightnesses: (sb (n1d^2), total)."""
        c = np.ascontiguousarray(center, dtype=np.float64)
        p = np.ascontiguousarray(params, dtype=np.float64)
        sb = np.zeros(n1d * n1d)
        tot = oracle_lib().orc_gridmap_adaptive_sb(self.h, n1d, _ptr(c), range_rad, int(kind), _ptr(p), _ptr(sb))
        return sb, tot

    def plane_force(self, j: int, xx: np.ndarray) -> np.ndarray:
        L = oracle_lib()
        xx = np.ascontiguousarray(xx, dtype=np.float64).reshape(-1, 2)
        n = len(xx)
        a = np.zeros((n, 2)); k = np.zeros(n); g = np.zeros((n, 3)); ph = np.zeros(n)
        L.orc_lens_plane_force(self.h, j, n, _ptr(xx), _ptr(a), _ptr(k), _ptr(g), _ptr(ph))
        return np.concatenate([a, k[:, None], g, ph[:, None]], axis=1)

    def __del__(self):
        try:
            oracle_lib().orc_lens_free(self.h)
        except Exception:
            pass


def oracle_source_sb(kind, params, y):
    """orc_source_sb: params = {x, y, ...} as glb_gridmap_surface_brightness takes them."""
    y = np.ascontiguousarray(y, dtype=np.float64).reshape(-1, 2)
    p = np.ascontiguousarray(params, dtype=np.float64)
    out = np.zeros(len(y))
    oracle_lib().orc_source_sb(int(kind), _ptr(p), len(y), _ptr(y), _ptr(out))
    return out


def oracle_smoothing(particles: np.ndarray, nsmooth: int) -> np.ndarray:
    """orc_calculate_smoothing on a copy of the records -> the float32 sizes."""
    p = np.array(particles, dtype=synth.PARTICLE_DTYPE, copy=True)
    rc = oracle_lib().orc_calculate_smoothing(_ptr(p), len(p), int(nsmooth))
    if rc != 0:
        raise ValueError(f"orc_calculate_smoothing: {rc}")
    return p["Size"].copy()


# ------------------------------------------- error attribution (GPU, library)
class PlaneRecursion:
    """The multi-plane recursion of include/lens.h:1003-1066 restated in numpy
    over per-plane forces computed by the library on the GPU (a
    TreeQuadParticles per particle plane with LensHaloParticles' parameters,
    the analytic haloes' force_halo).  The deflection and the shear/convergence
    of each plane can come from different precision forms, and the deflection
    can be perturbed, which separates the split form's per-plane evaluation
    error from the error that earlier planes' deflections carry into later
    planes' positions.  Particle and analytic (NSIE / NFW) planes only."""

    def __init__(self, spec: synth.LensSpec, lens):
        import slsimlib_b200 as glb
        self.glb = glb
        self.z, self.Dl, self.dDl = lens.planes()
        self.np = lens.getNplanes()
        self.charge = 4 * np.pi * synth.GRAV
        cosmo = synth.Cosmology()
        self.halos = [[] for _ in range(self.np)]
        for h in spec.halos:
            if isinstance(h, synth.FieldPlane):
                raise TypeError("field planes are not supported")
            zh = float(np.float32(h.z)) if isinstance(h, synth.ParticlePlane) else float(h.z)
            j = int(np.argmin(np.abs(self.z[:self.np] - zh)))
            off = np.array(h.theta) * cosmo.angdist(zh)
            if isinstance(h, synth.ParticlePlane):
                obj = glb.TreeQuadParticles(h.particles, inv_area=h.inv_area, bucket=20, theta_force=0.1,
                                            inv_screening_scale=h.max_range)
            else:
                obj = glb.halo_from_spec(h)
            self.halos[j].append((isinstance(h, synth.ParticlePlane), obj, off))

    def plane_force(self, j, xx, prec):
        """Plane j at physical positions xx: (alpha (n,2) with the sign of
        LensPlaneSingular::force, kappa, gamma0, gamma1)."""
        import torch
        n = len(xx)
        al = np.zeros((n, 2)); kap = np.zeros(n); g0 = np.zeros(n); g1 = np.zeros(n)
        for part, obj, off in self.halos[j]:
            xc = np.ascontiguousarray(xx - off)
            if part:
                r = torch.from_numpy(xc).cuda()
                o = torch.empty((n, 5), dtype=torch.float64, device="cuda")
                torch.cuda.synchronize()
                obj.force_device(n, r.data_ptr(), o.data_ptr(), prec, None)
                torch.cuda.synchronize()
                o = o.cpu().numpy()
                # force_halo negates the walk's alpha, force subtracts it
                al += o[:, :2]; kap += o[:, 2]; g0 += o[:, 3]; g1 += o[:, 4]
            else:
                a, k, g, _ = obj.force_halo(xc)
                al -= a; kap += k; g0 += g[:, 0]; g1 += g[:, 1]
        return al, kap, g0, g1

    def shoot(self, x, alpha_prec, G_prec, noise=0.0, seed=0, g_noise=0.0):
        """y (n,2), A (n,4) with the deflection from alpha_prec (times
        1 + noise * N(0,1) per component) and kappa/gamma from G_prec (times
        1 + g_noise * N(0,1) per component), both evaluated at the positions
        this recursion produces."""
        rs = np.random.default_rng(seed)
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 2)
        n = len(x)
        th, sa = x.copy(), x.copy()
        A = np.tile([1.0, 0.0, 0.0, 1.0], (n, 1))
        s = A.copy()
        z, Dl, dDl, ch = self.z, self.Dl, self.dDl, self.charge
        for j in range(self.np):
            xx = th * (Dl[j] / (1 + z[j]))
            fa = self.plane_force(j, xx, alpha_prec)
            fg = fa if G_prec == alpha_prec else self.plane_force(j, xx, G_prec)
            al = fa[0] * (1 + noise * rs.standard_normal(fa[0].shape)) if noise else fa[0]
            Gf = ch * Dl[j] / (1 + z[j])
            kap, g0, g1 = fg[1], fg[2], fg[3]
            if g_noise:
                kap, g0, g1 = (v * (1 + g_noise * rs.standard_normal(v.shape)) for v in (kap, g0, g1))
            G0, G1, G3 = Gf * (kap + g0), Gf * g1, Gf * (kap - g0)
            sa = sa - ch * al
            aa, bb = dDl[j + 1] / Dl[j + 1], Dl[j] / Dl[j + 1]
            th = bb * th + aa * sa
            s = np.stack([s[:, 0] - (G0 * A[:, 0] + G1 * A[:, 2]), s[:, 1] - (G0 * A[:, 1] + G1 * A[:, 3]),
                          s[:, 2] - (G1 * A[:, 0] + G3 * A[:, 2]), s[:, 3] - (G1 * A[:, 1] + G3 * A[:, 3])], 1)
            A = A * bb + s * aa
        return th, A


def error_stats(x, y, A, yref, Aref, kappa_floor=1e-3, gamma_floor=1e-3):
    """Median and 99.9th percentile of the relative errors of alpha = x - y,
    kappa = 1 - (a0 + a3)/2, |gamma| and invmag = det A against a reference
    result.  Denominators: |alpha_ref| (rays below 1e-6 of the median |alpha|
    left out), max(|kappa_ref|, kappa_floor), max(|gamma_ref|, gamma_floor);
    invmag only away from critical curves, |invmag_ref| > 0.05."""
    a, ar = x - y, x - yref
    na = np.hypot(ar[:, 0], ar[:, 1])
    keep = na > 1e-6 * np.median(na)
    ea = np.hypot(*(a - ar).T)[keep] / na[keep]

    def der(M):
        return (1 - (M[:, 0] + M[:, 3]) / 2, np.hypot((M[:, 0] - M[:, 3]) / 2, (M[:, 1] + M[:, 2]) / 2),
                M[:, 0] * M[:, 3] - M[:, 1] * M[:, 2])
    k, g, inv = der(A)
    kr, gr, invr = der(Aref)
    m = np.abs(invr) > 0.05
    out = {}
    for name, e in (("alpha", ea), ("kappa", np.abs(k - kr) / np.maximum(np.abs(kr), kappa_floor)),
                    ("gamma", np.abs(g - gr) / np.maximum(np.abs(gr), gamma_floor)),
                    ("invmag", np.abs(inv - invr)[m] / np.abs(invr[m]))):
        out[name] = {"median": float(np.median(e)) if len(e) else 0.0,
                     "p999": float(np.percentile(e, 99.9)) if len(e) else 0.0}
    return out


def uniform_map_restated(x, values, map_center, nx, ny, rng):
    """GridMap::writePixelMapUniform restated (include/gridmap.h:506-690;
    PixelMap's lower corner and find_index, ImageProcessing/pixelmap.cpp): the
    grid points in order, each writing its value into its pixel (truncation
    toward zero), the last write kept."""
    res = rng / (nx - 1)
    p1 = np.array(map_center) - np.array([nx, ny]) * res / 2.0
    out = np.zeros(nx * ny)
    for i in range(len(x)):
        ix, iy = int((x[i, 0] - p1[0]) / res), int((x[i, 1] - p1[1]) / res)
        if 0 <= ix < nx and 0 <= iy < ny:
            out[ix + nx * iy] = values[i]
    return out.reshape(ny, nx)


# ------------------------------------------------------- reference driver
def ref_available() -> bool:
    return os.path.exists(REF_BIN)


class RefDriver:
    """Runs commands against the reference compiled in place (oracle/_ref);
    binary=DROPIN_BIN runs the same reference code with the GPU drop-in as
    its rayshooter."""

    def __init__(self, binary: str = REF_BIN):
        self.bin = binary
        self.tmp = tempfile.mkdtemp(prefix="glamer_ref_")
        self.lines = []
        self.k = 0

    def _file(self, arr: Optional[np.ndarray] = None) -> str:
        self.k += 1
        f = os.path.join(self.tmp, f"a{self.k}.bin")
        if arr is not None:
            np.ascontiguousarray(arr).tofile(f)
        return f

    def run(self, lines, timeout=3600):
        script = "\n".join(lines) + "\n"
        r = subprocess.run([self.bin], input=script.encode(), stdout=subprocess.PIPE,
                           stderr=subprocess.PIPE, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"glamer_ref failed: {r.stderr.decode()[-2000:]}")

    def tree_force(self, particles, rays, bucket=5, theta=0.1, inv_area=0.0, max_range=-1.0,
                   periodic=False, inv_screening=0.0, export=False):
        pf = self._file(particles)
        rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 2)
        rf = self._file(rays)
        of = self._file()
        ef = self._file() if export else ""
        self.run([f"tree {pf} {len(particles)} {bucket} {theta!r} {inv_area!r} {max_range!r} "
                  f"{int(periodic)} {inv_screening!r} {rf} {len(rays)} {of} {ef}"])
        out = np.fromfile(of).reshape(-1, 7)
        if export:
            return out, np.fromfile(ef).reshape(-1, 16)
        return out

    def halo_force(self, h, xcm, screening=None):
        """force_halo of an NFW / NSIE halo; screening given: with
        subtract_point = true and that screening."""
        xcm = np.ascontiguousarray(xcm, dtype=np.float64).reshape(-1, 2)
        xf = self._file(xcm)
        of = self._file()
        sub = "" if screening is None else f" {float(screening)!r}"
        if isinstance(h, synth.NFWHalo):
            cmd = f"nfw {h.mass!r} {h.rsize!r} {h.z!r} {h.conc!r} 1 0 {xf} {len(xcm)} {of}{sub}"
        else:
            cmd = (f"nsie {h.mass!r} {h.z!r} {h.sigma!r} {h.rcore!r} {h.fratio!r} {h.pa!r} "
                   f"{xf} {len(xcm)} {of}{sub}")
        self.run([cmd])
        o = np.fromfile(of)
        return o[:-3].reshape(-1, 7), tuple(o[-3:])

    def smoothing(self, particles, nsmooth):
        """LensHaloParticles::calculate_smoothing in the reference -> (sizes, seconds)."""
        pf = self._file(np.ascontiguousarray(particles, dtype=synth.PARTICLE_DTYPE))
        of, tf = self._file(), self._file()
        self.run([f"smooth {pf} {len(particles)} {int(nsmooth)} {of} {tf}"])
        return np.fromfile(of).astype(np.float32), float(np.fromfile(tf)[0])

    def make_particles(self, filename, fmt, nsmooth, recenter=False, cut=0, center=(0.0, 0.0, 0.0), radius=0.0):
        """MakeParticleLenses in the reference (then radialCut for cut 1,
        cylindricalCut for cut 2) -> (records, meta) or (None, None) when it
        throws; meta = {cm[3], bbox_ll[3], bbox_ur[3], z_original, nparticles[6],
        densest_particle[3]}."""
        of = self._file()
        c = " ".join(repr(float(v)) for v in center)
        self.run([f"makeparticles {filename} {int(fmt)} {int(nsmooth)} {int(recenter)} {of} {int(cut)} {c} "
                  f"{float(radius)!r}"])
        meta = np.fromfile(of + ".meta")
        if meta[0] == 0:
            return None, None
        return np.fromfile(of, dtype=synth.PARTICLE_DTYPE), meta[1:]

    def write_sizes(self, particles, nsmooth, filename):
        pf = self._file(np.ascontiguousarray(particles, dtype=synth.PARTICLE_DTYPE))
        self.run([f"writesizes {pf} {len(particles)} {int(nsmooth)} {filename}"])

    def read_sizes(self, filename, n, nsmooth, min_size):
        """readSizesFile -> sizes, None (not found / other Nsmooth) or 'throw'."""
        of = self._file()
        self.run([f"readsizes {filename} {int(n)} {int(nsmooth)} {float(min_size)!r} {of}"])
        o = np.fromfile(of)
        if o[0] < 0:
            return "throw"
        return o[1:].astype(np.float32) if o[0] == 1 else None

    def field_plane(self, fp: "synth.FieldPlane", xx):
        """LensPlaneTree::force of a field plane at plane positions xx -> (n, 7)."""
        rows = []
        for h in fp.halos:
            if isinstance(h, synth.NFWHalo):
                rows.append([0, h.mass, h.rsize, h.conc, 0, 0, h.theta[0], h.theta[1]])
            else:
                rows.append([1, h.mass, h.sigma, h.rcore, h.fratio, h.pa, h.theta[0], h.theta[1]])
        hf = self._file(np.asarray(rows, dtype=np.float64))
        xx = np.ascontiguousarray(xx, dtype=np.float64).reshape(-1, 2)
        xf = self._file(xx)
        of = self._file()
        self.run([f"fieldplane {hf} {len(rows)} {fp.z!r} {fp.sigma_back!r} {fp.inv_screening!r} {xf} {len(xx)} {of}"])
        return np.fromfile(of).reshape(-1, 7)

    def source_sb(self, kind, p7, y):
        """The reference's Source::SurfaceBrightness at source positions y ->
        (values, total flux); p7 as the driver's sourcesb command reads them."""
        y = np.ascontiguousarray(y, dtype=np.float64).reshape(-1, 2)
        yf = self._file(y)
        of = self._file()
        self.run([f"sourcesb {kind} " + " ".join(repr(float(v)) for v in p7) + f" {yf} {len(y)} {of}"])
        o = np.fromfile(of)
        return o[:-1], float(o[-1])

    def adaptive(self, spec, n1d, center, range_rad, kind, p7):
        """GridMap + AdaptiveRefreshSurfaceBrightnesses in the reference -> total."""
        of = self._file()
        self.run(self.lens_lines(spec) + [f"adaptive {n1d} {center[0]!r} {center[1]!r} {range_rad!r} {kind} " +
                                          " ".join(repr(float(v)) for v in p7) + f" {of}"])
        return float(np.fromfile(of)[0])

    def lens_lines(self, spec: synth.LensSpec):
        lines = [f"lens {spec.zsource!r}"]
        for h in spec.halos:
            if isinstance(h, synth.ParticlePlane):
                pf = self._file(h.particles)
                lines.append(f"particles {pf} {len(h.particles)} {h.z!r} {h.inv_area!r} "
                             f"{h.max_range!r} {h.theta[0]!r} {h.theta[1]!r}")
            elif isinstance(h, synth.NSIEHalo):
                lines.append(f"addnsie {h.mass!r} {h.z!r} {h.sigma!r} {h.rcore!r} {h.fratio!r} "
                             f"{h.pa!r} {h.theta[0]!r} {h.theta[1]!r}")
            elif isinstance(h, synth.NFWHalo):
                lines.append(f"addnfw {h.mass!r} {h.rsize!r} {h.z!r} {h.conc!r} "
                             f"{h.theta[0]!r} {h.theta[1]!r}")
        return lines

    def grid(self, spec, n1d, center=(0.0, 0.0), range_rad=30 * synth.ARCSEC):
        of = self._file()
        tf = self._file()
        self.run(self.lens_lines(spec) + [f"grid {n1d} {center[0]!r} {center[1]!r} {range_rad!r} {of} {tf}"])
        o = np.fromfile(of).reshape(-1, 6)
        return o[:, :2], o[:, 2:], float(np.fromfile(tf)[0])

    def rays(self, spec, x, zs=None):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 2)
        xf = self._file(x)
        of = self._file()
        tf = self._file()
        if zs is None:
            cmd = f"points {xf} {len(x)} {of} {tf}"
        else:
            zf = self._file(np.ascontiguousarray(zs, dtype=np.float64))
            cmd = f"rays {xf} {len(x)} {zf} {of} {tf}"
        self.run(self.lens_lines(spec) + [cmd])
        o = np.fromfile(of).reshape(-1, 6)
        return o[:, :2], o[:, 2:], float(np.fromfile(tf)[0])

    def rays_batches(self, spec, xs, timeout=3600):
        """One reference process: the lens is built once, then
        Lens::rayshooterInternal(n, Point*) runs on each ray array of xs in
        turn -> [(y, A, seconds of that call)]."""
        cmds, files = [], []
        for x in xs:
            x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 2)
            xf, of, tf = self._file(x), self._file(), self._file()
            cmds.append(f"points {xf} {len(x)} {of} {tf}")
            files.append((of, tf))
        self.run(self.lens_lines(spec) + cmds, timeout=timeout)
        out = []
        for of, tf in files:
            o = np.fromfile(of).reshape(-1, 6)
            out.append((o[:, :2], o[:, 2:], float(np.fromfile(tf)[0])))
        return out

    def threads(self) -> int:
        """The thread count the reference's rayshooterInternal uses on this host."""
        tf = self._file()
        self.run([f"threads {tf}"])
        return int(np.fromfile(tf)[0])
