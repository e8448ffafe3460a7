"""B200-native ray shooting for GLAMER / SLsimLib lenses.

Python mirror of the reference's interface for the ray-shooting path, over the
C ABI of ``libglamer_b200.so`` (include/glamer_b200.h).  Class and method
names follow the reference:

* ``TreeQuadParticles(particles, ...)`` / ``force2D_recur(rays)``
  (include/quadTree.h:49-68, 932-987);
* ``LensHaloParticles``, ``LensHaloNFW``, ``LensHaloRealNSIE`` with
  ``force_halo(xcm)`` and ``setTheta`` (include/particle_halo.h,
  include/lens_halos.h);
* ``Lens(zsource)`` with ``insertMainHalo`` / ``moveinMainHalo``,
  ``ResetSourcePlane`` and ``rayshooterInternal`` (include/lens.h);
* ``GridMap(lens, N, center, range)`` (include/gridmap.h:35).

There is no CPU path: without a CUDA device every call raises
``GlamerError`` (status GLB_ERR_NO_DEVICE).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

from .synth import PARTICLE_DTYPE

__all__ = [
    "GlamerError", "load_library", "TreeQuadParticles", "LensHaloParticles", "LensHaloNFW",
    "LensHaloRealNSIE", "Lens", "GridMap", "GridBatch", "Server", "PREC_FP64", "PREC_SPLIT", "PARTICLE_DTYPE",
]

HERE = os.path.dirname(os.path.abspath(__file__))
# SLSIMLIB_B200_LIB selects another build of the library (e.g. for A/B timing of kernel variants)
LIB_PATH = os.environ.get("SLSIMLIB_B200_LIB") or os.path.join(HERE, "libglamer_b200.so")

PREC_FP64 = 0
PREC_SPLIT = 1
PREC_FP32 = 2

# per-ray status bytes of Lens.rayshooterInternal_status
RAY_OK = 0
RAY_SKIPPED = 1
RAY_NONFINITE = 2

GLB_ERR_ARG = -1
GLB_ERR_CUDA = -2
GLB_ERR_OOM = -3
GLB_ERR_SAME_PLACE = -4
GLB_ERR_DEPTH = -5
GLB_ERR_UNSUPPORTED = -6
GLB_ERR_NO_DEVICE = -7
GLB_ERR_TIMEOUT = -8

# every symbol include/glamer_b200.h declares
EXPORTED = [
    "glb_last_error", "glb_version", "glb_set_option",
    "glb_tree_create", "glb_tree_destroy", "glb_tree_force2D_recur", "glb_tree_force_device", "glb_tree_export",
    "glb_tree_build_ms", "glb_direct_sum_device",
    "glb_halo_particles", "glb_halo_nfw", "glb_halo_nsie", "glb_halo_set_theta", "glb_halo_force", "glb_halo_force_ex",
    "glb_halo_params", "glb_halo_destroy", "glb_halo_field_plane", "glb_halo_nsie_state",
    "glb_lens_create", "glb_lens_destroy", "glb_lens_insert_halo", "glb_lens_insert_field_plane",
    "glb_lens_nplanes", "glb_lens_planes",
    "glb_lens_reset_source", "glb_lens_rayshoot", "glb_lens_rayshoot_device", "glb_lens_rayshoot_status",
    "glb_lens_rayshoot_device_status", "glb_gridmap", "glb_gridmap_pixelmap", "glb_gridmap_pixelmap_uniform",
    "glb_gridmap_surface_brightness", "glb_gridmap_adaptive_surface_brightness",
    "glb_lens_last_timing", "glb_lens_count_interactions", "glb_lens_rayshoot_noalloc",
    "glb_batch_create_grids", "glb_batch_run", "glb_batch_autotune", "glb_batch_set_block", "glb_batch_info",
    "glb_batch_result", "glb_batch_destroy", "glb_batch_tile", "glb_batch_set_tile",
    "glb_server_create", "glb_server_submit", "glb_server_wait", "glb_server_poll", "glb_server_stats",
    "glb_server_destroy", "glb_server_admission",
    "glb_particles_smoothing", "glb_particles_smoothing_device",
]


class GlamerError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_vp = C.c_void_p
_lib = None


def load_library():
    """Loads libglamer_b200.so (built in-tree by slsimlib_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise GlamerError(GLB_ERR_NO_DEVICE,
                          f"{LIB_PATH} is missing: run `python -m slsimlib_b200.build` first")
    L = C.CDLL(LIB_PATH)
    L.glb_last_error.restype = C.c_char_p
    L.glb_version.restype = C.c_char_p
    L.glb_set_option.argtypes = [C.c_int, C.c_longlong]
    L.glb_tree_create.argtypes = [_vp, C.c_size_t, C.c_float, C.c_float, C.c_double, C.c_int, C.c_double,
                                  C.c_int, C.c_double, C.c_double, C.POINTER(_vp)]
    L.glb_tree_destroy.argtypes = [_vp]
    L.glb_tree_force2D_recur.argtypes = [_vp, C.c_size_t, _vp, _vp, _vp, _vp, _vp]
    L.glb_tree_export.argtypes = [_vp, C.POINTER(C.c_size_t), _vp]
    L.glb_tree_force_device.argtypes = [_vp, C.c_size_t, _vp, _vp, C.c_int, _vp]
    L.glb_direct_sum_device.argtypes = [_vp, C.c_size_t, C.c_double, _vp, C.c_size_t, _vp, _vp]
    L.glb_tree_build_ms.argtypes = [_vp, C.POINTER(C.c_double)]
    L.glb_halo_particles.argtypes = [_vp, C.c_size_t, C.c_double, C.c_double, C.c_double, C.POINTER(_vp)]
    L.glb_halo_nfw.argtypes = [C.c_float, C.c_float, C.c_double, C.c_float, C.c_float, C.c_float, C.POINTER(_vp)]
    L.glb_halo_nsie.argtypes = [C.c_float, C.c_double, C.c_float, C.c_float, C.c_float, C.c_float,
                                C.POINTER(_vp)]
    L.glb_halo_set_theta.argtypes = [_vp, C.c_double, C.c_double]
    L.glb_halo_force.argtypes = [_vp, C.c_size_t, _vp, _vp, _vp, _vp, _vp]
    L.glb_halo_force_ex.argtypes = [_vp, C.c_size_t, _vp, _vp, _vp, _vp, _vp, C.c_int, C.c_double]
    L.glb_halo_params.argtypes = [_vp, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.glb_halo_destroy.argtypes = [_vp]
    L.glb_halo_field_plane.argtypes = [_vp, C.c_int, C.c_double, C.c_double, C.c_double, C.POINTER(_vp)]
    L.glb_lens_insert_field_plane.argtypes = [_vp, _vp]
    L.glb_lens_create.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.POINTER(_vp)]
    L.glb_lens_destroy.argtypes = [_vp]
    L.glb_lens_insert_halo.argtypes = [_vp, _vp, C.c_int]
    L.glb_lens_nplanes.argtypes = [_vp, C.POINTER(C.c_int)]
    L.glb_lens_planes.argtypes = [_vp, _vp, _vp, _vp]
    L.glb_lens_reset_source.argtypes = [_vp, C.c_double, C.c_int, C.POINTER(C.c_int)]
    L.glb_lens_rayshoot.argtypes = [_vp, C.c_size_t, _vp, _vp, _vp, _vp, C.c_int]
    L.glb_lens_rayshoot_device.argtypes = [_vp, C.c_size_t, _vp, _vp, _vp, _vp, C.c_int, _vp]
    L.glb_lens_rayshoot_status.argtypes = [_vp, C.c_size_t, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int]
    L.glb_lens_rayshoot_device_status.argtypes = [_vp, C.c_size_t, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int, _vp]
    L.glb_gridmap.argtypes = [_vp, C.c_size_t, _vp, C.c_double, _vp, _vp, C.c_int]
    L.glb_gridmap_pixelmap.argtypes = [_vp, C.c_size_t, _vp, C.c_double, C.c_int, _vp, C.c_int]
    L.glb_gridmap_pixelmap_uniform.argtypes = [_vp, C.c_size_t, _vp, C.c_double, _vp, C.c_size_t, C.c_size_t,
                                               C.c_int, _vp, C.c_int]
    L.glb_gridmap_surface_brightness.argtypes = [_vp, C.c_size_t, _vp, C.c_double, C.c_int, _vp, _vp,
                                                 C.POINTER(C.c_double), C.c_int]
    L.glb_gridmap_adaptive_surface_brightness.argtypes = [_vp, C.c_size_t, _vp, C.c_double, C.c_int, _vp, _vp,
                                                          C.POINTER(C.c_double), C.c_int]
    L.glb_lens_last_timing.argtypes = [_vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.glb_lens_count_interactions.argtypes = [_vp, C.c_size_t, _vp, _vp, _vp]
    L.glb_lens_rayshoot_noalloc.argtypes = [_vp, C.c_size_t, _vp, _vp, _vp, _vp, C.c_int, _vp]
    L.glb_batch_create_grids.argtypes = [_vp, C.c_int, _vp, _vp, _vp, C.c_int, C.POINTER(_vp)]
    L.glb_batch_run.argtypes = [_vp, C.c_int]
    L.glb_batch_autotune.argtypes = [_vp, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.glb_batch_set_block.argtypes = [_vp, C.c_int]
    L.glb_batch_tile.argtypes = [_vp, C.POINTER(C.c_int)]
    L.glb_batch_set_tile.argtypes = [_vp, C.c_int]
    L.glb_batch_info.argtypes = [_vp, C.POINTER(C.c_size_t), C.POINTER(C.c_double), C.POINTER(C.c_int)]
    L.glb_batch_result.argtypes = [_vp, C.c_int, _vp, _vp]
    L.glb_batch_destroy.argtypes = [_vp]
    L.glb_server_create.argtypes = [_vp, C.c_int, C.c_size_t, C.c_int, C.c_int, C.POINTER(_vp)]
    L.glb_server_submit.argtypes = [_vp, C.c_int, C.c_size_t, _vp, C.c_double, _vp, _vp,
                                    C.POINTER(C.c_longlong)]
    L.glb_server_wait.argtypes = [_vp, C.c_longlong, C.c_double, _vp]
    L.glb_server_poll.argtypes = [_vp, C.c_longlong, C.POINTER(C.c_int)]
    L.glb_server_stats.argtypes = [_vp, _vp]
    L.glb_server_admission.argtypes = [_vp, _vp, _vp]
    L.glb_server_destroy.argtypes = [_vp]
    L.glb_particles_smoothing.argtypes = [_vp, C.c_size_t, C.c_int]
    L.glb_particles_smoothing_device.argtypes = [_vp, C.c_size_t, C.c_int, _vp, _vp, _vp]
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        raise GlamerError(rc, load_library().glb_last_error().decode())


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_vp)


def _f64(a, shape=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a if shape is None else a.reshape(shape)


def _particles(p) -> np.ndarray:
    p = np.ascontiguousarray(p)
    if p.dtype != PARTICLE_DTYPE:
        raise TypeError("particles must be a ParticleType<float> record array (slsimlib_b200.PARTICLE_DTYPE)")
    return p


def _forces(n):
    return (np.zeros((n, 2)), np.zeros(n), np.zeros((n, 3)), np.zeros(n))


# ------------------------------------------------------------------- trees
class TreeQuadParticles:
    """TreeQuadParticles<ParticleType<float>> (include/quadTree.h:49-60)."""

    def __init__(self, particles, mass_fixed=-1.0, size_fixed=-1.0, inv_area=0.0, bucket=5, theta_force=0.1,
                 periodic_buffer=False, inv_screening_scale=0.0, maximum_range=-1.0, keep_export=False):
        L = load_library()
        p = _particles(particles)
        h = _vp()
        if keep_export:
            _check(L.glb_set_option(1, 1))
        try:
            _check(L.glb_tree_create(_p(p), len(p), mass_fixed, size_fixed, inv_area, bucket, theta_force,
                                     int(periodic_buffer), inv_screening_scale, maximum_range, C.byref(h)))
        finally:
            if keep_export:
                L.glb_set_option(1, 0)
        self._h = h

    def force2D_recur(self, rays):
        """alpha (n,2), kappa (n,), gamma (n,3), phi (n,) at rays (n,2) in physical Mpc."""
        r = _f64(rays, (-1, 2))
        a, k, g, ph = _forces(len(r))
        _check(load_library().glb_tree_force2D_recur(self._h, len(r), _p(r), _p(a), _p(k), _p(g), _p(ph)))
        return a, k, g, ph

    def force_device(self, n: int, rays_ptr: int, out_ptr: int, precision=PREC_FP64, stream=None):
        """force2D_recur on device rays (raw pointers): out = 5 doubles per ray."""
        _check(load_library().glb_tree_force_device(self._h, n, rays_ptr, out_ptr, precision, stream))

    def export(self) -> np.ndarray:
        L = load_library()
        nb = C.c_size_t(0)
        _check(L.glb_tree_export(self._h, C.byref(nb), None))
        out = np.zeros((nb.value, 16))
        _check(L.glb_tree_export(self._h, C.byref(nb), _p(out)))
        return out

    def build_ms(self) -> float:
        v = C.c_double(0)
        _check(load_library().glb_tree_build_ms(self._h, C.byref(v)))
        return v.value

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            load_library().glb_tree_destroy(self._h)
            self._h = None


# ------------------------------------------------------------------- halos
class _Halo:
    """Common part of the halo classes: a description that can create the
    C-side halo (Lens.insertMainHalo copies, as the reference does)."""

    theta = (0.0, 0.0)

    def setTheta(self, tx, ty=None):
        if ty is None:
            tx, ty = tx
        self.theta = (float(tx), float(ty))

    def _create(self):
        raise NotImplementedError

    def _make(self):
        h = self._create()
        _check(load_library().glb_halo_set_theta(h, self.theta[0], self.theta[1]))
        return h

    def force_halo(self, xcm, subtract_point=False, screening=1.0):
        """LensHalo::force_halo at positions xcm (n,2) relative to the halo
        centre, physical Mpc: alpha (n,2), kappa, gamma (n,3), phi."""
        L = load_library()
        x = _f64(xcm, (-1, 2))
        h = self._make()
        try:
            a, k, g, ph = _forces(len(x))
            _check(L.glb_halo_force_ex(h, len(x), _p(x), _p(a), _p(k), _p(g), _p(ph), int(bool(subtract_point)),
                                       float(screening)))
            return a, k, g, ph
        finally:
            L.glb_halo_destroy(h)

    def params(self):
        L = load_library()
        h = self._make()
        try:
            m, rs, rm = C.c_float(), C.c_float(), C.c_float()
            _check(L.glb_halo_params(h, C.byref(m), C.byref(rs), C.byref(rm)))
            return m.value, rs.value, rm.value
        finally:
            L.glb_halo_destroy(h)


class LensHaloParticles(_Halo):
    """LensHaloParticles(std::vector<ParticleType<float>>&, float redshift,
    cosmo, Point_2d(0,0), recenter=false, inv_area, MinPSize=0, max_range)
    (include/particle_halo.h:58-75)."""

    def __init__(self, particles, redshift, inv_area=0.0, max_range=-1.0):
        self.particles = _particles(particles)
        self.z = float(redshift)
        self.inv_area = float(inv_area)
        self.max_range = float(max_range)

    def _create(self):
        h = _vp()
        _check(load_library().glb_halo_particles(_p(self.particles), len(self.particles), self.z, self.inv_area,
                                                 self.max_range, C.byref(h)))
        return h


def calculate_smoothing(Nsmooth: int, pp: np.ndarray, Npoints: Optional[int] = None) -> None:
    """LensHaloParticles<ParticleType<float>>::calculate_smoothing(Nsmooth, pp,
    Npoints) (include/particle_halo.h:683-730) on the GPU: sets pp[i].Size, in
    place, to the distance to the particle's Nsmooth-th nearest neighbour (the
    (Nsmooth+1)-th nearest particle, itself counted), as
    TreeSimple::NNDistance returns it.  Npoints (default len(pp)) smooths the
    first Npoints records only, as the reference does for one particle type."""
    if not isinstance(pp, np.ndarray) or pp.dtype != PARTICLE_DTYPE or not pp.flags.c_contiguous:
        raise TypeError("pp must be a C-contiguous ParticleType<float> record array (slsimlib_b200.PARTICLE_DTYPE)")
    n = len(pp) if Npoints is None else int(Npoints)
    if n < 0 or n > len(pp):
        raise ValueError("Npoints out of range")
    _check(load_library().glb_particles_smoothing(_p(pp), n, int(Nsmooth)))


def calculate_smoothing_device(Nsmooth: int, n: int, particles_ptr: int, size_ptr: int, stream: int = 0):
    """glb_particles_smoothing_device on raw device pointers (n records in,
    n floats out); returns the device milliseconds (sort + boxes, search)."""
    ms = (C.c_float * 2)()
    _check(load_library().glb_particles_smoothing_device(_vp(particles_ptr), int(n), int(Nsmooth), _vp(size_ptr),
                                                         _vp(stream) if stream else None, ms))
    return float(ms[0]), float(ms[1])


class LensHaloNFW(_Halo):
    """LensHaloNFW(float mass, float Rsize, z, float concentration, float fratio,
    float pa, cosmo) (MultiPlane/lens_halos.cpp:389-431)."""

    def __init__(self, mass, Rsize, zlens, concentration, fratio=1.0, pa=0.0):
        self.args = (float(mass), float(Rsize), float(zlens), float(concentration), float(fratio), float(pa))

    def _create(self):
        h = _vp()
        m, r, z, c, f, pa = self.args
        _check(load_library().glb_halo_nfw(m, r, z, c, f, pa, C.byref(h)))
        return h


class LensHaloRealNSIE(_Halo):
    """LensHaloRealNSIE(float mass, z, float sigma, float rcore, float fratio,
    float pa, cosmo) (MultiPlane/lens_halos.cpp:1043-1078)."""

    def __init__(self, mass, zlens, sigma, rcore, fratio, pa):
        self.args = (float(mass), float(zlens), float(sigma), float(rcore), float(fratio), float(pa))

    def _create(self):
        h = _vp()
        _check(load_library().glb_halo_nsie(*self.args, C.byref(h)))
        return h


class LensPlaneTree(_Halo):
    """LensPlaneTree(z, halos, n, sigma_background, inv_screening_scale)
    (MultiPlane/planes.cpp:13-18): a plane of NFW / NSIE field haloes walked
    as TreeQuadHalos (include/quadTreeHalos.h).  force_halo gives
    LensPlaneTree::force at plane positions; Lens.insertFieldPlane adds the
    plane to a lens as Lens::createFieldPlanes does."""

    def __init__(self, z, halos, sigma_background=0.0, inv_screening_scale=0.0):
        self.z = float(z)
        self.halos = list(halos)
        self.sigma_background = float(sigma_background)
        self.inv_screening_scale = float(inv_screening_scale)

    def _create(self):
        L = load_library()
        members = [m._make() for m in self.halos]
        arr = (_vp * max(1, len(members)))(*members)
        h = _vp()
        rc = L.glb_halo_field_plane(arr, len(members), self.z, self.sigma_background, self.inv_screening_scale,
                                    C.byref(h))
        if rc != 0:
            msg = L.glb_last_error().decode()
            for m in members:
                L.glb_halo_destroy(m)
            raise GlamerError(rc, msg)
        return h

    def _make(self):  # a field plane has no position of its own
        return self._create()


# -------------------------------------------------------------------- lens
class Lens:
    """Lens(long *seed, z_source, COSMOLOGY) (MultiPlane/lens.cpp:59-77) for a
    flat LambdaCDM cosmology."""

    def __init__(self, zsource, omega_m=0.3, omega_l=0.7, hubble=0.7):
        L = load_library()
        h = _vp()
        _check(L.glb_lens_create(float(zsource), omega_m, omega_l, hubble, C.byref(h)))
        self._h = h

    def insertMainHalo(self, halo: _Halo, addplanes: bool = True):
        """Lens::insertMainHalo / moveinMainHalo (include/lens.h:149-185)."""
        _check(load_library().glb_lens_insert_halo(self._h, halo._make(), int(addplanes)))

    moveinMainHalo = insertMainHalo

    def insertFieldPlane(self, plane: LensPlaneTree):
        """A LensPlaneTree among the lens planes (Lens::createFieldPlanes,
        MultiPlane/lens.cpp:443-452; combinePlanes sorts all planes by distance)."""
        _check(load_library().glb_lens_insert_field_plane(self._h, plane._make()))

    def getNplanes(self) -> int:
        n = C.c_int(0)
        _check(load_library().glb_lens_nplanes(self._h, C.byref(n)))
        return n.value

    def planes(self):
        n = self.getNplanes()
        z, Dl, dDl = np.zeros(n + 1), np.zeros(n + 1), np.zeros(n + 1)
        _check(load_library().glb_lens_planes(self._h, _p(z), _p(Dl), _p(dDl)))
        return z, Dl, dDl

    def ResetSourcePlane(self, z, nearest=False) -> int:
        j = C.c_int(0)
        _check(load_library().glb_lens_reset_source(self._h, float(z), int(nearest), C.byref(j)))
        return j.value

    def rayshooterInternal(self, x, source_zs=None, precision=PREC_FP64):
        """x (n,2) image-plane angles (radians) -> y (n,2) source-plane angles,
        A (n,4) Jacobian.  source_zs: one source redshift per ray (the
        LinkedPoint / RAY overloads), or None for the lens's source plane."""
        x = _f64(x, (-1, 2))
        n = len(x)
        zs = None
        if source_zs is not None:
            zs = _f64(source_zs)
            if len(zs) != n:
                raise ValueError("missing redshifts")  # internal_rayshooter_multi.cpp:130-133
        y = np.zeros((n, 2))
        A = np.zeros((n, 4))
        _check(load_library().glb_lens_rayshoot(self._h, n, _p(x), _p(zs), _p(y), _p(A), precision))
        return y, A

    def rayshooterInternal_status(self, x, source_zs=None, skip=None, y=None, A=None, precision=PREC_FP64):
        """rayshooterInternal with per-ray flags: skip (n,) bool -- those rays'
        y and A keep the values passed in (the reference's in_image == MAYBE
        points); returns y, A and a status byte per ray (RAY_OK, RAY_SKIPPED,
        RAY_NONFINITE)."""
        x = _f64(x, (-1, 2))
        n = len(x)
        zs = None if source_zs is None else _f64(source_zs)
        if zs is not None and len(zs) != n:
            raise ValueError("missing redshifts")
        sk = None if skip is None else np.ascontiguousarray(skip, dtype=np.uint8)
        y = np.zeros((n, 2)) if y is None else np.array(y, dtype=np.float64, copy=True).reshape(n, 2)
        A = np.zeros((n, 4)) if A is None else np.array(A, dtype=np.float64, copy=True).reshape(n, 4)
        st = np.zeros(n, dtype=np.uint8)
        _check(load_library().glb_lens_rayshoot_status(self._h, n, _p(x), _p(zs), _p(sk), _p(y), _p(A), _p(st),
                                                       precision))
        return y, A, st

    def rayshoot_device(self, n, x_ptr, zs_ptr, y_ptr, A_ptr, precision=PREC_FP64, stream=None):
        """Device-buffer form (raw CUDA pointers)."""
        _check(load_library().glb_lens_rayshoot_device(self._h, n, x_ptr, zs_ptr, y_ptr, A_ptr, precision,
                                                       stream))

    def count_interactions(self, x, source_zs=None) -> np.ndarray:
        """Interaction counts (nodes tested, far cells, leaf point masses,
        big-particle checks, B-splines) summed over rays and planes, then the
        node-loop and leaf-particle-loop iterations summed over lanes."""
        x = _f64(x, (-1, 2))
        zs = None if source_zs is None else _f64(source_zs)
        out = np.zeros(7, dtype=np.uint64)
        _check(load_library().glb_lens_count_interactions(self._h, len(x), _p(x), _p(zs), _p(out)))
        return out

    def last_timing(self):
        k, t = C.c_double(0), C.c_double(0)
        _check(load_library().glb_lens_last_timing(self._h, C.byref(k), C.byref(t)))
        return k.value, t.value

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            load_library().glb_lens_destroy(self._h)
            self._h = None


class GridMap:
    """GridMap(LensHndl, N1d, center, range) (TreeCode_link/gridmap.cpp:93-120):
    an N1d x N1d grid, x fastest, shot through the lens on construction."""

    def __init__(self, lens: Lens, N1d: int, center: Sequence[float], range_: float, precision=PREC_FP64):
        self.N = int(N1d)
        self.center = np.ascontiguousarray(center, dtype=np.float64)
        self.range = float(range_)
        n = self.N * self.N
        self.y = np.zeros((n, 2))
        self.A = np.zeros((n, 4))
        _check(load_library().glb_gridmap(lens._h, self.N, _p(self.center), self.range, _p(self.y), _p(self.A),
                                          precision))

    def positions(self) -> np.ndarray:
        from .synth import grid_positions
        return grid_positions(self.N, tuple(self.center), self.range)

    # LensingVariable outputs of GridMap::writePixelMap (include/gridmap.h:532-600)
    def kappa(self):
        return 1 - (self.A[:, 0] + self.A[:, 3]) / 2

    def gamma1(self):
        return (self.A[:, 0] - self.A[:, 3]) / 2

    def gamma2(self):
        return (self.A[:, 1] + self.A[:, 2]) / 2

    def gamma3(self):
        return (self.A[:, 2] - self.A[:, 1]) / 2

    def invmag(self):
        return self.A[:, 0] * self.A[:, 3] - self.A[:, 1] * self.A[:, 2]

    def alpha(self):
        return self.positions() - self.y


# LensingVariable, include/standard.h:89-102
DELAYT, ALPHA, ALPHA1, ALPHA2, KAPPA, GAMMA, GAMMA1, GAMMA2, GAMMA3, INVMAG, PHI, SURF_BRIGHTNESS = range(12)


def writePixelMap(lens: Lens, N1d: int, center: Sequence[float], range_: float, lensvar: int,
                  precision=PREC_FP64) -> np.ndarray:
    """GridMap(lens, N1d, center, range).writePixelMap(lensvar)
    (include/gridmap.h:529-598) computed on the GPU: an (N1d, N1d) map, rows
    of constant y; only the map comes back to the host."""
    c = np.ascontiguousarray(center, dtype=np.float64)
    out = np.zeros(int(N1d) * int(N1d))
    _check(load_library().glb_gridmap_pixelmap(lens._h, int(N1d), _p(c), float(range_), int(lensvar), _p(out),
                                               precision))
    return out.reshape(int(N1d), int(N1d))


def writePixelMapUniform(lens: Lens, N1d: int, center: Sequence[float], range_: float, map_center: Sequence[float],
                         Nx: int, Ny: int, lensvar: int, precision=PREC_FP64) -> np.ndarray:
    """GridMap(lens, N1d, center, range).writePixelMapUniform(map_center, Nx, Ny,
    lensvar) (include/gridmap.h:98-102,506-690) computed on the GPU: an
    (Ny, Nx) map of pixel side range / (Nx - 1); grid points write their value
    into the pixel containing them (the largest grid index where several do)."""
    c = np.ascontiguousarray(center, dtype=np.float64)
    mc = np.ascontiguousarray(map_center, dtype=np.float64)
    out = np.zeros(int(Nx) * int(Ny))
    _check(load_library().glb_gridmap_pixelmap_uniform(lens._h, int(N1d), _p(c), float(range_), _p(mc), int(Nx),
                                                       int(Ny), int(lensvar), _p(out), precision))
    return out.reshape(int(Ny), int(Nx))


SOURCE_UNIFORM, SOURCE_GAUSSIAN, SOURCE_SERSIC = 0, 1, 2


def refreshSurfaceBrightnesses(lens: Lens, N1d: int, center: Sequence[float], range_: float, kind: int,
                               params: Sequence[float], precision=PREC_FP64):
    """GridMap(lens, N1d, center, range).RefreshSurfaceBrightnesses(&source)
    (TreeCode_link/gridmap.cpp:174-187) on the GPU: (sb as an (N1d, N1d) map,
    total flux).  params per kind as glb_gridmap_surface_brightness documents:
    SOURCE_UNIFORM (x, y, radius), SOURCE_GAUSSIAN (x, y, r_size),
    SOURCE_SERSIC (x, y, flux, Reff_arcsec, PA, index, q, sb_limit)."""
    c = np.ascontiguousarray(center, dtype=np.float64)
    prm = np.ascontiguousarray(params, dtype=np.float64)
    sb = np.zeros(int(N1d) * int(N1d))
    tot = C.c_double()
    _check(load_library().glb_gridmap_surface_brightness(lens._h, int(N1d), _p(c), float(range_), int(kind), _p(prm),
                                                         _p(sb), C.byref(tot), precision))
    return sb.reshape(int(N1d), int(N1d)), tot.value


def adaptiveRefreshSurfaceBrightnesses(lens: Lens, N1d: int, center: Sequence[float], range_: float, kind: int,
                                       params: Sequence[float], precision=PREC_FP64):
    """GridMap(lens, N1d, center, range).AdaptiveRefreshSurfaceBrightnesses(lens,
    source) (TreeCode_link/gridmap.cpp:189-258) with the refinement rays shot
    in batches on the GPU: (refined sb as an (N1d, N1d) map, total flux)."""
    c = np.ascontiguousarray(center, dtype=np.float64)
    prm = np.ascontiguousarray(params, dtype=np.float64)
    sb = np.zeros(int(N1d) * int(N1d))
    tot = C.c_double()
    _check(load_library().glb_gridmap_adaptive_surface_brightness(lens._h, int(N1d), _p(c), float(range_), int(kind),
                                                                  _p(prm), _p(sb), C.byref(tot), precision))
    return sb.reshape(int(N1d), int(N1d)), tot.value


def direct_sum_device(n: int, particles_ptr: int, inv_area: float, nrays: int, rays_ptr: int, out_ptr: int,
                      stream=None):
    """FP64 direct summation (no tree) over device particles at device rays."""
    _check(load_library().glb_direct_sum_device(particles_ptr, n, inv_area, rays_ptr, nrays, out_ptr, stream))


# ----------------------------------------------------------- batched lenses
class GridBatch:
    """GridMaps of many lenses shot by one persistent launch (optionally
    replayed from a CUDA graph).  The lenses must outlive the batch."""

    def __init__(self, lenses: Sequence[Lens], n1d: Sequence[int], centers, ranges, precision=PREC_SPLIT):
        L = load_library()
        self.lenses = list(lenses)
        self.n1d = np.ascontiguousarray(n1d, dtype=np.uint64)
        c = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 2)
        r = np.ascontiguousarray(ranges, dtype=np.float64)
        handles = (_vp * len(self.lenses))(*[l._h for l in self.lenses])
        h = _vp()
        _check(L.glb_batch_create_grids(handles, len(self.lenses), _p(self.n1d), _p(c), _p(r), precision,
                                        C.byref(h)))
        self._h = h

    def run(self, use_graph=True) -> float:
        """Shoots every grid; returns the device milliseconds of the launch."""
        L = load_library()
        _check(L.glb_batch_run(self._h, int(use_graph)))
        return self.info()[1]

    def autotune(self):
        b, ms = C.c_int(0), C.c_double(0)
        _check(load_library().glb_batch_autotune(self._h, C.byref(b), C.byref(ms)))
        return b.value, ms.value

    def set_block(self, block: int):
        _check(load_library().glb_batch_set_block(self._h, block))

    def tile(self) -> int:
        """Width in rays of the warp tile (8, 16, 32; height 32 / width)."""
        w = C.c_int(0)
        _check(load_library().glb_batch_tile(self._h, C.byref(w)))
        return w.value

    def set_tile(self, width: int):
        _check(load_library().glb_batch_set_tile(self._h, width))

    def info(self):
        n, ms, b = C.c_size_t(0), C.c_double(0), C.c_int(0)
        _check(load_library().glb_batch_info(self._h, C.byref(n), C.byref(ms), C.byref(b)))
        return n.value, ms.value, b.value

    def result(self, i: int):
        n = int(self.n1d[i]) ** 2
        y, A = np.zeros((n, 2)), np.zeros((n, 4))
        _check(load_library().glb_batch_result(self._h, i, _p(y), _p(A)))
        return y, A

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            load_library().glb_batch_destroy(self._h)
            self._h = None


# ---------------------------------------------------------- served requests
class Server:
    """Resident request loop over lenses kept on the device, with continuous
    batching (see glb_server_create).  The models must outlive the server."""

    def __init__(self, models: Sequence[Lens], max_rays_per_batch: int = 0, precision=PREC_SPLIT, nslots: int = 3):
        L = load_library()
        self.models = list(models)
        handles = (_vp * len(self.models))(*[m._h for m in self.models])
        h = _vp()
        _check(L.glb_server_create(handles, len(self.models), max_rays_per_batch, precision, nslots, C.byref(h)))
        self._h = h
        self._live = {}

    def submit(self, model: int, x, zs: float = -1.0) -> int:
        x = _f64(x, (-1, 2))
        n = len(x)
        y, A = np.zeros((n, 2)), np.zeros((n, 4))
        t = C.c_longlong(0)
        _check(load_library().glb_server_submit(self._h, model, n, _p(x), float(zs), _p(y), _p(A), C.byref(t)))
        self._live[t.value] = (x, y, A)
        return t.value

    def wait(self, ticket: int, timeout: float = 0.0):
        """-> (y, A, (t_submit, t_start, t_done))"""
        times = np.zeros(3)
        rc = load_library().glb_server_wait(self._h, ticket, timeout, _p(times))
        if rc == GLB_ERR_TIMEOUT:
            raise TimeoutError(load_library().glb_last_error().decode())
        x, y, A = self._live.pop(ticket)
        _check(rc)
        return y, A, tuple(times)

    def poll(self, ticket: int) -> bool:
        d = C.c_int(0)
        _check(load_library().glb_server_poll(self._h, ticket, C.byref(d)))
        return bool(d.value)

    def stats(self):
        s = np.zeros(6)
        _check(load_library().glb_server_stats(self._h, _p(s)))
        w, f = C.c_double(0), C.c_double(0)
        _check(load_library().glb_server_admission(self._h, C.byref(w), C.byref(f)))
        return dict(rays=s[0], requests=s[1], batches=s[2], busy_s=s[3], ray_budget=s[4], pending=s[5],
                    memory_waits=w.value, min_free_gb=f.value)

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            load_library().glb_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def halo_from_spec(h):
    """The library halo for a halo description of slsimlib_b200.synth
    (ParticlePlane, NFWHalo, NSIEHalo, FieldPlane)."""
    from slsimlib_b200 import synth
    if isinstance(h, synth.ParticlePlane):
        out = LensHaloParticles(h.particles, h.z, h.inv_area, h.max_range)
    elif isinstance(h, synth.NSIEHalo):
        out = LensHaloRealNSIE(h.mass, h.z, h.sigma, h.rcore, h.fratio, h.pa)
    elif isinstance(h, synth.NFWHalo):
        out = LensHaloNFW(h.mass, h.rsize, h.z, h.conc)
    elif isinstance(h, synth.FieldPlane):
        return LensPlaneTree(h.z, [halo_from_spec(m) for m in h.halos], h.sigma_back, h.inv_screening)
    else:
        raise TypeError(h)
    out.setTheta(*h.theta)
    return out


def lens_from_spec(spec) -> Lens:
    """A Lens holding the haloes of a synth.LensSpec in insertion order (field
    planes through insertFieldPlane, the rest through insertMainHalo)."""
    lens = Lens(spec.zsource)
    for h in spec.halos:
        g = halo_from_spec(h)
        if isinstance(g, LensPlaneTree):
            lens.insertFieldPlane(g)
        else:
            lens.insertMainHalo(g, True)
    return lens
