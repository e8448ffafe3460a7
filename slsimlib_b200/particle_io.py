"""Particle files of the reference, read and written on the host, with the
adaptive smoothing they trigger done on the GPU.

Formats (records are ParticleType<float>, 24 bytes: float x[3], float Mass,
float Size, int type):
  * glmb -- MakeParticleLenses::writeSizesB / readSizesB
    (include/particle_halo.h:1036-1073): int Nsmooth, size_t ntot,
    size_t numbytype[6], double redshift, then ntot records, native byte order;
  * sizes cache -- LensHaloParticles::writeSizes / readSizesFile
    (include/particle_halo.h:734-762, 557-632): "# nparticles N",
    "# nsmooth NS", then one Size per line as std::ostream prints a float
    (6 significant digits, %g);
  * ascii positions -- LensHaloParticles::readPositionFileASCII
    (include/particle_halo.h:445-547): "# nparticles N" (and "# mass M" for
    single-mass files) header lines, then x y z [mass] per line;
  * csv -- MakeParticleLenses::readCSV (MultiPlane/particle_lens.cpp:211-341):
    optional '#' lines, then x,y,z[,mass[,size[,type]]] per line.

Numbers are parsed through double and rounded to float (the reference parses
straight to float); the two agree except for decimals within half a double
ulp of a float rounding boundary.
"""
from __future__ import annotations

import os
import struct
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .synth import PARTICLE_DTYPE

GLMB_HEADER = struct.Struct("=iQ6Qd")  # Nsmooth, ntot, numbytype[6], redshift (68 bytes)


# ------------------------------------------------------------------- glmb
def write_glmb(filename: str, data: np.ndarray, nsmooth: int, numbytype: Sequence[int], redshift: float) -> None:
    """MakeParticleLenses::writeSizesB (include/particle_halo.h:1036-1053)."""
    if len(numbytype) != 6:
        raise ValueError("numbytype must have 6 entries")
    data = np.ascontiguousarray(data, dtype=PARTICLE_DTYPE)
    try:
        with open(filename, "wb") as f:
            f.write(GLMB_HEADER.pack(int(nsmooth), len(data), *[int(k) for k in numbytype], float(redshift)))
            f.write(data.tobytes())
    except OSError as e:
        raise RuntimeError(f"file writing error: {filename}") from e


def read_glmb(filename: str) -> Optional[Tuple[np.ndarray, int, List[int], float]]:
    """MakeParticleLenses::readSizesB (include/particle_halo.h:1056-1073):
    (records, Nsmooth, numbytype[6], redshift), or None when the file cannot
    be read."""
    try:
        with open(filename, "rb") as f:
            head = f.read(GLMB_HEADER.size)
            if len(head) < 4:
                return None
            head = head + b"\0" * (GLMB_HEADER.size - len(head))
            ns, ntot, *rest = GLMB_HEADER.unpack(head)
            numbytype, z = list(rest[:6]), rest[6]
            raw = f.read(ntot * PARTICLE_DTYPE.itemsize)
    except OSError:
        return None
    data = np.zeros(ntot, dtype=PARTICLE_DTYPE)
    got = np.frombuffer(raw, dtype=PARTICLE_DTYPE, count=len(raw) // PARTICLE_DTYPE.itemsize)
    data[: len(got)] = got
    return data, int(ns), numbytype, float(z)


# ----------------------------------------------------------- sizes cache
def write_sizes(filename: str, nsmooth: int, sizes: np.ndarray) -> None:
    """LensHaloParticles::writeSizes (include/particle_halo.h:734-762)."""
    sizes = np.asarray(sizes, dtype=np.float32)
    try:
        with open(filename, "w") as f:
            f.write(f"# nparticles {len(sizes)}\n# nsmooth {int(nsmooth)}\n")
            f.write("".join("%g\n" % float(s) for s in sizes))
    except OSError as e:
        raise RuntimeError(f"file writing error: {filename}") from e


def read_sizes_file(filename: str, npoints: int, nsmooth: int, min_size: float) -> Optional[np.ndarray]:
    """LensHaloParticles::readSizesFile (include/particle_halo.h:557-632): the
    sizes (floats, raised to min_size), or None when the file is missing or
    was made with another Nsmooth.  A particle count that differs, missing
    header lines or a wrong number of rows raise RuntimeError, as the
    reference throws."""
    if not os.path.exists(filename):
        return None
    with open(filename) as f:
        lines = f.read().split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    count, i = 0, 0
    while i < len(lines):
        tok = lines[i].split()
        i += 1
        if tok and tok[0] == "#":
            if len(tok) > 1 and tok[1] == "nparticles":
                if int(tok[2]) != npoints:
                    raise RuntimeError("file reading error: number of particles does not match")
                count += 1
            if len(tok) > 1 and tok[1] == "nsmooth":
                if int(tok[2]) != nsmooth:
                    return None
                count += 1
        else:
            break
        if count == 2:
            break
    if count != 2:
        raise RuntimeError("file reading error: missing header lines")
    vals = []
    for ln in lines[i:]:
        if ln.startswith("#"):
            continue
        tok = ln.split()
        vals.append(float(tok[0]) if tok else 0.0)
    if len(vals) != npoints:
        raise RuntimeError("file reading error: number of data rows does not match")
    s = np.asarray(vals, dtype=np.float64).astype(np.float32)
    return np.where(np.float64(min_size) > s.astype(np.float64), np.float32(min_size), s).astype(np.float32)


# ------------------------------------------------------- ascii positions
def read_positions_ascii(filename: str, multimass: bool) -> Tuple[np.ndarray, float]:
    """LensHaloParticles::readPositionFileASCII (include/particle_halo.h:445-547):
    (records, header mass).  Multi-mass files carry a fourth column of masses.
    The reference never stores the header mass of a single-mass file in the
    records (their Mass stays 0); it is returned so that callers can."""
    if not os.path.exists(filename):
        raise RuntimeError(f"file reading error: unable to open {filename}")
    with open(filename) as f:
        lines = f.read().split("\n")
    npoints, mass, count, i = 0, 0.0, 0, 0
    while i < len(lines):
        tok = lines[i].split()
        i += 1
        if tok and tok[0] == "#":
            if len(tok) > 1 and tok[1] == "nparticles":
                npoints = int(tok[2])
                count += 1
            if not multimass and len(tok) > 1 and tok[1] == "mass":
                mass = float(tok[2])
                count += 1
        else:
            break
        if (multimass and count == 1) or (not multimass and count == 2):
            break
    if count == 0:
        raise RuntimeError("file reading error: missing header lines")
    p = np.zeros(npoints, dtype=PARTICLE_DTYPE)
    row = 0
    ncol = 4 if multimass else 3
    for ln in lines[i:]:
        if row >= npoints:
            break
        if ln.startswith("#"):
            continue
        tok = ln.split()
        vals = [float(t) for t in tok[:ncol]] + [0.0] * max(0, ncol - len(tok))
        p["x"][row] = np.asarray(vals[:3], dtype=np.float64).astype(np.float32)
        if multimass:
            p["Mass"][row] = np.float32(vals[3])
        row += 1
    if row != npoints:
        raise RuntimeError("file reading error: number of data rows does not match")
    return p, mass


# ------------------------------------------------------------------- csv
def read_csv(filename: str, columns_used: int, nsmooth: int) -> Tuple[np.ndarray, List[int]]:
    """MakeParticleLenses::readCSV (MultiPlane/particle_lens.cpp:211-341):
    (records, particles per type).  3 columns: unit masses; 4: masses; 5:
    masses and sizes; 6: also types.  With fewer than 5 columns the sizes
    are the adaptive smoothing lengths of every type (on the GPU).  As in the
    reference, a 6-column file counts every particle as type 0 (the count
    reads the type of the record after the one just parsed) and is not
    re-ordered by type."""
    with open(filename) as f:
        lines = f.read().split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    i = 0
    while i < len(lines) and lines[i].startswith("#"):
        i += 1
    body = lines[i:]
    if not body or len(body[0].split(",")) < columns_used:
        raise ValueError(f"file {filename} does not have enough columns.")
    rows = [ln.split(",") for ln in body]
    n = len(rows)
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    try:
        cols = np.array([[float(r[k]) for k in range(min(columns_used, 5))] for r in rows], dtype=np.float64)
    except (ValueError, IndexError) as e:
        raise ValueError(f"bad line in {filename}") from e
    p["x"] = cols[:, :3].astype(np.float32)
    p["Mass"] = np.float32(1.0) if columns_used == 3 else cols[:, 3].astype(np.float32)
    if columns_used >= 5:
        p["Size"] = cols[:, 4].astype(np.float32)
    if columns_used == 6:
        p["type"] = np.array([int(r[5]) for r in rows], dtype=np.int32)
    nparticles = [n, 0, 0, 0, 0, 0]
    if columns_used < 5:
        from . import calculate_smoothing
        calculate_smoothing(nsmooth, p)
    return p, nparticles


# ------------------------------------------------------ MakeParticleLenses
class MakeParticleLenses:
    """MakeParticleLenses (include/particle_halo.h:975-1035,
    MultiPlane/particle_lens.cpp:22-210) for glmb and csv files.

    MakeParticleLenses(filename, fmt, Nsmooth, recenter): fmt "glmb" reads the
    file; "csv3", "csv4", "csv5" read <filename>_S<Nsmooth>.glmb when it
    exists, otherwise the csv file (smoothing on the GPU) and write that glmb
    file for the next time.  "csv6" is refused as in the reference, whose
    switch falls through to its error branch.  MakeParticleLenses(filename,
    recenter=...) with fmt None reads a glmb file."""

    def __init__(self, filename: str, fmt: Optional[str] = None, Nsmooth: int = 0, recenter: bool = False):
        self.filename = filename
        self.Nsmooth = int(Nsmooth)
        self.halos = []
        self.masses = [0.0] * 6
        self.z_original = -1.0
        if fmt in (None, "glmb"):
            r = read_glmb(filename)
            if r is None:
                raise ValueError(f"Can't find file {filename}")
            self.data, self.Nsmooth, self.nparticles, self.z_original = r
        elif fmt in ("csv3", "csv4", "csv5"):
            sizefile = f"{filename}_S{self.Nsmooth}.glmb"
            r = read_glmb(sizefile) if os.path.exists(sizefile) else None
            if r is not None:
                self.data, self.Nsmooth, self.nparticles, self.z_original = r
            else:
                self.data, self.nparticles = read_csv(filename, int(fmt[3]), self.Nsmooth)
                write_glmb(sizefile, self.data, self.Nsmooth, self.nparticles, self.z_original)
        else:
            raise ValueError("Data file format is not supported in MakeParticleLenses.")
        # the glmb-only constructor (particle_lens.cpp:109-137) starts its
        # bounding box at the origin instead of the first particle
        self._moments(from_origin=fmt is None)
        if recenter:
            self.Recenter(self.cm)

    def _moments(self, from_origin: bool):
        # cm sums the float products x*Mass in double, particle by particle
        x = self.data["x"]
        m = self.data["Mass"]
        cm = np.zeros(3)
        for k in range(3):
            cm[k] = float(np.cumsum((x[:, k] * m).astype(np.float64))[-1]) if len(x) else 0.0
        self.cm = cm / (float(np.cumsum(m.astype(np.float64))[-1]) if len(x) else 0.0)
        lo = x.min(axis=0).astype(np.float64) if len(x) else np.zeros(3)
        hi = x.max(axis=0).astype(np.float64) if len(x) else np.zeros(3)
        if from_origin:
            lo, hi = np.minimum(lo, 0.0), np.maximum(hi, 0.0)
        self.bbox_ll, self.bbox_ur = lo, hi

    def Recenter(self, x: Sequence[float]) -> None:
        """particle_lens.cpp:139-151: shifts records, bounding box and centre
        of mass by -x (records rounded to float) and drops the haloes."""
        x = np.asarray(x, dtype=np.float64).copy()
        self.data["x"] = (self.data["x"].astype(np.float64) - x).astype(np.float32)
        self.bbox_ll = self.bbox_ll - x
        self.bbox_ur = self.bbox_ur - x
        self.cm = self.cm - x
        self.halos = []

    def _cut(self, r2: np.ndarray, radius: float) -> None:
        # particle_lens.cpp:447-478 / 497-520: a particle beyond the radius is
        # swapped with the last one still kept, and the scan goes on from the
        # same place; the kept records are then sorted by type if more than one
        # type has particles (stable here; the reference's std::sort leaves the
        # order within a type unspecified)
        # The scan's result in closed form: with K records kept, a kept record
        # at a position below K stays there, and the removed records' places
        # below K, in ascending order, receive the kept records at K and above
        # taken from the end backwards (each swap brings in the last record
        # not yet scanned).
        d = self.data
        out = r2 > float(radius) * float(radius)
        for t, c in zip(*np.unique(d["type"][out], return_counts=True)):
            self.nparticles[int(t)] -= int(c)
        K = int(np.count_nonzero(~out))
        order = np.arange(K)
        order[np.nonzero(out[:K])[0]] = (np.nonzero(~out[K:])[0] + K)[::-1]
        d = d[order]
        if sum(1 for k in self.nparticles if k > 0) > 1:
            d = d[np.argsort(d["type"], kind="stable")]
        self.data = d

    def radialCut(self, center: Sequence[float], radius: float) -> None:
        """Removes the particles farther than radius (Mpc/h) from center."""
        c = np.asarray(center, dtype=np.float64)
        x = self.data["x"].astype(np.float64)
        a, b, e = x[:, 0] - c[0], x[:, 1] - c[1], x[:, 2] - c[2]
        self._cut(a * a + b * b + e * e, radius)

    def cylindricalCut(self, center: Sequence[float], radius: float) -> None:
        """Removes the particles farther than radius (Mpc/h) from center in x, y."""
        c = np.asarray(center, dtype=np.float64)
        x = self.data["x"].astype(np.float64)
        a, b = x[:, 0] - c[0], x[:, 1] - c[1]
        self._cut(a * a + b * b, radius)

    def densest_particle(self) -> np.ndarray:
        """particle_lens.cpp:480-495: position of the largest Mass/Size^3
        (float arithmetic, first maximum)."""
        m, sz = self.data["Mass"], self.data["Size"]
        with np.errstate(divide="ignore", invalid="ignore"):
            d = ((m / sz) / sz) / sz
        best, x = -1.0, np.zeros(3)
        for i in range(len(d)):
            if float(d[i]) > best:
                best = float(d[i])
                x = self.data["x"][i].astype(np.float64)
        return x

    def getnp(self) -> List[int]:
        return list(self.nparticles)

    def getCenterOfMass(self) -> np.ndarray:
        return self.cm.copy()

    def getBoundingBox(self) -> Tuple[np.ndarray, np.ndarray]:
        return self.bbox_ll.copy(), self.bbox_ur.copy()

    def getZoriginal(self) -> float:
        return self.z_original

    def CreateHalos(self, hubble: float, redshift: float, inv_area: float):
        """particle_lens.cpp:153-209: records to comoving Mpc and Msun (x,
        Size and Mass divided by h, in float), one LensHaloParticles per
        particle type present."""
        from . import LensHaloParticles
        unit = 1.0 / float(np.float32(hubble))  # float h, double 1/h
        d = self.data
        d["x"] = (d["x"].astype(np.float64) * unit).astype(np.float32)
        d["Size"] = (d["Size"].astype(np.float64) * unit).astype(np.float32)
        d["Mass"] = (d["Mass"].astype(np.float64) * unit).astype(np.float32)
        self.halos = []
        skip = 0
        for k in range(6):
            nk = int(self.nparticles[k])
            if nk > 0:
                self.halos.append(LensHaloParticles(d[skip:skip + nk].copy(), redshift, inv_area=inv_area))
            skip += nk
        return self.halos


# ------------------------------------------- LensHaloParticles from a file
def lens_halo_particles_from_file(filename: str, redshift: float, Nsmooth: int, theta_rotate=(0.0, 0.0),
                                  recenter: bool = False, multimass: bool = True, inv_area: float = 0.0,
                                  MinPSize: float = 0.0, massscaling: float = 1.0):
    """LensHaloParticles(simulation_filename, SimFileFormat::ascii, redshift,
    Nsmooth, cosmo, theta_rotate, recenter, multimass, inv_area, MinPSize,
    massscaling) (include/particle_halo.h:229-340): reads the ascii positions,
    takes the sizes from <filename>.<Nsmooth>sizes or computes them (GPU) and
    writes that file, then as the reference: sizes below MinPSize raised to it,
    masses of all particles but the first multiplied by massscaling, positions
    from comoving to physical (1/(1+z)), optional recentring on the centre of
    mass, rotation, and a particle lens whose tree has no screening.  Returns
    (slsimlib_b200.LensHaloParticles, the particle records used)."""
    from . import LensHaloParticles, calculate_smoothing
    pp, _ = read_positions_ascii(filename, multimass)
    n = len(pp)
    sizefile = f"{filename}.{int(Nsmooth)}sizes"
    mn = float(MinPSize)
    s = read_sizes_file(sizefile, n, Nsmooth, mn)
    if s is None:
        calculate_smoothing(Nsmooth, pp)
        write_sizes(sizefile, Nsmooth, pp["Size"])
        pp["Size"] = np.where(pp["Size"].astype(np.float64) < mn, np.float32(mn), pp["Size"])
    else:
        pp["Size"] = s
    if n > 1:
        pp["Mass"][1:] = (pp["Mass"][1:].astype(np.float64) * float(massscaling)).astype(np.float32)
    sf = 1.0 / (1.0 + float(redshift))
    pp["x"] = (pp["x"].astype(np.float64) * sf).astype(np.float32)
    m = pp["Mass"] if multimass else np.full(n, pp["Mass"][0], dtype=np.float32)
    mc = np.array([float(np.cumsum((pp["x"][:, k] * m).astype(np.float64))[-1]) for k in range(3)])
    mass = float(np.cumsum(m.astype(np.float64))[-1])
    mc = mc / mass
    if recenter:
        pp["x"] = (pp["x"].astype(np.float64) - mc).astype(np.float32)
    tx, ty = float(theta_rotate[0]), float(theta_rotate[1])
    if tx != 0.0 or ty != 0.0:
        cx, sx, cy, sy = np.cos(tx), np.sin(tx), np.cos(ty), np.sin(ty)
        coord = np.array([[cy, 0.0, -sy], [-sy * sx, cx, -cy * sx], [cx, sx, cy * cx]])
        x = pp["x"].astype(np.float64)
        t = np.zeros_like(x)
        for r in range(3):
            for j in range(3):
                t[:, r] += coord[r, j] * x[:, j]
        pp["x"] = t.astype(np.float32)
    return LensHaloParticles(pp, redshift, inv_area=inv_area, max_range=0.0), pp
