"""Benchmark of the ray-shooting path on the multi-plane light cone.

Workload (one "step" = one GridMap pass): 10 particle planes at
z = 0.1, 0.3, ..., 1.9 holding 320 NFW haloes sampled as 4,194,304 equal-mass
particles (softening 0.5 kpc, opening angle 0.1) plus a main NSIE lens at
z = 0.5 (sigma 250 km/s, q 0.7, core 0.05 arcsec); 2048 x 2048 rays over
60 arcsec; source at z = 2.5.  Inputs are seeded synthetic data of that shape.

Lines printed by rank 0 (one JSON line):
  value  rays/s of the split-precision (FP32 walk + FP64 recursion) form, all
         GPUs, inputs resident in HBM, CUDA events on the launching stream;
  e2e    the same metric through the host C ABI (glb_lens_rayshoot: host
         x in, host y and A out, copies inside the timed region);
  roofline of the plane-step kernel (k_plane_step_split_g; algorithmic FP32 flops from the counted
         interactions / kernel time vs the FP32 CUDA-core peak);
  cpu_baseline: the reference compiled in place (oracle/_ref) on host cores.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--small]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "rays/s/GPU at rel. deflection err <=1e-5 vs plain FP64 GPU form"
N1D = 2048
FIELD_ARCSEC = 60.0

# algorithmic FP32 flops per event of one ray-plane tree evaluation
# (nodes tested V, far-field cells F, leaf point masses P, big-particle checks B,
# B-spline corrections S) and per ray-plane recursion
FLOPS = {"V": 8, "F": 60, "P": 29, "B": 8, "S": 65, "rec": 50}
# DRAM bytes (read + write) per ray of one split plane launch, from an ncu capture of
# `bench.py --no-cpu --no-served --n1d 1536` (184.3 MB for one 1,179,648-ray slab of a
# plane, k_plane_step_split_g): the 96 B ray state read and written once and the plane's
# L2-resident tree
DRAM_BYTES_PER_RAY_PLANE = 156


def workload(small: bool):
    from slsimlib_b200 import synth
    if small:
        return synth.light_cone(seed=2, n_total=262_144), 512
    return synth.light_cone(seed=2), N1D


def make_lens(spec):
    import slsimlib_b200 as glb
    return glb.lens_from_spec(spec)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.rows = []
        self.stop = threading.Event()
        self.t = threading.Thread(target=self.run, daemon=True)

    def run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([c.strip() for c in out.split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def fp32_peak_tflops(sm_mhz):
    # 148 SMs x 128 FP32 lanes x 2 flops per FMA at the sampled SM clock
    return 148 * 128 * 2 * sm_mhz * 1e6 / 1e12


def error_stats(x, y, A, yref, Aref):
    """Relative errors of alpha, kappa, gamma and invmag against a reference
    result (median, 99.9th percentile); floors of 1e-3 on the kappa and gamma
    denominators, invmag where |invmag_ref| > 0.05."""
    from tests.harness import error_stats as es
    return es(x, y, A, yref, Aref)


def attribution(spec, lens, x, nsample=16384, seed=78):
    """Where the split form's kappa/gamma/invmag error comes from, on a seeded
    sample of the grid's rays (tests.harness.PlaneRecursion: the recursion over
    the library's per-plane GPU forces):
      evaluation   -- split kappa/gamma at the FP64 form's plane positions
                      (deflection from the FP64 form);
      propagated   -- split deflection, FP64 kappa/gamma at the positions it
                      gives;
      fp64_noise_* -- the FP64 form with every plane's deflection perturbed by
                      relative Gaussian noise of that size (the conditioning of
                      the light cone: no error in kappa/gamma evaluation);
      fp64_G_noise_6e-8 -- the FP64 form with every plane's kappa/gamma
                      perturbed by FP32 unit roundoff;
    all against the unperturbed FP64 recursion, plus the sample's final fields."""
    import slsimlib_b200 as glb
    from tests.harness import PlaneRecursion
    xs = x[sample_indices(int(round(np.sqrt(len(x)))), nsample, seed)]
    R = PlaneRecursion(spec, lens)
    F, S = glb.PREC_FP64, glb.PREC_SPLIT
    y0, A0 = R.shoot(xs, F, F)
    out = {"rays": len(xs)}
    for name, (pa, pg, eps, geps) in {"evaluation": (F, S, 0.0, 0.0), "propagated": (S, F, 0.0, 0.0),
                                      "fp64_noise_1e-8": (F, F, 1e-8, 0.0), "fp64_noise_1e-10": (F, F, 1e-10, 0.0),
                                      "fp64_G_noise_6e-8": (F, F, 0.0, 6e-8)}.items():
        y, A = R.shoot(xs, pa, pg, noise=eps, seed=5, g_noise=geps)
        out[name] = error_stats(xs, y, A, y0, A0)
    k = 1 - (A0[:, 0] + A0[:, 3]) / 2
    inv = A0[:, 0] * A0[:, 3] - A0[:, 1] * A0[:, 2]
    out["fields"] = {"kappa_median": float(np.median(k)), "invmag_median": float(np.median(inv)),
                     "frac_abs_invmag_below_0.05": float(np.mean(np.abs(inv) < 0.05))}
    return out


def sample_indices(n1d, nsample, seed):
    n = n1d * n1d
    return np.sort(np.random.default_rng(seed).choice(n, size=min(nsample, n), replace=False))


def cpu_reference(spec, n1d, nsample, seed=77):
    """Times the reference (oracle/_ref) Lens::rayshooterInternal on a seeded
    sample of the grid's rays; returns (rays/s, threads, seconds, sample
    description, sample indices, y, A) -- y and A are the reference's results
    for those rays, kept for the parity check of the GPU's FP64 form."""
    from tests import harness as H
    from slsimlib_b200 import synth
    if not H.ref_available():
        return None
    x = synth.grid_positions(n1d, range_rad=FIELD_ARCSEC * synth.ARCSEC)
    idx = sample_indices(n1d, nsample, seed)
    R = H.RefDriver()
    threads = R.threads()
    y, A, secs = R.rays(spec, x[idx])
    return (len(idx) / secs, threads, secs, f"{len(idx)} seeded rays of the {n1d}x{n1d} grid, all planes", idx,
            y, A)


def parity_vs_reference(y_gpu, A_gpu, y_ref, A_ref):
    """The GPU's FP64 form against the reference's own rayshooterInternal on
    the same rays: relative source-position error (max, p99.9) and the largest
    absolute Jacobian difference."""
    ey = np.hypot(*(y_gpu - y_ref).T) / np.hypot(*y_ref.T)
    return {"rays": int(len(y_ref)), "y_max_rel": float(ey.max()), "y_p999_rel": float(np.percentile(ey, 99.9)),
            "A_max_abs": float(np.max(np.abs(A_gpu - A_ref)))}


def run_reference_arm(args, rank):
    """The reference's own CPU rayshooter (oracle/_ref: Lens::rayshooterInternal
    compiled from the reference's sources) on the host cores: one process
    builds the lens once, then each warm-up and timed step shoots a new seeded
    sample of the grid's rays through the reference's Point* overload."""
    if rank != 0:
        return
    from tests import harness as H
    from slsimlib_b200 import synth
    if not H.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/glamer_ref not built"}))
        return
    spec, n1d = workload(args.small)
    nsample = 2048 if args.small else 16384
    x = synth.grid_positions(n1d, range_rad=FIELD_ARCSEC * synth.ARCSEC)
    R = H.RefDriver()
    threads = R.threads()
    res = R.rays_batches(spec, [x[sample_indices(n1d, nsample, 100 + s)] for s in range(args.warmup + args.steps)])
    vals = [nsample / r[2] for r in res[args.warmup:]]
    v = float(np.median(vals))
    n = n1d * n1d
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "rays/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": n / v * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded light cone)",
            "config": {"workload": f"light cone: 10 planes, 4,194,304 particles + NSIE, {n1d}^2 rays over 60 arcsec",
                       "sample_rays_per_step": nsample},
            "cpu_baseline": {"value": v, "unit": "rays/s", "cores": threads, "kind": "reference",
                             "sample": f"{nsample} seeded rays of the grid per step (a new sample each step), all "
                                       f"planes, rate extrapolated per ray; lens built once in one reference "
                                       f"process, each step one rayshooterInternal(n, Point*) call"},
            "e2e": {"value": v, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ------------------------------------------------------------ other workloads
def _tile_order(n1d):
    """Grid indices (x fastest) reordered into 8 x 4 tiles, one tile per warp."""
    ix = np.arange(n1d)
    iy = np.arange(n1d)
    X, Y = np.meshgrid(ix, iy)
    key = ((Y // 4) * ((n1d + 7) // 8) + (X // 8)) * 32 + (Y % 4) * 8 + (X % 8)
    return np.argsort(key.ravel(), kind="stable")


def _timed(fn, stream, steps):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _base_line(args, metric, unit, value, ms, dtype, workload, **extra):
    d = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
         "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
         "data": "synthetic (seeded)", "config": {"workload": workload}}
    d.update(extra)
    return d


def run_single(args):
    """One NFW particle plane (2^18 particles, 1e14 Msun, c=5, z=0.3, 1 kpc),
    512^2 rays over 30 arcsec, z_s=2, through GridMap in the plain FP64 form."""
    import torch
    import slsimlib_b200 as glb
    from slsimlib_b200 import synth
    spec = synth.single_plane_nfw(seed=1)
    lens = make_lens(spec)
    n1d, rng = 512, 30 * synth.ARCSEC
    x_host = synth.grid_positions(n1d, range_rad=rng)
    n = n1d * n1d
    x = torch.from_numpy(x_host).cuda()
    y = torch.empty((n, 2), dtype=torch.float64, device="cuda")
    A = torch.empty((n, 4), dtype=torch.float64, device="cuda")
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    out = {}
    for prec in (glb.PREC_FP64, glb.PREC_SPLIT):
        f = lambda: lens.rayshoot_device(n, x.data_ptr(), None, y.data_ptr(), A.data_ptr(), prec, st.cuda_stream)
        for _ in range(args.warmup):
            f()
        torch.cuda.synchronize()
        out[prec] = (_timed(f, st, args.steps), y.cpu().numpy().copy(), A.cpu().numpy().copy())
    ms = out[glb.PREC_FP64][0]
    line = _base_line(args, "rays/s/GPU (plain FP64 form)", "rays/s", n / (ms / 1e3), ms, "f64",
                      "single NFW particle plane: 2^18 particles, 512^2 rays over 30 arcsec, z_l=0.3, z_s=2")
    line["split"] = {"value": n / (out[glb.PREC_SPLIT][0] / 1e3), "unit": "rays/s",
                     "errors_vs_fp64": error_stats(x_host, out[1][1], out[1][2], out[0][1], out[0][2])}
    if not args.no_cpu:
        from tests import harness as H
        if H.ref_available():
            R = H.RefDriver()
            tf = R._file()
            R.run([f"threads {tf}"])
            thr = int(np.fromfile(tf)[0])
            yr, Ar, secs = R.grid(spec, n1d, range_rad=rng)
            line["cpu_baseline"] = {"value": n / secs, "unit": "rays/s", "cores": thr, "kind": "reference",
                                    "sample": "the full 512^2 GridMap"}
            line["parity_vs_reference"] = {
                "y_max_rel": float(np.max(np.abs(out[0][1] - yr) / np.abs(yr))),
                "A_max_abs": float(np.max(np.abs(out[0][2] - Ar)))}
    print(json.dumps(line))


def run_field(args):
    """The 10-plane light cone plus nine field planes between its particle
    planes (z = 0.2, 0.4, ..., 1.8), each of 400 NFW haloes (1e10-1e13 Msun)
    and 4 NSIE haloes over the 60 arcsec field (LensPlaneTree, no screening);
    2048^2 rays, split and plain FP64 forms."""
    import torch
    import slsimlib_b200 as glb
    from slsimlib_b200 import synth
    spec, n1d = workload(args.small)
    for i in range(9):
        z = 0.2 + 0.2 * i
        spec.halos.append(synth.FieldPlane(z, synth.field_halos(600 + i, 400, z, n_nsie=4)))
    lens = make_lens(spec)
    x_host = synth.grid_positions(n1d, range_rad=FIELD_ARCSEC * synth.ARCSEC)
    n = n1d * n1d
    x = torch.from_numpy(x_host).cuda()
    y = torch.empty((n, 2), dtype=torch.float64, device="cuda")
    A = torch.empty((n, 4), dtype=torch.float64, device="cuda")
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    out = {}
    for prec in (glb.PREC_FP64, glb.PREC_SPLIT):
        f = lambda: lens.rayshoot_device(n, x.data_ptr(), None, y.data_ptr(), A.data_ptr(), prec, st.cuda_stream)
        for _ in range(args.warmup if prec == glb.PREC_SPLIT else 1):
            f()
        torch.cuda.synchronize()
        steps = args.steps if prec == glb.PREC_SPLIT else 1
        out[prec] = (_timed(f, st, steps), y.cpu().numpy().copy(), A.cpu().numpy().copy())
    ms = out[glb.PREC_SPLIT][0]
    line = _base_line(args, "rays/s/GPU, light cone with field planes (split form)", "rays/s", n / (ms / 1e3), ms,
                      "f32+f64", f"light cone (10 particle planes, 4,194,304 particles, NSIE) + 9 field planes of "
                                 f"404 haloes, {n1d}^2 rays over 60 arcsec" + (" [reduced]" if args.small else ""))
    line["planes"] = lens.getNplanes()
    line["plain_fp64"] = {"value": n / (out[glb.PREC_FP64][0] / 1e3), "unit": "rays/s"}
    line["errors_vs_fp64"] = error_stats(x_host, out[1][1], out[1][2], out[0][1], out[0][2])
    print(json.dumps(line))


def run_sweep(args):
    """Precision sweep on one large plane: 2^24 triaxial-NFW particles
    (1e15 Msun, c=4, axes 1/0.8/0.6) + 10% uniform background, 4096^2 rays
    over 40 arcsec at z_l=0.3; opening angles 0.05/0.1/0.3; FP64, split and
    plain FP32 trees; errors against an FP64 direct sum on 1000 seeded rays."""
    import torch
    import slsimlib_b200 as glb
    from slsimlib_b200 import synth
    rs = np.random.default_rng(3)
    cosmo = synth.Cosmology()
    n_halo = 2 ** 24 if not args.small else 2 ** 20
    p = synth.nfw_particles(rs, n_halo, 1e15, 4.0, 0.3, 1e-3, cosmo=cosmo, axis_ratios=(0.8, 0.6))
    nb = int(round(0.1 * n_halo))
    lo = p["x"][:, :2].min(axis=0)
    hi = p["x"][:, :2].max(axis=0)
    bg = np.zeros(nb, dtype=synth.PARTICLE_DTYPE)
    bg["x"][:, :2] = rs.uniform(lo, hi, size=(nb, 2)).astype(np.float32)
    bg["Mass"] = p["Mass"][0]
    bg["Size"] = np.float32(1e-3)
    parts = np.concatenate([p, bg])
    n1d = 4096 if not args.small else 1024
    da = cosmo.angdist(0.3)
    ang = synth.grid_positions(n1d, range_rad=40 * synth.ARCSEC)
    rays = (ang * da)[_tile_order(n1d)]
    n = len(rays)
    dr = torch.from_numpy(np.ascontiguousarray(rays)).cuda()
    out = torch.empty((n, 5), dtype=torch.float64, device="cuda")
    sub = np.random.default_rng(4).choice(n, size=1000, replace=False)
    drs = dr[torch.from_numpy(sub).cuda()].contiguous()
    pdev = torch.from_numpy(parts.view(np.uint8)).cuda()
    ds = torch.empty((1000, 5), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    glb.direct_sum_device(len(parts), pdev.data_ptr(), 0.0, 1000, drs.data_ptr(), ds.data_ptr(), None)
    torch.cuda.synchronize()
    ds = ds.cpu().numpy()
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    results = []
    for theta in (0.05, 0.1, 0.3):
        tree = glb.TreeQuadParticles(parts, bucket=20, theta_force=theta)
        for prec, name in ((glb.PREC_FP64, "fp64"), (glb.PREC_SPLIT, "split"), (glb.PREC_FP32, "fp32")):
            f = lambda: tree.force_device(n, dr.data_ptr(), out.data_ptr(), prec, st.cuda_stream)
            f()
            torch.cuda.synchronize()
            ms = _timed(f, st, max(1, args.steps // 2))
            o = out.cpu().numpy()[sub]
            na = np.hypot(ds[:, 0], ds[:, 1])
            e = np.hypot(o[:, 0] - ds[:, 0], o[:, 1] - ds[:, 1]) / na
            results.append({"theta": theta, "form": name, "rays_per_s": n / (ms / 1e3), "ms": ms,
                            "alpha_err_vs_direct": {"median": float(np.median(e)), "p999": float(np.percentile(e, 99.9))},
                            "build_ms": tree.build_ms()})
        del tree
    best = [r for r in results if r["theta"] == 0.1 and r["form"] == "split"][0]
    line = _base_line(args, "rays/s/GPU of the split tree at theta=0.1 (one plane)", "rays/s", best["rays_per_s"],
                      best["ms"], "f32+f64", f"precision sweep: {len(parts)} particles, {n1d}^2 rays over 40 arcsec")
    line["sweep"] = results
    print(json.dumps(line))


def smoothing_particles(n, seed=31):
    """A simulated cluster snapshot: a triaxial NFW halo (1e15 Msun, c = 4,
    axes 1 / 0.8 / 0.6) sampled by 90 % of n particles plus 10 % uniform in its
    bounding box (physical Mpc)."""
    from slsimlib_b200 import synth
    r = np.random.default_rng(seed)
    nh = n - n // 10
    p = synth.nfw_particles(r, nh, 1e15, 4.0, 0.3, 0.0, axis_ratios=(0.8, 0.6))
    bg = np.zeros(n - nh, dtype=synth.PARTICLE_DTYPE)
    lo, hi = p["x"].min(axis=0), p["x"].max(axis=0)
    bg["x"] = r.uniform(lo, hi, size=(n - nh, 3)).astype(np.float32)
    bg["Mass"] = p["Mass"][0]
    return np.concatenate([p, bg])


def run_smoothing(args):
    """Adaptive kNN smoothing (LensHaloParticles::calculate_smoothing,
    Nsmooth = 64) of a 4,194,304-particle cluster snapshot: particles/s with the
    records resident in HBM (value), through the host C ABI with the records in
    host memory (e2e), and the reference's threaded calculate_smoothing on a
    524,288-particle snapshot of the same shape on the host cores."""
    import torch
    import slsimlib_b200 as glb
    n = 4_194_304 if not args.small else 524_288
    ns = 64
    p = smoothing_particles(n)
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    dev = torch.from_numpy(p.view(np.uint8).copy()).cuda()
    out = torch.empty(n, dtype=torch.float32, device="cuda")
    split = []
    f = lambda: split.append(glb.calculate_smoothing_device(ns, n, dev.data_ptr(), out.data_ptr(), st.cuda_stream))
    for _ in range(args.warmup):
        f()
    split.clear()
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms = _timed(f, st, args.steps)
    clocks = clk.summary()
    sort_ms = float(np.median([s[0] for s in split]))
    search_ms = float(np.median([s[1] for s in split]))
    # e2e: host records in, Size written back into them
    q = p.copy()
    glb.calculate_smoothing(ns, q)
    t = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        glb.calculate_smoothing(ns, q)
        t.append(time.perf_counter() - t0)
    e2e_s = float(np.median(t))
    assert np.array_equal(q["Size"], out.cpu().numpy())
    line = _base_line(args, "particles/s, adaptive kNN smoothing (Nsmooth = 64)", "particles/s", n / (ms / 1e3), ms,
                      "f32 coords, f64 distances",
                      f"kNN smoothing of {n} particles (triaxial NFW cluster + 10% background), Nsmooth {ns}",
                      clocks=clocks, kernels_ms={"morton_sort_and_boxes": sort_ms, "search": search_ms},
                      # own kernels per call: bbox, Morton keys, gather, bucket boxes, chunk boxes, log2(P) box
                      # levels, search (the radix sort's kernels are the library's)
                      gpu_launches=args.steps * (6 + int(np.ceil(np.log2(max(1, n // 128))))),
                      e2e={"value": n / e2e_s, "unit": "particles/s", "h2d_bytes_per_step": 24 * n,
                           "d2h_bytes_per_step": 4 * n})
    if not args.no_cpu:
        from tests import harness as H
        if H.ref_available():
            nc = 524_288 if not args.small else 65_536
            pc = smoothing_particles(nc, seed=32)
            R = H.RefDriver()
            tf = R._file()
            R.run([f"threads {tf}"])
            _, secs = R.smoothing(pc, ns)
            line["cpu_baseline"] = {"value": nc / secs, "unit": "particles/s", "cores": int(np.fromfile(tf)[0]),
                                    "kind": "reference",
                                    "sample": f"calculate_smoothing of a {nc}-particle snapshot of the same shape"}
    print(json.dumps(line))


def _random_lens_c4(seed):
    from slsimlib_b200 import synth
    r = np.random.default_rng(seed)
    n_p = int(2 ** r.uniform(14, 20))
    m = 10 ** r.uniform(12, 15)
    c = r.uniform(3, 10)
    side = int(round(2 ** r.uniform(6, 10)))
    zs = r.uniform(1, 3)
    three = r.random() < 0.5
    zl = r.uniform(0.2, 0.8)
    zls = [zl - 0.15, zl, zl + 0.15] if three else [zl]
    halos = []
    for z in zls:
        k = n_p // len(zls)
        halos.append(synth.ParticlePlane(synth.nfw_particles(r, k, m / len(zls), c, z, 1e-3), z))
    return synth.LensSpec(zsource=max(zs, zls[-1] + 0.05), halos=halos), side


def run_batched(args):
    """256 independent single- or three-plane NFW particle lenses (N_p in
    2^14-2^20, M in 1e12-1e15, c in 3-10, grid side in 64-1024, z_s in 1-3)
    shot by one persistent launch replayed from a CUDA graph, block size
    picked by the autotuner; split precision."""
    import multiprocessing as mp
    import slsimlib_b200 as glb
    from slsimlib_b200 import synth
    nl = 256 if not args.small else 32
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        specs = pool.map(_random_lens_c4, [4000 + i for i in range(nl)])
    lenses = [make_lens(s) for s, _ in specs]
    sides = [side for _, side in specs]
    rng = 30 * synth.ARCSEC
    b = glb.GridBatch(lenses, sides, [(0.0, 0.0)] * nl, [rng] * nl, glb.PREC_SPLIT)
    block, tune_ms = b.autotune()
    for _ in range(args.warmup):
        b.run(True)
    ms = [b.run(True) for _ in range(args.steps)]
    total = sum(s * s for s in sides)
    rp = sum(s * s * l.getNplanes() for s, l in zip(sides, lenses))
    # the FP64 form of the same batch, for the error of the split form
    b64 = glb.GridBatch(lenses, sides, [(0.0, 0.0)] * nl, [rng] * nl, glb.PREC_FP64)
    ms64 = b64.run(True)
    errs = []
    for i in range(0, nl, max(1, nl // 16)):
        y, A = b.result(i)
        y64, A64 = b64.result(i)
        x = synth.grid_positions(sides[i], range_rad=rng)
        errs.append(error_stats(x, y, A, y64, A64)["alpha"])
    m = float(np.median(ms))
    line = _base_line(args, "rays/s/GPU, batched uneven lenses in one persistent launch", "rays/s", total / (m / 1e3),
                      m, "f32+f64", f"{nl} lens realisations, {total} rays, {rp} ray-planes, CUDA graph",
                      ray_planes_per_s=rp / (m / 1e3), autotune={"block": block, "tile": f"{b.tile()}x{32 // b.tile()}",
                                                                  "ms": tune_ms},
                      plain_fp64={"value": total / (ms64 / 1e3), "unit": "rays/s"},
                      errors_vs_fp64_alpha={"median_of_medians": float(np.median([e["median"] for e in errs])),
                                            "max_p999": float(max(e["p999"] for e in errs))})
    print(json.dumps(line))


def _c5_model(seed):
    from slsimlib_b200 import synth
    return synth.light_cone(seed=seed)


def served_sweep(models, rates, nreq, seed=5, nslots=3):
    """Poisson request streams at the given rates against resident light-cone
    models: request sizes log-uniform in 1e3-5e5 rays in 1-8 Gaussian blobs
    (sigma 0.05-1 arcsec), z_s uniform in 1-3, split precision.  Returns the
    per-rate rays/s and p50/p99 request latency (submit to results), the
    server's statistics and the deflection error of a few served requests
    against the plain FP64 form."""
    import slsimlib_b200 as glb
    from slsimlib_b200 import synth
    nm = len(models)
    srv = glb.Server(models, max_rays_per_batch=2_000_000, precision=glb.PREC_SPLIT, nslots=nslots)
    r = np.random.default_rng(seed)
    half = 30 * synth.ARCSEC

    def request():
        n = int(10 ** r.uniform(3, np.log10(5e5)))
        nb = int(r.integers(1, 9))
        cen = r.uniform(-half, half, size=(nb, 2))
        sig = 10 ** r.uniform(np.log10(0.05), 0) * synth.ARCSEC
        which = r.integers(0, nb, size=n)
        x = cen[which] + r.normal(0, sig, size=(n, 2))
        return int(r.integers(0, nm)), x, float(r.uniform(1, 3))

    sweep = []
    for lam in rates:
        reqs = [request() for _ in range(nreq)]
        gaps = r.exponential(1 / lam, size=nreq)
        tickets = []
        t0 = time.perf_counter()
        tnext = t0
        for (m, x, zs), g in zip(reqs, gaps):
            tnext += g
            d = tnext - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets.append(srv.submit(m, x, zs))
        lat, rays = [], 0
        for (m, x, zs), t in zip(reqs, tickets):
            y, A, tm = srv.wait(t, timeout=600)
            lat.append((tm[2] - tm[0]) * 1e3)
            rays += len(x)
        wall = time.perf_counter() - t0
        sweep.append({"rate_req_per_s": lam, "requests": nreq, "rays": rays, "rays_per_s": rays / wall,
                      "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))})
    st = srv.stats()
    errs = []
    for _ in range(3):
        m, x, zs = request()
        y, A, _ = srv.wait(srv.submit(m, x, zs), timeout=600)
        y64, A64 = models[m].rayshooterInternal(x, np.full(len(x), zs), precision=glb.PREC_FP64)
        errs.append(error_stats(x, y, A, y64, A64)["alpha"])
    srv.close()
    return sweep, st, {"median": float(np.median([e["median"] for e in errs])),
                       "max_p999": float(max(e["p999"] for e in errs))}


def run_served(args):
    """32 resident light-cone models; Poisson request stream at swept rates;
    request sizes log-uniform in 1e3-5e5 rays in 1-8 Gaussian blobs
    (sigma 0.05-1 arcsec); z_s uniform in 1-3; split precision."""
    import multiprocessing as mp
    nm = 32 if not args.small else 4
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        specs = pool.map(_c5_model, [5000 + i for i in range(nm)])
    models = [make_lens(s) for s in specs]
    sweep, st, err = served_sweep(models, (5.0, 20.0, 60.0), 120 if not args.small else 30)
    top = max(sweep, key=lambda s: s["rays_per_s"])
    line = _base_line(args, "rays/s/GPU served; p50/p99 request ms", "rays/s", top["rays_per_s"],
                      None, "f32+f64", f"{nm} resident light-cone models, Poisson request stream",
                      sweep=sweep, server=st, errors_vs_fp64_alpha=err)
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="a reduced workload for quick checks")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-served", action="store_true", help="skip the served-stream leg of the default line")
    ap.add_argument("--n1d", type=int, default=0,
                    help="rays per side of the light-cone grid (default 2048; a profiling size, not a bench line)")
    ap.add_argument("--workload", default="lightcone",
                    choices=["lightcone", "single", "sweep", "batched", "served", "field", "smoothing"],
                    help="lightcone (default): the 10-plane light cone; the others are the single plane, the "
                         "precision sweep, batched uneven lenses, the served request stream and the light cone "
                         "with field planes, and adaptive kNN smoothing of a particle snapshot")
    args = ap.parse_args()
    if args.impl == "ours" and args.workload != "lightcone":
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        return {"single": run_single, "sweep": run_sweep, "batched": run_batched, "served": run_served,
                "field": run_field, "smoothing": run_smoothing}[
            args.workload](args)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank)

    import torch
    import torch.distributed as dist
    import slsimlib_b200 as glb
    from slsimlib_b200 import synth
    from slsimlib_b200.replicas import max_over_ranks

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    spec, n1d = workload(args.small)
    if args.n1d:
        n1d = args.n1d
    n = n1d * n1d
    lens = make_lens(spec)
    x_host = synth.grid_positions(n1d, range_rad=FIELD_ARCSEC * synth.ARCSEC)
    dev = torch.device("cuda", local)
    x = torch.from_numpy(x_host).to(dev)
    y = torch.empty((n, 2), dtype=torch.float64, device=dev)
    A = torch.empty((n, 4), dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream(device=dev)  # a real stream handle (the library maps NULL to its own)
    torch.cuda.set_stream(stream)

    def shoot(prec):
        lens.rayshoot_device(n, x.data_ptr(), None, y.data_ptr(), A.data_ptr(), prec, stream.cuda_stream)

    served = None
    if rank == 0 and not args.no_served:
        # the served form on a few resident models: this light cone and three
        # more of the same kind (seeds 5000-5002), two Poisson rates; measured
        # first, with its own clock record
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(3) as pool:
            extra = pool.map(_c5_model, [5000, 5001, 5002] if not args.small else [5000])
        models = [lens] + [make_lens(sp) for sp in extra]
        # three repetitions of the same seeded streams, reported per rate as the
        # median of each figure (the overloaded rate varies between runs)
        reps = []
        with ClockSampler(local) as sclk:
            for _ in range(3 if not args.small else 1):
                reps.append(served_sweep(models, (20.0, 60.0), 120 if not args.small else 20))
        sw = []
        for i, first in enumerate(reps[0][0]):
            row = dict(first)
            for key in ("rays_per_s", "p50_ms", "p99_ms"):
                row[key] = float(np.median([r[0][i][key] for r in reps]))
            row["repetitions"] = [{key: r[0][i][key] for key in ("rays_per_s", "p50_ms", "p99_ms")} for r in reps]
            sw.append(row)
        sst, serr = reps[-1][1], reps[-1][2]
        served = {"models": len(models), "sweep": sw, "server": sst, "errors_vs_fp64_alpha": serr,
                  "request_rays": "log-uniform 1e3-5e5 in 1-8 Gaussian blobs (0.05-1 arcsec), z_s uniform 1-3",
                  "latency": "submit to results on the host (ms)", "clocks": sclk.summary(),
                  "statistic": "median of 3 repetitions per rate"}
        del models, extra

    # FP64 form (the error reference) and its timing
    shoot(glb.PREC_FP64)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    shoot(glb.PREC_FP64)
    e1.record(stream)
    torch.cuda.synchronize()
    fp64_ms = e0.elapsed_time(e1)
    y64, A64 = y.cpu().numpy().copy(), A.cpu().numpy().copy()

    # interaction counts (identical for both forms: same opening decisions)
    counts = lens.count_interactions(x_host) if rank == 0 else None

    for _ in range(args.warmup):
        shoot(glb.PREC_SPLIT)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    kernel_ms = []
    with ClockSampler(local) as clk:
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.steps):
            shoot(glb.PREC_SPLIT)
        t1.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(t0.elapsed_time(t1), device=dev)
    if world > 1:
        dist.barrier()
    # per-launch plane-step time from the library's events (last step)
    shoot(glb.PREC_SPLIT)
    torch.cuda.synchronize()
    k_ms, tot_ms = lens.last_timing()
    y32, A32 = y.cpu().numpy(), A.cpu().numpy()
    errs = error_stats(x_host, y32, A32, y64, A64)
    attrib = attribution(spec, lens, x_host) if rank == 0 and not args.small else None

    # end to end through the host C ABI (pinned host buffers, copies timed)
    xp = torch.from_numpy(x_host).pin_memory()
    yp = torch.empty((n, 2), dtype=torch.float64).pin_memory()
    Ap = torch.empty((n, 4), dtype=torch.float64).pin_memory()
    L = glb.load_library()

    def shoot_host():
        glb._check(L.glb_lens_rayshoot(lens._h, n, xp.data_ptr(), None, yp.data_ptr(), Ap.data_ptr(),
                                       glb.PREC_SPLIT))
    shoot_host()
    if world > 1:
        dist.barrier()
    h0 = time.perf_counter()
    for _ in range(args.steps):
        shoot_host()
    e2e_s = max_over_ranks(time.perf_counter() - h0, device=dev)

    if rank == 0:
        clocks = clk.summary()
        value = world * n * args.steps / (ms / 1e3)
        nplanes = lens.getNplanes()
        V, F, P, B, S, Wn, Wp = [int(c) for c in counts]
        alg_flops = (FLOPS["V"] * V + FLOPS["F"] * F + FLOPS["P"] * P + FLOPS["B"] * B + FLOPS["S"] * S
                     + FLOPS["rec"] * n * nplanes)
        sm = clocks.get("sm_mhz") or 1965.0
        peak = fp32_peak_tflops(sm)
        achieved = alg_flops / (k_ms / 1e3) / 1e12
        cpu = None if args.no_cpu else cpu_reference(spec, n1d, 4096 if args.small else 65536)
        line = {
            "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded light cone)",
            "config": {"workload": f"light cone: 10 particle planes (4,194,304 particles) + NSIE at z=0.5, "
                                   f"{n1d}^2 rays over 60 arcsec, z_s=2.5" + (" [reduced]" if args.small else ""),
                       "rays_per_step": n, "planes": nplanes, "particles": spec.n_particles(),
                       "precision": "FP32 walk (block-compensated) + FP64 offsets/recursion",
                       "l2": "inputs larger than L2 (x 2n + 12n recursion state doubles)",
                       "parallelism": f"replicated lens, one full grid per GPU"},
            "plain_fp64": {"value": n / (fp64_ms / 1e3), "unit": "rays/s", "ms": fp64_ms},
            "errors_vs_fp64": errs,
            "kappa_gamma_attribution": attrib,
            "served": served,
            "e2e": {"value": world * n * args.steps / e2e_s, "unit": "rays/s", "h2d_bytes_per_step": 16 * n,
                    "d2h_bytes_per_step": 48 * n},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": DRAM_BYTES_PER_RAY_PLANE * n,
                         "traffic_note": "dram read+write bytes per plane (both slabs): ncu capture of one "
                                         "1,179,648-ray slab launch at 1536^2 (156 B/ray) scaled by rays",
                         "kernel": "k_plane_step_split_g", "kernel_ms_per_step": k_ms,
                         "peak_note": "FP32 CUDA-core FMA rate at the sampled SM clock (148 SMs x 128 lanes x 2)",
                         "alg_flops_per_step": alg_flops,
                         "counts": {"V": V, "F": F, "P": P, "B": B, "S": S},
                         "lane_efficiency": {"nodes": V / max(Wn, 1), "leaf_particles": P / max(Wp, 1)}},
            # per step: ray bbox, Morton keys, the 6 kernels of the CUB radix sort compiled into the
            # library, and per slab of rays (two from 2^21 rays on) state init, one plane step per
            # plane, finish (ncu launch list)
            "gpu_launches": args.steps * (8 + (2 if n >= (1 << 21) else 1) * (2 + nplanes)),
            "clocks": clocks,
        }
        if cpu:
            line["cpu_baseline"] = {"value": cpu[0], "unit": "rays/s", "cores": cpu[1], "kind": "reference",
                                    "sample": cpu[3], "seconds": cpu[2]}
            # the plain FP64 GPU form against the reference's own results on the sampled rays
            line["parity_vs_reference"] = parity_vs_reference(y64[cpu[4]], A64[cpu[4]], cpu[5], cpu[6])
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
