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
  roofline of the plane-step kernel (algorithmic FP32 flops from the counted
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


def workload(small: bool):
    from slsimlib_b200 import synth
    if small:
        return synth.light_cone(seed=2, n_total=262_144), 512
    return synth.light_cone(seed=2), N1D


def make_lens(spec):
    import slsimlib_b200 as glb
    from slsimlib_b200 import synth
    lens = glb.Lens(spec.zsource)
    for h in spec.halos:
        if isinstance(h, synth.ParticlePlane):
            lens.insertMainHalo(glb.LensHaloParticles(h.particles, h.z, h.inv_area, h.max_range), True)
        elif isinstance(h, synth.NSIEHalo):
            lens.insertMainHalo(glb.LensHaloRealNSIE(h.mass, h.z, h.sigma, h.rcore, h.fratio, h.pa), True)
        else:
            lens.insertMainHalo(glb.LensHaloNFW(h.mass, h.rsize, h.z, h.conc), True)
    return lens


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
    for name, e in (("alpha", ea), ("kappa", np.abs(k - kr) / np.abs(kr)), ("gamma", np.abs(g - gr) / np.abs(gr)),
                    ("invmag", np.abs(inv - invr)[m] / np.abs(invr[m]))):
        out[name] = {"median": float(np.median(e)), "p999": float(np.percentile(e, 99.9))}
    return out


def cpu_reference(spec, n1d, nsample, seed=77):
    """Times the reference (oracle/_ref) Lens::rayshooterInternal on a seeded
    sample of the grid's rays; returns (rays/s, threads, seconds, sample)."""
    from tests import harness as H
    from slsimlib_b200 import synth
    if not H.ref_available():
        return None
    x = synth.grid_positions(n1d, range_rad=FIELD_ARCSEC * synth.ARCSEC)
    idx = np.sort(np.random.default_rng(seed).choice(len(x), size=nsample, replace=False))
    R = H.RefDriver()
    tf = R._file()
    R.run([f"threads {tf}"])
    threads = int(np.fromfile(tf)[0])
    _, _, secs = R.rays(spec, x[idx])
    return nsample / secs, threads, secs, f"{nsample} seeded rays of the {n1d}x{n1d} grid, all planes"


def run_reference_arm(args, rank):
    if rank != 0:
        return
    from tests import harness as H
    if not H.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/glamer_ref not built"}))
        return
    spec, n1d = workload(args.small)
    vals = []
    nsample = 2048 if args.small else 4096
    threads = 0
    for s in range(args.warmup + args.steps):
        r = cpu_reference(spec, n1d, nsample, seed=100 + s)
        if s >= args.warmup:
            vals.append(r[0])
        threads = r[1]
    v = float(np.median(vals))
    n = n1d * n1d
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "rays/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": n / v * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded light cone)",
            "config": {"workload": f"light cone: 10 planes, 4,194,304 particles + NSIE, {n1d}^2 rays over 60 arcsec",
                       "sample_rays_per_step": nsample},
            "cpu_baseline": {"value": v, "unit": "rays/s", "cores": threads, "kind": "reference",
                             "sample": f"{nsample} seeded rays per step, all 11 planes, rate extrapolated per ray"},
            "e2e": {"value": v, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="a reduced workload for quick checks")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank)

    import torch
    import torch.distributed as dist
    import slsimlib_b200 as glb
    from slsimlib_b200 import synth

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    spec, n1d = workload(args.small)
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
    ms = t0.elapsed_time(t1)
    if world > 1:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
        dist.barrier()
    # per-launch plane-step time from the library's events (last step)
    shoot(glb.PREC_SPLIT)
    torch.cuda.synchronize()
    k_ms, tot_ms = lens.last_timing()
    y32, A32 = y.cpu().numpy(), A.cpu().numpy()
    errs = error_stats(x_host, y32, A32, y64, A64)

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
    e2e_s = time.perf_counter() - h0
    if world > 1:
        tt = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())

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
            "e2e": {"value": world * n * args.steps / e2e_s, "unit": "rays/s", "h2d_bytes_per_step": 16 * n,
                    "d2h_bytes_per_step": 48 * n},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "k_plane_step<split>", "kernel_ms_per_step": k_ms,
                         "peak_note": "FP32 CUDA-core FMA rate at the sampled SM clock (148 SMs x 128 lanes x 2)",
                         "alg_flops_per_step": alg_flops,
                         "counts": {"V": V, "F": F, "P": P, "B": B, "S": S},
                         "lane_efficiency": {"nodes": V / max(Wn, 1), "leaf_particles": P / max(Wp, 1)}},
            "gpu_launches": args.steps * (4 + nplanes),
            "clocks": clocks,
        }
        if cpu:
            line["cpu_baseline"] = {"value": cpu[0], "unit": "rays/s", "cores": cpu[1], "kind": "reference",
                                    "sample": cpu[3], "seconds": cpu[2]}
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
