#!/usr/bin/env python
"""Benchmark of the distance-driven fan-beam projector pair on B200.

Workload (the batched 2D fan-beam workload): 64 independent 512x512 slices at
0.7 mm, 888-channel arc detector (1.2858 mm pitch at 1085.6 mm), source at
595 mm, each slice with a seeded uneven view count in [576, 1152] over 360
degrees; random-ellipse phantoms.  One step = DD forward projection of every
view of every slice followed by the matched (exact-transpose) backprojection
of that sinogram -- the projector work of one OS-SQS pass.

Metric: Gray/s = 1e9 footprint updates per second, where an update is one
ray-line integration of the forward projector (nominal count
views x channels x lines, the reference's loop count) or one pixel-view
integration of the backprojector (views x pixels).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 is launched with torch.distributed.run (one process per GPU); every
rank processes its own batch (weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DD proj+BP Gray/s & % HBM roofline; OS-SQS time-to-RMSE learned vs TV, 1 B200"
UNIT = "Gray/s"
BYTES_PER_UPDATE = 8          # two FP32 prefix samples per footprint
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--slices", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ossqs", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the Siddon, tomosynthesis, cone and filter measurements")
    ap.add_argument("--ossqs-iters", type=int, default=30)
    ap.add_argument("--extra", choices=["siddon", "tomo", "cone", "filter", "ossqs", "cyl", "cfg0", "prior", "conv"],
                    help="run only this extra measurement (one GPU) and print its JSON object")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def workload(rank, nslices):
    from reconnet_b200 import phantom as P
    geom = P.geom_fan512()
    counts = P.batch_view_counts(nslices, seed=1 + rank)
    angles = np.concatenate([P.uniform_angles(int(n)) for n in counts])
    rng = np.random.default_rng(100 + rank)
    imgs = np.stack([P.ellipse_phantom(geom.nx, geom.ny, geom.dx, geom.dy, rng) for _ in range(nslices)])
    return geom, counts, angles, imgs


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def ncu_counts(kernel):
    """Per-launch ncu counters of `kernel` at the bench size from the committed
    summary (profiles/ncu_counts_bench.txt: `<kernel> <dram_bytes> <warp_inst>`);
    None where the file or the kernel's line is missing."""
    p = os.path.join(ROOT, "profiles", "ncu_counts_bench.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        parts = line.split()
        if len(parts) >= 3 and parts[0] == kernel and not line.startswith("#"):
            try:
                return {"dram_bytes": float(parts[1]), "warp_inst": float(parts[2])}
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def bench_config(nslices, counts, world):
    """The workload description both arms print (the same config on each)."""
    nview = int(np.sum(counts))
    return {"workload": "batched 2D fan-beam DD forward projection + matched backprojection: "
                        f"{nslices} slices 512x512 @0.7 mm, 888 ch @1.2858 mm, "
                        "views U[576,1152] per slice over 360 deg",
            "slices_per_gpu": nslices, "total_views_per_gpu": nview,
            "fp_updates_per_step": nview * 888 * 512, "bp_updates_per_step": nview * 512 * 512,
            "l2": "inputs larger than L2 (64 MB image batch, "
                  f"{nview * 888 * 4 / 1e6:.0f} MB sinogram, ~1.2 GB scratch per step)",
            "parallelism": f"dp{world} (independent slice batches)"}


def cpu_baseline_sample(geom, counts, angles, imgs, target_s=12.0):
    """FP32 OpenMP port of the oracle on whole slices of the workload (all of
    each slice's views, FP + matched BP), slice after slice until about
    `target_s` seconds; returns (Gray/s, threads, description)."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    offs = np.concatenate([[0], np.cumsum(counts)])
    upd, dt, done = 0, 0.0, 0
    for s in range(len(counts)):
        sel = np.ascontiguousarray(angles[offs[s]:offs[s + 1]])
        img = imgs[s][None, :, :, None, None]
        t0 = time.perf_counter()
        p = O.fan_fp(img, sel, geom, geom.nu, 1, dtype=np.float32)
        O.fan_bp(p, sel, geom, (geom.nx, geom.ny, 1), 2, dtype=np.float32)
        dt += time.perf_counter() - t0
        upd += sel.size * (geom.nu * geom.ny + geom.nx * geom.ny)
        done += 1
        if dt >= target_s:
            break
    desc = (f"{done} of the {len(counts)} slices (all their views), FP + matched BP, FP32 OpenMP port of the "
            f"oracle, {threads} threads, {dt:.1f} s")
    return upd / dt / 1e9, threads, desc


def run_reference(args):
    """Reference arm: the CPU port of the reference DD loop on the host cores
    (rank 0 only), plus the reference's own CUDA library (built from its
    sources into oracle/_ref) on the same GPU for context.  Nothing here loads
    this repository's sm_100a library: the workload comes from
    reconnet_b200.phantom / .geometry, which import no native code."""
    rank, local, world = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O
    geom, counts, angles, imgs = workload(0, args.slices)
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    n0 = int(counts[0])
    # per step: one slice, a view subset sized for ~4 s (pilot-calibrated)
    img = imgs[0][None, :, :, None, None]

    def step(nv):
        sel = angles[:n0][:: max(1, n0 // nv)][:nv].copy()
        p = O.fan_fp(img, sel, geom, geom.nu, 1, dtype=np.float32)
        O.fan_bp(p, sel, geom, (geom.nx, geom.ny, 1), 0, dtype=np.float32)
        return sel.size * (geom.nu * geom.ny + geom.nx * geom.ny)

    t0 = time.perf_counter()
    step(4)
    per_view = (time.perf_counter() - t0) / 4
    nv = int(max(4, min(n0, 4.0 / max(per_view, 1e-6))))
    for _ in range(args.warmup):
        step(nv)
    upd, t0 = 0, time.perf_counter()
    for _ in range(args.steps):
        upd += step(nv)
    dt = time.perf_counter() - t0
    value = upd / dt / 1e9
    sample = (f"per step: 1 slice 512x512, 888 ch, {nv} of its {n0} views: the reference's DD forward projection "
              f"(DDFPFanKernelX/Y) and its iterative backprojection (DDBPFanKernelX/Y, typeProjector 0), as the "
              f"oracle's FP32 OpenMP port (the reference has no CPU DD path), {threads} threads")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded random-ellipse phantoms",
            "config": bench_config(args.slices, counts, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    import torch
    if torch.cuda.is_available():
        line["reference_gpu"] = reference_gpu(geom, counts, angles, imgs, min(3, args.steps))
        if not args.no_extras:
            line["reference_gpu_extras"] = reference_gpu_extras(geom, counts, angles, imgs)
    print(json.dumps(line), flush=True)


def tomo_geometry(nview=25):
    """The tomosynthesis workload of `tomo_run` / `cone_run`: 25 sources on a
    +-20 deg arc at 650 mm, the detector centre 80 mm below the isocentre,
    detector axes along x and y."""
    import math
    src = np.zeros((nview, 3), np.float32)
    dc = np.zeros((nview, 3), np.float32)
    for k in range(nview):
        a = (k - (nview - 1) / 2) / ((nview - 1) / 2) * math.radians(20)
        src[k] = (650 * math.sin(a), 0.0, 650 * math.cos(a))
        dc[k] = (0.0, 0.0, -80.0)
    du = np.tile(np.float32([1, 0, 0]), (nview, 1))
    dv = np.tile(np.float32([0, 1, 0]), (nview, 1))
    return dc, du, dv, src


def reference_gpu_extras(geom, counts, angles, imgs):
    """The reference library's other paths on the workloads of the extras in
    this arm's counterpart, through its C entry points with host arrays (so
    including its per-call allocations and copies; the kernel-only times come
    from an ncu launch list of this command): the Siddon fan pair and the
    pixel-driven backprojection on two slices of the fan batch, the
    tomosynthesis DD pair and the Siddon cone pair on the tomosynthesis
    workload."""
    path = os.path.join(ROOT, "oracle", "_ref", "libreconnet_ref.so")
    if not os.path.exists(path):
        return {"unavailable": "reference library not built (make -C oracle ref)"}
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden
    lib = make_golden.load_ref(path)
    p = make_golden.p
    out = {}
    offs = np.concatenate([[0], np.cumsum(counts)])

    def timed(fn):
        fn()
        t0 = time.perf_counter()
        fn()
        return (time.perf_counter() - t0) * 1e3

    # fan batch, 2 slices
    fan_upd = {"fp": 0, "bp": 0}
    calls = []
    for s in range(2):
        n = int(counts[s])
        img = np.ascontiguousarray(imgs[s][None, :, :, None, None])
        ang = np.ascontiguousarray(angles[offs[s]:offs[s + 1]])
        sino = np.zeros((1, geom.nu, n, 1, 1), np.float32)
        bp = np.zeros_like(img)
        a = (1, 1, geom.nx, geom.ny, 1, geom.dx, geom.dy, geom.dz, geom.nu, n, 1, geom.da, geom.dv, 0.0, 0.0,
             geom.dsd, geom.dso, 0)
        calls.append((img, ang, sino, bp, a))
        fan_upd["fp"] += n * geom.nu * geom.ny
        fan_upd["bp"] += n * geom.nx * geom.ny
    for name, sym, fn in (
            ("siddon_fp", "cSiddonFanProjection", lambda c: lib.cSiddonFanProjection(p(c[2]), p(c[0]), p(c[1]), *c[4])),
            ("siddon_bp", "cSiddonFanBackprojection",
             lambda c: lib.cSiddonFanBackprojection(p(c[3]), p(c[2]), p(c[1]), *c[4])),
            ("pixel_bp", "cPixelDrivenFanBackprojection",
             lambda c: lib.cPixelDrivenFanBackprojection(p(c[3]), p(c[2]), p(c[1]), *c[4]))):
        if not hasattr(lib, sym):
            continue
        ms = timed(lambda: [fn(c) for c in calls])
        upd = fan_upd["fp"] if name.endswith("fp") else fan_upd["bp"]
        out[name] = {"ms": ms, "gupd_s_host_call": upd / ms / 1e6, "workload": "2 slices of the fan batch"}
    # tomosynthesis workload
    nx, ny, nz, nu, nv, nview = 512, 512, 128, 736, 736, 25
    dc, du, dv, src = tomo_geometry(nview)
    vol = np.random.default_rng(11).random((1, nx, ny, nz, 1)).astype(np.float32)
    prj = np.zeros((1, nu, nview, nv, 1), np.float32)
    back = np.zeros_like(vol)
    targs = (1, 1, nx, ny, nz, 0.8, 0.8, 1.0, 0.0, 0.0, 0.0, nu, nview, nv, 0.6, 0.6, 0.0, 0.0)
    pairs = [("tomo_fp", lambda: lib.cDistanceDrivenTomoProjection(p(prj), p(vol), p(dc), p(src), *targs),
              nview * nu * nv * nz),
             ("tomo_bp", lambda: lib.cDistanceDrivenTomoBackprojection(p(back), p(prj), p(dc), p(src), *targs),
              nx * ny * nz * nview)]
    if hasattr(lib, "cSiddonConeProjectionAbitrary"):
        pairs += [("cone_fp", lambda: lib.cSiddonConeProjectionAbitrary(p(prj), p(vol), p(dc), p(du), p(dv), p(src),
                                                                         *targs), nview * nu * nv * nz),
                  ("cone_bp", lambda: lib.cSiddonConeBackprojectionAbitrary(p(back), p(prj), p(dc), p(du), p(dv),
                                                                             p(src), *targs), nx * ny * nz * nview)]
    for name, fn, upd in pairs:
        ms = timed(fn)
        out[name] = {"ms": ms, "gupd_s_host_call": upd / ms / 1e6, "workload": "the tomosynthesis workload"}
    # the ramp filter on the filter extra's workload (64 sinograms of 888 x 1152,
    # Ram-Lak): cFilterFanFilter plans cuFFT and stages host arrays per call
    fB, fview = 64, 1152
    fs = np.random.default_rng(12).random((fB, geom.nu, fview, 1, 1), dtype=np.float32)
    fo = np.zeros_like(fs)
    fargs = (fB, 1, geom.nu, fview, 1, geom.da, geom.dv, 0.0, 0.0, geom.dsd, geom.dso, 0, 0)
    ms = timed(lambda: lib.cFilterFanFilter(p(fo), p(fs), *fargs))
    out["filter"] = {"ms": ms, "views_per_s_host_call": fB * fview / (ms * 1e-3),
                     "workload": "64 fan sinograms of 888 channels x 1152 views, Ram-Lak (host arrays, cuFFT)"}
    out["note"] = ("reference CUDA library (oracle/_ref) through its C entry points with host arrays: wall time "
                   "of the second of two calls, including its allocations and copies")
    return out


def reference_gpu(geom, counts, angles, imgs, steps):
    """The reference CUDA library on the full workload, called as its Python
    wrapper does (python/ReconNet_no_tf.py:133-200): per slice, FP then BP
    through cDistanceDrivenFan{Projection,Backprojection} with host arrays."""
    path = os.path.join(ROOT, "oracle", "_ref", "libreconnet_ref.so")
    if not os.path.exists(path):
        return {"unavailable": "reference library not built (make -C oracle ref)"}
    import ctypes
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden
    lib = make_golden.load_ref(path)
    p = make_golden.p
    offs = np.concatenate([[0], np.cumsum(counts)])
    sinos = [np.zeros((1, geom.nu, int(n), 1, 1), np.float32) for n in counts]
    bps = [np.zeros((1, geom.nx, geom.ny, 1, 1), np.float32) for _ in counts]
    imgs5 = [np.ascontiguousarray(im[None, :, :, None, None]) for im in imgs]
    angs = [np.ascontiguousarray(angles[offs[s]:offs[s + 1]]) for s in range(len(counts))]

    def one_step():
        for s, n in enumerate(counts):
            a = (1, 1, geom.nx, geom.ny, 1, geom.dx, geom.dy, geom.dz, geom.nu, int(n), 1, geom.da, geom.dv,
                 0.0, 0.0, geom.dsd, geom.dso, 0)
            lib.cDistanceDrivenFanProjection(p(sinos[s]), p(imgs5[s]), p(angs[s]), *a)
            lib.cDistanceDrivenFanBackprojection(p(bps[s]), p(sinos[s]), p(angs[s]), *a)

    one_step()
    t0 = time.perf_counter()
    for _ in range(steps):
        one_step()
    dt = (time.perf_counter() - t0) / steps
    upd = int(np.sum(counts)) * (geom.nu * geom.ny + geom.nx * geom.ny)
    return {"value": upd / dt / 1e9, "unit": UNIT, "ms_per_step": dt * 1e3, "steps": steps,
            "note": "reference CUDA kernels (ReconNet4D_no_tf sources built for sm_100a into oracle/_ref), "
                    "per-slice host calls FP + iterative BP incl. its per-call allocation and copies, same B200"}


def ossqs_run(plan, geom, counts, angles, truth, n_iter, dev, n_subsets=24, I0=5e4):
    """TV-regularised OS-SQS on the same batch: Poisson data at I0 (weights =
    counts), 24 interleaved subsets, one iteration captured in a CUDA graph
    and replayed n_iter times; returns time per iteration and RMSE in HU."""
    import torch

    from reconnet_b200.ossqs import BatchedOSSQS, tv_terms
    from reconnet_b200.phantom import HU
    gen = torch.Generator(device=dev).manual_seed(7)
    with torch.no_grad():
        line_int = plan.project(truth)
        counts_t = torch.poisson(I0 * torch.exp(-line_int.double()), generator=gen).clamp_min(1.0)
        b = (-torch.log(counts_t / I0)).float()
        w = counts_t.float()
    t_setup = time.perf_counter()
    solver = BatchedOSSQS(geom, counts, angles, b, w, n_subsets=n_subsets, beta=0.0, lb=0.0, ub=None,
                          device=dev)
    # TV weight: 5% of the data curvature against the TV curvature of a flat image
    _, n_flat = tv_terms(torch.zeros((1, 8, 8), device=dev))
    solver.beta = float(0.05 * solver.norm_img.median() / n_flat[0, 4, 4])
    x0 = torch.zeros_like(truth)
    solver.run(x0, 1)   # capture + warm-up
    setup_s = time.perf_counter() - t_setup
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(st)
    x = solver.run(x0, n_iter)
    e1.record(st)
    torch.cuda.synchronize(dev)
    solver.check()
    ms = e0.elapsed_time(e1)
    rmse = lambda a: float(torch.sqrt(((a - truth) ** 2).mean())) / HU
    starved = float((counts_t <= 1.0).double().mean())
    # the same solver on noise-free, unweighted data (b = line integrals, W = 1):
    # separates the solver's convergence from the photon starvation of rays
    # through the densest ellipse overlaps
    with torch.no_grad():
        solver_nf = BatchedOSSQS(geom, counts, angles, line_int, torch.ones_like(line_int),
                                 n_subsets=n_subsets, beta=0.0, lb=0.0, ub=None, device=dev)
        x_nf = solver_nf.run(x0, n_iter)
        solver_nf.check()
    return {"iterations": n_iter, "subsets": n_subsets, "I0": I0, "beta": solver.beta,
            "ms_per_iteration": ms / n_iter, "ms_total": ms, "setup_s": setup_s,
            "tuning": dict(zip(("fp_views", "fp_lines", "bp_parts"), solver.tuning)),
            "rmse_hu_initial": rmse(x0), "rmse_hu_final": rmse(x),
            "starved_ray_fraction": starved, "rmse_hu_final_noise_free_unweighted": rmse(x_nf),
            "note": "graph replay of one full iteration (24 subset updates: FP, residual, matched BP, "
                    "TV + SQS step); includes the start-up copy of x0.  Rays with at most one photon "
                    "(starved_ray_fraction) carry a clipped, biased line integral, which bounds the noisy RMSE"}


def cfg0_run(dev, cpu_sample=True, n_iter=20, n_subsets=12, I0=1e5):
    """The 2D fan workload end to end: a 256x256 random-ellipse phantom (1.0 mm
    pixels), 736 channels at 1.2858 mm, 720 views over 360 degrees; its DD
    projection, Poisson counts at I0 = 1e5, the ramp-filtered FBP (Ram-Lak,
    pixel-driven backprojection) and 20 iterations of TV OS-SQS with 12
    subsets started from the FBP image.  The same pipeline runs on the host
    cores as the FP32 OpenMP port of the oracle (the reference has no CPU DD
    path; this is the "host C++ build" of the workload)."""
    import torch

    from reconnet_b200 import phantom as P
    from reconnet_b200.ossqs import BatchedOSSQS, interleaved_subsets, tv_terms
    from reconnet_b200.torch_ops import FanPlan, fbp
    geom = P.geom_fan256()
    nview = 720
    ang = P.uniform_angles(nview)
    truth = P.ellipse_phantom(geom.nx, geom.ny, geom.dx, geom.dy, np.random.default_rng(2)).astype(np.float32)
    t = torch.from_numpy(truth[None, :, :, None, None]).to(dev)
    plan = FanPlan(geom, ang, device=dev)
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    times = {}

    def timed(name, fn):
        fn()
        torch.cuda.synchronize(dev)
        e0, e1 = ev()
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize(dev)
        times[name] = e0.elapsed_time(e1)
        return r

    line = timed("fp_ms", lambda: plan.project(t))
    rng = np.random.default_rng(3)
    b_np, cnt_np = P.poisson_sinogram(line.cpu().numpy(), I0, rng)
    b, w = torch.from_numpy(b_np).to(dev), torch.from_numpy(cnt_np).to(dev)
    timed("bp_ms", lambda: plan.backproject(b, 2))
    x_fbp = timed("fbp_ms", lambda: fbp(b, plan, geom, 0))
    solver = BatchedOSSQS(geom, [nview], ang, b.reshape(-1), w.reshape(-1), n_subsets=n_subsets, lb=0.0, device=dev)
    _, n_flat = tv_terms(torch.zeros((1, 8, 8), device=dev))
    solver.beta = float(0.05 * solver.norm_img.median() / n_flat[0, 4, 4])
    x0 = x_fbp[:, :, :, 0, 0].clamp_min(0).contiguous()
    x = timed("ossqs_ms", lambda: solver.run(x0, n_iter))
    solver.check()
    rmse = lambda a: float(np.sqrt(np.mean((np.asarray(a, np.float64) - truth) ** 2)) / P.HU)
    out = {"workload": "256x256 @1.0 mm, 736 ch @1.2858 mm, 720 views over 360 deg: DD FP, matched BP, Ram-Lak FBP, "
                       f"{n_iter} TV OS-SQS iterations ({n_subsets} subsets) from the FBP image, I0 = {I0:g}",
           "gpu_ms": times, "gpu_pipeline_ms": times["fp_ms"] + times["fbp_ms"] + times["ossqs_ms"],
           "rmse_hu_fbp": rmse(x_fbp[0, :, :, 0, 0].cpu().numpy()), "rmse_hu_ossqs": rmse(x[0].cpu().numpy()),
           "beta": solver.beta}
    if cpu_sample:
        from oracle import oracle as O
        O.set_threads(os.cpu_count() or 1)
        c = {}
        t0 = time.perf_counter()
        O.fan_fp(truth[None, :, :, None, None], ang, geom, geom.nu, 1, dtype=np.float32)
        c["fp_s"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        filt = O.filter_sino(b_np, geom, 0).astype(np.float32)
        xf = O.pixel_bp(filt, ang, geom, (geom.nx, geom.ny, 1), dtype=np.float32)[0, :, :, 0, 0]
        c["fbp_s"] = time.perf_counter() - t0
        sino, wsn = b_np[0, :, :, 0, 0], cnt_np[0, :, :, 0, 0]
        ones = np.ones((1, geom.nx, geom.ny, 1, 1), np.float32)
        a1 = (O.fan_fp(ones, ang, geom, geom.nu, 1, dtype=np.float32)[0, :, :, 0, 0] * wsn).astype(np.float32)
        norm = O.fan_bp(a1[None, :, :, None, None], ang, geom, (geom.nx, geom.ny, 1), 2,
                        dtype=np.float32)[0, :, :, 0, 0]
        xc = np.maximum(xf, 0).astype(np.float32)
        t0 = time.perf_counter()
        iters = 0
        while iters < n_iter:
            for views in interleaved_subsets(nview, n_subsets):
                xc = O.sqs_subset_update(xc, sino, wsn, norm, ang, views, geom, n_subsets, beta=solver.beta, lb=0.0,
                                         dtype=np.float32).astype(np.float32)
            iters += 1
            if time.perf_counter() - t0 > 20.0:
                break
        c["ossqs_s_per_iteration"] = (time.perf_counter() - t0) / iters
        c["ossqs_iterations_run"] = iters
        c["pipeline_s"] = c["fp_s"] + c["fbp_s"] + c["ossqs_s_per_iteration"] * n_iter
        c["rmse_hu_after_run"] = rmse(xc)
        out["cpu_baseline"] = {"value": c["pipeline_s"], "unit": "s", "cores": os.cpu_count() or 1, "kind": "port",
                               "sample": f"the same pipeline on the host, FP32 OpenMP oracle; OS-SQS timed over "
                                         f"{iters} of the {n_iter} iterations (capped at ~20 s) and scaled",
                               "stages": c}
        out["speedup_vs_cpu"] = c["pipeline_s"] * 1e3 / out["gpu_pipeline_ms"]
    return out


def conv_roofline(dev, n=16, hw=512):
    """The 32 -> 32 channel BF16 3x3 convolution layer of the prior (the
    dominant layer: 3 of 5) forward, input-gradient and weight-gradient
    kernels on n images of hw x hw, timed with CUDA events; FLOPs 2 * pixels
    * 32 * 288 per kernel, against the measured dense BF16 peak."""
    import torch

    from reconnet_b200.learned_prior import ConvKernels, pack_dgrad_weights, pack_weights
    k = ConvKernels(dev)
    x = (torch.rand((n, 4, hw, hw, 8), device=dev) - 0.5).to(torch.bfloat16)
    w = torch.randn(32, 3, 3, 32, device=dev) * 0.05
    b = torch.zeros(32, device=dev)
    pk, pkd = pack_weights(w), pack_dgrad_weights(w)
    out = torch.empty_like(x)
    flops = 2.0 * n * hw * hw * 32 * 288
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(p))["bf16_tflops"] if os.path.exists(p) else 1590.0
    res = {"workload": f"{n} images {hw}x{hw}, 32 -> 32 channels, BF16 in / FP32 accumulation",
           "flops_per_launch": flops, "peak_tflops": peak}
    for name, fn in (("forward", lambda: k.conv(x, pk, b, 32, 32, 0, out=out)),
                     ("input_gradient", lambda: k.conv(x, pkd, None, 32, 32, 2, aux=x, out=out)),
                     ("weight_gradient", lambda: k.wgrad(x, x, 32, 32))):
        fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / 5
        tf = flops / (ms * 1e-3) / 1e12
        hbm = 2 * x.numel() * 2 / (ms * 1e-3) / 1e9
        res[name] = {"ms": ms, "tflops": tf, "frac_of_bf16_peak": tf / peak, "activation_gbs": hbm}
    k.check()
    return res


def prior_run(dev, n_train=256, n_eval=32, train_steps=4000, tv_iters=100, n_val=8):
    """The learned prior against plain TV-SQS (the learned-prior workload at
    reduced slice counts): 512x512 slices @0.7 mm, 888 channels, 1152 views;
    the CNN (5 layers, 32 channels, BF16 tcgen05 convolutions) is trained here
    on n_train pairs (inputs: 4 OS-SQS iterations at I0 = 1e4; targets: 100
    TV-SQS iterations at I0 = 1e6), then n_eval held-out slices at I0 = 1e4
    are reconstructed by (a) TV-SQS for tv_iters iterations, (b) 4 OS-SQS
    iterations + the network and (c) OS-SQS iterations with the network
    between them, on a schedule chosen on n_val validation slices.  Time-to-RMSE: the target is TV-SQS's final
    RMSE + 1 HU; TV's time is that of its first iteration within the target.
    Two references for the RMSE: the high-dose reconstruction of the held-out slices (100 TV-SQS
    iterations at I0 = 1e6, the training targets' definition), and the
    phantom itself; at I0 = 1e4 a part of the rays through these phantoms is
    photon-starved, which leaves every reconstruction hundreds of HU from the
    phantom, so the high-dose reference is the one the 1 HU margin is read on."""
    import torch

    from reconnet_b200 import learned_prior as LP
    from reconnet_b200.phantom import HU, ellipse_phantom, geom_fan512
    geom = geom_fan512()
    nview = 1152
    t0 = time.perf_counter()
    x_in, x_tg, _ = LP.make_training_pairs(geom, nview, n_train, seed=5)
    gen_s = time.perf_counter() - t0
    net = LP.PriorCNN(dev, seed=0)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    losses = net.train(x_in, x_tg, steps=train_steps, batch=8, lr=1e-3, log_every=500)
    torch.cuda.synchronize(dev)
    train_s = time.perf_counter() - t0
    rng = np.random.default_rng(77)
    truth = torch.from_numpy(np.stack([ellipse_phantom(geom.nx, geom.ny, geom.dx, geom.dy, rng)
                                       for _ in range(n_eval)]).astype(np.float32)).to(dev)
    ang_hd, b_hd, w_hd = LP.simulate(geom, nview, truth, 1e6, seed=98)
    x_hd, _ = LP.os_sqs(geom, nview, ang_hd, b_hd, w_hd, n_eval, 100)
    del ang_hd, b_hd, w_hd
    ang, b, w = LP.simulate(geom, nview, truth, 1e4, seed=99)
    rmse = lambda a: float(torch.sqrt(((a - truth) ** 2).mean())) / HU
    rmse_hd = lambda a: float(torch.sqrt(((a - x_hd) ** 2).mean())) / HU
    # TV-SQS trajectory (untimed), then its timing (graph replay, CUDA events)
    from reconnet_b200.ossqs import BatchedOSSQS
    solver = BatchedOSSQS(geom, [nview] * n_eval, ang, b, w, n_subsets=24, lb=0.0, device=dev)
    solver.beta = LP.tv_weight(solver)
    x = torch.zeros_like(truth)
    traj, traj_hd = [], []
    for k in range(tv_iters):
        x = solver.run(x, 1)
        traj.append(rmse(x))
        traj_hd.append(rmse_hd(x))
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    e0, e1 = ev()
    e0.record()
    solver.run(torch.zeros_like(truth), tv_iters)
    e1.record()
    torch.cuda.synchronize(dev)
    tv_ms_per_iter = e0.elapsed_time(e1) / tv_iters
    solver.check()
    target = traj[-1] + 1.0

    def time_to_target(tr, r_l, l_ms):
        tgt = tr[-1] + 1.0
        k_reach = next((k for k, r in enumerate(tr) if r <= tgt), None)
        t_ms = None if k_reach is None else (k_reach + 1) * tv_ms_per_iter
        sp = None if (t_ms is None or r_l > tgt) else t_ms / l_ms
        return tgt, t_ms, sp

    def timed(schedule):
        LP.run_schedule(net, solver, torch.zeros_like(truth), schedule)   # warm (graph capture)
        e0, e1 = ev()
        e0.record()
        y = LP.run_schedule(net, solver, torch.zeros_like(truth), schedule)
        e1.record()
        torch.cuda.synchronize(dev)
        return y, e0.elapsed_time(e1)

    # The learned path with the network trained for: 4 iterations + the network.
    y, learned_ms = timed((4, "N"))
    net.k.check()
    x4 = solver.run(torch.zeros_like(truth), 4)
    r_learned, r_learned_hd = rmse(y), rmse_hd(y)
    target, tv_ms_to_target, speedup = time_to_target(traj, r_learned, learned_ms)
    target_hd, tv_ms_to_target_hd, speedup_hd = time_to_target(traj_hd, r_learned_hd, learned_ms)

    # Learned-prior OS-SQS with the network between iterations: the schedule
    # (iterations and network passes, LP.SCHEDULES) is chosen on n_val
    # validation slices of their own seeds -- the cheapest one whose RMSE
    # against their high-dose reconstruction is at most TV-SQS's 100-iteration
    # RMSE, the target's 1 HU kept as margin for the step to other slices --
    # and then timed and scored on the held-out slices above.
    rng_v = np.random.default_rng(177)
    truth_v = torch.from_numpy(np.stack([ellipse_phantom(geom.nx, geom.ny, geom.dx, geom.dy, rng_v)
                                         for _ in range(n_val)]).astype(np.float32)).to(dev)
    a_v, b_v, w_v = LP.simulate(geom, nview, truth_v, 1e6, seed=198)
    x_hd_v, _ = LP.os_sqs(geom, nview, a_v, b_v, w_v, n_val, 100)
    a_v, b_v, w_v = LP.simulate(geom, nview, truth_v, 1e4, seed=199)
    solver_v = BatchedOSSQS(geom, [nview] * n_val, a_v, b_v, w_v, n_subsets=24, lb=0.0, device=dev)
    solver_v.beta = LP.tv_weight(solver_v)
    tv_v = solver_v.run(torch.zeros_like(truth_v), tv_iters)
    tv_v_rmse = float(torch.sqrt(((tv_v - x_hd_v) ** 2).mean()))
    chosen, val_err, val_excess = LP.choose_schedule(net, solver_v, x_hd_v, tv_v)
    del solver_v, a_v, b_v, w_v
    y_s, sched_ms = timed(chosen)
    net.k.check()
    solver.check()
    r_s, r_s_hd = rmse(y_s), rmse_hd(y_s)
    _, _, speedup_s = time_to_target(traj, r_s, sched_ms)
    _, _, speedup_s_hd = time_to_target(traj_hd, r_s_hd, sched_ms)
    its, passes = LP.schedule_cost(chosen)
    conv = conv_roofline(dev)
    sched_name = lambda sch: " ".join("net" if t == "N" else f"{t}it" for t in sch)
    return {"conv_32x32": conv,
            "workload": f"512x512 @0.7 mm, 888 ch, {nview} views; train {n_train} slices (4-iteration OS-SQS at "
                        f"I0=1e4 -> 100-iteration TV-SQS at I0=1e6), evaluate {n_eval} held-out slices at I0=1e4",
            "scaled_from": "4,000 training and 256 held-out slices in the workload's definition",
            "data_generation_s": gen_s, "train_s": train_s, "train_steps": train_steps, "train_loss": losses,
            "tv_iterations": tv_iters, "tv_ms_per_iteration": tv_ms_per_iter, "tv_rmse_hu_final": traj[-1],
            "tv_rmse_hu_at": {str(k + 1): traj[k] for k in (0, 3, 9, 19, 49, tv_iters - 1) if k < tv_iters},
            "lr_schedule": "Adam, 1e-3 cosine-decayed to 1e-5, batch 8, the eight orientations of the square",
            "learned_ms": learned_ms,
            "against_high_dose": {
                "reference": "100-iteration TV-SQS at I0=1e6 of the held-out slices",
                "tv_rmse_hu_final": traj_hd[-1],
                "tv_rmse_hu_at": {str(k + 1): traj_hd[k] for k in (0, 3, 9, 19, 49, tv_iters - 1) if k < tv_iters},
                "rmse_target_hu": target_hd, "tv_ms_to_target": tv_ms_to_target_hd,
                "learned_rmse_hu": r_learned_hd, "os_sqs4_rmse_hu": rmse_hd(x4),
                "speedup_time_to_rmse": speedup_hd,
                "target_met": bool(speedup_hd is not None and speedup_hd >= 3.0)},
            "against_phantom": {
                "rmse_target_hu": target, "tv_ms_to_target": tv_ms_to_target,
                "learned_rmse_hu": r_learned, "os_sqs4_rmse_hu": rmse(x4),
                "speedup_time_to_rmse": speedup,
                "target_met": bool(speedup is not None and speedup >= 3.0)},
            "scheduled": {
                "what": "OS-SQS iterations with the network between them, the schedule chosen on "
                        f"{n_val} validation slices (their own seeds) as the cheapest whose RMSE against their "
                        "high-dose reconstruction is at most TV-SQS's 100-iteration RMSE (the target's 1 HU kept "
                        "as margin for the step to the held-out slices)",
                "validation_rmse_hu": {sched_name(k): v / HU for k, v in val_err.items()},
                "validation_excess_over_tv_hu": {sched_name(k): v / HU for k, v in val_excess.items()},
                "validation_tv_rmse_hu": tv_v_rmse / HU,
                "schedule": sched_name(chosen), "iterations": its, "network_passes": passes, "ms": sched_ms,
                "against_high_dose": {"rmse_hu": r_s_hd, "rmse_target_hu": target_hd,
                                      "speedup_time_to_rmse": speedup_s_hd,
                                      "target_met": bool(speedup_s_hd is not None and speedup_s_hd >= 3.0)},
                "against_phantom": {"rmse_hu": r_s, "rmse_target_hu": target, "speedup_time_to_rmse": speedup_s,
                                    "target_met": bool(speedup_s is not None and speedup_s >= 3.0)}},
            "target_met": bool((speedup_hd is not None and speedup_hd >= 3.0) or
                               (speedup_s_hd is not None and speedup_s_hd >= 3.0))}


def tomo_run(dev, cpu_sample=True):
    """Tomosynthesis DD pair (DistanceDriven3D) on a 512x512x128 volume:
    512x512x128 voxels of 0.8x0.8x1.0 mm, a 736x736 flat detector of 0.6 mm
    cells 80 mm below the isocentre, 25 sources on a +-20 deg arc at 650 mm.
    Updates: FP = views * nu * nv * nz ray-plane integrals, BP = voxels * views;
    algorithmic bytes 16 B per update (the reference's 4 summed-area-table
    corners, 4 B each)."""
    import ctypes
    import math

    import torch

    from reconnet_b200 import _native as N
    nx, ny, nz, nu, nv, nview = 512, 512, 128, 736, 736, 25
    dx, dy, dz, du, dv = 0.8, 0.8, 1.0, 0.6, 0.6
    dc = np.zeros((nview, 3), np.float32)
    src = np.zeros((nview, 3), np.float32)
    for k in range(nview):
        a = (k - (nview - 1) / 2) / ((nview - 1) / 2) * math.radians(20)
        src[k] = (650 * math.sin(a), 0.0, 650 * math.cos(a))
        dc[k] = (0.0, 0.0, -80.0)
    rng = np.random.default_rng(11)
    from reconnet_b200.phantom import ellipsoid_phantom
    img = ellipsoid_phantom(nx, ny, nz, dx, dy, dz, rng, device=dev)[None, :, :, :, None].contiguous()
    prj = torch.empty((1, nu, nview, nv, 1), device=dev)
    back = torch.empty_like(img)
    fpb, bpb = ctypes.c_size_t(), ctypes.c_size_t()
    N.lib.rn_tomo_sat_bytes(nx, ny, nz, nu, nview, nv, ctypes.byref(fpb), ctypes.byref(bpb))
    sat = torch.empty(max(fpb.value, bpb.value) // 8 + 1, dtype=torch.float64, device=dev)
    ddc, dsrc = torch.from_numpy(dc).to(dev), torch.from_numpy(src).to(dev)
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    geo = (1, 1, nx, ny, nz, dx, dy, dz, 0.0, 0.0, 0.0, nu, nview, nv, du, dv, 0.0, 0.0)
    st = lambda: ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    fp = lambda: N.check(N.lib.rn_tomo_project(P(prj), P(img), P(ddc), P(dsrc), P(sat), *geo, st()))
    bp = lambda: N.check(N.lib.rn_tomo_backproject(P(back), P(prj), P(ddc), P(dsrc), P(sat), *geo, 1, st()))
    peak, kind = measured_peaks()
    out = {"workload": "tomosynthesis: 512x512x128 @0.8x0.8x1.0 mm, 736x736 flat detector @0.6 mm, 25 views "
                       "over +-20 deg (the reference's 3D DD pair is this flat-detector, z-main geometry; a 360-deg "
                       "cylindrical-detector scan has no reference kernel)",
           "model": "16 B per update (the reference's 4 summed-area-table corners)"}
    for name, f, upd in (("fp", fp, nview * nu * nv * nz), ("bp", bp, nx * ny * nz * nview)):
        f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            f()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        ach = 16.0 * upd / (ms * 1e-3) / 1e9
        out[name] = {"ms": ms, "updates": upd, "gupd_s": upd / ms / 1e6,
                     "roofline": {"achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                  "peak_kind": kind}}
    if cpu_sample:
        from oracle import oracle as O
        from types import SimpleNamespace
        O.set_threads(os.cpu_count() or 1)
        g = SimpleNamespace(dx=dx, dy=dy, dz=dz, cx=0.0, cy=0.0, cz=0.0, du=du, dv=dv, off_u=0.0, off_v=0.0)
        vol = img.cpu().numpy()
        t0 = time.perf_counter()
        O.tomo_fp(vol, dc[:1], src[:1], g, nu, nv)
        t1 = time.perf_counter()
        O.tomo_bp(np.ones((1, nu, 1, nv, 1), np.float32), dc[:1], src[:1], g, (nx, ny, nz), 1)
        t2 = time.perf_counter()
        out["cpu_baseline"] = {"fp_gupd_s": nu * nv * nz / (t1 - t0) / 1e9, "bp_gupd_s": nx * ny * nz / (t2 - t1) / 1e9,
                               "cores": os.cpu_count() or 1, "kind": "port",
                               "sample": "1 of the 25 views, FP64 OpenMP oracle (the reference has no CPU path)"}
    return out


def cyl_run(dev, cpu_sample=True):
    """The cone-beam workload: the cylindrical-detector DD pair (csrc/cyl.cu)
    on 512x512x128 voxels of 0.8x0.8x1.0 mm, 736 x 64 cells (1.2858 mm x
    1.0 mm at the detector), 984 views over 360 degrees, source at 595 mm and
    the detector at 1085.6 mm; random ellipsoids of 0-0.04/mm.  Updates:
    FP = views x cells x planes (984 x 736 x 64 x 512), BP = voxels x views.
    The bound is instruction issue, not HBM: the FP reads a band of z
    prefix sums per voxel column and the BP per-view row tables, both from
    L2.  `roofline` is the kernel's warp instructions per projection (ncu,
    profiles/ncu_counts_bench.txt) over its CUDA-event time against one warp
    instruction per clock on each scheduler at the sampled SM clock; the
    compulsory-bytes fraction of HBM is reported beside it."""
    import torch

    from reconnet_b200.phantom import ellipsoid_phantom
    from reconnet_b200.torch_ops import CylGeometry, CylPlan
    g = CylGeometry()
    nview = 984
    ang = (np.arange(nview) * 2 * np.pi / nview).astype(np.float32)
    plan = CylPlan(g, ang, device=dev)
    vol = ellipsoid_phantom(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, np.random.default_rng(21), device=dev)[None].contiguous()
    prj = torch.empty(plan.prj_shape, device=dev)
    back = torch.empty(plan.vol_shape, device=dev)
    peak, kind = measured_peaks()
    vol_b, prj_b = vol.numel() * 4, prj.numel() * 4
    tab_b = nview * g.nu * (g.nv + 1) * 8
    out = {"workload": "cylindrical-detector cone-beam DD pair: 512x512x128 @0.8x0.8x1.0 mm, 736x64 cells "
                       "(1.2858 x 1.0 mm at the detector), 984 views over 360 deg, dso 595 / dsd 1085.6 mm",
           "data": "synthetic: 10 seeded random ellipsoids, 0-0.04/mm"}
    fp_upd = nview * g.nu * g.nv * g.ny       # planes per ray: ny (X-class) or nx (Y-class), equal here
    bp_upd = g.nx * g.ny * g.nz * nview
    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    for name, kern, f, upd, hbm in (("fp", "cyl_fp_kernel", lambda: plan.project(vol, out=prj), fp_upd, vol_b + prj_b),
                                    ("bp", "cyl_bp_kernel", lambda: plan.backproject(prj, out=back), bp_upd,
                                     prj_b + 2 * tab_b + vol_b)):
        f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(dev.index if dev.index is not None else 0) as clk:
            e0.record()
            for _ in range(3):
                f()
            e1.record()
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        t = ms * 1e-3
        clocks = clk.summary()
        mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz")
        counts = ncu_counts(kern)
        roof = {"bound": "issue", "kernel": kern, "unit": "Gwarp-inst/s", "achieved": None, "peak": None, "frac": None,
                "traffic": None, "peak_source": f"{n_sm} SMs x 4 schedulers x 1 warp instruction per clock at the "
                                                "sampled SM clock", "sm_mhz": mhz,
                "compulsory_hbm": {"bytes": hbm, "achieved": hbm / t / 1e9, "peak": peak, "unit": "GB/s",
                                   "frac": hbm / t / 1e9 / peak, "peak_kind": kind}}
        if counts is not None:
            roof["traffic"] = counts["dram_bytes"]
            if mhz:
                roof["achieved"] = counts["warp_inst"] / t / 1e9
                roof["peak"] = n_sm * 4 * mhz * 1e6 / 1e9
                roof["frac"] = roof["achieved"] / roof["peak"]
        out[name] = {"ms": ms, "updates": upd, "gupd_s": upd / ms / 1e6, "roofline": roof, "clocks": clocks}
    y = torch.rand(plan.prj_shape, device=dev)
    aty = plan.backproject(y)
    ax = plan.project(vol)
    lhs, rhs = float((ax.double() * y.double()).sum()), float((vol.double() * aty.double()).sum())
    out["adjoint_rel"] = abs(lhs - rhs) / abs(lhs)
    if cpu_sample:
        from oracle import oracle as O
        O.set_threads(os.cpu_count() or 1)
        v = vol.cpu().numpy()
        t0 = time.perf_counter()
        O.cyl_fp(v, ang[:1], g)
        t1 = time.perf_counter()
        out["cpu_baseline"] = {"fp_gupd_s": g.nu * g.nv * g.ny / (t1 - t0) / 1e9, "cores": os.cpu_count() or 1,
                               "kind": "port", "sample": "1 of the 984 views, FP64 OpenMP oracle (no reference CPU path)"}
    return out


def siddon_run(plan, x, p, b, geom, angles, counts, cpu_sample=True):
    """Siddon fan pair (Siddon.cu, the reference OS-SQS projector) on the
    bench's slice batch: FP of every view of every slice, then the Siddon
    transpose BP.  Updates are counted as for DD: FP = views * nu * ny
    ray-band integrals, BP = views * nx * ny pixel-view gathers; the byte
    model is the same 8 B per update (two prefix samples per band)."""
    import torch

    from reconnet_b200 import _native as N
    peak, kind = measured_peaks()
    out = {"workload": "the fan batch above, Siddon ray-length pair (FP, then its exact transpose)",
           "model": f"{BYTES_PER_UPDATE} B per update"}
    for name, f, upd in (("fp", lambda: plan.project(x, out=p, siddon=True), plan.fp_updates()),
                         ("bp", lambda: plan.backproject(p, N.RN_TYPE_SIDDON, out=b), plan.bp_updates())):
        f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            f()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        ach = BYTES_PER_UPDATE * upd / (ms * 1e-3) / 1e9
        out[name] = {"ms": ms, "updates": upd, "gupd_s": upd / ms / 1e6,
                     "roofline": {"achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                  "peak_kind": kind}}
    plan.check()
    if cpu_sample:
        from oracle import oracle as O
        O.set_threads(os.cpu_count() or 1)
        nvw = 128
        sel = np.ascontiguousarray(angles[:nvw])
        img = x[0].cpu().numpy()[None, :, :, None, None]
        t0 = time.perf_counter()
        s = O.siddon_fp(img, sel, geom, geom.nu, 1)
        t1 = time.perf_counter()
        O.siddon_bp(s.astype(np.float32), sel, geom, (geom.nx, geom.ny, 1))
        t2 = time.perf_counter()
        out["cpu_baseline"] = {"fp_gupd_s": nvw * geom.nu * geom.ny / (t1 - t0) / 1e9,
                               "bp_gupd_s": nvw * geom.nx * geom.ny / (t2 - t1) / 1e9,
                               "cores": os.cpu_count() or 1, "kind": "port",
                               "sample": f"{nvw} views of slice 0, FP64 OpenMP oracle (exact crossings)"}
    return out


def cone_run(dev, cpu_sample=True):
    """Siddon cone pair with per-view geometry (SiddonCone.cu) on the
    tomosynthesis workload of `tomo_run`: 512x512x128 voxels of 0.8x0.8x1.0 mm,
    a 736x736 flat detector of 0.6 mm cells 80 mm below the isocentre, 25
    sources on a +-20 deg arc at 650 mm.  Updates as for the DD pair: FP =
    views * nu * nv * nz ray-slab steps, BP = voxels * views; the byte model
    is one 4-byte voxel (FP) or sinogram (BP) read per piece, about 1.3 pieces
    per update (5.2 B)."""
    import torch

    from reconnet_b200.phantom import ellipsoid_phantom
    from reconnet_b200.torch_ops import ConeGeometry, ConePlan
    nx, ny, nz, nu, nv, nview = 512, 512, 128, 736, 736, 25
    g = ConeGeometry(nx=nx, ny=ny, nz=nz, dx=0.8, dy=0.8, dz=1.0, nu=nu, nv=nv, du=0.6, dv=0.6)
    dc, du, dv, src = tomo_geometry(nview)
    plan = ConePlan(g, dc, du, dv, src, device=dev)
    img = ellipsoid_phantom(nx, ny, nz, 0.8, 0.8, 1.0, np.random.default_rng(11), device=dev)[None, :, :, :, None]
    img = img.contiguous()
    prj = plan.project(img)
    back = torch.empty_like(img)
    peak, kind = measured_peaks()
    out = {"workload": "the tomosynthesis workload above (512x512x128 @0.8x0.8x1.0 mm, 736x736 @0.6 mm, 25 views "
                       "over +-20 deg), Siddon ray lengths: FP, then its exact transpose",
           "model": "5.2 B per update (one 4-byte read per piece, ~1.3 pieces)"}
    for name, f, upd in (("fp", lambda: plan.project(img, out=prj), nview * nu * nv * nz),
                         ("bp", lambda: plan.backproject(prj, out=back), nx * ny * nz * nview)):
        f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            f()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        ach = 5.2 * upd / (ms * 1e-3) / 1e9
        out[name] = {"ms": ms, "updates": upd, "gupd_s": upd / ms / 1e6,
                     "roofline": {"achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                  "peak_kind": kind}}
    if cpu_sample:
        from oracle import oracle as O
        from types import SimpleNamespace
        O.set_threads(os.cpu_count() or 1)
        gg = SimpleNamespace(dx=0.8, dy=0.8, dz=1.0, cx=0.0, cy=0.0, cz=0.0, du=0.6, dv=0.6, off_u=0.0, off_v=0.0)
        vol = img.cpu().numpy()
        # one view, the central 128 detector rows (the sample's rows are
        # centred on the detector centre like the full detector's)
        t0 = time.perf_counter()
        O.cone_fp(vol, dc[:1], du[:1], dv[:1], src[:1], gg, nu, 128)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"fp_gupd_s": nu * 128 * nz / dt / 1e9, "cores": os.cpu_count() or 1, "kind": "port",
                               "sample": "the central 128 detector rows of one view, FP64 OpenMP oracle "
                                         "(exact crossings)"}
    del plan
    return out


def host_calls_run(geom, counts, angles, imgs):
    """The drop-in path: every slice of the batch through the reference-named
    host entry points cDistanceDrivenFanProjection + ...Backprojection
    (typeProjector 0, as the reference arm's `reference_gpu` calls the
    reference's library), host arrays in and out, one call pair per slice
    (each slice has its own angles, so each call builds its plan)."""
    from reconnet_b200.reconnet import ReconNet
    rn = ReconNet()
    for k in ("nx", "ny", "dx", "dy", "nu", "da", "dsd", "dso"):
        setattr(rn, k, getattr(geom, k))
    rn.nz, rn.nv, rn.dz, rn.dv, rn.off_a, rn.off_v = 1, 1, geom.dz, geom.dv, geom.off_a, geom.off_v
    offs = np.concatenate([[0], np.cumsum(counts)])
    imgs5 = [np.ascontiguousarray(im[None, :, :, None, None]) for im in imgs]
    angs = [np.ascontiguousarray(angles[offs[s]:offs[s + 1]]) for s in range(len(counts))]

    def one_step():
        for s in range(len(counts)):
            sino = rn.cDDFanProjection4d(imgs5[s], angs[s])
            rn.cDDFanBackprojection4d(sino, angs[s], type_projector=0)

    one_step()
    t0 = time.perf_counter()
    one_step()
    dt = time.perf_counter() - t0
    upd = int(np.sum(counts)) * (geom.nu * geom.ny + geom.nx * geom.ny)
    return {"value": upd / dt / 1e9, "unit": UNIT, "ms_per_step": dt * 1e3,
            "api": "reference-named host entry points, per slice, host arrays (numpy) in and out, "
                   "typeProjector 0; wall time of one step after one warm-up step"}


def filter_run(dev, cpu_sample=True):
    """Ramp filter (Filter.cu): 64 fan sinograms of 888 channels x 1152 views,
    Ram-Lak window.  The filter is a linear convolution of every view with the
    (2 nu - 1)-tap kernel, run as an FFT of length 2048 per pair of views in
    shared memory; the roofline is the memory one (every sample read and
    written once), and the rate of the direct convolution (nu^2 multiply-adds
    per view) is given for comparison."""
    import torch

    from reconnet_b200.phantom import geom_fan512
    from reconnet_b200.torch_ops import filter_sino
    geom = geom_fan512()
    B, nu, nview = 64, geom.nu, 1152
    rng = np.random.default_rng(12)
    sino = torch.from_numpy(rng.random((B, nu, nview, 1, 1), dtype=np.float32)).to(dev)
    filter_sino(sino, geom)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        filter_sino(sino, geom)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 5
    direct_flops = 2.0 * nu * nu * nview * B
    nbytes = 2 * 4 * nu * nview * B
    peak, kind = measured_peaks()
    achieved = nbytes / (ms * 1e-3) / 1e9
    out = {"workload": f"{B} fan sinograms, {nu} channels x {nview} views, Ram-Lak",
           "ms": ms, "views_per_s": B * nview / (ms * 1e-3),
           "direct_equivalent_tflops": direct_flops / (ms * 1e-3) / 1e12,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_kind": kind,
                        "model": "4 B read + 4 B written per sinogram sample"}}
    if cpu_sample:
        from oracle import oracle as O
        O.set_threads(os.cpu_count() or 1)
        sample = sino[:1, :, :64].cpu().numpy()
        t0 = time.perf_counter()
        O.filter_sino(sample, geom, 0, True)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"views_per_s": 64 / dt, "cores": os.cpu_count() or 1, "kind": "port",
                               "sample": "64 views of one sinogram, FP64 OpenMP oracle"}
    return out


def fan_roofline(kernel, dur_ms, updates, io_bytes, clocks, dev):
    """Roofline of the dominant fan kernel against its real bound.

    The DD kernels are not HBM-bound: they read their prefix samples from
    shared memory and move ~1 GB of DRAM per launch (under 1% of peak).  They
    are bound by instruction issue (and the L1/shared pipe behind it).  So the
    headline fraction is issue-rate: the kernel's warp instructions per launch
    (ncu, profiles/ncu_counts_bench.txt) over its CUDA-event launch time,
    against one warp instruction per clock on each of the 4 schedulers of
    every SM at the SM clock sampled during the timed region.  Beside it:
    `hbm`, the measured DRAM bytes over the same time against the measured
    HBM peak, and `effective_onchip`, the 8 B-per-footprint model (two FP32
    prefix samples per update) that these kernels serve from shared memory."""
    import torch
    counts = ncu_counts(kernel)
    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    peak_hbm, peak_kind = measured_peaks()
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz")
    t = dur_ms * 1e-3
    onchip = BYTES_PER_UPDATE * updates + io_bytes
    out = {"bound": "issue", "kernel": kernel, "launch_ms": dur_ms, "unit": "Gwarp-inst/s",
           "achieved": None, "peak": None, "frac": None, "traffic": None,
           "peak_source": f"{n_sm} SMs x 4 schedulers x 1 warp instruction per clock at the sampled SM clock",
           "hbm": {"achieved": None, "peak": peak_hbm, "unit": "GB/s", "frac": None, "peak_kind": peak_kind},
           "effective_onchip": {"bytes_per_launch": onchip, "gbs": onchip / t / 1e9,
                                "model": f"{BYTES_PER_UPDATE} B per footprint update (two FP32 prefix samples, "
                                         "read from shared memory) + 4 B per image/sinogram element"}}
    if counts is not None:
        out["traffic"] = counts["dram_bytes"]
        out["hbm"]["achieved"] = counts["dram_bytes"] / t / 1e9
        out["hbm"]["frac"] = out["hbm"]["achieved"] / peak_hbm
        if mhz:
            peak_inst = n_sm * 4 * mhz * 1e6
            out["achieved"] = counts["warp_inst"] / t / 1e9
            out["peak"] = peak_inst / 1e9
            out["frac"] = counts["warp_inst"] / t / peak_inst
            out["sm_mhz"] = mhz
    return out


def run_b200(args):
    import torch
    import torch.distributed as dist

    from reconnet_b200.torch_ops import FanPlan

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    geom, counts, angles, imgs = workload(rank, args.slices)
    plan = FanPlan(geom, angles, nbatches=args.slices, nview_per_slice=counts, device=dev)
    x = torch.from_numpy(imgs).to(dev)
    p = torch.empty(plan.sino_shape, device=dev)
    b = torch.empty(plan.img_shape, device=dev)
    fp_upd, bp_upd = plan.fp_updates(), plan.bp_updates()
    updates = fp_upd + bp_upd

    def step():
        plan.project(x, out=p)
        plan.backproject(p, 2, out=b)

    for _ in range(max(3, args.warmup)):
        step()
    plan.check()
    torch.cuda.synchronize()

    # ---- device-timed region ----
    barrier()
    torch.cuda.synchronize()
    l0 = plan.launches()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(st)
        for _ in range(args.steps):
            step()
        e1.record(st)
        torch.cuda.synchronize()
    barrier()
    launches = plan.launches() - l0
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = updates * world / (ms_step * 1e-3) / 1e9
    plan.check()

    # ---- per-kernel timing (CUDA events around each launch) for the roofline ----
    plan.set_timing(True)
    prof_steps = 3
    for _ in range(prof_steps):
        step()
    kt, _ = plan.read_timing()
    plan.set_timing(False)
    fp_ms = kt["fp"][0] / max(kt["fp"][1], 1)
    bp_ms = kt["bp"][0] / max(kt["bp"][1], 1)
    dominant = "fan_fp_kernel" if kt["fp"][0] >= kt["bp"][0] else "fan_bp_kernel"
    roofline = fan_roofline(dominant, fp_ms if dominant == "fan_fp_kernel" else bp_ms,
                            fp_upd if dominant == "fan_fp_kernel" else bp_upd, 4 * (x.numel() + p.numel()),
                            clk.summary(), dev)
    roofline["kernels_ms"] = {k: (v[0] / max(v[1], 1)) for k, v in kt.items() if v[1]}

    # ---- end to end through the public API with host buffers ----
    # StreamedFanPair: pinned host images in, pinned host backprojections out,
    # every step; double-buffered device copies on two copy streams, so a
    # step's H2D and D2H run beside the FP + BP of the neighbouring steps
    from reconnet_b200.torch_ops import StreamedFanPair
    xh = torch.from_numpy(imgs).pin_memory()
    bh = torch.empty(plan.img_shape, dtype=torch.float32).pin_memory()
    pair = StreamedFanPair(geom, angles, counts, groups=1, device=dev)
    assert pair.updates() == updates
    e2e_steps = max(3, args.steps // 2)

    def timed(fn, n, finish=lambda: None):
        for _ in range(2):
            fn()
        barrier()
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(n):
            fn()
        finish()
        e1.record(st)
        torch.cuda.synchronize()
        barrier()
        t_ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([t_ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_ms = float(t.item())
        return t_ms

    # the timed region ends when the last step's result is in host memory
    ms_e2e = timed(lambda: pair(xh, bh), e2e_steps, finish=lambda: st.wait_event(pair.done))
    pair.check()
    # the same with the copies serialised on the compute stream, for reference
    xs = torch.empty_like(x)

    def serial_step():
        xs.copy_(xh, non_blocking=True)
        plan.project(xs, out=p)
        plan.backproject(p, 2, out=b)
        bh.copy_(b, non_blocking=True)

    ms_serial = timed(serial_step, e2e_steps)
    e2e = {"value": updates * world / (ms_e2e / e2e_steps * 1e-3) / 1e9, "unit": UNIT,
           "h2d_bytes_per_step": int(xh.numel() * 4), "d2h_bytes_per_step": int(bh.numel() * 4),
           "ms_per_step": ms_e2e / e2e_steps,
           "api": "reconnet_b200.torch_ops.StreamedFanPair: double-buffered device inputs/outputs, each step's "
                  "H2D and D2H on two copy streams overlapping the FP + BP of the neighbouring steps",
           "serial_ms_per_step": ms_serial / e2e_steps}

    host_calls = host_calls_run(geom, counts, angles, imgs) if rank == 0 and not args.no_extras else None
    ossqs = None if args.no_ossqs else ossqs_run(plan, geom, counts, angles, x, args.ossqs_iters, dev)
    extras = {}
    if rank == 0 and not args.no_extras:
        extras["siddon"] = siddon_run(plan, x, p, b, geom, angles, counts, cpu_sample=world == 1)
        extras["tomo"] = tomo_run(dev, cpu_sample=world == 1)
        extras["siddon_cone"] = cone_run(dev, cpu_sample=world == 1)
        extras["filter"] = filter_run(dev, cpu_sample=world == 1)
        extras["cone_cyl"] = cyl_run(dev, cpu_sample=world == 1)
        extras["fan2d_pipeline"] = cfg0_run(dev, cpu_sample=world == 1)
        extras["learned_prior"] = prior_run(dev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cores, desc = cpu_baseline_sample(geom, counts, angles, imgs)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32",
                "data": "synthetic: seeded random-ellipse phantoms (10 ellipses, 5-120 mm, 0-0.04/mm)",
                "config": bench_config(args.slices, counts, world),
                "roofline": roofline, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clk.summary()}
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if host_calls is not None:
            line["e2e_host_calls"] = host_calls
        if ossqs is not None:
            line["ossqs_tv"] = ossqs
        line.update(extras)
        print(json.dumps(line), flush=True)
    del plan
    if world > 1:
        dist.destroy_process_group()


def run_extra(args):
    """One extra measurement alone (for profiling a single kernel family)."""
    import torch
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    cpu = not args.no_cpu_baseline
    if args.extra in ("siddon", "ossqs"):
        from reconnet_b200.torch_ops import FanPlan
        geom, counts, angles, imgs = workload(0, args.slices)
        plan = FanPlan(geom, angles, nbatches=args.slices, nview_per_slice=counts, device=dev)
        x = torch.from_numpy(imgs).to(dev)
        if args.extra == "ossqs":
            out = ossqs_run(plan, geom, counts, angles, x, args.ossqs_iters, dev)
        else:
            p = torch.empty(plan.sino_shape, device=dev)
            b = torch.empty(plan.img_shape, device=dev)
            out = siddon_run(plan, x, p, b, geom, angles, counts, cpu_sample=cpu)
    elif args.extra == "tomo":
        out = tomo_run(dev, cpu_sample=cpu)
    elif args.extra == "cone":
        out = cone_run(dev, cpu_sample=cpu)
    elif args.extra == "cyl":
        out = cyl_run(dev, cpu_sample=cpu)
    elif args.extra == "cfg0":
        out = cfg0_run(dev, cpu_sample=cpu)
    elif args.extra == "prior":
        out = prior_run(dev)
    elif args.extra == "conv":
        out = conv_roofline(dev)
    else:
        out = filter_run(dev, cpu_sample=cpu)
    print(json.dumps({args.extra: out}), flush=True)


def main():
    args = parse()
    if args.extra and args.impl == "b200":
        run_extra(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
