#!/usr/bin/env python3
"""Path-tracing throughput benchmark (Msamples/s) on the large-mesh workload.

Workload (one "step"): render 1024 x 1024 pixels x 64 samples of the seeded
spheres scene - three displaced level-7 icospheres (983,040 triangles), a
ground plane and a tessellated spherical area light of radius 0.3, 984,322
triangles in all, per-triangle Lambert albedo in [0.2, 0.9] - through a pinhole
camera (40 degree fov), max path depth 10, SAH kd-tree (traversal cost 1,
intersection cost 1.5, leaves of <= 4 triangles).  One sample is one camera
path.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl xyz|reference]

Prints one JSON line on rank 0.  `value` is device-timed with the scene resident
in HBM; `e2e` is the same metric through the C ABI with host buffers (scene
arrays uploaded, tree built and film read back every step).  Multi-GPU: one
process per GPU under torchrun; every rank renders its own 64 samples per pixel
(sample offset rank * 64) and the films are summed on rank 0 with one NCCL
reduce per step (weak scaling).
"""

from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

W_PIX, H_PIX, SPP, MAX_DEPTH, SEED = 1024, 1024, 64, 10, 0
METRIC = "Msamples/s on 1 B200 (path samples per second, 1M-triangle scene)"
UNIT = "Msamples/s"
L2_FLUSH_BYTES = 256 << 20
TRI_BYTES_ALGO = 36   # v0, e1, e2 as the reference stores a triangle
NODE_BYTES = 8
REF_BYTES = 4
RAY_IO_BYTES = 32 + 16


def workload_config():
    """The workload, identical in both arms' lines (the GPU arm's kd-tree
    statistics, parallelism and waves go beside it)."""
    cfg = {
        "workload": "spheres-1M: 3 displaced level-7 icospheres + ground + spherical light r=0.3, "
                    "984,322 triangles, 1024x1024, 64 spp, max depth 10, pinhole fov 40, "
                    "SAH kd-tree (64 bins, Ct=1, Ci=1.5, leaf<=4, no empty bonus), Lambert + NEE/MIS + Russian roulette, "
                    "XYZ film",
        "triangles": 984322, "width": W_PIX, "height": H_PIX, "spp": SPP, "max_depth": MAX_DEPTH,
        "seed": SEED, "l2_flush": "256 MiB buffer written between timed steps",
    }
    return cfg


# kd-tree of the workload as the configuration states it: SAH with traversal
# cost 1, intersection cost 1.5 and leaves of at most 4 triangles (64 bins,
# no empty-side bonus: the library's defaults otherwise)
WORKLOAD_BUILD = dict(leaf_max_tris=4, cost_traversal=1.0, cost_intersect=1.5)


def pinned_scene(sd):
    """A copy of the scene whose arrays live in page-locked host memory (the
    inputs a caller streams to the device each step)."""
    import dataclasses
    import torch
    out = {}
    for f in dataclasses.fields(sd):
        v = getattr(sd, f.name)
        if isinstance(v, np.ndarray) and v.nbytes >= 4096:
            t = torch.empty(v.shape, dtype=torch.from_numpy(v[:0]).dtype, pin_memory=True)
            a = t.numpy()
            a[...] = v
            out[f.name] = a
    return dataclasses.replace(sd, **out)


def make_scene():
    """The workload's scene as the XYZ renderer takes it: XYZ albedos only (the
    generator also makes 31-bin albedo spectra for the spectral modes, 122 MB
    for this scene, which an XYZ render never reads)."""
    from xyz_b200 import scenes
    sd = scenes.spheres_scene(level=7, n_spheres=3, seed=SEED)
    sd.albedo_spd = None
    sd.light_power_spd = None
    return sd


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(device_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


# ----------------------------------------------------------------- CPU arms
def reference_lib():
    """The reference's own renderer built from its sources (oracle/_ref), else
    the C restatement (oracle/_port)."""
    from oracle import refbind
    if refbind.fast_ref_available():
        return refbind.RefLib(pinhole=True, fast=True), "reference"
    if refbind.ref_available(pinhole=True):
        return refbind.RefLib(pinhole=True), "reference"
    if not refbind.port_available():
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "port"], check=True,
                       stdout=subprocess.DEVNULL)
    return refbind.PortLib(), "port"


def cpu_setup(sd):
    lib, kind = reference_lib()
    threads = lib.max_threads()
    t0 = time.perf_counter()
    lib.scene_create(sd)
    build_s = time.perf_counter() - t0
    lib.set_camera(sd.camera, W_PIX, H_PIX)
    lib.set_path_params(max_depth=MAX_DEPTH)
    return lib, kind, threads, build_s


def cpu_plan(lib, threads, target_s):
    """(rows, spp): a centre band of rows and a number of samples per pixel
    that take about target_s seconds on `threads` threads."""
    y0 = H_PIX // 2 - 32
    t0 = time.perf_counter()
    lib.render(1, seed=SEED + 7, y0=y0, y1=y0 + 64, nthreads=threads)
    dt = max(time.perf_counter() - t0, 1e-3)
    rows = int(64 * target_s / dt)
    if rows <= H_PIX:
        return max(16, rows), 1
    spp = int(math.ceil(target_s / (dt * H_PIX / 64)))
    return H_PIX, max(1, min(SPP, spp))


def cpu_sample(lib, threads, rows, spp, s0):
    y0 = max(0, H_PIX // 2 - rows // 2)
    t0 = time.perf_counter()
    lib.render(spp, seed=SEED, s0=s0, y0=y0, y1=y0 + rows, nthreads=threads)
    dt = time.perf_counter() - t0
    return rows * W_PIX * spp / dt / 1e6, dt


def cpu_baseline(sd, target_s=12.0):
    lib, kind, threads, build_s = cpu_setup(sd)
    rows, spp = cpu_plan(lib, threads, target_s)
    v, dt = cpu_sample(lib, threads, rows, spp, 0)
    # the same renderer on one host thread: the same rows, one sample per pixel
    rows1, spp1 = rows, 1
    v1, dt1 = cpu_sample(lib, 1, rows1, spp1, 0)
    return {"value": round(v, 4), "unit": UNIT, "cores": threads, "kind": kind,
            "build": getattr(lib, "build", "-O2"),
            "sample": f"{spp} spp over {rows} of 1024 rows (centre band) of the same scene and "
                      f"camera, {rows * W_PIX * spp} paths in {dt:.1f} s; tree build {build_s:.1f} s untimed",
            "single_core_value": round(v1, 4),
            "single_core_sample": f"{spp1} spp over the same {rows1} rows, "
                                  f"{rows1 * W_PIX * spp1} paths in {dt1:.1f} s on 1 thread"}


def run_reference_arm(args, rank):
    if rank != 0:
        return
    sd = make_scene()
    lib, kind, threads, build_s = cpu_setup(sd)
    per_step_s = max(2.0, min(15.0, 100.0 / max(1, args.steps + args.warmup)))
    rows, spp = cpu_plan(lib, threads, per_step_s)
    for w in range(args.warmup):
        cpu_sample(lib, threads, max(16, rows // 4), 1, 1000 + w)
    times = []
    for k in range(args.steps):
        _, dt = cpu_sample(lib, threads, rows, spp, k * spp)
        times.append(dt)
    total = sum(times)
    value = rows * W_PIX * spp * args.steps / total / 1e6
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * total / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene generator)", "config": workload_config(),
        "impl": "reference",
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads, "kind": kind,
                         "build": getattr(lib, "build", "-O2"),
                         "sample": f"each step: {spp} spp over {rows} of 1024 rows (centre band), "
                                   f"{rows * W_PIX * spp} paths; tree build {build_s:.1f} s untimed"},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- GPU arm
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_bf16_sustained():
    """Dense bf16 TFLOP/s of a seconds-long cuBLAS loop (MEASURED_PEAKS.json),
    the denominator for a kernel timed inside a long step; else the fallback."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        if "bf16_tflops_sustained" in d:
            return float(d["bf16_tflops_sustained"]), "measured"
    return 1400.0, "fallback"


def adjoint_bench(steps: int, warmup: int):
    """Differentiable-rendering iteration on the 19,392-triangle room: render
    512 x 512 x 32 spp, L2 loss gradient to a target, 32 spp path-replay adjoint
    on the next 32 samples, max depth 6, Russian roulette off.  Returns
    ms per iteration (primal + adjoint, CUDA events, each iteration enqueued
    behind a lead kernel) and its split."""
    import torch
    from xyz_b200 import api, diff, scenes
    W = H = 512
    spp = 32
    ds = scenes.diff_scene()
    with api.Scene(ds.scene) as s:
        R = diff.Renderer(s, ds.scene.camera, W, H, spp, adjoint_spp=spp, adjoint_offset=spp,
                          max_depth=6, rr_threshold=0.0)
        s.set_materials(ds.target_albedo, ds.target_emission)
        target = R.render()
        s.set_materials(ds.albedo, ds.emission)

        def iteration():
            img = R.render()
            d_img = 2.0 * (img - target)
            return R.gradient(d_img)

        for _ in range(warmup):
            iteration()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        prim = adj = 0.0
        for _ in range(steps):
            # the iteration is enqueued behind a lead kernel, so the host's
            # enqueueing time does not show as idle GPU time between the events
            gpu_lead(20.0)
            ev[0].record()
            img = R.render()
            d_img = 2.0 * (img - target)
            ev[1].record()
            R.gradient(d_img)
            ev[2].record()
            torch.cuda.synchronize()
            prim += ev[0].elapsed_time(ev[1])
            adj += ev[1].elapsed_time(ev[2])
        samples = W * H * spp
        return {"ms_per_iter": round((prim + adj) / steps, 3), "primal_ms": round(prim / steps, 3),
                "adjoint_ms": round(adj / steps, 3),
                "adjoint_msamples_per_s": round(samples / (adj / steps / 1000.0) / 1e6, 1),
                "config": "room + 3 displaced level-4 spheres, 19,392 triangles (one material each), "
                          "512x512, 32 spp primal + 32 spp replay adjoint (next 32 samples), "
                          "max depth 6, Russian roulette off, gradients of albedo (3 per triangle) "
                          "and emission (32 light triangles)"}


def batch_bench(steps: int, warmup: int):
    """Batched workload: 64 scenes (seeds 0-63, 1k-500k triangles, displaced
    icospheres and box stacks), resolutions in {128,256,512,1024}^2, 4-64 spp,
    max depth 8, in one graph launch after autotuning (the wave and bounce
    loops are conditional nodes the device runs); against the same 64
    renders issued one xyzgpu_render call after another.  Device time."""
    import torch
    from xyz_b200 import api, scenes
    work = scenes.batch_workload(64)
    sc = [api.Scene(e.scene) for e in work]
    try:
        paths = sum(e.width * e.height * e.spp for e in work)
        jobs = [api.BatchJob(s, e.scene.camera, e.width, e.height, e.spp, seed=k, max_depth=e.max_depth)
                for k, (s, e) in enumerate(zip(sc, work))]
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def singles():
            for k, (s, e) in enumerate(zip(sc, work)):
                s.render(e.scene.camera, e.width, e.height, e.spp, seed=k, max_depth=e.max_depth,
                         film=jobs[k].film)

        singles()
        ev0.record()
        singles()
        ev1.record()
        torch.cuda.synchronize()
        single_ms = ev0.elapsed_time(ev1)
        with api.Batch(jobs) as b:
            chosen = b.autotune(trials=1, probe_spp=4)
            for _ in range(warmup):
                b.launch()
            torch.cuda.synchronize()
            ev0.record()
            for _ in range(steps):
                b.launch()
            ev1.record()
            torch.cuda.synchronize()
            ms = ev0.elapsed_time(ev1) / steps
            st = b.stats()
        return {"msamples_per_s": round(paths / ms / 1e3, 1), "ms_per_launch": round(ms, 3),
                "sequential_renders_msamples_per_s": round(paths / single_ms / 1e3, 1),
                "paths": paths, "triangles": int(sum(e.scene.n_tris for e in work)),
                "waves": st["waves"], "graph_nodes": st["graph_nodes"],
                "graph_top_nodes": st["graph_top_nodes"], "host_calls_per_launch": 1,
                "device_kernel_launches_per_launch": st["kernel_launches_per_launch"], "autotuned": chosen,
                "config": "64 scenes (seeds 0-63), 1k-500k triangles log-uniform, displaced icospheres "
                          "(odd) and box stacks (even), 128^2..1024^2, 4-64 spp, max depth 8"}
    finally:
        for s in sc:
            s.close()


GUIDE_CAMERA = ((0.0, 1.5, 1.2), (0.0, 1.1, -2.0), 60.0)


def relmse_estimator(half_a, half_b):
    """relMSE on Y against a reference given as two independent half
    estimates A and B (arrays of Y, numpy or torch): the reference is
    R = (A + B) / 2, the image is exposed so that mean(R) = 1, and
    relMSE(I) = mean((I - R)^2 / (R^2 + 1e-2)) - mean(Var(R) / (R^2 + 1e-2)) with
    Var(R) = (A - B)^2 / 4, which removes the reference's own noise from the
    measured error (for an image I independent of A and B the result is an
    unbiased estimate of mean(Var(I) / (R^2 + 1e-2))).  Returns (relmse, the
    subtracted noise term, the exposure scale); relmse takes the image's Y."""
    ref_y = (half_a + half_b) / 2
    scale = 1.0 / float(ref_y.mean())
    ry = ref_y * scale
    den = ry ** 2 + 1e-2
    ref_noise = float((((half_a - half_b) * scale) ** 2 / 4 / den).mean())

    def relmse(img_y):
        return float((((img_y * scale - ry) ** 2) / den).mean()) - ref_noise

    return relmse, ref_noise, scale


GUIDE_FP64_FIXTURE = os.path.join(ROOT, "tests", "golden", "guide_reference_fp64.npz")


def fp64_cpu_reference(rows, gpu_ref_y, gpu_ref_spp):
    """The converged image of the FP64 CPU oracle (65,536 samples per pixel
    of the oracle's restatement of the reference estimator, sums in double,
    on the 32 x 32 pixel grid x, y = 16, 48, ..., 1008 of the same scene and
    camera; tests/golden/make_guide_reference.py): how the GPU reference
    (`gpu_ref_y`: Y of the measured rows, a torch tensor) agrees with it per
    pixel, and relmse(img) of an image of the measured rows against it on
    those pixels (exposed and with the reference's own noise removed as in
    relmse_estimator).  None when the fixture is absent."""
    if not os.path.exists(GUIDE_FP64_FIXTURE):
        return None
    fx = np.load(GUIDE_FP64_FIXTURE)
    row_of = {y: i for i, y in enumerate(range(*rows))}
    if not all(int(y) in row_of for y in fx["py"]):
        return None
    ri = np.array([row_of[int(y)] for y in fx["py"]])
    px = np.asarray(fx["px"])
    n = int(fx["spp"])
    mean_c = fx["acc"][:, 1] / n
    var_mean_c = np.maximum(fx["acc"][:, 3] / n - mean_c ** 2, 0.0) / n
    scale = 1.0 / mean_c.mean()
    ry = mean_c * scale
    den = ry ** 2 + 1e-2
    noise = float((var_mean_c * scale ** 2 / den).mean())
    g = gpu_ref_y.cpu().numpy()[ri, px]
    z = (g - mean_c) / np.sqrt(np.maximum(fx["acc"][:, 3] / n - mean_c ** 2, 0.0) * (1.0 / gpu_ref_spp + 1.0 / n)
                               + 1e-30)

    def relmse(img):
        iy = img[..., 1].cpu().numpy()[ri, px] * scale
        return float(((iy - ry) ** 2 / den).mean()) - noise

    return {"relmse": relmse,
            "summary": {"pixels": int(px.size), "spp": n, "sums": "float64",
                        "tracer": "CPU oracle (C restatement of the reference's estimator), seed 77",
                        "own_relmse": round(noise, 5),
                        "gpu_reference_vs_oracle": {
                            "mean_y_ratio": round(float(g.mean() / mean_c.mean()), 5),
                            "fraction_beyond_3_sigma": round(float((np.abs(z) > 3).mean()), 4)}}}


GUIDE_SETTINGS = dict(train_bounces=5, guide_bounces=9, alpha=0.5, steps_per_pass=512, batch_size=16384)
# forward flops of one guide query, 2 (192 * 64 + 3 * 64 * 64 + 64 * 40)
GUIDE_QUERY_FLOPS = 2 * (192 * 64 + 3 * 64 * 64 + 64 * 40)


def guide_bench(band: int = 32, ref_spp: int = 65536, pass_spp: int = 64, plan_spp: int = 2048,
                max_seconds: float = 30.0, guide_cfg=None, variants=(), repeats: int = 3):
    """Time to relative MSE 0.01, guided vs plain, on the indirect-lit room
    (196,146 triangles; light only through a 0.1 m gap), 1024 x 1024 camera,
    max depth 10, Russian roulette 0.2.  The error is measured on `band` image
    rows spread evenly over the frame (rows 16, 48, ..., 1008 for 32: every
    32nd row; both tracers render exactly those rows of the full image, the
    same pixels and paths as a full render), against a `ref_spp` plain render
    of those rows (float64 accumulation),
    relMSE = mean((Y - Y_ref)^2 / (Y_ref^2 + 1e-2)) with the image exposed so
    that the rows' mean reference Y is 1, minus the reference's own share of
    that error (estimated from the difference of its two independent halves
    A and B: var(Y_ref) = E[(A - B)^2] / 4).  Both tracers render passes of
    `pass_spp` until the error reaches 0.01; each pass is timed with CUDA
    events around the render call (the error evaluation is not timed).  The
    reported time is the sum of the pass times (the guided tracer's training
    passes included); passes x median pass time is reported beside it.  Each
    tracer's buffers are allocated before its first timed pass (the guide's by
    xyzgpu_guide_reserve, as the plain tracer's wave buffers are by the
    untimed warm-up).  The guided tracer trains during the first 25 % of
    a planned `plan_spp` (Adam steps after every training pass); as in path
    guiding practice the training passes' samples, drawn while the guide is
    still immature, are left out of the image, but their time counts.  Plain
    and guided runs alternate `repeats` times and each tracer reports its
    faster run.  A tracer that has not reached 0.01 after `max_seconds`
    reports the time extrapolated from relMSE ~ 1 / spp.  `variants`: further guide settings (dicts of
    guide_cfg overrides, optionally with their own plan_spp) measured against
    the same reference and plain run."""
    import torch
    from xyz_b200 import api, scenes
    W = H = 1024
    step = H // band
    rows = (step // 2, H, step)
    row_list = list(range(*rows))
    depth = 10
    sd = scenes.occluded_room()
    cam = scenes.Camera.with_fov(*GUIDE_CAMERA, pinhole=True)
    cfg = dict(GUIDE_SETTINGS)
    cfg.update(guide_cfg or {})
    with api.Scene(sd) as s:
        halves = [torch.zeros((band, W, 3), dtype=torch.float64, device="cuda") for _ in range(2)]
        chunk = 4096
        t0 = time.perf_counter()
        for k in range(0, ref_spp, chunk):
            f = s.render(cam, W, H, chunk, seed=99, spp_offset=k, max_depth=depth, rows=rows)
            halves[(k // chunk) & 1] += f[row_list].double()
        torch.cuda.synchronize()
        ref_s = time.perf_counter() - t0
        a, b = (h[..., 1] / (ref_spp // 2) for h in halves)
        relmse_y, ref_noise, _ = relmse_estimator(a, b)

        def relmse(img):
            return relmse_y(img[..., 1])

        cpu_ref = fp64_cpu_reference(rows, (a + b) / 2, ref_spp)

        def run(render_pass, train_passes=0):
            acc = torch.zeros((band, W, 3), dtype=torch.float64, device="cuda")
            film = torch.zeros((H, W, 3), dtype=torch.float32, device="cuda")
            times, p, e = [], 0, float("inf")
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            while True:
                torch.cuda.synchronize()
                gpu_lead(5.0)
                e0.record()
                render_pass(p, film)
                e1.record()
                torch.cuda.synchronize()
                times.append(e0.elapsed_time(e1) * 1e-3)
                p += 1
                if p <= train_passes:
                    continue
                acc += film[row_list].double()
                e = relmse(acc / ((p - train_passes) * pass_spp))
                tr, rd = times[:train_passes], times[train_passes:]
                robust = len(tr) * (statistics.median(tr) if tr else 0.0) + len(rd) * (statistics.median(rd) if rd else 0.0)
                total = sum(times)
                out = {"spp": p * pass_spp, "image_spp": (p - train_passes) * pass_spp, "relmse": round(e, 5),
                       "passes": p, "training_passes": train_passes,
                       "training_seconds": round(sum(tr), 4),
                       "median_pass_ms": round(statistics.median(rd if rd else tr) * 1e3, 3),
                       "passes_times_median_seconds": round(robust, 3)}
                if cpu_ref is not None and (e <= 0.01 or total > max_seconds):
                    out["relmse_vs_fp64_cpu_oracle"] = round(cpu_ref["relmse"](acc / ((p - train_passes) * pass_spp)), 5)
                if e <= 0.01:
                    return {"seconds": round(total, 3), "reached": True} | out
                if total > max_seconds:
                    return {"seconds": round(total * e / 0.01, 3), "reached": False} | out

        def plain_pass(p, film):
            s.render(cam, W, H, pass_spp, seed=1, spp_offset=p * pass_spp, max_depth=depth, film=film, rows=rows)

        # untimed warm-up of both tracers (module loading, first-use allocations)
        s.render(cam, W, H, pass_spp, seed=7, max_depth=depth, rows=rows)
        with api.Guide(s, **cfg) as g0:
            g0.reserve(W * band * pass_spp, train=True)
            g0.render(cam, W, H, pass_spp, seed=7, max_depth=depth, rows=rows, train=True)
        torch.cuda.synchronize()
        def guided_run(gcfg, gplan):
            train_passes = max(1, (gplan // 4) // pass_spp)
            with api.Guide(s, **gcfg) as g:
                g.reserve(W * band * pass_spp, train=True)

                def guided_pass(p, film):
                    g.render(cam, W, H, pass_spp, seed=1, spp_offset=p * pass_spp, max_depth=depth, film=film,
                             rows=rows, train=p < train_passes)

                res = run(guided_pass, train_passes)
                info = gcfg | g.stats() | {"training_spp": train_passes * pass_spp}
                # one profiled pass of the trained guide: the network's share
                # and its rate (queries = extension-queue entries of the
                # guided bounces; the last bounce and those past guide_bounces
                # run no inference)
                g.render(cam, W, H, pass_spp, seed=5, max_depth=depth, rows=rows, profile=1)
                pr = s.render_profile()
                nb = min(depth - 1, gcfg.get("guide_bounces", depth))
                queries = sum(pr["ext_rays_by_iter"][:nb])
                gms = pr["ms"]["guide"]
                tf = queries * GUIDE_QUERY_FLOPS / (gms * 1e-3) / 1e12 if gms > 0 else None
                bf16, bf16_kind = measured_bf16_sustained()
                info["profiled_pass"] = {
                    "ms": {k: round(v, 3) for k, v in pr["ms"].items()},
                    "guide_queries": queries,
                    "guide_inference_tflops": round(tf, 1) if tf else None,
                    "guide_inference_frac_of_bf16_sustained": round(tf / bf16, 4) if tf else None,
                    "bf16_sustained_tflops": bf16, "bf16_peak_source": bf16_kind}
                return res, info

        def importon_run(particles):
            """The reference's non-learned guide: the light-importance map
            (particles traced and sorted into the grid, CUDA-event time of the
            build included in the total), then importance-driven passes."""
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            with api.Importons(s, particles=particles, seed=3) as m:
                e1.record()
                torch.cuda.synchronize()
                build_s = e0.elapsed_time(e1) * 1e-3

                def imp_pass(p, film):
                    m.render(cam, W, H, pass_spp, seed=1, spp_offset=p * pass_spp, max_depth=depth, film=film,
                             rows=rows)

                res = run(imp_pass)
                n_imp = m.count()
            res["map_seconds"] = round(build_s, 4)
            res["seconds"] = round(res["seconds"] + build_s, 3)
            return res | {"particles": particles, "importons": n_imp}

        plains, guideds = [], []
        for _ in range(max(1, repeats)):
            plains.append(run(plain_pass))
            guideds.append(guided_run(cfg, plan_spp))
        plain = min(plains, key=lambda r: r["seconds"])
        guided, ginfo = min(guideds, key=lambda r: r[0]["seconds"])
        importon = [importon_run(n) for n in (100000, 1000000)]
        more = []
        for v in variants:
            v = dict(v)
            vplan = v.pop("plan_spp", plan_spp)
            r, info = guided_run(cfg | v, vplan)
            more.append({"guide": info, "guided": r, "speedup": round(plain["seconds"] / r["seconds"], 2)})
    out = {"metric": "seconds to relMSE 0.01 (lower is better)",
           "plain": plain, "guided": guided,
           "speedup": round(plain["seconds"] / guided["seconds"], 2),
           "guide": ginfo,
           "importance_driven": [r | {"speedup": round(plain["seconds"] / r["seconds"], 2)} for r in importon],
           "runs": {"plain_seconds": [r["seconds"] for r in plains],
                    "guided_seconds": [r[0]["seconds"] for r in guideds],
                    "guided_spp": [r[0]["spp"] for r in guideds]},
           "reference": {"spp": ref_spp, "seconds": round(ref_s, 2), "own_relmse": round(ref_noise, 5),
                         "tracer": "plain GPU path tracer, float64 sums",
                         "fp64_cpu_oracle": cpu_ref["summary"] if cpu_ref else None},
           "time": "sum of the CUDA-event times of every pass (training passes included)",
           "config": f"occluded room, 196,146 triangles, 1024x1024 camera, {band} rows spread over the frame "
                     f"(rows {rows[0]}, {rows[0] + rows[2]}, ..., {row_list[-1]}), max depth 10, "
                     f"Russian roulette 0.2, passes of {pass_spp} spp, exposure: mean reference Y = 1"}
    if more:
        out["variants"] = more
    return out


def pinhole_rays(cam, width, height, n, rng):
    """n pinhole rays through uniformly jittered random pixels of a width x
    height image of `cam` (its eye, look-at point and vertical field of view
    film_size / focal_length), as rows o.xyz, tmin, d.xyz, tmax."""
    eye = np.asarray(cam.eye, np.float64)
    fwd = np.asarray(cam.at, np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, (0.0, 1.0, 0.0))
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    pix = rng.integers(0, width * height, n)
    x = ((pix % width) + rng.random(n)) / width
    y = ((pix // width) + rng.random(n)) / height
    film = cam.film_size
    d = (np.outer((x - 0.5) * film * width / height, right) + np.outer((0.5 - y) * film, up) +
         cam.focal_length * fwd)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.empty((n, 8), np.float32)
    r[:, 0:3] = eye
    r[:, 3] = 1e-5
    r[:, 4:7] = d
    r[:, 7] = np.inf
    return r


def cosine_bounce_rays(sd, prim, hits, n, rng):
    """n rays leaving recorded hit points (drawn with replacement from the
    primary rays that hit) in cosine-weighted directions about the hit
    triangle's geometric normal, turned to face the incoming ray."""
    ids = hits[:, 3].view(np.int32)
    hit = np.flatnonzero(ids >= 0)
    sel = rng.choice(hit, n, replace=True)
    tri = ids[sel] >> 1
    o = prim[sel, 0:3].astype(np.float64) + hits[sel, 0:1].astype(np.float64) * prim[sel, 4:7]
    v = sd.positions[sd.tris[tri]].astype(np.float64)
    ng = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
    ng /= np.linalg.norm(ng, axis=1, keepdims=True)
    ng[np.einsum("ij,ij->i", ng, prim[sel, 4:7]) > 0] *= -1.0
    a = np.where(np.abs(ng[:, 0:1]) > 0.9, [[0.0, 1.0, 0.0]], [[1.0, 0.0, 0.0]])
    t1 = np.cross(ng, a)
    t1 /= np.linalg.norm(t1, axis=1, keepdims=True)
    t2 = np.cross(ng, t1)
    u1, u2 = rng.random(n), rng.random(n)
    rr, ph = np.sqrt(u1), 2.0 * np.pi * u2
    d = (t1 * (rr * np.cos(ph))[:, None] + t2 * (rr * np.sin(ph))[:, None] +
         ng * np.sqrt(np.maximum(0.0, 1.0 - u1))[:, None])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.empty((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = 1e-5
    r[:, 4:7] = d
    r[:, 7] = np.inf
    return r


def trace_micro_bench(scene, sd, n=1 << 24, seed=0, reps=5):
    """Closest-hit throughput of xyzgpu_trace_closest on 2^24 rays of the
    workload's scene: half pinhole camera rays, half cosine bounces from
    recorded hit points of those (seed 0), resident on the device (512 MB of
    rays, larger than L2).  CUDA-event time per launch (median of reps), work
    per ray from one counted launch."""
    import torch
    rng = np.random.default_rng(seed)
    half = n // 2
    prim = pinhole_rays(sd.camera, W_PIX, H_PIX, half, rng)
    rays = torch.from_numpy(prim).cuda()
    hits = torch.empty((half, 4), dtype=torch.float32, device="cuda")
    scene.trace_device(rays, hits)
    h = hits.cpu().numpy()
    bounce = cosine_bounce_rays(sd, prim, h, half, rng)
    all_rays = torch.from_numpy(np.concatenate([prim, bounce])).cuda()
    all_hits = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    del rays, hits
    peak, peak_kind = measured_peaks()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(r, hts):
        scene.trace_device(r, hts)
        out = []
        for _ in range(reps):
            e0.record()
            scene.trace_device(r, hts)
            e1.record()
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1))
        return statistics.median(out)

    res = {}
    for name, lo, hi in (("all", 0, n), ("primary", 0, half), ("bounce", half, n)):
        r, hts = all_rays[lo:hi], all_hits[lo:hi]
        ms = timed(r, hts)
        c = scene.trace_device(r, hts, counted=True)
        nr = max(1, c["rays"])
        algo = (RAY_IO_BYTES * c["rays"] + NODE_BYTES * c["nodes_visited"] +
                (REF_BYTES + TRI_BYTES_ALGO) * c["tri_tests"]) / nr
        gbs = algo * (hi - lo) / (ms * 1e-3) / 1e9
        res[name] = {"rays": hi - lo, "ms": round(ms, 3), "mrays_per_s": round((hi - lo) / ms / 1e3, 1),
                     "hit_rate": round(c["hits"] / nr, 4),
                     "per_ray": {"nodes": round(c["nodes_visited"] / nr, 2),
                                 "leaves": round(c["leaves_visited"] / nr, 2),
                                 "tri_tests": round(c["tri_tests"] / nr, 2)},
                     "algorithmic_bytes_per_ray": round(algo, 1),
                     "achieved_gbs": round(gbs, 1), "frac_of_hbm": round(gbs / peak, 4)}
    res["peak_gbs"] = peak
    res["peak_source"] = peak_kind
    res["config"] = ("2^24 rays of the workload's scene and kd-tree: 2^23 pinhole camera rays through "
                     "jittered random pixels, 2^23 cosine-weighted bounces from their recorded hit points "
                     "(seed 0); device-resident, xyzgpu_trace_closest")
    del all_rays, all_hits
    return res


def guide_profile_case():
    """The guide's kernels on a small case for ncu: one Adam step on 65,536
    synthetic training rows (k_guide_gradient), then one guided 64-spp pass
    over rows 496-528 of the occluded room at 1024 x 1024 (k_guide_infer at
    every bounce; the first launch sees the 2,097,152 camera hits)."""
    import numpy as np
    import torch
    from xyz_b200 import api, scenes
    W = H = 1024
    rows = (H // 2 - 16, H // 2 + 16)
    sd = scenes.occluded_room()
    cam = scenes.Camera.with_fov(*GUIDE_CAMERA, pinhole=True)
    rng = np.random.default_rng(0)
    n = 1 << 16
    rec = np.zeros((n, 10), np.float32)
    rec[:, 0:3] = rng.uniform(-2.0, 2.0, (n, 3))
    for c in (3, 6):
        v = rng.normal(size=(n, 3))
        rec[:, c:c + 3] = v / np.linalg.norm(v, axis=1, keepdims=True)
    rec[:, 9] = rng.exponential(1.0, n)
    with api.Scene(sd) as s, api.Guide(s, **GUIDE_SETTINGS) as g:
        g.train_step(torch.from_numpy(rec).cuda())
        f = g.render(cam, W, H, 64, seed=5, max_depth=10, rows=rows)
        torch.cuda.synchronize()
        print(json.dumps({"guide_profile_case": "ok", "film_sum": float(f.sum())}))


def adjoint_profile_case():
    """The adjoint's kernels on a small case for ncu: one primal render and
    one path-replay adjoint of the 19,392-triangle room at 256 x 256, 8 spp
    each, max depth 6 (the benchmark's iteration at a sixteenth of its
    samples)."""
    import torch
    from xyz_b200 import api, diff, scenes
    ds = scenes.diff_scene()
    with api.Scene(ds.scene) as s:
        R = diff.Renderer(s, ds.scene.camera, 256, 256, 8, adjoint_spp=8, adjoint_offset=8, max_depth=6,
                          rr_threshold=0.0)
        s.set_materials(ds.albedo, ds.emission)
        img = R.render()
        g = R.gradient(2.0 * img)
        torch.cuda.synchronize()
        print(json.dumps({"adjoint_profile_case": "ok", "film_sum": float(img.sum()),
                          "grad_norm": float(sum(float(t.double().norm()) for t in g if t is not None))}))


def gpu_lead(ms: float = 100.0):
    """Occupies the current stream for about `ms` (torch's spin kernel,
    outside any timed region) so that the host can enqueue the timed work
    behind it: a host thread descheduled while enqueueing then cannot leave
    the GPU idle inside the timed region."""
    import torch
    torch.cuda._sleep(int(ms * 1e-3 * 1.9e9))


def profiled_traffic(key: str = "dram_bytes_per_ray"):
    """Bytes per traced ray of the trace kernel (`key`: dram_bytes_per_ray or
    l2_bytes_per_ray) from the committed ncu summary
    (profiles/trace_queue_spheres1m.txt), if present."""
    p = os.path.join(ROOT, "profiles", "trace_queue_spheres1m.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def measure_l2_copy_gbs(mib: int = 32, reps: int = 100):
    """L2 bandwidth of a device copy whose buffers (2 x `mib` MiB) stay in
    the 126 MB L2: `reps` copies captured in one CUDA graph (so that launch
    gaps do not count), read + write bytes over the graph's CUDA-event time,
    best of three replays."""
    import torch
    n = mib * (1 << 20) // 4
    a = torch.ones(n, device="cuda")
    b = torch.empty_like(a)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(3):
            b.copy_(a)
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(reps):
            b.copy_(a)
    best = 0.0
    for _ in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * a.nbytes * reps / (e0.elapsed_time(e1) * 1e-3) / 1e9)
    del g
    return best


def run_gpu_arm(args, rank, world):
    import torch
    from xyz_b200 import api

    dev = torch.cuda.current_device()
    dist = None
    if world > 1:
        import torch.distributed as dist

    sd = make_scene()
    scene = api.Scene(sd, **WORKLOAD_BUILD)
    stats = scene.stats()
    cam = sd.camera
    film = torch.zeros((H_PIX, W_PIX, 3), dtype=torch.float32, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    from xyz_b200.distributed import render_and_reduce, weak_range
    offset, _ = weak_range(SPP, rank)

    def step(s_off, profile=0):
        render_and_reduce(lambda first, count: scene.render(
            cam, W_PIX, H_PIX, count, seed=SEED, spp_offset=first, max_depth=MAX_DEPTH,
            film=film, profile=profile), s_off, SPP)
        flush.zero_()

    for _ in range(args.warmup):
        step(offset)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()

    clocks = ClockSampler(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t_wall = time.perf_counter()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    # the K steps are enqueued back to back behind a lead kernel, with no
    # host synchronisation in between, so the device time does not depend on
    # host scheduling
    gpu_lead()
    ev0.record()
    for k in range(args.steps):
        step(offset)
    ev1.record()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    wall_ms = 1000 * (time.perf_counter() - t_wall)
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    samples_per_step = W_PIX * H_PIX * SPP
    value = samples_per_step * world * args.steps / (ms / 1000.0) / 1e6

    # per-kernel-class times and launch counts from one profiled step (CUDA
    # events around every launch), outside the timed region
    step(offset, profile=1)
    prof = scene.render_profile()
    ms_cls = {c: prof["ms"][c] * args.steps for c in api.KERNEL_CLASSES}
    n_cls = {c: prof["launches"][c] * args.steps for c in api.KERNEL_CLASSES}
    launches = scene.render_counters()["kernel_launches"] * args.steps
    # work per ray from one counted render (outside the timed region)
    step(offset, profile=2)
    cp = scene.render_profile()
    counters = scene.render_counters()
    ext_bytes = (cp["ext_rays"] * RAY_IO_BYTES + cp["ext_nodes"] * NODE_BYTES +
                 cp["ext_tri_tests"] * (REF_BYTES + TRI_BYTES_ALGO))
    sh_bytes = (cp["shadow_rays"] * RAY_IO_BYTES + cp["shadow_nodes"] * NODE_BYTES +
                cp["shadow_tri_tests"] * (REF_BYTES + TRI_BYTES_ALGO))
    trace_ms = (ms_cls["trace_extension"] + ms_cls["trace_shadow"]) / max(1, args.steps)
    trace_launches = (n_cls["trace_extension"] + n_cls["trace_shadow"]) / max(1, args.steps)
    peak, peak_kind = measured_peaks()
    achieved = (ext_bytes + sh_bytes) / (trace_ms / 1000.0) / 1e9 if trace_ms > 0 else 0.0
    rays = cp["ext_rays"] + cp["shadow_rays"]
    per_ray_traffic = profiled_traffic()
    traffic = None
    if per_ray_traffic is not None and trace_launches:
        traffic = per_ray_traffic * rays / trace_launches
    roofline = {
        "bound": "hbm", "kernel": "k_trace_queue (extension + shadow closest hit)",
        "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
        "frac": round(achieved / peak, 4), "peak_source": peak_kind,
        "traffic": traffic,
        "algorithmic_bytes_per_ray": round((ext_bytes + sh_bytes) / max(1, rays), 1),
        "per_ray": {"nodes": round((cp["ext_nodes"] + cp["shadow_nodes"]) / max(1, rays), 2),
                    "tri_tests": round((cp["ext_tri_tests"] + cp["shadow_tri_tests"]) / max(1, rays), 2),
                    "extension": {"rays": cp["ext_rays"],
                                  "nodes": round(cp["ext_nodes"] / max(1, cp["ext_rays"]), 2),
                                  "leaves": round(cp["ext_leaves"] / max(1, cp["ext_rays"]), 2),
                                  "tri_tests": round(cp["ext_tri_tests"] / max(1, cp["ext_rays"]), 2)},
                    "shadow": {"rays": cp["shadow_rays"],
                               "nodes": round(cp["shadow_nodes"] / max(1, cp["shadow_rays"]), 2),
                               "leaves": round(cp["shadow_leaves"] / max(1, cp["shadow_rays"]), 2),
                               "tri_tests": round(cp["shadow_tri_tests"] / max(1, cp["shadow_rays"]), 2)}},
        "rays_per_step": rays,
        "rays_by_iteration": {"extension": cp["ext_rays_by_iter"], "shadow": cp["shadow_rays_by_iter"]},
        "trace_ms_per_step": round(trace_ms, 3),
        "kernel_ms_per_step": {c: round(ms_cls[c] / max(1, args.steps), 3) for c in api.KERNEL_CLASSES},
        "kernel_share": {c: round(ms_cls[c] / max(1e-9, sum(ms_cls.values())), 4) for c in api.KERNEL_CLASSES},
        "grays_per_s": round(rays / (trace_ms / 1000.0) / 1e9, 3) if trace_ms > 0 else None,
    }
    # the traversal's working set (tree and triangles, about 100 MB) lives in
    # L2, so its roof is also stated against a copy that stays in L2
    l2_per_ray = profiled_traffic("l2_bytes_per_ray")
    if l2_per_ray is not None and trace_ms > 0:
        l2_peak = measure_l2_copy_gbs()
        l2_ach = l2_per_ray * rays / (trace_ms * 1e-3) / 1e9
        roofline["l2"] = {"achieved": round(l2_ach, 1), "peak": round(l2_peak, 1), "unit": "GB/s",
                          "frac": round(l2_ach / l2_peak, 4), "bytes_per_ray": l2_per_ray,
                          "peak_source": "measured in this run: 100 device copies of 2 x 32 MiB buffers (in L2) in one CUDA graph",
                          "bytes_source": "lts__t_bytes per ray, profiles/trace_queue_spheres1m.txt"}

    # end to end through the C ABI with host buffers: upload + build + render +
    # read back; the step's inputs and its film live in page-locked host memory
    e2e = None
    if not args.no_e2e:
        sd = pinned_scene(sd)
        h2d = sum(int(a.nbytes) for a in (sd.positions, sd.tris, sd.tri_mat, sd.albedo_xyz, sd.is_light))
        for extra in (sd.normals, sd.albedo_spd, sd.material_kind, sd.shininess):
            if extra is not None:
                h2d += int(extra.nbytes)
        host_film = torch.zeros((H_PIX, W_PIX, 3), dtype=torch.float32, pin_memory=True).numpy()
        torch.cuda.synchronize()
        # wall time per step (the leg includes host work: the scene arrays'
        # upload, the build's per-level reads, the film read-back); the value
        # uses the median step so that a host stall on a shared machine does
        # not stand for the path's cost; the total is reported beside it
        step_s, parts = [], []
        for k in range(args.steps):
            t0 = time.perf_counter()
            s2 = api.Scene(sd, **WORKLOAD_BUILD)
            t1 = time.perf_counter()
            try:
                s2.render(cam, W_PIX, H_PIX, SPP, seed=SEED, spp_offset=offset, max_depth=MAX_DEPTH,
                          film=host_film)
                t2 = time.perf_counter()
            finally:
                s2.close()
            torch.cuda.synchronize()
            t3 = time.perf_counter()
            step_s.append(t3 - t0)
            parts.append((t1 - t0, t2 - t1, t3 - t2))
        e2e_s, total_s = statistics.median(step_s), sum(step_s)
        if dist is not None:
            t = torch.tensor([e2e_s, total_s], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s, total_s = (float(x) for x in t.tolist())
        e2e = {"value": round(samples_per_step * world / e2e_s / 1e6, 3), "unit": UNIT,
               "host_memory": "page-locked (scene arrays and film)",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(host_film.nbytes),
               "median_step_ms": round(e2e_s * 1e3, 2),
               "median_ms": {name: round(statistics.median(p[i] for p in parts) * 1e3, 2)
                             for i, name in enumerate(("scene_create", "render_with_film_copies", "scene_destroy"))},
               "value_from_total_time": round(samples_per_step * world * args.steps / total_s / 1e6, 3),
               "includes": "scene upload + kd-tree build + render + film read-back, every step"}

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(sd)
    adjoint = batch = guiding = micro = None
    if rank == 0 and world == 1 and not args.no_extras:
        micro = trace_micro_bench(scene, sd)
        adjoint = adjoint_bench(args.steps, args.warmup)
        batch = batch_bench(args.steps, args.warmup)
        guiding = guide_bench()

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene generator)",
            "config": workload_config(),
            "kd_tree": {"nodes": stats["n_nodes"], "leaf_refs": stats["n_leaf_refs"],
                        "depth": stats["max_depth"], "build_ms": round(stats["build_ms"], 1)},
            "parallelism": f"sample-parallel x{world}", "waves_per_step": counters["waves"],
            "roofline": roofline, "cpu_baseline": base, "e2e": e2e, "gpu_launches": launches,
            "trace_micro": micro, "adjoint": adjoint, "batch": batch, "guiding": guiding,
            "clocks": clk, "wall_ms_timed_region": round(wall_ms, 1),
            "render_counters": counters,
        }
        print(json.dumps(line), flush=True)
    scene.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["xyz", "reference"], default="xyz")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the differentiable-rendering, batched-rendering and guided-rendering measurements")
    ap.add_argument("--spp", type=int, default=None,
                    help="samples per pixel per step (default 64; smaller for profiler captures)")
    ap.add_argument("--guide-profile-case", action="store_true",
                    help="run only the guide kernels' small profiling case (for ncu) and exit")
    ap.add_argument("--adjoint-profile-case", action="store_true",
                    help="run only the adjoint kernels' small profiling case (for ncu) and exit")
    args = ap.parse_args()
    if args.spp is not None:
        global SPP
        SPP = max(1, args.spp)
    if args.guide_profile_case:
        guide_profile_case()
        return
    if args.adjoint_profile_case:
        adjoint_profile_case()
        return
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    try:
        run_gpu_arm(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
