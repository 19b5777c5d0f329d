#!/usr/bin/env python
"""Benchmark of the B200 path tracer on the single-large-scene workload.

Workload (one "step" = one full frame): a seeded geodesic icosphere of
frequency 229 (1,048,820 triangles) radially displaced by 4-octave value
noise (amplitude 0.1), binned-SAH BVH, 64 metallic-roughness materials
hashed per triangle, 8 procedural 2048^2 textures with full mips (RGBA16F
atlas), 16 punctual lights, 512 emissive triangles, a 1024x512 analytic sky
with a sun disk; 1920x1080, 64 spp, max_bounces 12. Synthetic data.

metric: Msamples/s (camera paths per second, whole job). One process per
GPU; with N > 1 every rank renders its own frame (seed = rank): weak
scaling, no collective on the data path; the time is the max over ranks.

The JSON line also carries:
  e2e          the same metric through the C ABI with host buffers: per
               step, upload of the flat scene buffers from pinned host
               memory, tables and params, refine, resolve and the RGBA8
               readback, all inside the timed region;
  roofline     the trace kernel's algorithmic bytes (32 B per AABB tested,
               48 B per triangle tested, 192 B of attributes and 544 B of
               material record per shaded hit; counted by the counting build
               of the kernel) per launch over its CUDA-event duration, against
               the measured HBM copy bandwidth;
  cpu_baseline the CPU oracle (the same estimator, C++, all host threads) on
               a bounded sample of the same frame (N = 1, rank 0 only).
`--impl reference` times that CPU implementation alone: the reference's own
CPU tracer is an external Rust crate that cannot be built without a Rust
toolchain, so its C++ restatement stands in for it.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import __graft_entry__  # noqa: E402

BYTES_AABB, BYTES_TRI, BYTES_ATTR, BYTES_MAT = 32, 48, 192, 544


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--freq", type=int, default=229)
    ap.add_argument("--tex", type=int, default=2048)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-tolerance-plan", action="store_true",
                    help="skip timing the tolerance plan (four-wide closest hits) beside the exact one")
    ap.add_argument("--mode", default="auto", choices=["auto", "mega", "wave", "split"],
                    help="execution plan; auto = the library default")
    ap.add_argument("--slots", type=int, default=0, help="wavefront paths in flight (0 = default)")
    ap.add_argument("--no-tune", action="store_true", help="library default plan (no tuner, no fixed plan)")
    ap.add_argument("--tune", action="store_true", help="single workload: run the autotuner instead of the "
                    "fixed plan (tuner.LARGE_SCENE_PLAN, the plan the headline parity test runs)")
    ap.add_argument("--wave-items", type=int, default=0, help="wavefront paths per launch round (0: the plan's)")
    ap.add_argument("--trace-variant", type=int, default=-1, help="override the plan's traversal kernels "
                    "(0-2 local-memory stacks, 3-5 shared-memory short stacks)")
    ap.add_argument("--refill", type=int, default=0, help="override the plan's traversal refill threshold")
    ap.add_argument("--graphs", type=int, default=-1, choices=[-1, 0, 1],
                    help="override the plan's CUDA graphs (0: host-driven loop, e.g. for profilers that cannot "
                         "see kernels inside graphs with conditional nodes)")
    ap.add_argument("--shadow-postpone", type=int, default=-1, choices=[-1, 0, 1],
                    help="four-wide shadow walks park leaves until the warp has no node work (1) or not (0)")
    ap.add_argument("--l2-window", type=int, default=0, choices=[0, 1],
                    help="1: the traversal kernels mark the tree nodes they read as persisting L2 lines "
                         "(oxpt_diag_set_l2_window)")
    ap.add_argument("--ray-order", type=int, default=-1, choices=[-1, 0, 1, 2, 3],
                    help="reorder ray queues before the walks: 1 continuation rays (origin cell, direction "
                         "octant), 2 shadow rays (light, origin cell), 3 both")
    ap.add_argument("--nee-mask", type=int, default=-1, choices=[-1, 0, 1],
                    help="split plan's NEE results as per-slot visibility bits (1, default) or per-job records (0)")
    ap.add_argument("--nee-variant", type=int, default=-1, help="serve workload: the executor's NEE kernel "
                    "(-1: the serving executor's default, job-major)")
    ap.add_argument("--shadow-walk", default="auto", choices=["auto", "four", "binary"],
                    help="shadow rays' tree with --mode wave/split (auto: the library default, four-wide)")
    ap.add_argument("--requests", type=int, default=300, help="serve workload: requests in the stream")
    ap.add_argument("--rate", type=float, default=40.0, help="serve workload: Poisson arrival rate per second")
    ap.add_argument("--repeats", type=int, default=1, help="serve workload: independent streams (seeds) to run")
    ap.add_argument("--spp-scale", type=int, default=16,
                    help="serve workload: spp targets {4..1024} divided by this (one GPU cannot keep up with the "
                         "full stream)")
    ap.add_argument("--nrc-plain-training", default="0,16", help="nrc workload: comma list of counts of first "
                    "frames rendered as plain frames whose every path trains the cache (0: cache frames from the "
                    "first); one arm per pair with --nrc-frames-per-wave")
    ap.add_argument("--serve-idle-views", type=int, default=2, help="serve workload: closed sessions' views kept "
                    "per scene for the next request (0: every session makes and frees its own)")
    ap.add_argument("--frames", type=int, default=512, help="nrc workload: frames of 1 spp")
    ap.add_argument("--ref-spp", type=int, default=16384, help="nrc workload: spp of the plain reference")
    ap.add_argument("--nrc-scene", default="large", choices=["large", "cornell"], help="nrc workload: scene")
    ap.add_argument("--nrc-train-one-in", type=int, default=4, help="nrc workload: one training path in this many")
    ap.add_argument("--nrc-query-bounce", type=int, default=2, help="nrc workload: first bounce at which paths may "
                    "end into the cache")
    ap.add_argument("--nrc-spread", type=float, default=0.01, help="nrc workload: path-spread constant (0: every "
                    "path ends at the query bounce)")
    ap.add_argument("--nrc-frames-per-wave", default="1,4,8", help="nrc workload: comma list of cache frames traced "
                    "as one wavefront (one training step per wave); the line reports the fastest to 35 dB and "
                    "lists every one")
    ap.add_argument("--workload", default="single",
                    choices=["single", "batch", "cornell", "cornell16", "serve", "nrc", "prepare", "walk-sweep"],
                    help="single: the large scene (headline); batch: 64 mixed scenes in batched launches; "
                         "cornell: the reference's own Cornell benchmark shape (256^2, 8 bounces); "
                         "cornell16: the Cornell box at 256^2, 16 spp, 8 bounces, roulette from 3, seed 0, "
                         "device-timed with the CPU oracle beside it")
    ap.add_argument("--scenes", type=int, default=64, help="batch workload: number of scenes")
    ap.add_argument("--split", default="rows", choices=["rows", "replicas"],
                    help="single workload on N > 1 GPUs: rows = one frame in contiguous row tiles, one per rank, "
                         "with an NCCL all-gather of the accumulator tiles every step (strong scaling); replicas = "
                         "one frame per GPU, no collective (weak scaling)")
    return ap.parse_args()


def workload(pkg, a, seed=1):
    scene = pkg.Scene.icosphere(freq=a.freq, seed=seed, n_materials=64, n_textures=8, tex_size=a.tex,
                                n_punctual=16, n_emissive=512, material_mix=0)
    env = pkg.EnvironmentMap.sky(1024, 512, sun_dir=(0.3, 0.8, -0.5), sun_radiance=2000.0)
    return scene, env


def options(pkg, a, seed=0, spp=None):
    return pkg.RenderOptions(width=a.width, height=a.height, scene_camera=0,
                             path_trace=pkg.PathTraceOptions(samples_per_pixel=spp or a.spp, max_bounces=12,
                                                             rr_start=3, seed=seed))


def config(a, n_gpus, rows=False):
    par = (f"rows{n_gpus} (one frame in contiguous row tiles, one per GPU; NCCL all-gather of the accumulator "
           "tiles every step)" if rows else f"replicas{n_gpus} (one frame per GPU)")
    return {"workload": "single large scene, plain tracer", "triangles": 20 * a.freq * a.freq,
            "materials": 64, "textures": f"8 x {a.tex}^2 RGBA16F + mips", "punctual_lights": 16,
            "emissive_triangles": 512, "environment": "1024x512 RGBA32F sky + sun",
            "resolution": f"{a.width}x{a.height}", "spp": a.spp, "max_bounces": 12,
            "parallelism": par,
            "l2": "inputs (0.6 GB of scene buffers) larger than L2; no flush between steps"}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(pkg, oracle, prep, a, budget_s: float):
    """Oracle (same estimator, all host threads) on whole rows of the same
    frame at the same spp, sized to about `budget_s` of CPU work."""
    threads = os.cpu_count() or 1
    h, w = a.height, a.width
    probe_rows = min(h, max(16, 2 * threads))
    acc = np.zeros((h, w, 4), np.float32)
    t0 = time.perf_counter()
    oracle.dispatch(prep, prep.params, (0, 1, (h - probe_rows) // 2, probe_rows), acc, threads)
    per_path = (time.perf_counter() - t0) / (probe_rows * w)
    rows = int(max(1, min(h, budget_s / max(per_path * w * a.spp, 1e-9))))
    spp = a.spp
    if rows == 1 and per_path * w * a.spp > budget_s:
        spp = max(1, int(budget_s / (per_path * w)))
    y0 = max(0, h // 2 - rows // 2)
    acc[:] = 0
    t0 = time.perf_counter()
    oracle.dispatch(prep, prep.params, (0, spp, y0, rows), acc, threads)
    dt = time.perf_counter() - t0
    paths = rows * w * spp
    return {"value": paths / dt / 1e6, "unit": "Msamples/s", "cores": threads, "kind": "port",
            "sample": f"rows {y0}..{y0 + rows - 1} of the {w}x{h} frame at {spp} spp ({paths} paths, {dt:.1f} s)"}


def run_reference(a):
    """--impl reference: the reference estimator's CPU restatement (the
    reference's own CPU tracer is an external Rust crate that cannot be
    built here) on all host threads, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    __graft_entry__.build(load=False)
    pkg = __graft_entry__.load_package()
    pkg._native.select_host_only()  # CPU scene preparation only: no CUDA library in this process
    import oracle
    scene, env = workload(pkg, a)
    prep = pkg.prepare(scene, options(pkg, a), env)
    threads = os.cpu_count() or 1
    h, w = a.height, a.width
    acc = np.zeros((h, w, 4), np.float32)
    t0 = time.perf_counter()
    oracle.dispatch(prep, prep.params, (0, 1, h // 2, 2), acc, threads)
    per_row = (time.perf_counter() - t0) / 2
    rows = int(max(1, min(h, 4.0 / max(per_row, 1e-9))))
    times = []
    for i in range(a.warmup + a.steps):
        acc[:] = 0
        t0 = time.perf_counter()
        oracle.dispatch(prep, prep.params, (0, 1, (i * rows) % (h - rows + 1), rows), acc, threads)
        if i >= a.warmup:
            times.append(time.perf_counter() - t0)
    paths = rows * w
    value = paths * len(times) / sum(times) / 1e6
    line = {"metric": "Msamples/s", "value": value, "unit": "Msamples/s", "impl": "reference",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config(a, 1),
            "cpu_baseline": {"value": value, "unit": "Msamples/s", "cores": threads, "kind": "port",
                             "sample": f"{rows} rows x {w} px x 1 spp per step"},
            "e2e": {"value": value, "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


BATCH_RES = [(256, 256), (512, 512), (768, 432), (1024, 1024)]
BATCH_SPP = [16, 64, 256]


def batch_workload(pkg, a, seed=2):
    """64 seeded scenes: triangle counts log-uniform in [1e3, 5e5] (displaced
    icospheres and box fields alternating), the mixed material model (20%
    volume transmission, 20% clearcoat, 10% sheen), resolutions from
    {256^2, 512^2, 768x432, 1024^2} and spp from {16, 64, 256}."""
    rng = np.random.default_rng(seed)
    items = []
    for k in range(a.scenes):
        tris = float(np.exp(rng.uniform(np.log(1e3), np.log(5e5))))
        if k % 2 == 0:
            freq = max(8, int(round(np.sqrt(tris / 20.0))))
            scene = pkg.Scene.icosphere(freq=freq, seed=100 + k, n_materials=16, n_textures=2, tex_size=256,
                                        n_punctual=4, n_emissive=16, material_mix=1)
        else:
            scene = pkg.Scene.box_field(max(1, int(tris / 12)), seed=100 + k, material_mix=1)
        w, h = BATCH_RES[int(rng.integers(len(BATCH_RES)))]
        spp = BATCH_SPP[int(rng.integers(len(BATCH_SPP)))]
        items.append((scene, w, h, spp))
    return items


def run_batch(a):
    """Batched launches of the 64-scene workload against the same scenes
    refined one after another, each by its own plain refine."""
    import torch
    torch.cuda.set_device(0)
    __graft_entry__.build()
    pkg = __graft_entry__.load_package()
    from oxideav_render_vulkan_b200 import tuner
    items = batch_workload(pkg, a)
    env = pkg.EnvironmentMap.sky(256, 128)
    tracers = []
    for scene, w, h, spp in items:
        t = pkg.GpuPathTracer(0)
        t.set_environment(env)
        t.sync(scene, pkg.RenderOptions(width=w, height=h, scene_camera=0,
                                        path_trace=pkg.PathTraceOptions(samples_per_pixel=spp, max_bounces=8)))
        t.prepared()
        tracers.append(t)
    spps = [it[3] for it in items]
    paths = sum(it[1] * it[2] * it[3] for it in items)
    ex = pkg.GpuPathTracer(0)
    tune_log = []
    plan = tuner.tune_batch(tracers, ex, log=tune_log)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            for t in tracers:
                t.reset()
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(steps):
            for t in tracers:
                t.reset()
            for t in tracers:
                t.finish()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record()
            fn()
            for t in tracers:
                t.finish()
            e1.record()
            torch.cuda.synchronize()
            ms.append(max(e0.elapsed_time(e1), 1e3 * (time.perf_counter() - t0)))
        return ms

    batch_ms = timed(lambda: pkg.refine_batch(tracers, spps, executor=ex), a.steps, a.warmup)
    accs = [t.read_accum().copy() for t in tracers[:4]]
    serial_ms = timed(lambda: [t.refine(n) for t, n in zip(tracers, spps)], max(1, a.steps - 1), 1)
    same = all(np.array_equal(x.view(np.uint32), t.read_accum().view(np.uint32)) for x, t in zip(accs, tracers))
    value = paths / (statistics.median(batch_ms) / 1e3) / 1e6
    serial = paths / (statistics.median(serial_ms) / 1e3) / 1e6
    line = {"metric": "Msamples/s", "value": value, "unit": "Msamples/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": statistics.median(batch_ms), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batched {a.scenes} scenes (triangles log-uniform 1e3..5e5, mixed materials, "
                                   "resolutions 256^2..1024^2, spp 16/64/256)",
                       "paths_per_step": paths, "triangles": sum(int(it[0].triangle_count()) for it in items),
                       "timing": "host wall clock around the step (includes launch gaps), max with CUDA events"},
            "serial_plain_value": serial, "speedup_vs_serial": value / serial,
            "serial_matches_batch": same, "plan": tuner.describe(plan), "tuner_trials": len(tune_log)}
    print(json.dumps(line), flush=True)


def run_cornell(a):
    """The reference's pt_bench shape: procedural Cornell box, 256x256,
    8 bounces, roulette from bounce 3, seed 0, `--spp` samples (64 by
    default); refine alone and refine + image() readback."""
    import torch
    torch.cuda.set_device(0)
    __graft_entry__.build()
    pkg = __graft_entry__.load_package()
    from oxideav_render_vulkan_b200 import tuner
    spp = a.spp
    pt = pkg.GpuPathTracer(0)
    opts = pkg.RenderOptions(width=256, height=256,
                             path_trace=pkg.PathTraceOptions(samples_per_pixel=spp, max_bounces=8, rr_start=3,
                                                             seed=0))
    pt.sync(pkg.Scene.cornell(), opts)
    pt.prepared()
    tune_log = []
    plan = None
    if not a.no_tune:
        plan = tuner.tune(pt, spp=spp, repeats=3, log=tune_log)  # the measured frame itself: 13 ms a trial

    def measure(with_image):
        ms = []
        for i in range(a.warmup + a.steps):
            pt.reset()
            pt.finish()
            t0 = time.perf_counter()
            pt.refine(spp)
            if with_image:
                pt.image()
            pt.finish()
            if i >= a.warmup:
                ms.append(1e3 * (time.perf_counter() - t0))
        return statistics.median(ms)

    refine_ms = measure(False)
    render_ms = measure(True)
    paths = 256 * 256 * spp
    line = {"metric": "Msamples/s", "value": paths / refine_ms / 1e3, "unit": "Msamples/s", "n_gpus": 1,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": refine_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "procedural Cornell box (36 triangles), 256x256, 8 bounces, roulette from 3, "
                                   f"seed 0, {spp} spp", "timing": "host wall clock, median, refine + finish"},
            "render_ms": render_ms, "refine_ms": refine_ms,
            "reference_rtx5080_context": {"refine_ms_64spp": 31.8, "render_ms_64spp": 32.2,
                                          "note": "published on RTX 5080 through Vulkan; cross-hardware context only"},
            "plan": plan_of(pt), "tuner_trials": len(tune_log)}
    print(json.dumps(line), flush=True)


def run_cornell16(a):
    """The procedural Cornell box (36 triangles, one emissive quad, no
    punctual light) at 256x256, 16 spp, 8 bounces, roulette from bounce 3,
    seed 0, FP32 accumulator. Its 3 KB of scene data sit in L1/L2, so the
    kernels are issue-bound rather than HBM-bound; the line reports the
    device time per frame (CUDA events on the tracer's stream, L2 flushed
    between frames outside the timed windows), the end-to-end render()
    (prepare + upload + refine + RGBA8 readback, host wall clock) and the
    CPU oracle on all host threads over the same frame."""
    import torch
    torch.cuda.set_device(0)
    __graft_entry__.build()
    pkg = __graft_entry__.load_package()
    L = pkg._native.lib()
    from oxideav_render_vulkan_b200 import tuner
    spp, w, h = 16, 256, 256
    scene = pkg.Scene.cornell()
    opts = pkg.RenderOptions(width=w, height=h, path_trace=pkg.PathTraceOptions(samples_per_pixel=spp, max_bounces=8,
                                                                                rr_start=3, seed=0))
    pt = pkg.GpuPathTracer(0)
    stream = torch.cuda.Stream(device=0)
    assert L.oxpt_set_stream(pt.ctx, C.c_void_p(stream.cuda_stream)) == 0
    pt.sync(scene, opts)
    prep = pt.prepared()
    tune_log = []
    if not a.no_tune:
        tuner.tune(pt, spp=spp, repeats=3, log=tune_log)
    if a.mode != "auto":
        pt.set_tuning(mode={"mega": 0, "wave": 1, "split": 2}[a.mode])
    if a.slots:
        pt.set_tuning(wave_slots=a.slots)
    if a.graphs >= 0:
        pt.set_tuning(graphs=a.graphs)
    if a.trace_variant >= 0:
        pt.set_tuning(trace_variant=a.trace_variant)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    frames = max(20, a.steps)
    for _ in range(a.warmup):
        pt.reset()
        pt.refine(spp)
    pt.finish()
    n0 = C.c_uint64()
    L.oxpt_diag_launch_count(pt.ctx, C.byref(n0))
    ms = []
    with Clocks(0) as clk:
        for _ in range(frames):
            with torch.cuda.stream(stream):
                flush.fill_(1)  # L2 flush, outside the timed window
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            pt.reset()
            e0.record(stream)
            pt.refine(spp)
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
    n1 = C.c_uint64()
    L.oxpt_diag_launch_count(pt.ctx, C.byref(n1))
    frame_ms = statistics.median(ms)
    paths = w * h * spp
    # End to end: the reference's render() (sync with a re-prepared scene,
    # refine, image readback), host wall clock.
    e2e_ms = []
    for i in range(3 + frames):
        pt.invalidate_scene()
        pt.finish()
        t0 = time.perf_counter()
        pt.sync(scene, opts)
        pt.refine(spp)
        img = pt.image()
        if i >= 3:
            e2e_ms.append(1e3 * (time.perf_counter() - t0))
    h2d = prep.geom.nbytes + prep.attrs.nbytes + prep.tables.nbytes + prep.atlas.nbytes
    # Algorithmic bytes (counting build, untimed): nodes, triangles, shaded hits.
    cnt = (C.c_uint64 * 8)()
    assert L.oxpt_diag_refine_counted(pt.ctx, 1 << 20, spp, cnt) == 0
    c = [int(x) for x in cnt]
    alg = BYTES_AABB * c[3] + BYTES_TRI * c[5] + (BYTES_ATTR + BYTES_MAT) * c[6]
    peak, peak_kind = measured_peak()
    achieved = alg / (frame_ms * 1e-3) / 1e9
    cpu = None
    if not a.no_cpu_baseline:
        import oracle
        threads = os.cpu_count() or 1
        acc = np.zeros((h, w, 4), np.float32)
        t0 = time.perf_counter()
        oracle.dispatch(prep, prep.params, (0, spp, 0, h), acc, threads)
        dt = time.perf_counter() - t0
        cpu = {"value": paths / dt / 1e6, "unit": "Msamples/s", "cores": threads, "kind": "port",
               "sample": f"the whole 256x256 frame at 16 spp ({paths} paths, {dt:.2f} s)"}
    line = {"metric": "Msamples/s", "value": paths / frame_ms / 1e3, "unit": "Msamples/s", "n_gpus": 1,
            "steps": frames, "warmup": a.warmup, "ms_per_step": frame_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "procedural Cornell box (36 triangles, emissive ceiling quad, no punctual light), "
                                   "256x256, 16 spp, 8 bounces, roulette from 3, seed 0",
                       "l2": "flushed (256 MB write) before every timed frame",
                       "timing": "CUDA events around each frame's refine on the tracer's stream; median"},
            "mrays_per_s": (c[1] + c[2]) / c[0] * paths / frame_ms / 1e3,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "kernel": "whole frame (all kernels)", "peak_kind": peak_kind,
                         "note": "3 KB of scene data: served from L1/L2, so the frame is issue-bound; issue-slot "
                                 "use and active lanes are in the committed ncu summary for this workload"},
            "e2e": {"value": paths / statistics.median(e2e_ms) / 1e3, "unit": "Msamples/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": w * h * 4, "ms": statistics.median(e2e_ms),
                    "path": "render(): invalidate_scene + sync (prepare + upload) + refine + image()"},
            "cpu_baseline": cpu, "gpu_launches": int(n1.value - n0.value), "clocks": clk.summary(),
            "plan": plan_of(pt), "tuner_trials": len(tune_log)}
    print(json.dumps(line), flush=True)


def run_walk_sweep(a):
    """Traversal-kernel sweep on the single large scene: per-launch CUDA-event
    times of the extension and shadow kernels, summed over a `--spp` refine
    of the frame (graphs off, so every launch is timed), for each traversal
    variant (0-2 local-memory stacks at 6 / 8 / 10 blocks per SM; 3-5
    shared-memory short stacks at 6 / 8 / 10), stack entries kept on chip and
    staged top nodes, and the tolerance plan. One JSON line per point."""
    import torch
    torch.cuda.set_device(0)
    __graft_entry__.build()
    pkg = __graft_entry__.load_package()
    L = pkg._native.lib()
    from oxideav_render_vulkan_b200 import tuner
    scene, env = workload(pkg, a)
    t = pkg.GpuPathTracer(0)
    t.set_environment(env)
    t.sync(scene, options(pkg, a))
    tuner.apply(t, tuner.LARGE_SCENE_PLAN)
    t.set_tuning(graphs=0, wave_items=tuner.LARGE_SCENE_WAVE_ITEMS)
    t.prepared()
    ctx = t.ctx
    spp = min(a.spp, 8)
    line_extra = {}

    def run(tv, lim, stage, closest=0):
        t.set_tuning(trace_variant=tv, closest_walk=closest)
        L.oxpt_diag_set_walk(ctx, lim, stage)
        t.reset()
        t.refine(spp)
        t.finish()
        L.oxpt_diag_set_timing(ctx, 1)
        L.oxpt_diag_timing(ctx, None, None, None, None)
        t.reset()
        t.refine(spp)
        t.finish()
        L.oxpt_diag_timing(ctx, None, None, None, None)
        L.oxpt_diag_set_timing(ctx, 0)
        kms, kn = (C.c_double * 12)(), (C.c_uint64 * 12)()
        L.oxpt_diag_timing_kinds(ctx, kms, kn)
        line = {"workload": f"traversal sweep, single large scene 1920x1080, {spp} spp, graphs off",
                "trace_variant": tv, "stack_entries_on_chip": lim, "staged_nodes": stage, "closest_walk": closest,
                "extend_ms": kms[3], "shadow_ms": kms[4], "order_ms": kms[10],
                "frame_kernels_ms": sum(kms[k] for k in (2, 3, 4, 5, 6, 10))}
        line.update(line_extra)
        print(json.dumps(line), flush=True)

    for tv in (0, 1, 2):
        run(tv, 2, 0)
    for tv in (3, 4, 5):
        for lim in (0, 2, 4, 8, 16):
            for stage in (0, 127, 511):
                run(tv, lim, stage)
    for tv in (3, 4):
        for lim in (2, 8):
            run(tv, lim, 0, closest=1)
    # Refill threshold and postponed shadow leaves on the chosen kernels.
    L.oxpt_diag_set_walk(ctx, 2, 0)
    for post in (0, 1):
        L.oxpt_diag_set_shadow_postpone(ctx, post)
        for refill in (2, 4, 8, 16, 32):
            t.set_tuning(refill=refill)
            line_extra["refill"] = refill
            line_extra["shadow_postpone"] = post
            run(4, 2, 0)
    L.oxpt_diag_set_shadow_postpone(ctx, 0)
    line_extra.clear()
    # Ray queues reordered before the walks (1: continuation rays, 2: shadow rays, 3: both).
    for mode in (1, 2, 3):
        L.oxpt_diag_set_ray_order(ctx, mode)
        line_extra["ray_order"] = mode
        run(4, 2, 0)
    run(4, 2, 0, closest=1)
    L.oxpt_diag_set_ray_order(ctx, 0)
    line_extra.clear()


def _leaf_depth_sum(geom, nodes):
    """Sum over triangles of the depth of their leaf (root = 1): the levels
    each triangle takes part in during a level-by-level build."""
    w = geom[: nodes * 8].reshape(-1, 8)
    first, count = w[:, 3].astype(np.int64), w[:, 7].astype(np.int64)
    total, level, depth = 0, np.array([0], np.int64), 1
    while level.size:
        c = count[level]
        total += int(c[c > 0].sum()) * depth
        inner = level[c == 0]
        level = np.concatenate([first[inner], first[inner] + 1])
        depth += 1
    return total


def run_prepare(a):
    """Scene preparation on the device (oxpt_build_scene behind
    GpuPathTracer.sync with set_gpu_prepare): the large scene from host
    memory to device-ready buffers, against the host preparation."""
    import torch
    torch.cuda.set_device(0)
    __graft_entry__.build()
    pkg = __graft_entry__.load_package()
    scene, env = workload(pkg, a)
    opts = options(pkg, a, spp=1)
    tris = 20 * a.freq * a.freq
    pt = pkg.GpuPathTracer(0)
    pt.set_environment(env)
    pt.set_gpu_prepare(True)
    wall, phases = [], []
    with Clocks(0) as clk:
        for i in range(a.warmup + a.steps):
            pt.invalidate_scene()
            pt.finish()
            t0 = time.perf_counter()
            pt.sync(scene, opts)
            pt.finish()
            dt = time.perf_counter() - t0
            if i >= a.warmup:
                wall.append(dt)
                phases.append(pt.prepare_timing())
    prep = pt.prepared()
    level_tris = _leaf_depth_sum(prep.geom, prep.node_count)
    med = {k: statistics.median(p[k] for p in phases) for k in phases[0]}
    build_ms = med["bvh"] + med["flatten"]
    e2e_s = statistics.median(wall)
    # Source bytes that go up per step: positions, attribute streams, level-0 texels.
    h2d = tris * (36 + 36 + 24)  # positions, normals, uv0 (the icosphere's streams)
    h2d += 8 * a.tex * a.tex * 16  # level-0 texels of the 8 textures
    d2h = 512 * 4  # leaf slots of the emissive triangles (the four-wide tree is collapsed on the device)
    # Host preparation of the same scene (bounded sample: one run).
    host = pkg.GpuPathTracer(0)
    host.set_gpu_prepare(False)
    host.set_environment(env)
    t0 = time.perf_counter()
    host.sync(scene, opts)
    host.finish()
    host_s = time.perf_counter() - t0
    hp = host.prepared()
    same = (np.array_equal(hp.geom, prep.geom) and np.array_equal(hp.attrs.view(np.uint32), prep.attrs.view(np.uint32))
            and np.array_equal(hp.atlas, prep.atlas) and np.array_equal(hp.tables, prep.tables))
    peak, peak_kind = measured_peak()
    # BVH roofline: per level every triangle still in an inner node reads its
    # box and centroid (48 B) and its id (4 B) and writes its id (4 B).
    alg = level_tris * 56
    achieved = alg / (med["bvh"] * 1e-3) / 1e9
    line = {"metric": "Mtriangles/s prepared", "value": tris / (build_ms * 1e-3) / 1e6, "unit": "Mtriangles/s",
            "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * e2e_s,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"scene preparation of the single large scene ({tris} triangles, 8 x {a.tex}^2 "
                                   "textures + mips, 64 materials, 512 emissive triangles)",
                       "value": "BVH build + slot flattening on sources resident in HBM (CUDA events)",
                       "e2e": "GpuPathTracer.sync from host memory to device-ready buffers (host wall clock): "
                              "source upload, BVH, flattening, atlas, four-wide tree, tables",
                       "l2": "sources and outputs (0.9 GB) larger than L2; no flush"},
            "phases_ms": med, "identical_to_host": bool(same),
            "e2e": {"value": tris / e2e_s / 1e6, "unit": "Mtriangles/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "kernel": "BVH build (all levels)",
                         "peak_kind": peak_kind},
            "cpu_baseline": {"value": tris / host_s / 1e6, "unit": "Mtriangles/s", "cores": 1, "kind": "port",
                             "sample": f"host preparation of the same scene, one run ({host_s:.1f} s): binned-SAH BVH, "
                                       "slot flattening, mip chains and atlas on one thread, then the upload"},
            "clocks": clk.summary(), "gpu_launches": int(med["launches"])}
    print(json.dumps(line), flush=True)


SERVE_RES = [(128, 128), (256, 256), (512, 512), (1280, 720), (1920, 1080)]
SERVE_SPP = [4, 16, 64, 256, 1024]


def serve_stream(serve, a, n_scenes, seed=3):
    """Poisson arrivals at `rate`; each new session picks a resident scene,
    a resolution and an spp target (scaled by 1/spp_scale); 30% of requests
    are camera moves on an already opened session."""
    rng = np.random.default_rng(seed)
    reqs, opened, t = [], [], 0.0
    for rid in range(a.requests):
        t += float(rng.exponential(1.0 / a.rate))
        if opened and rng.random() < 0.3:
            base = reqs[opened[int(rng.integers(len(opened)))]]
            key = base.session if base.session is not None else base.rid
            spp = max(1, SERVE_SPP[int(rng.integers(len(SERVE_SPP)))] // a.spp_scale)
            ang = float(rng.uniform(-0.6, 0.6))
            cam = ((2.6 * np.sin(ang), 0.4, 2.6 * np.cos(ang)), (0.0, 0.0, 0.0))
            reqs.append(serve.Request(rid, t, base.scene, base.width, base.height, spp, cam, key))
        else:
            w, h = SERVE_RES[int(rng.integers(len(SERVE_RES)))]
            spp = max(1, SERVE_SPP[int(rng.integers(len(SERVE_SPP)))] // a.spp_scale)
            reqs.append(serve.Request(rid, t, int(rng.integers(n_scenes)), w, h, spp))
            opened.append(rid)
    return reqs


def run_serve(a):
    """The served stream: continuous batching against serial plain launches."""
    import torch
    torch.cuda.set_device(0)
    __graft_entry__.build()
    pkg = __graft_entry__.load_package()
    from oxideav_render_vulkan_b200 import serve
    rng = np.random.default_rng(5)
    n_scenes = a.scenes
    env = pkg.EnvironmentMap.sky(256, 128)
    owners, tris = [], 0
    for k in range(n_scenes):
        t_k = float(np.exp(rng.uniform(np.log(1e3), np.log(2e6))))
        if k % 2 == 0:
            sc = pkg.Scene.icosphere(freq=max(8, int(round(np.sqrt(t_k / 20.0)))), seed=300 + k, n_materials=16,
                                     n_textures=2, tex_size=256, n_punctual=4, n_emissive=16, material_mix=1)
        else:
            sc = pkg.Scene.box_field(max(1, int(t_k / 12)), seed=300 + k, material_mix=1)
        tris += int(sc.triangle_count())
        o = pkg.GpuPathTracer(0)
        o.set_environment(env)
        o.sync(sc, pkg.RenderOptions(width=64, height=64, scene_camera=0,
                                     path_trace=pkg.PathTraceOptions(samples_per_pixel=1, max_bounces=8)))
        o.refine(1)  # binds tables and params
        o.finish()
        owners.append(o)
    def options(r):
        return pkg.RenderOptions(width=r.width, height=r.height, scene_camera=0,
                                 path_trace=pkg.PathTraceOptions(samples_per_pixel=r.spp, max_bounces=8))

    runs = []
    for rep in range(max(1, a.repeats)):
        reqs = serve_stream(serve, a, n_scenes, seed=3 + rep)
        check = set(int(x) for x in np.random.default_rng(9 + rep).choice(a.requests, size=8, replace=False))
        ex = serve.GpuExecutor(pkg, owners, options, keep=lambda o: o.rid in check, idle_views=a.serve_idle_views)
        ex.exe.set_tuning(mode=2, graphs=1)
        if a.nee_variant >= 0:
            ex.exe.set_tuning(nee_variant=a.nee_variant)
        budget = 150 << 30
        # device time of the ticks (CUDA events around each batched step)
        L = pkg._native.lib()
        L.oxpt_diag_set_timing(ex.exe.ctx, 1)
        L.oxpt_diag_timing(ex.exe.ctx, None, None, None, None)
        served = serve.Server(ex, budget, tick_paths=1 << 24).run(reqs)
        L.oxpt_diag_timing(ex.exe.ctx, None, None, None, None)  # folds the ticks' event pairs
        kms, kn = (C.c_double * 12)(), (C.c_uint64 * 12)()
        L.oxpt_diag_timing_kinds(ex.exe.ctx, kms, kn)
        L.oxpt_diag_set_timing(ex.exe.ctx, 0)
        busy_s = kms[0] / 1e3
        ex2 = serve.GpuExecutor(pkg, owners, options, idle_views=a.serve_idle_views)
        serial = serve.run_serial(ex2, reqs)
        by = {r.rid: r for r in reqs}
        same = []
        for rid, acc in ex.kept.items():
            v = ex2.open(by[rid])
            v.refine(by[rid].spp)
            same.append(bool(np.array_equal(acc.view(np.uint32), v.read_accum().view(np.uint32))))
        runs.append({"stream_seed": 3 + rep, "msamples_per_s": served.msamples_per_s(),
                     "p50_latency_s": served.percentile(50), "p99_latency_s": served.percentile(99),
                     "completed": len(served.completed()), "superseded": sum(o.superseded for o in served.outcomes),
                     "ticks": served.ticks, "peak_device_bytes_accounted": served.peak_bytes,
                     "served_wall_s": served.wall, "gpu_busy_s": busy_s,
                     "gpu_busy_frac": busy_s / max(served.wall, 1e-9),
                     "serial_plain": {"msamples_per_s": serial.msamples_per_s(),
                                      "p50_latency_s": serial.percentile(50), "p99_latency_s": serial.percentile(99),
                                      "completed": len(serial.completed()), "wall_s": serial.wall},
                     "throughput_vs_serial": served.msamples_per_s() / serial.msamples_per_s(),
                     "same_alone_and_in_mix": same})
        del ex, ex2
    ratios = [r["throughput_vs_serial"] for r in runs]
    mid = sorted(runs, key=lambda r: r["throughput_vs_serial"])[len(runs) // 2]
    line = {"metric": "Msamples/s", "value": mid["msamples_per_s"], "unit": "Msamples/s", "n_gpus": 1,
            "steps": len(runs), "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"served stream: {a.requests} requests, Poisson {a.rate}/s, {n_scenes} resident "
                                   "scenes (1e3..2e6 triangles log-uniform), resolutions 128^2..1920x1080, spp "
                                   f"targets {{4,16,64,256,1024}}/{a.spp_scale}, 30% camera moves, 150 GB budget",
                       "triangles": tris, "repeats": f"{len(runs)} streams (seeds 3..{2 + len(runs)}); value and "
                                                    "latencies are the median-ratio run's",
                       "idle_views_per_scene": a.serve_idle_views},
            "p50_latency_s": mid["p50_latency_s"], "p99_latency_s": mid["p99_latency_s"],
            "throughput_vs_serial": {"median": statistics.median(ratios), "min": min(ratios), "max": max(ratios)},
            "same_alone_and_in_mix": all(all(r["same_alone_and_in_mix"]) for r in runs),
            "runs": runs}
    print(json.dumps(line), flush=True)


def _psnr(a, b):
    d = a[..., :3].astype(np.float64) - b[..., :3].astype(np.float64)
    mse = float(np.mean(d * d))
    return float("inf") if mse == 0 else 10.0 * np.log10(255.0 * 255.0 / mse)


def _hdr_mean(t):
    acc = t.read_accum()
    return acc[..., :3] / np.maximum(acc[..., 3:4], 1.0)


def run_nrc(a):
    """Radiance-cache frames against the plain tracer on the large scene with
    the mixed materials: 1 spp per frame, PSNR (RGBA8 images) and relative
    MSE (HDR) against a high-spp plain reference after each doubling of the
    frame count, and each method's wall time to reach 35 dB."""
    import torch
    torch.cuda.set_device(0)
    __graft_entry__.build()
    pkg = __graft_entry__.load_package()
    from oxideav_render_vulkan_b200.nrc import RadianceCache
    if a.nrc_scene == "cornell":
        scene, env = pkg.Scene.cornell(), None
    else:
        scene = pkg.Scene.icosphere(freq=a.freq, seed=1, n_materials=64, n_textures=8, tex_size=a.tex,
                                    n_punctual=16, n_emissive=512, material_mix=1)
        env = pkg.EnvironmentMap.sky(1024, 512, sun_dir=(0.3, 0.8, -0.5), sun_radiance=2000.0)

    def tracer():
        t = pkg.GpuPathTracer(0)
        if env is not None:
            t.set_environment(env)
        t.sync(scene, pkg.RenderOptions(width=a.width, height=a.height, scene_camera=0,
                                        path_trace=pkg.PathTraceOptions(samples_per_pixel=a.ref_spp, max_bounces=12,
                                                                        rr_start=3)))
        t.set_tuning(mode=2)
        t.prepared()
        return t

    ref = tracer()
    t0 = time.perf_counter()
    done = 0
    while done < a.ref_spp:
        n = min(256, a.ref_spp - done)
        ref.refine(n)
        done += n
    ref.finish()
    ref_s = time.perf_counter() - t0
    ref_img, ref_hdr = ref.image(), _hdr_mean(ref)
    del ref

    checkpoints = [1 << k for k in range(20) if (1 << k) <= a.frames]

    def progress(t, step, warm=None):
        # untimed first: one call of every chunk size the timed loop makes,
        # so that allocations and the CUDA graph of each refine shape (and
        # the cache's buffers) are not part of the comparison; the cache
        # warms up without training, so it starts the timed loop untrained
        sizes, done_ = [], 0
        for c in checkpoints:
            sizes.append(c - done_)
            done_ = c
        for n in sorted(set(sizes)):
            (warm or step)(n)
        t.finish()
        t.reset()
        out, wall, frames = [], 0.0, 0
        for c in checkpoints:
            t0 = time.perf_counter()
            step(c - frames)
            t.finish()
            wall += time.perf_counter() - t0
            frames = c
            img = t.image()
            hdr = _hdr_mean(t)
            out.append({"frames": c, "seconds": wall, "psnr_db": _psnr(img, ref_img),
                        "rel_mse": float(np.mean((hdr - ref_hdr) ** 2 / (ref_hdr ** 2 + 0.01)))})
        return out

    plain = tracer()
    plain.set_tuning(wave_slots=1 << 21, graphs=1)  # the plain tracer's best 1-spp plan
    plain_curve = progress(plain, lambda n: plain.refine(n))
    del plain
    # Where a frame's time goes (CUDA events per launch, 8 more frames of
    # each; the plain tracer without its graph so its launches are timed).
    L = pkg._native.lib()
    names = {0: "trace", 1: "reduce", 2: "logic", 3: "extend", 4: "shadow", 5: "shade", 6: "nee",
             7: "cache_inference", 8: "cache_train_forward", 9: "cache_backward"}

    def breakdown(t, fn, frames=8):
        t.finish()
        L.oxpt_diag_set_timing(t.ctx, 1)
        L.oxpt_diag_timing(t.ctx, None, None, None, None)
        fn(frames)
        t.finish()
        L.oxpt_diag_timing(t.ctx, None, None, None, None)
        L.oxpt_diag_set_timing(t.ctx, 0)
        kms, kn = (C.c_double * 12)(), (C.c_uint64 * 12)()
        L.oxpt_diag_timing_kinds(t.ctx, kms, kn)
        return {names[k]: kms[k] / frames for k in names if kn[k] and k != 0}

    def time_to(curve, db):
        prev = None
        for p in curve:
            if p["psnr_db"] >= db:
                if prev is None:
                    return p["seconds"]
                f = (db - prev["psnr_db"]) / max(p["psnr_db"] - prev["psnr_db"], 1e-9)
                return prev["seconds"] + f * (p["seconds"] - prev["seconds"])
            prev = p
        return None

    frame_ms = lambda c: 1e3 * c[-1]["seconds"] / c[-1]["frames"]
    runs = {}
    arms = [(int(g), int(w)) for g in a.nrc_frames_per_wave.split(",") for w in a.nrc_plain_training.split(",")]
    for per_wave, warm in arms:
        nt = tracer()
        cache = RadianceCache(nt)
        cache.configure(train_one_in=a.nrc_train_one_in, query_bounce=a.nrc_query_bounce, spread=a.nrc_spread,
                        frames_per_wave=per_wave)
        state = {"frames": 0}

        def cache_step(n):
            # the first `warm` frames: every path a training path, so the
            # frames are the plain tracer's while the cache learns
            while n > 0:
                if state["frames"] < warm:
                    m = min(n, warm - state["frames"])
                    cache.refine_training(m)
                else:
                    m = n
                    cache.refine(m)
                state["frames"] += m
                n -= m

        def untrained(n):
            cache.configure(train=0)
            cache.refine(n)
            cache.configure(train=1)
            state["frames"] = 0

        curve = progress(nt, cache_step, untrained)
        q, smp = cache.frame_counts()
        key = str(per_wave) if not warm else f"{per_wave}+plain{warm}"
        runs[key] = {"per_wave": per_wave, "plain_training_frames": warm, "curve": curve, "queries": q,
                     "samples": smp, "seconds_to_35db": time_to(curve, 35.0), "ms_per_frame": frame_ms(curve),
                     "kernel_ms_per_frame": breakdown(nt, lambda n: cache.refine(n))}
        del nt, cache
    best = min(runs, key=lambda g: runs[g]["seconds_to_35db"] if runs[g]["seconds_to_35db"] else 1e30)
    nrc_curve, q, smp = runs[best]["curve"], runs[best]["queries"], runs[best]["samples"]
    cache_ms = runs[best]["kernel_ms_per_frame"]
    plain2 = tracer()
    plain2.set_tuning(wave_slots=1 << 21)
    plain_ms = breakdown(plain2, lambda n: [plain2.refine(1) for _ in range(n)])
    del plain2

    tp, tn = time_to(plain_curve, 35.0), time_to(nrc_curve, 35.0)
    line = {"metric": "seconds to 35 dB PSNR", "value": tn, "unit": "s", "n_gpus": 1, "steps": a.frames,
            "warmup": 0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f32",
            "data": "synthetic",
            "config": {"workload": ("radiance cache: procedural Cornell box" if a.nrc_scene == "cornell" else
                                    "radiance cache: large scene (20 x freq^2 triangles) with the mixed material model")
                                   + f", {a.width}x{a.height}, 1 spp per frame, {a.frames} frames, 12 bounces",
                       "reference": f"plain tracer {a.ref_spp} spp ({ref_s:.1f} s)",
                       "cache": "5 x 64 ReLU MLP, BF16 tcgen05, 12-frequency encoding, paths end into the cache from "
                                f"bounce {a.nrc_query_bounce} when the path spread exceeds {a.nrc_spread} x the "
                                "primary vertex's, "
                                f"1 in {a.nrc_train_one_in} paths trains (suffix of 4 bounces into the cache), "
                                f"<= 65536 samples and one Adam step (lr 1e-2) per wave of {runs[best]['per_wave']} "
                                f"frame(s); the first {runs[best]['plain_training_frames']} frames plain, every path "
                                "training",
                       "timing": "host wall clock with a device sync per checkpoint; one untimed call of every chunk size first"},
            "plain_seconds_to_35db": tp, "ratio_to_plain": (tn / tp) if (tn and tp) else None,
            "plain_ms_per_frame": frame_ms(plain_curve), "cache_ms_per_frame": frame_ms(nrc_curve),
            "plain": plain_curve, "cache": nrc_curve,
            "last_frame_queries": q, "last_frame_training_samples": smp,
            "kernel_ms_per_frame": {"plain": plain_ms, "cache": cache_ms},
            "frames_per_wave": runs[best]["per_wave"], "plain_training_frames": runs[best]["plain_training_frames"],
            "by_frames_per_wave": {str(g): {"seconds_to_35db": r["seconds_to_35db"], "ms_per_frame": r["ms_per_frame"],
                                            "psnr_db_last": r["curve"][-1]["psnr_db"],
                                            "rel_mse_last": r["curve"][-1]["rel_mse"],
                                            "kernel_ms_per_frame": r["kernel_ms_per_frame"]}
                                   for g, r in runs.items()}}
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    if a.workload == "nrc":
        run_nrc(a)
        return
    if a.workload == "serve":
        run_serve(a)
        return
    if a.workload == "cornell":
        run_cornell(a)
        return
    if a.workload == "cornell16":
        run_cornell16(a)
        return
    if a.workload == "walk-sweep":
        run_walk_sweep(a)
        return
    if a.workload == "prepare":
        run_prepare(a)
        return
    if a.impl == "reference":
        run_reference(a)
        return
    if a.workload == "batch":
        run_batch(a)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    if rank == 0:
        __graft_entry__.build()
    if world > 1:
        dist.barrier()
    pkg = __graft_entry__.load_package()
    L = pkg._native.lib()

    scene, env = workload(pkg, a)
    rows_mode = world > 1 and a.split == "rows"
    opts = options(pkg, a, seed=0 if rows_mode else rank)
    pt = pkg.GpuPathTracer(local)
    stream = torch.cuda.Stream(device=local)
    assert L.oxpt_set_stream(pt.ctx, C.c_void_p(stream.cuda_stream)) == 0
    pt.set_environment(env)
    pt.sync(scene, opts)
    tune_log = []
    from oxideav_render_vulkan_b200 import tuner
    if a.tune:
        tuner.tune(pt, spp=min(a.spp, 4), repeats=3, log=tune_log)  # best of three per trial: steadier picks
    elif not a.no_tune:
        tuner.apply(pt, tuner.LARGE_SCENE_PLAN)  # the tuner's pick on this scene, and the tested plan
        pt.set_tuning(wave_items=tuner.LARGE_SCENE_WAVE_ITEMS)
    # Overrides on top of the plan.
    if a.mode != "auto":
        pt.set_tuning(mode={"mega": 0, "wave": 1, "split": 2}[a.mode])
    if a.slots:
        pt.set_tuning(wave_slots=a.slots)
    if a.shadow_walk != "auto":
        pt.set_tuning(shadow_walk={"four": 0, "binary": 1}[a.shadow_walk])
    if a.wave_items:
        pt.set_tuning(wave_items=a.wave_items)
    if a.trace_variant >= 0:
        pt.set_tuning(trace_variant=a.trace_variant)
    if a.refill:
        pt.set_tuning(refill=a.refill)
    if a.graphs >= 0:
        pt.set_tuning(graphs=a.graphs)
    if a.nee_mask >= 0:
        L.oxpt_diag_set_nee_mask(pt.ctx, a.nee_mask)
    if a.shadow_postpone >= 0:
        L.oxpt_diag_set_shadow_postpone(pt.ctx, a.shadow_postpone)
    if a.ray_order >= 0:
        L.oxpt_diag_set_ray_order(pt.ctx, a.ray_order)
    l2_granted = C.c_uint64(0)
    if a.l2_window:
        assert L.oxpt_diag_set_l2_window(pt.ctx, 1, C.byref(l2_granted)) == 0, L.oxpt_last_error(pt.ctx).decode()
    prep = pt.prepared()

    # Algorithmic bytes per path from the counting build (untimed, 1 spp):
    # traversal kernels 32 B per AABB and 48 B per triangle tested, shading
    # 192 B of attributes + 544 B of material record per shaded hit.
    cnt = (C.c_uint64 * 8)()
    assert L.oxpt_diag_refine_counted(pt.ctx, 1 << 20, 1, cnt) == 0
    c = [int(x) for x in cnt]
    split = (C.c_uint64 * 16)()
    L.oxpt_diag_counters_split(pt.ctx, split)
    h0, h1 = [int(x) for x in split[:8]], [int(x) for x in split[8:]]
    npaths = max(c[0], 1)
    bytes_per_path = (BYTES_AABB * c[3] + BYTES_TRI * c[5] + (BYTES_ATTR + BYTES_MAT) * c[6]) / npaths
    kernel_bytes = {  # algorithmic bytes per camera path, per kernel
        "trace_paths": bytes_per_path,
        "wave_logic": (BYTES_ATTR + BYTES_MAT) * c[6] / npaths,
        "wave_extend": (BYTES_AABB * h0[3] + BYTES_TRI * h0[5]) / npaths,
        "wave_shadow": (BYTES_AABB * h1[3] + BYTES_TRI * h1[5]) / npaths,
        "split_logic": 0.0,
        "split_shade": (BYTES_ATTR + BYTES_MAT) * c[6] / npaths,
        "split_nee": 0.0,
    }
    kernel_bytes["walk_extend"] = kernel_bytes["wave_extend"]  # on-chip-stack kernels (trace_variant 3-5)
    kernel_bytes["walk_shadow"] = kernel_bytes["wave_shadow"]
    rays_per_path = (c[1] + c[2]) / npaths

    from oxideav_render_vulkan_b200 import shard
    y0, rows = shard.row_tile(a.height, rank, world) if rows_mode else (0, a.height)
    gather = TileGather(pkg, pt, stream, rank, world, local, torch) if rows_mode else None

    def step():
        pt.reset()
        if rows_mode:
            assert L.oxpt_tracer_refine_rows(pt._h, a.spp, y0, rows) == 0
            gather.run()
        else:
            pt.refine(a.spp)

    for _ in range(a.warmup):
        step()
    pt.finish()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    L.oxpt_diag_set_timing(pt.ctx, 1)
    L.oxpt_diag_timing(pt.ctx, None, None, None, None)
    n0 = C.c_uint64()
    L.oxpt_diag_launch_count(pt.ctx, C.byref(n0))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(a.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    elapsed = ev0.elapsed_time(ev1) / 1e3
    tms, tn, rms, rn = C.c_double(), C.c_uint64(), C.c_double(), C.c_uint64()
    L.oxpt_diag_timing(pt.ctx, C.byref(tms), C.byref(tn), C.byref(rms), C.byref(rn))
    L.oxpt_diag_set_timing(pt.ctx, 0)
    n1 = C.c_uint64()
    L.oxpt_diag_launch_count(pt.ctx, C.byref(n1))
    pt.finish()
    t_max = elapsed
    if world > 1:
        t = torch.tensor([elapsed], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    paths_step = a.width * a.height * a.spp
    frames = 1 if rows_mode else world  # frames all ranks trace per step
    value = frames * a.steps * paths_step / t_max / 1e6

    # Roofline of the dominant kernel: its algorithmic bytes over the timed
    # region / its summed CUDA-event time (kernel launches on the tracer's
    # stream), against the measured HBM copy bandwidth.
    peak, peak_kind = measured_peak()
    kms, kn = (C.c_double * 12)(), (C.c_uint64 * 12)()
    L.oxpt_diag_timing_kinds(pt.ctx, kms, kn)
    kernel_timing = "timed region"
    if pt.tuning().graphs:
        # A graph step records no per-kernel events: time the same kernels
        # over the same number of frames with the graph off (untimed for
        # `value`), one event pair per launch.
        pt.set_tuning(graphs=0)
        L.oxpt_diag_set_timing(pt.ctx, 1)
        L.oxpt_diag_timing(pt.ctx, None, None, None, None)
        for _ in range(a.steps):
            step()
        pt.finish()
        L.oxpt_diag_timing(pt.ctx, None, None, None, None)
        L.oxpt_diag_set_timing(pt.ctx, 0)
        L.oxpt_diag_timing_kinds(pt.ctx, kms, kn)
        pt.set_tuning(graphs=1)
        kernel_timing = "same frames re-run without the graph (per-launch CUDA events)"
    paths_timed = paths_step * a.steps
    mode = pt.tuning().mode
    walk = pt.tuning().trace_variant >= 3
    ext_name, sh_name = ("walk_extend", "walk_shadow") if walk else ("wave_extend", "wave_shadow")
    kinds = {0: ((0, "trace_paths"),), 1: ((2, "wave_logic"), (3, ext_name), (4, sh_name)),
             2: ((2, "split_logic"), (5, "split_shade"), (6, "split_nee"), (3, ext_name),
                 (4, sh_name))}[mode]
    traffic_db = {}
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        traffic_db = json.loads(tf.read_text())
    kernels = {}
    for k, name in kinds:
        if not kn[k]:
            continue
        b = kernel_bytes[name] * paths_timed
        per_launch = b / kn[k]
        tr = traffic_db.get(name, {}).get("dram_bytes_per_path")
        kernels[name] = {"ms_total": kms[k], "launches": int(kn[k]), "launch_ms": kms[k] / kn[k],
                         "algorithmic_bytes_per_launch": per_launch,
                         "achieved_gbs": b / (kms[k] / 1e3) / 1e9 if kms[k] else None,
                         "traffic_bytes_per_launch": tr * paths_timed / kn[k] if tr else None}
    dom = max(kernels, key=lambda n: kernels[n]["ms_total"])
    kd = kernels[dom]
    achieved = kd["achieved_gbs"]

    # End to end through the C ABI with host buffers.
    e2e = None
    if not a.no_e2e:
        e2e = e2e_measure(pkg, L, pt, prep, a, stream, torch, rank, (y0, rows), gather)
        if world > 1:
            t = torch.tensor([e2e["seconds"]], device=f"cuda:{local}", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e["seconds"] = float(t.item())
        e2e = {"value": frames * a.steps * paths_step / e2e["seconds"] / 1e6, "unit": "Msamples/s",
               "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"],
               "upload_sync_ms": e2e["upload_sync_ms"], "upload_staged_ms": e2e["upload_staged_ms"],
               "h2d_gbs_sync": e2e["h2d_gbs_sync"], "steps_identical": e2e["steps_identical"],
               "graph_builds_in_timed_steps": e2e["graph_builds_in_timed_steps"],
               "pipeline": "scene staged into a second buffer set during the previous step's trace; "
                           "image read back on the copy stream"}

    # The tolerance plan (closest hits over the four-wide tree: images within
    # 60 dB of the CPU tracer, hit ids equal except near-ties, not bit-exact)
    # on the same frames, device-timed the same way; `value` stays the
    # bit-exact plan's.
    tolerance = None
    if not a.no_tolerance_plan:
        saved = pt.tuning()
        tv = saved.trace_variant if saved.trace_variant >= 3 else 3
        fast = 1 if saved.mode == 2 else 0  # the fast-math shading build is the split plan's

        def timed_plan(**kw):
            pt.set_tuning(trace_variant=tv, **kw)
            for _ in range(max(1, a.warmup // 2)):
                step()
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(a.steps):
                step()
            e1.record(stream)
            torch.cuda.synchronize()
            tsec = e0.elapsed_time(e1) / 1e3
            if world > 1:
                t = torch.tensor([tsec], device=f"cuda:{local}", dtype=torch.float64)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                tsec = float(t.item())
            return tsec

        t_walk = timed_plan(closest_walk=1, fast_shading=0)
        # the fast build's shading kernel compiles to other register counts,
        # so its occupancy variant is chosen here by measurement
        by_shade = {}
        for sv in ((0, 1, 2) if fast else (saved.shade_variant,)):
            by_shade[sv] = timed_plan(closest_walk=1, fast_shading=fast, shade_variant=sv)
        best_sv = min(by_shade, key=by_shade.get)
        tsec = by_shade[best_sv]
        pt.set_tuning(shade_variant=best_sv)
        # its kernels, as for the exact plan: frames re-run without the graph
        tol_steps = min(a.steps, 4)
        pt.set_tuning(graphs=0)
        L.oxpt_diag_set_timing(pt.ctx, 1)
        L.oxpt_diag_timing(pt.ctx, None, None, None, None)
        for _ in range(tol_steps):
            step()
        pt.finish()
        L.oxpt_diag_timing(pt.ctx, None, None, None, None)
        L.oxpt_diag_set_timing(pt.ctx, 0)
        tms_, tn_ = (C.c_double * 12)(), (C.c_uint64 * 12)()
        L.oxpt_diag_timing_kinds(pt.ctx, tms_, tn_)
        pt.set_tuning(graphs=saved.graphs)
        tol_kernels = {name: {"ms_per_step": tms_[k] / tol_steps, "launch_ms": tms_[k] / tn_[k]}
                       for k, name in kinds if tn_[k]}
        tolerance = {"value": frames * a.steps * paths_step / tsec / 1e6, "unit": "Msamples/s",
                     "ms_per_step": 1e3 * tsec / a.steps, "plan": plan_of(pt),
                     "closest_walk_only": {"value": frames * a.steps * paths_step / t_walk / 1e6,
                                           "ms_per_step": 1e3 * t_walk / a.steps},
                     "kernels": tol_kernels,
                     "ms_per_step_by_shade_variant": {str(k): 1e3 * v / a.steps for k, v in by_shade.items()},
                     "checks": "tests/test_gpu_tolerance.py, tests/test_gpu_headline.py: ids on 10^6 rays equal "
                               "except ties within 1e-6 relative t; >= 60 dB PSNR against the libm oracle"}
        pt.set_tuning(trace_variant=saved.trace_variant, closest_walk=saved.closest_walk,
                      fast_shading=saved.fast_shading, shade_variant=saved.shade_variant)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        import oracle
        cpu = cpu_baseline(pkg, oracle, prep, a, a.cpu_seconds)

    if world > 1:
        dist.barrier()
    if rank == 0:
        line = {"metric": "Msamples/s", "value": value, "unit": "Msamples/s", "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": 1e3 * t_max / a.steps, "higher_is_better": True,
                "scaling": "strong" if rows_mode else "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": dict(config(a, world, rows_mode),
                                                    l2_persisting_bytes=int(l2_granted.value)),
                "mrays_per_s": value * rays_per_path,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": kd["traffic_bytes_per_launch"],
                             "kernel": dom, "peak_kind": peak_kind,
                             "dram_gbs": (kd["traffic_bytes_per_launch"] / (kd["launch_ms"] * 1e-3) / 1e9
                                          if kd["traffic_bytes_per_launch"] else None),
                             "dram_frac": (kd["traffic_bytes_per_launch"] / (kd["launch_ms"] * 1e-3) / 1e9 / peak
                                           if kd["traffic_bytes_per_launch"] else None),
                             "l1_l2_served_share": (1.0 - kd["traffic_bytes_per_launch"] /
                                                    kd["algorithmic_bytes_per_launch"]
                                                    if kd["traffic_bytes_per_launch"] else None),
                             "limiter": "dependent-load latency and SIMD divergence of the walks: node and "
                                        "triangle bytes are served mostly by L1/L2 (see l1_l2_served_share), "
                                        "so frac is an effective bandwidth against the HBM copy peak, and "
                                        "dram_frac the kernel's real HBM use",
                             "algorithmic_bytes_per_launch": kd["algorithmic_bytes_per_launch"],
                             "launch_ms": kd["launch_ms"], "launches": kd["launches"],
                             "algorithmic_bytes_per_path": bytes_per_path, "kernels": kernels,
                             "trace_phase_ms": tms.value, "reduce_ms_total": rms.value,
                             "kernel_timing": kernel_timing},
                "cpu_baseline": cpu, "e2e": e2e, "tolerance_plan": tolerance,
                "gpu_launches": int(n1.value - n0.value),
                "clocks": clk.summary(), "rays_per_path": rays_per_path,
                "plan": plan_of(pt), "tuner_trials": len(tune_log)}
        print(json.dumps(line), flush=True)
    del pt
    if world > 1:
        dist.destroy_process_group()


def plan_of(pt):
    t = pt.tuning()
    return {"mode": ["megakernel", "wavefront", "wavefront-split"][t.mode], "wave_slots": t.wave_slots,
            "shade_variant": t.shade_variant, "trace_variant": t.trace_variant, "stack": t.stack,
            "nee_variant": t.nee_variant, "shadow_walk": ["four-wide", "binary"][t.shadow_walk],
            "refill": t.refill, "graphs": t.graphs,
            "closest_walk": ["binary (exact)", "four-wide (tolerance plan)"][t.closest_walk],
            "shading": ["exact build", "fast-math build (tolerance plan)"][t.fast_shading]}


class TileGather:
    """The row split's exchange (shard.gather_row_tiles on the tracer's
    stream, zero copy): each rank's accumulator rows go to every rank with
    one NCCL all-gather of equal-sized (padded) tiles."""

    def __init__(self, pkg, pt, stream, rank, world, local, torch):
        from oxideav_render_vulkan_b200 import shard
        self.torch, self.stream, self.shard, self.pt = torch, stream, shard, pt
        self.acc = shard.accumulator_tensor(pt, local)
        self.h = self.acc.shape[0]
        self.world, self.rank = world, rank

    def run(self):
        with self.torch.cuda.stream(self.stream):
            self.shard.gather_row_tiles(self.acc, self.h)


def e2e_measure(pkg, L, pt, prep, a, stream, torch, rank, tile=None, gather=None):
    """Per step through the C ABI: the flat scene buffers and tables go up
    from pinned host memory (oxpt_stage_scene, into the context's second
    buffer set while the previous step still traces), params, reset,
    refine, resolve and the RGBA8 readback into pinned memory on the copy
    stream (oxpt_resolve_async). Steps overlap as a renderer's frames do;
    the timed region ends when the last image is in host memory. Also
    times one synchronous upload (oxpt_upload_scene + oxpt_set_tables, the
    reference's order) and the staged one on their own, for the record."""
    N = pkg._native
    pin = {k: torch.from_numpy(getattr(prep, k)).pin_memory() for k in ("geom", "attrs", "tables", "atlas")}
    imgs = [torch.empty((a.height, a.width, 4), dtype=torch.uint8).pin_memory() for _ in range(2)]
    desc = N.SceneDesc(pin["geom"].data_ptr(), prep.geom.size, pin["attrs"].data_ptr(), prep.attrs.size,
                       pin["atlas"].data_ptr(), prep.atlas_side, prep.atlas_layers, prep.node_count, prep.slot_count)
    params = prep.params
    rp = pt.resolve_params(False)
    rp.exposure[1] = float(a.spp)
    ctx = pt.ctx
    tables = C.c_void_p(pin["tables"].data_ptr())
    h2d = prep.geom.nbytes + prep.attrs.nbytes + prep.atlas.nbytes + prep.tables.nbytes
    d2h = a.width * a.height * 4

    def check(st):
        if st != 0:
            raise RuntimeError(L.oxpt_last_error(ctx).decode())

    y0, rows = tile or (0, a.height)

    def step(i):
        check(L.oxpt_stage_scene(ctx, C.byref(desc), tables, prep.tables.size))
        check(L.oxpt_set_params(ctx, C.byref(params)))
        check(L.oxpt_reset(ctx))
        check(L.oxpt_dispatch(ctx, C.byref(N.Frame(0, a.spp, y0, rows))))
        if gather is not None:
            gather.run()
        check(L.oxpt_resolve_async(ctx, C.byref(rp), 0, C.c_void_p(imgs[i % 2].data_ptr())))

    # Upload alone, each way (untimed for e2e): host wall clock of the call.
    L.oxpt_finish(ctx)
    t0 = time.perf_counter()
    check(L.oxpt_upload_scene(ctx, C.byref(desc)))
    check(L.oxpt_set_tables(ctx, tables, prep.tables.size))
    sync_ms = 1e3 * (time.perf_counter() - t0)
    t0 = time.perf_counter()
    check(L.oxpt_stage_scene(ctx, C.byref(desc), tables, prep.tables.size))
    staged_ms = 1e3 * (time.perf_counter() - t0)
    for i in range(2):
        step(i)
    check(L.oxpt_resolve_wait(ctx))
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b0, b1 = C.c_uint64(), C.c_uint64()
    L.oxpt_diag_graph_builds(ctx, C.byref(b0))
    t0 = time.perf_counter()
    ev0.record(stream)
    for i in range(a.steps):
        step(i)
    check(L.oxpt_resolve_wait(ctx))
    L.oxpt_diag_graph_builds(ctx, C.byref(b1))
    ev1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    # The last image is in host memory when resolve_wait returns; the events
    # bracket the stream, the host clock the whole loop: take the longer.
    seconds = max(ev0.elapsed_time(ev1) / 1e3, wall)
    same = bool(torch.equal(imgs[0], imgs[1]))  # every step renders the same frame
    return {"seconds": seconds, "h2d": h2d, "d2h": d2h, "upload_sync_ms": sync_ms, "upload_staged_ms": staged_ms,
            "h2d_gbs_sync": h2d / (sync_ms * 1e-3) / 1e9, "steps_identical": same,
            "graph_builds_in_timed_steps": int(b1.value - b0.value)}


if __name__ == "__main__":
    main()
