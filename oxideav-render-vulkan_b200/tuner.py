"""Autotuner for the tracer's execution plan.

Chooses, per scene and resolution, between the megakernel and the
wavefront, and within the wavefront the shading kernel's register budget
(shade_variant), the traversal kernels' occupancy target (trace_variant),
the traversal stack depth, the number of paths in flight (wave_slots) and
the shadow rays' tree (the four-wide any-hit tree or the binary walk).
Every plan yields bit-identical accumulators, so the tuner only measures
time: each candidate runs a short refine at sample indices far from any
real render's, timed with CUDA events on the tracer's stream, and the
accumulator is reset afterwards. The search is coordinate descent (one knob
at a time, keeping the best), which needs ~10 short runs instead of the full
product.
"""
from __future__ import annotations

import ctypes as C
import json
import time
from dataclasses import asdict, dataclass
from typing import Callable, Dict, List, Optional

from . import _native as N

TUNE_FIRST_SAMPLE = 1 << 30  # sample indices the tuner uses (not rendered by users)


@dataclass
class Plan:
    mode: int = N.MODE_WAVEFRONT
    shade_variant: int = 1
    trace_variant: int = 4
    stack: int = 0
    wave_slots: int = 1 << 20
    nee_variant: int = 3
    shadow_walk: int = 0
    graphs: int = 0
    refill: int = 8
    closest_walk: int = 0  # 1: the tolerance plan (four-wide closest-hit walk), never chosen by the tuner
    fast_shading: int = 0  # 1: the tolerance plan's fast-math shading kernels, never chosen by the tuner

    def key(self):
        return (self.mode, self.shade_variant, self.trace_variant, self.stack, self.wave_slots, self.nee_variant,
                self.shadow_walk, self.graphs, self.refill, self.closest_walk, self.fast_shading)


SPACE = {
    "mode": [N.MODE_WAVEFRONT, N.MODE_WAVEFRONT_SPLIT, N.MODE_MEGAKERNEL],
    "shade_variant": [0, 1, 2],
    "trace_variant": [0, 1, 2, 3, 4, 5],
    "stack": [0, 64],
    "wave_slots": [1 << 19, 1 << 20, 1 << 21, 1 << 22],
    "nee_variant": [0, 1, 2, 3, 4, 5],
    "shadow_walk": [0, 1],
    "refill": [1, 8, 16, 32],
    "graphs": [0, 1],
}
# The plan of the single-large-scene workload (1,048,820 triangles, 1920x1080,
# 64 spp, 12 bounces): the tuner's pick on that scene. The benchmark runs it
# by default and the GPU parity test of that workload runs exactly it, so
# the measured plan is the tested plan.
LARGE_SCENE_PLAN = Plan(mode=N.MODE_WAVEFRONT_SPLIT, shade_variant=0, trace_variant=4, stack=64,
                        wave_slots=1 << 22, nee_variant=3, shadow_walk=0, graphs=1, refill=16)
LARGE_SCENE_WAVE_ITEMS = 1 << 27  # paths per launch round: a whole frame

WAVE_ONLY = ("shade_variant", "trace_variant", "stack", "wave_slots", "nee_variant", "shadow_walk", "graphs",
             "refill")
SPLIT_ONLY = ("nee_variant",)


def coordinate_descent(measure: Callable[[Plan], float], start: Optional[Plan] = None,
                       space: Dict[str, List[int]] = SPACE, log: Optional[list] = None) -> Plan:
    """Minimise `measure` (seconds) one knob at a time."""
    best = start or Plan()
    cache = {}

    def cost(p: Plan) -> float:
        k = p.key()
        if k not in cache:
            cache[k] = measure(p)
            if log is not None:
                log.append({"plan": asdict(p), "seconds": cache[k]})
        return cache[k]

    best_cost = cost(best)
    for knob, values in space.items():
        if knob in WAVE_ONLY and best.mode == N.MODE_MEGAKERNEL:
            continue
        if knob in SPLIT_ONLY and best.mode != N.MODE_WAVEFRONT_SPLIT:
            continue
        for v in values:
            if getattr(best, knob) == v:
                continue
            cand = Plan(**{**asdict(best), knob: v})
            c = cost(cand)
            if c < best_cost:
                best, best_cost = cand, c
    return best


def apply(tracer, plan: Plan):
    tracer.set_tuning(mode=plan.mode, shade_variant=plan.shade_variant, trace_variant=plan.trace_variant,
                      stack=plan.stack, wave_slots=plan.wave_slots, nee_variant=plan.nee_variant,
                      shadow_walk=plan.shadow_walk, graphs=plan.graphs, refill=plan.refill,
                      closest_walk=plan.closest_walk, fast_shading=plan.fast_shading)


def tune(tracer, spp: int = 1, repeats: int = 1, log: Optional[list] = None) -> Plan:
    """Tune `tracer` (already synced to its scene and options) in place and
    return the chosen plan. Leaves the accumulation reset."""
    L = N.lib()
    ctx = tracer.ctx
    tracer.prepared()  # binds tables and params

    def measure(p: Plan) -> float:
        apply(tracer, p)
        best = float("inf")
        for r in range(repeats + 1):
            L.oxpt_diag_set_timing(ctx, 1)
            L.oxpt_diag_timing(ctx, None, None, None, None)
            t0 = time.perf_counter()
            st = L.oxpt_refine(ctx, TUNE_FIRST_SAMPLE + 97 * r, spp)
            if st != N.OK:
                raise RuntimeError(L.oxpt_last_error(ctx).decode())
            ms = C.c_double()
            L.oxpt_diag_timing(ctx, C.byref(ms), None, None, None)
            L.oxpt_diag_set_timing(ctx, 0)
            if r > 0 or repeats == 0:  # the first run warms caches and buffers
                best = min(best, ms.value / 1e3 if ms.value > 0 else time.perf_counter() - t0)
        return best

    plan = coordinate_descent(measure, log=log)
    apply(tracer, plan)
    tracer.reset()
    return plan


def tune_batch(tracers, executor, spp: int = 1, log: Optional[list] = None,
               space: Dict[str, List[int]] = None) -> Plan:
    """Tune `executor`'s plan for batched refinement of `tracers` (already
    synced): each candidate traces `spp` samples of every tracer at the
    tuner's sample indices as one batch, timed with CUDA events on the
    executor's stream; the tracers' accumulations are reset afterwards.
    The megakernel is not a batch plan."""
    L = N.lib()
    ctx = executor.ctx
    frames = (N.BatchFrame * len(tracers))()
    for k, t in enumerate(tracers):
        t.prepared()  # binds tables and params
        w, h = t.size()
        frames[k] = N.BatchFrame(t.ctx, TUNE_FIRST_SAMPLE, spp, 0, h)
    space = space or {k: v for k, v in SPACE.items() if k != "mode"}
    space = {"mode": [N.MODE_WAVEFRONT_SPLIT, N.MODE_WAVEFRONT], **space}

    def measure(p: Plan) -> float:
        apply(executor, p)
        best = float("inf")
        for r in range(2):
            L.oxpt_diag_set_timing(ctx, 1)
            L.oxpt_diag_timing(ctx, None, None, None, None)
            t0 = time.perf_counter()
            st = L.oxpt_refine_batch(ctx, frames, len(tracers))
            if st != N.OK:
                raise RuntimeError(L.oxpt_last_error(ctx).decode())
            ms = C.c_double()
            L.oxpt_diag_timing(ctx, C.byref(ms), None, None, None)
            L.oxpt_diag_set_timing(ctx, 0)
            if r > 0:
                best = min(best, ms.value / 1e3 if ms.value > 0 else time.perf_counter() - t0)
        return best

    plan = coordinate_descent(measure, start=Plan(mode=N.MODE_WAVEFRONT_SPLIT), space=space, log=log)
    apply(executor, plan)
    for t in tracers:
        t.reset()
    return plan


def describe(plan: Plan) -> dict:
    d = asdict(plan)
    d["mode"] = {N.MODE_WAVEFRONT: "wavefront", N.MODE_WAVEFRONT_SPLIT: "wavefront-split"}.get(plan.mode,
                                                                                           "megakernel")
    return d


def dumps(plan: Plan) -> str:
    return json.dumps(describe(plan))
