"""The autotuner's search (coordinate descent) on a synthetic cost model,
without a GPU; the GPU test runs it on a real tracer and checks the plan
does not change results."""
from __future__ import annotations

import numpy as np
import pytest


def _tuner(pkg):
    import importlib
    return importlib.import_module("oxideav_render_vulkan_b200.tuner")


def test_coordinate_descent_finds_the_separable_optimum(pkg):
    tuner = _tuner(pkg)
    N = pkg._native
    target = {"shade_variant": 2, "trace_variant": 0, "stack": 64, "wave_slots": 1 << 21}

    def cost(p):
        c = 10.0 if p.mode == N.MODE_MEGAKERNEL else 1.0
        for k, v in target.items():
            c += 0.0 if getattr(p, k) == v else 0.1
        return c

    log = []
    best = tuner.coordinate_descent(cost, log=log)
    assert best.mode == N.MODE_WAVEFRONT
    for k, v in target.items():
        assert getattr(best, k) == v
    assert len(log) <= 1 + sum(len(v) - 1 for v in tuner.SPACE.values())


def test_megakernel_skips_wavefront_knobs(pkg):
    tuner = _tuner(pkg)
    N = pkg._native
    seen = []

    def cost(p):
        seen.append(p)
        return 0.5 if p.mode == N.MODE_MEGAKERNEL else 1.0

    best = tuner.coordinate_descent(cost)
    assert best.mode == N.MODE_MEGAKERNEL
    assert len(seen) == 3


@pytest.mark.gpu
def test_tuned_plan_keeps_results_bit_exact(pkg, oracle):
    import scenes
    tuner = _tuner(pkg)
    t = pkg.GpuPathTracer(0)
    opts = pkg.RenderOptions(width=64, height=48, path_trace=pkg.PathTraceOptions(samples_per_pixel=4))
    t.sync(scenes.materials_scene(pkg), opts)
    log = []
    plan = tuner.tune(t, spp=1, repeats=0, log=log)
    assert len(log) >= 2 and t.samples() == 0
    t.refine(4)
    gpu = t.read_accum()
    cpu, _ = oracle.render(t.prepared(), 4)
    assert np.array_equal(gpu.view(np.uint32), cpu.view(np.uint32)), tuner.describe(plan)
