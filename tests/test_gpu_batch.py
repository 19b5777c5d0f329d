"""Batched refinement (oxpt_batch.h) against each scene refined alone.

One executor traces the frames of several scenes (different geometry,
materials, light counts, environments, resolutions and sample counts) as a
single wavefront. Every tracer's accumulator must be bit-identical to the
one its own refine() gives, across execution plans, with rounds and row
bands forced small, with the executor inside or outside the batch, and
when a second batch continues the first's samples.
"""
from __future__ import annotations

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu


def _cases(pkg):
    """(scene factory, environment factory or None, width, height, spp)."""
    return [
        (lambda: pkg.Scene.cornell(), None, 48, 40, 3),
        (lambda: scenes.materials_scene(pkg), None, 40, 30, 2),
        (lambda: scenes.alpha_scene(pkg), None, 52, 20, 4),
        (lambda: scenes.env_scene(pkg), lambda: pkg.EnvironmentMap(scenes.sky(), 1.0), 36, 24, 2),
        (lambda: pkg.Scene.icosphere(freq=8, seed=5, n_materials=8, n_textures=2, tex_size=64, n_punctual=16,
                                     n_emissive=4, material_mix=1), None, 33, 17, 3),
    ]


def _tracer(pkg, case, bounces=8):
    scene, env, w, h, spp = case
    t = pkg.GpuPathTracer(0)
    if env is not None:
        t.set_environment(env())
    opts = pkg.RenderOptions(width=w, height=h,
                             path_trace=pkg.PathTraceOptions(samples_per_pixel=64, max_bounces=bounces))
    assert t.sync(scene(), opts)
    return t


def _alone(pkg, cases, chunks):
    out = []
    for c in cases:
        t = _tracer(pkg, c)
        for n in chunks(c):
            t.refine(n)
        out.append(t.read_accum())
    return out


@pytest.mark.parametrize("plan", [
    dict(mode=2),
    dict(mode=1, shadow_walk=1),
    dict(mode=2, wave_items=3000, wave_slots=700),   # many rounds, row bands, slot reuse across frames
    dict(mode=0),                                     # a megakernel executor runs the split wavefront
    dict(mode=2, graphs=1),                           # one CUDA graph, device-side while loops
    dict(mode=1, graphs=1, wave_items=3000, wave_slots=700),
    dict(mode=2, nee_variant=3, wave_items=3000, wave_slots=700),  # vertex-major NEE, per-scene job counts
    dict(mode=2, nee_variant=5, graphs=1),
])
def test_batch_matches_each_scene_alone(pkg, plan):
    cases = _cases(pkg)
    want = _alone(pkg, cases, lambda c: [c[4]])
    tracers = [_tracer(pkg, c) for c in cases]
    tracers[0].set_tuning(**plan)
    pkg.refine_batch(tracers, [c[4] for c in cases])
    for k, (t, w) in enumerate(zip(tracers, want)):
        assert t.samples() == cases[k][4]
        got = t.read_accum()
        assert np.array_equal(got.view(np.uint32), w.view(np.uint32)), f"scene {k} differs"


def test_second_batch_continues_the_samples_with_an_outside_executor(pkg):
    cases = _cases(pkg)
    want = _alone(pkg, cases, lambda c: [c[4], 2])
    tracers = [_tracer(pkg, c) for c in cases]
    ex = pkg.GpuPathTracer(0)
    ex.set_tuning(mode=2, wave_items=5000)
    pkg.refine_batch(tracers, [c[4] for c in cases], executor=ex)
    pkg.refine_batch(tracers, 2, executor=ex)
    for k, (t, w) in enumerate(zip(tracers, want)):
        assert t.samples() == cases[k][4] + 2
        assert np.array_equal(t.read_accum().view(np.uint32), w.view(np.uint32)), f"scene {k} differs"
    # images resolve on each tracer's own stream after the batch
    assert tracers[0].image().shape == (cases[0][3], cases[0][2], 4)


def test_batch_matches_the_oracle(pkg, oracle):
    cases = _cases(pkg)[:3]
    tracers = [_tracer(pkg, c) for c in cases]
    pkg.refine_batch(tracers, [c[4] for c in cases])
    for t, c in zip(tracers, cases):
        cpu, _ = oracle.render(t.prepared(), c[4])
        assert np.array_equal(t.read_accum().view(np.uint32), cpu.view(np.uint32))


def test_batch_rejects_a_frame_without_a_scene(pkg):
    import ctypes as C
    N = pkg._native
    L = N.lib()
    t = _tracer(pkg, _cases(pkg)[0])
    t.prepared()
    bare = C.c_void_p()
    assert L.oxpt_create(0, C.byref(bare)) == 0
    try:
        frames = (N.BatchFrame * 2)(N.BatchFrame(t.ctx, 0, 1, 0, 40), N.BatchFrame(bare, 0, 1, 0, 1))
        st = L.oxpt_refine_batch(t.ctx, frames, 2)
        assert st == N.E_INVALID
        assert b"batch frame 1" in L.oxpt_last_error(t.ctx)
    finally:
        L.oxpt_destroy(bare)


def test_graph_is_reused_while_the_step_shape_is_unchanged(pkg):
    """Two refine steps of the same shape: one graph instantiation, and the
    second step (new sample indices, read from device memory) still matches
    each scene refined alone."""
    import ctypes as C
    cases = _cases(pkg)
    want = _alone(pkg, cases, lambda c: [2, 2])
    tracers = [_tracer(pkg, c) for c in cases]
    ex = pkg.GpuPathTracer(0)
    ex.set_tuning(mode=2, graphs=1, wave_items=4000)
    L = pkg._native.lib()
    for _ in range(2):
        pkg.refine_batch(tracers, 2, executor=ex)
    builds = C.c_uint64()
    assert L.oxpt_diag_graph_builds(ex.ctx, C.byref(builds)) == 0
    assert builds.value == 1
    for k, (t, w) in enumerate(zip(tracers, want)):
        assert np.array_equal(t.read_accum().view(np.uint32), w.view(np.uint32)), f"scene {k} differs"
    launches, iters = C.c_uint64(), C.c_uint64()
    L.oxpt_diag_launch_count(ex.ctx, C.byref(launches))
    L.oxpt_diag_wave_iterations(ex.ctx, C.byref(iters))
    assert iters.value > 0 and launches.value > 5 * iters.value


@pytest.mark.parametrize("mode", [1, 2])
def test_single_tracer_graph_plan_matches_the_oracle(pkg, oracle, mode):
    """With graphs on, a tracer's own refine runs as a one-frame batch in a
    CUDA graph; refine(2) + refine(3) equals the oracle's 5 samples."""
    c = _cases(pkg)[1]
    t = _tracer(pkg, c)
    t.set_tuning(mode=mode, graphs=1, wave_slots=500)
    t.refine(2)
    t.refine(3)
    cpu, _ = oracle.render(t.prepared(), 5)
    assert np.array_equal(t.read_accum().view(np.uint32), cpu.view(np.uint32))
