"""The shared-memory short-stack traversal kernels (trace_variant 3-5)
against the oracle and against the local-memory kernels.

Same walks, storage moved on chip (walk stacks in shared-memory columns,
top nodes staged, alpha tests out of line), so:
* accumulators equal the oracle's bit for bit under every occupancy
  target, both execution plans, binary and four-wide shadow walks, and
  with the shared part of the stack cut to 0, 1 or 3 entries (entries
  spill to local memory much earlier: that path is exercised too);
* the traversal counters (boxes, leaves, triangles, pops) equal the
  oracle's for the binary walk and the local-memory kernels' for the
  four-wide walk;
* batched launches (one executor over several scenes, no node staging)
  equal each scene's own refine.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu


def _scene(pkg, which):
    if which == "materials":
        return scenes.materials_scene(pkg), None
    if which == "alpha":
        return scenes.alpha_scene(pkg), None
    if which == "textured":
        return scenes.textured_scene(pkg), None
    scene = pkg.Scene.icosphere(freq=16, seed=2, n_materials=12, n_textures=3, tex_size=64, n_punctual=3,
                                n_emissive=16, material_mix=1)
    return scene, pkg.EnvironmentMap.sky(64, 32)


def _tracer(pkg, scene, env, w=40, h=28, spp=6, bounces=10):
    t = pkg.GpuPathTracer(0)
    if env is not None:
        t.set_environment(env)
    assert t.sync(scene, pkg.RenderOptions(width=w, height=h, path_trace=pkg.PathTraceOptions(
        samples_per_pixel=spp, max_bounces=bounces)))
    return t


@pytest.mark.parametrize("walk", [0, 1])
@pytest.mark.parametrize("variant", [3, 4, 5])
@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("which", ["materials", "alpha", "layered", "textured"])
def test_short_stack_kernels_bit_exact(pkg, oracle, which, mode, variant, walk):
    scene, env = _scene(pkg, which)
    t = _tracer(pkg, scene, env)
    t.set_tuning(mode=mode, trace_variant=variant, shadow_walk=walk, wave_slots=333, wave_items=2000, refill=8)
    t.refine(6)
    cpu, _ = oracle.render(t.prepared(), 6)
    assert np.array_equal(t.read_accum().view(np.uint32), cpu.view(np.uint32))


@pytest.mark.parametrize("stage", [0, 200])
@pytest.mark.parametrize("lim", [0, 1, 3, 16])
@pytest.mark.parametrize("walk", [0, 1])
def test_stack_entries_in_local_memory_bit_exact(pkg, oracle, lim, walk, stage):
    """Fewer shared entries push the walk onto its local-memory part; staged
    top nodes serve the binary walk's first levels from shared memory."""
    scene = pkg.Scene.icosphere(freq=48, seed=5, n_materials=8, n_textures=2, tex_size=64, n_punctual=4,
                                n_emissive=32, material_mix=1)
    env = pkg.EnvironmentMap.sky(64, 32)
    t = _tracer(pkg, scene, env, w=48, h=32, spp=4, bounces=8)
    t.set_tuning(mode=2, trace_variant=4, shadow_walk=walk)
    L = pkg._native.lib()
    cur = (C.c_uint32 * 2)()
    assert L.oxpt_diag_get_walk(t.ctx, cur) == 0 and cur[0] > 0
    assert L.oxpt_diag_set_walk(t.ctx, lim, stage) == 0
    t.refine(4)
    cpu, _ = oracle.render(t.prepared(), 4)
    assert np.array_equal(t.read_accum().view(np.uint32), cpu.view(np.uint32))


@pytest.mark.parametrize("variant", [3, 5])
@pytest.mark.parametrize("mode", [1, 2])
def test_short_stack_counters_match(pkg, oracle, mode, variant):
    L = pkg._native.lib()
    scene, _ = _scene(pkg, "materials")
    opts = pkg.RenderOptions(width=48, height=32, path_trace=pkg.PathTraceOptions(samples_per_pixel=4))
    runs = {}
    for tv, walk in ((variant, 1), (variant, 0), (0, 0)):
        t = pkg.GpuPathTracer(0)
        assert t.sync(scene, opts)
        t.set_tuning(mode=mode, trace_variant=tv, shadow_walk=walk)
        p = t.prepared()
        out = (C.c_uint64 * 8)()
        assert L.oxpt_diag_refine_counted(t.ctx, 0, 4, out) == 0
        split = (C.c_uint64 * 16)()
        assert L.oxpt_diag_counters_split(t.ctx, split) == 0
        runs[(tv, walk)] = (list(out), list(split), t.read_accum())
    cpu, cnt = oracle.render(p, 4)
    assert runs[(variant, 1)][0] == [int(c) for c in cnt]  # binary walk: the reference's counters
    assert runs[(variant, 0)][1] == runs[(0, 0)][1]          # four-wide: the local-memory kernel's
    for k, (_, _, acc) in runs.items():
        assert np.array_equal(acc.view(np.uint32), cpu.view(np.uint32)), k


def test_short_stack_batch_equals_each_refine(pkg):
    items = [(scenes.materials_scene(pkg), None, 40, 28, 4), (scenes.alpha_scene(pkg), None, 33, 21, 6),
             _scene(pkg, "layered") + (48, 32, 5)]
    tracers, want = [], []
    for scene, env, w, h, spp in items:
        alone = _tracer(pkg, scene, env, w, h, spp)
        alone.set_tuning(mode=2, trace_variant=0)
        alone.refine(spp)
        want.append(alone.read_accum())
        t = _tracer(pkg, scene, env, w, h, spp)
        tracers.append(t)
    ex = pkg.GpuPathTracer(0)
    ex.set_tuning(mode=2, trace_variant=4, wave_slots=500, graphs=1)
    pkg.refine_batch(tracers, [it[4] for it in items], executor=ex)
    for t, w_ in zip(tracers, want):
        assert np.array_equal(t.read_accum().view(np.uint32), w_.view(np.uint32))


@pytest.mark.parametrize("mask", [0, 1])
@pytest.mark.parametrize("nee", [0, 3])
@pytest.mark.parametrize("which", ["materials", "layered", "alpha"])
def test_nee_visibility_masks_bit_exact(pkg, oracle, which, nee, mask):
    """The split plan's NEE results as per-slot visibility bits (1) or a
    pending record per job (0): the oracle's accumulator either way."""
    scene, env = _scene(pkg, which)
    t = _tracer(pkg, scene, env)
    t.set_tuning(mode=2, nee_variant=nee, trace_variant=4, wave_slots=333, wave_items=2000)
    assert pkg._native.lib().oxpt_diag_set_nee_mask(t.ctx, mask) == 0
    t.refine(6)
    cpu, _ = oracle.render(t.prepared(), 6)
    assert np.array_equal(t.read_accum().view(np.uint32), cpu.view(np.uint32))


@pytest.mark.parametrize("variant", [3, 4, 5])
@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("which", ["materials", "alpha", "layered"])
def test_postponed_leaf_shadow_walk_bit_exact(pkg, oracle, which, mode, variant):
    """Shadow rays that park leaves until their warp has no node work left
    (speculative traversal): occlusion is order-free, so the accumulator is
    the oracle's bit for bit; few slots and small refills mix lanes at
    every stage of the walk."""
    scene, env = _scene(pkg, which)
    t = _tracer(pkg, scene, env)
    t.set_tuning(mode=mode, trace_variant=variant, shadow_walk=0, wave_slots=333, wave_items=2000, refill=4)
    assert pkg._native.lib().oxpt_diag_set_shadow_postpone(t.ctx, 1) == 0
    t.refine(6)
    cpu, _ = oracle.render(t.prepared(), 6)
    assert np.array_equal(t.read_accum().view(np.uint32), cpu.view(np.uint32))


def test_postponed_leaf_shadow_walk_in_a_batch(pkg):
    items = [(scenes.materials_scene(pkg), None, 40, 28, 4), _scene(pkg, "layered") + (48, 32, 5)]
    tracers, want = [], []
    for scene, env, w, h, spp in items:
        alone = _tracer(pkg, scene, env, w, h, spp)
        alone.refine(spp)
        want.append(alone.read_accum())
        tracers.append(_tracer(pkg, scene, env, w, h, spp))
    ex = pkg.GpuPathTracer(0)
    ex.set_tuning(mode=2, trace_variant=4, wave_slots=500, graphs=1, refill=8)
    assert pkg._native.lib().oxpt_diag_set_shadow_postpone(ex.ctx, 1) == 0
    pkg.refine_batch(tracers, [it[4] for it in items], executor=ex)
    for t, w_ in zip(tracers, want):
        assert np.array_equal(t.read_accum().view(np.uint32), w_.view(np.uint32))


@pytest.mark.parametrize("variant", [0, 4])
@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("which", ["materials", "alpha", "layered"])
def test_reordered_continuation_rays_bit_exact(pkg, oracle, which, mode, variant):
    """Continuation rays sorted by origin cell and direction octant before
    the closest-hit walk, shadow rays walked in the order of their light and
    origin cell: every ray is walked alone, so the accumulator is the
    oracle's bit for bit."""
    scene, env = _scene(pkg, which)
    t = _tracer(pkg, scene, env)
    t.set_tuning(mode=mode, trace_variant=variant, wave_slots=333, wave_items=2000)
    assert pkg._native.lib().oxpt_diag_set_ray_order(t.ctx, 3) == 0  # both queues (shadow: variants 3-5)
    t.refine(6)
    cpu, _ = oracle.render(t.prepared(), 6)
    assert np.array_equal(t.read_accum().view(np.uint32), cpu.view(np.uint32))


def test_reordered_continuation_rays_in_a_graph_batch(pkg):
    items = [(scenes.materials_scene(pkg), None, 40, 28, 4), _scene(pkg, "layered") + (48, 32, 5)]
    tracers, want = [], []
    for scene, env, w, h, spp in items:
        alone = _tracer(pkg, scene, env, w, h, spp)
        alone.refine(spp)
        want.append(alone.read_accum())
        tracers.append(_tracer(pkg, scene, env, w, h, spp))
    ex = pkg.GpuPathTracer(0)
    ex.set_tuning(mode=2, trace_variant=4, wave_slots=500, graphs=1)
    assert pkg._native.lib().oxpt_diag_set_ray_order(ex.ctx, 3) == 0
    for _ in range(2):  # the second step reuses the graph
        for t in tracers:
            t.reset()
        pkg.refine_batch(tracers, [it[4] for it in items], executor=ex)
        for t, w_ in zip(tracers, want):
            assert np.array_equal(t.read_accum().view(np.uint32), w_.view(np.uint32))


@pytest.mark.parametrize("which", ["materials", "layered"])
@pytest.mark.parametrize("mode,variant", [(2, 4), (1, 3)])
def test_persisting_l2_window_bit_exact(pkg, oracle, which, mode, variant):
    """The walks' tree nodes marked as persisting L2 lines (an access-policy
    window on each traversal launch) change only where lines live: the
    accumulator is the oracle's bit for bit."""
    import ctypes as C
    scene, env = _scene(pkg, which)
    t = _tracer(pkg, scene, env)
    t.set_tuning(mode=mode, trace_variant=variant, wave_slots=333, wave_items=2000)
    granted = C.c_uint64(0)
    assert pkg._native.lib().oxpt_diag_set_l2_window(t.ctx, 1, C.byref(granted)) == 0
    assert granted.value > 0
    t.refine(6)
    cpu, _ = oracle.render(t.prepared(), 6)
    assert np.array_equal(t.read_accum().view(np.uint32), cpu.view(np.uint32))


def test_persisting_l2_window_in_a_graph_batch(pkg):
    import ctypes as C
    items = [(scenes.materials_scene(pkg), None, 40, 28, 4), _scene(pkg, "layered") + (48, 32, 5)]
    want, tracers = [], []
    for scene, env, w, h, spp in items:
        alone = _tracer(pkg, scene, env, w, h, spp)
        alone.refine(spp)
        want.append(alone.read_accum())
        tracers.append(_tracer(pkg, scene, env, w, h, spp))
    ex = pkg.GpuPathTracer(0)
    ex.set_tuning(mode=2, trace_variant=4, wave_slots=500, graphs=1)
    assert pkg._native.lib().oxpt_diag_set_l2_window(ex.ctx, 1, None) == 0
    for _ in range(2):
        for t in tracers:
            t.reset()
        pkg.refine_batch(tracers, [it[4] for it in items], executor=ex)
        for t, w_ in zip(tracers, want):
            assert np.array_equal(t.read_accum().view(np.uint32), w_.view(np.uint32))
    # one scene in the batch: the launches carry the window
    t = tracers[1]
    t.reset()
    pkg.refine_batch([t], [items[1][4]], executor=ex)
    assert np.array_equal(t.read_accum().view(np.uint32), want[1].view(np.uint32))
    assert pkg._native.lib().oxpt_diag_set_l2_window(ex.ctx, 0, None) == 0
