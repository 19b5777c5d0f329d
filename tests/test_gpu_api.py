"""The reference's behavioural tests (tests/pathtrace.rs:295-565) on the
CUDA tracer through its public API."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def opts(pkg, w, h, spp, bounces, **kw):
    return pkg.RenderOptions(width=w, height=h, scene_camera=0, background=(16, 16, 20, 255),
                             path_trace=pkg.PathTraceOptions(samples_per_pixel=spp, max_bounces=bounces, **kw))


@pytest.mark.parametrize("strategy", [0, 1, 2])
def test_white_furnace(pkg, strategy):
    g = json.loads((GOLDEN / "furnace.json").read_text())
    t = pkg.GpuPathTracer(0)
    o = opts(pkg, g["width"], g["height"], g["spp"], g["bounces"], strategy=strategy)
    o.ambient = 0.0
    img = t.render_hdr(pkg.Scene.furnace(g["rho"], g["le"]), o)
    m = img[..., :3].mean(axis=(0, 1))
    assert np.all(np.abs(m - g["expected"]) < g["tolerance"]), m


def test_deterministic_for_a_seed(pkg):
    t = pkg.GpuPathTracer(0)
    s = pkg.Scene.cornell()
    o = opts(pkg, 64, 64, 8, 8)
    a = t.render(s, o)
    b = t.render(s, o)
    assert np.array_equal(a, b)
    o.path_trace.seed = 7
    c = t.render(s, o)
    assert not np.array_equal(a, c)


def test_progressive_refines_add_up(pkg):
    t = pkg.GpuPathTracer(0)
    s = pkg.Scene.cornell()
    o = opts(pkg, 64, 48, 0, 8)
    t.sync(s, o)
    t.refine(3)
    t.refine(5)
    assert t.samples() == 8
    split = t.hdr()
    t.reset()
    assert t.samples() == 0
    t.refine(8)
    whole = t.hdr()
    assert np.array_equal(split.view(np.uint32), whole.view(np.uint32))


def test_refine_split_across_launches_is_bit_exact(pkg):
    """Launch splitting (a tiny per-launch path cap forces row and sample
    chunks) leaves every pixel's sum unchanged."""
    s = pkg.Scene.cornell()
    o = opts(pkg, 50, 37, 0, 8)
    a = pkg.GpuPathTracer(0)
    a.sync(s, o)
    a.refine(6)
    b = pkg.GpuPathTracer(0)
    assert pkg._native.lib().oxpt_diag_set_launch(b.ctx, 64, 1, 777) == 0
    b.sync(s, o)
    b.refine(6)
    assert np.array_equal(a.read_accum().view(np.uint32), b.read_accum().view(np.uint32))


def test_reset_rules_match_the_cpu_tracer(pkg):
    t = pkg.GpuPathTracer(0)
    s = pkg.Scene.cornell()
    o = opts(pkg, 32, 32, 16, 4)
    assert t.sync(s, o), "first sync prepares"
    t.refine(2)
    assert not t.sync(s, o), "no change, no reset"
    assert t.samples() == 2
    d = opts(pkg, 32, 32, 16, 4)
    d.background = (200, 0, 0, 255)
    d.tone_map = pkg.ToneMap.ACES_FITTED
    d.exposure = 2.0
    d.path_trace.samples_per_pixel = 999
    assert not t.sync(s, d)
    assert t.samples() == 2
    assert not t.is_converged()

    def seed(x):
        x.path_trace.seed = 3

    def bounces(x):
        x.path_trace.max_bounces = 2

    def width(x):
        x.width = 40

    def ambient(x):
        x.ambient = 0.5

    for change in (seed, bounces, width, ambient):
        t.refine(1)
        c = opts(pkg, 32, 32, 999, 4)
        c.background, c.tone_map, c.exposure = d.background, d.tone_map, d.exposure
        change(c)
        assert t.sync(s, c)
        assert t.samples() == 0
        t.sync(s, d)
    t.refine(1)
    t.invalidate_scene()
    assert t.sync(s, d)
    assert t.samples() == 0
    t.refine(1)
    t.set_environment(pkg.EnvironmentMap(scenes.sky()))
    assert t.samples() == 0
    t.refine(1)
    assert t.samples() == 1
    fresh = pkg.GpuPathTracer(0)
    fresh.refine(4)
    assert fresh.samples() == 0


def test_uncovered_pixels_keep_background_bytes(pkg, oracle):
    s = pkg.Scene()
    m = s.add_material(pkg.material(base_color=(0.8, 0.3, 0.2, 1), metallic=0.0))
    pos, nrm, uv = scenes.sphere(0.5, 16, 8)
    s.add_mesh(pos, m, normals=nrm, uv0=uv)
    s.add_light(0, direction=(0, -1, -1), intensity=3.0)
    s.add_camera((0, 0, 3), (0, 0, 0), 0.6)
    o = opts(pkg, 64, 48, 4, 2)
    o.background = (37, 99, 201, 180)
    t = pkg.GpuPathTracer(0)
    img = t.render(s, o)
    bg = np.all(img == np.array([37, 99, 201, 180], np.uint8), axis=2)
    assert bg.sum() > 100
    acc = t.read_accum()
    assert np.all(bg == (acc[..., 3] == 0))
    ref = oracle.resolve(acc, t.resolve_params(False), hdr=False)
    assert np.array_equal(img, ref)


def test_draw_texture_mode_and_registry(pkg):
    s = pkg.Scene.cornell()
    o = opts(pkg, 40, 30, 2, 2)
    t = pkg.GpuPathTracer(0)
    t.sync(s, o)
    t.refine(2)
    tex = t.draw_texture()
    assert (tex.width, tex.height, tex.format, tex.pitch_bytes) == (40, 30, "rgba8", 160)
    r = pkg.GpuRenderer(0)
    r.set_mode(pkg.GpuMode.PATH_TRACE)
    assert r.mode() is pkg.GpuMode.PATH_TRACE
    a = r.render(s, o)
    b = t.render(s, o)
    assert np.array_equal(a, b)
    reg = pkg.RenderRegistry()
    pkg.register_into(reg)
    assert pkg.PATHTRACE_BACKEND_NAME == "gpu-pathtrace"
    via = reg.make(pkg.PATHTRACE_BACKEND_NAME)
    assert np.array_equal(via.render(s, o), a)


def test_empty_scene_is_all_background(pkg):
    o = opts(pkg, 16, 12, 4, 4)
    o.scene_camera = None
    o.background = (1, 2, 3, 4)
    img = pkg.GpuPathTracer(0).render(pkg.Scene(), o)
    assert np.all(img == np.array([1, 2, 3, 4], np.uint8))


def test_image_before_sync_is_background(pkg):
    t = pkg.GpuPathTracer(0)
    img = t.image()
    assert img.shape == (1, 1, 4)


def test_oversized_image_is_invalid_options(pkg):
    t = pkg.GpuPathTracer(0)
    with pytest.raises(pkg.InvalidOptionsError):
        t.sync(pkg.Scene.cornell(), opts(pkg, 40000, 8, 1, 1))
