"""GPU parity for every texture-sampler and resolve mode, and for the row
tiles of the multi-GPU split, against the CPU oracle.

* Sampler (pathtrace.wgsl:306-420): min filters 0-5 (nearest, linear,
  nearest-mip-nearest, linear-mip-nearest, nearest-mip-linear,
  linear-mip-linear) x nearest / linear magnification x clamp / mirror /
  repeat wrap, on a minified texture (grazing floor, ray-cone LOD > 0) and
  on a magnified one (texels larger than pixels, LOD <= 0). Accumulators
  bit for bit.
* Resolve (resolve.wgsl:38-75, 138-188): tone maps clamp / Reinhard /
  ACES-fitted x exposure x background (opaque and translucent, over
  uncovered pixels) x RGBA8 / RGBA32F output, through oxpt_resolve on the
  device against oracle.resolve, bit for bit.
* Row tiles (src/pathtrace.rs:592-615 tiles by rows; the multi-GPU split
  gives each rank a contiguous tile): oxpt_tracer_refine_rows per tile of
  worlds 2, 3 and 8, each tile on its own tracer as each rank would, in two
  progressive refines; the stitched accumulator equals one whole-frame
  refine bit for bit.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu


def _opts(pkg, w, h, spp, bounces=6, **kw):
    return pkg.RenderOptions(width=w, height=h, path_trace=pkg.PathTraceOptions(samples_per_pixel=spp,
                                                                                max_bounces=bounces, **kw))


def _accum_vs_oracle(pkg, oracle, scene, opts, spp):
    t = pkg.GpuPathTracer(0)
    assert t.sync(scene, opts)
    t.refine(spp)
    t.finish()
    gpu = t.read_accum()
    cpu, _ = oracle.render(t.prepared(), spp)
    diff = gpu.view(np.uint32) != cpu.view(np.uint32)
    assert not diff.any(), f"{np.count_nonzero(diff.any(axis=2))} pixels differ"
    return gpu


@pytest.mark.parametrize("wrap", [(0, 0), (1, 1), (2, 2), (0, 1)])
@pytest.mark.parametrize("mag_linear", [False, True])
@pytest.mark.parametrize("minf", range(6))
def test_sampler_minified_bit_exact(pkg, oracle, minf, mag_linear, wrap):
    scene = scenes.textured_scene(pkg, min_filter=minf, wrap=wrap, mag_linear=mag_linear)
    _accum_vs_oracle(pkg, oracle, scene, _opts(pkg, 48, 32, 2), 2)


@pytest.mark.parametrize("wrap", [(0, 0), (1, 1), (2, 2)])
@pytest.mark.parametrize("mag_linear", [False, True])
@pytest.mark.parametrize("minf", [0, 5])
def test_sampler_magnified_bit_exact(pkg, oracle, minf, mag_linear, wrap):
    scene = scenes.textured_scene(pkg, min_filter=minf, wrap=wrap, mag_linear=mag_linear, tex_size=8)
    _accum_vs_oracle(pkg, oracle, scene, _opts(pkg, 96, 64, 2), 2)


def test_magnified_texture_changes_with_the_mag_filter(pkg, oracle):
    """The magnified case really takes the mag filter: nearest and linear
    magnification give different images."""
    a = _accum_vs_oracle(pkg, oracle, scenes.textured_scene(pkg, mag_linear=False, tex_size=8),
                         _opts(pkg, 96, 64, 1), 1)
    b = _accum_vs_oracle(pkg, oracle, scenes.textured_scene(pkg, mag_linear=True, tex_size=8),
                         _opts(pkg, 96, 64, 1), 1)
    assert not np.array_equal(a, b)


def _uncovered_scene(pkg):
    s = pkg.Scene()
    m = s.add_material(pkg.material(base_color=(0.8, 0.3, 0.2, 1), metallic=0.0))
    pos, nrm, uv = scenes.sphere(0.5, 16, 8)
    s.add_mesh(pos, m, normals=nrm, uv0=uv)
    s.add_light(1, position=(1.0, 1.5, 2.0), intensity=40.0)
    s.add_camera((0, 0, 3), (0, 0, 0), 0.6)
    return s


@pytest.mark.parametrize("which", ["materials", "uncovered"])
def test_resolve_modes_bit_exact(pkg, oracle, which):
    scene = scenes.materials_scene(pkg) if which == "materials" else _uncovered_scene(pkg)
    t = pkg.GpuPathTracer(0)
    assert t.sync(scene, _opts(pkg, 64, 48, 8))
    t.refine(8)
    t.finish()
    acc = t.read_accum()
    if which == "uncovered":
        assert (acc[..., 3] == 0).sum() > 100
    L = pkg._native.lib()
    checked = 0
    for hdr in (0, 1):
        for tone in (0, 1, 2):
            for exposure in (0.25, 1.0, 3.0):
                for bg in ((0.0, 0.0, 0.0, 1.0), (37 / 255, 99 / 255, 201 / 255, 180 / 255)):
                    rp = t.resolve_params(bool(hdr))
                    rp.cfg[2] = tone
                    rp.exposure[0] = exposure
                    for k in range(4):
                        rp.background[k] = bg[k]
                    out = np.empty((48, 64, 4), np.float32 if hdr else np.uint8)
                    assert L.oxpt_resolve(t.ctx, C.byref(rp), hdr, out.ctypes.data, None) == 0
                    want = oracle.resolve(acc, rp, hdr=bool(hdr))
                    assert np.array_equal(out.view(np.uint8), want.view(np.uint8)), (hdr, tone, exposure, bg)
                    checked += 1
    assert checked == 36


def test_tone_maps_differ(pkg, oracle):
    """The sweep is not vacuous: the three tone maps give three images."""
    t = pkg.GpuPathTracer(0)
    assert t.sync(scenes.materials_scene(pkg), _opts(pkg, 32, 24, 4))
    t.refine(4)
    L = pkg._native.lib()
    imgs = []
    for tone in (0, 1, 2):
        rp = t.resolve_params(False)
        rp.cfg[2] = tone
        out = np.empty((24, 32, 4), np.uint8)
        assert L.oxpt_resolve(t.ctx, C.byref(rp), 0, out.ctypes.data, None) == 0
        imgs.append(out)
    assert not np.array_equal(imgs[0], imgs[1]) and not np.array_equal(imgs[1], imgs[2])


@pytest.mark.parametrize("world", [2, 3, 8])
def test_row_tiles_stitch_to_the_whole_frame(pkg, world):
    from oxideav_render_vulkan_b200 import shard
    scene = pkg.Scene.icosphere(freq=16, seed=2, n_materials=12, n_textures=3, tex_size=64, n_punctual=3,
                                n_emissive=16, material_mix=1)
    env = pkg.EnvironmentMap.sky(64, 32)
    w, h = 61, 45
    opts = _opts(pkg, w, h, 5, bounces=10)
    whole = pkg.GpuPathTracer(0)
    whole.set_environment(env)
    assert whole.sync(scene, opts)
    whole.refine(5)
    want = whole.read_accum()
    got = np.full_like(want, np.nan)
    L = pkg._native.lib()
    for rank in range(world):
        y0, rows = shard.row_tile(h, rank, world)
        t = pkg.GpuPathTracer(0)
        t.set_environment(env)
        assert t.sync(scene, opts)
        for n in (2, 3):  # progressive: samples 0-1, then 2-4
            assert L.oxpt_tracer_refine_rows(t._h, n, y0, rows) == 0
        assert t.samples() == 5
        acc = t.read_accum()
        got[y0:y0 + rows] = acc[y0:y0 + rows]
        # rows outside the tile were never traced
        outside = np.ones(h, bool)
        outside[y0:y0 + rows] = False
        assert not acc[outside].any()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
