"""The tolerance plan (closest_walk = 1: continuation rays walk the
four-wide tree, nearest child first) against the oracle, on the north
star's own checks rather than bit equality:

* closest-hit triangle ids on 10^6 random rays equal the oracle's ordered
  binary walk except ties within 1e-6 relative t (where the ids agree, t
  and barycentrics are the same bits: the same triangle test);
* images at equal spp are within >= 60 dB PSNR of the oracle built with
  the C library's transcendentals (the CPU tracer's arithmetic), on the
  Cornell box at 256x256, 16 spp, 8 bounces, roulette from 3, and on the
  layered-material and alpha scenes;
* the same images with the shading kernels' fast-math build (FMA
  contraction, approximate division and square root, the CUDA library's
  transcendentals: fast_shading = 1), the rest of the tolerance plan.
"""
from __future__ import annotations

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu


def _rays(rng, n, lo, hi):
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.standard_normal((n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 3.0e38
    rays[: n // 4, 3] = rng.uniform(0.0, 2.0 * (hi - lo), n // 4).astype(np.float32)
    rays[:, 4:7] = d
    rays[:, 7] = np.frombuffer(np.full(n, 0xFFFFFFFF, np.uint32).tobytes(), np.float32)
    return rays


def check_ids(pkg, oracle, t, p, rays, min_hits):
    L = pkg._native.lib()
    n = rays.shape[0]
    for flags in (8, 10):  # four-wide closest hit; and as primary rays (back-face culling)
        slot = np.empty(n, np.uint32)
        gid = np.empty(n, np.uint32)
        tt = np.empty(n, np.float32)
        bary = np.empty((n, 3), np.float32)
        assert L.oxpt_diag_trace_rays(t.ctx, n, rays.ctypes.data, flags, slot.ctypes.data, gid.ctypes.data,
                                      tt.ctypes.data, bary.ctypes.data) == 0
        oslot, ogid, ot, obary, _ = oracle.trace_rays(p, rays, flags & 3)
        assert (ogid != 0xFFFFFFFF).sum() >= min_hits
        diff = gid != ogid
        if diff.any():
            both = diff & (gid != 0xFFFFFFFF) & (ogid != 0xFFFFFFFF)
            assert np.array_equal(diff, both), "a hit was found by one walk only"
            rel = np.abs(tt[diff] - ot[diff]) / np.maximum(np.abs(ot[diff]), 1e-30)
            assert np.all(rel <= 1e-6), f"{diff.sum()} ids differ beyond ties"
        same = ~diff
        assert np.array_equal(tt[same].view(np.uint32), ot[same].view(np.uint32))
        assert np.array_equal(bary[same].view(np.uint32), obary[same].view(np.uint32))


@pytest.mark.parametrize("which", ["icosphere", "boxes", "cornell", "alpha"])
def test_four_wide_closest_hit_ids_on_a_million_rays(pkg, oracle, which):
    if which == "icosphere":
        scene, lo, hi = pkg.Scene.icosphere(freq=64, seed=3, n_textures=0, n_punctual=0, n_emissive=16), -1.3, 1.3
    elif which == "boxes":
        scene, lo, hi = pkg.Scene.box_field(2000, seed=4, material_mix=0), -8.0, 8.0
    elif which == "alpha":
        scene, lo, hi = scenes.alpha_scene(pkg), -1.5, 1.5
    else:
        scene, lo, hi = pkg.Scene.cornell(), 0.01, 0.99
    t = pkg.GpuPathTracer(0)
    assert t.sync(scene, pkg.RenderOptions(width=16, height=16))
    p = t.prepared()
    check_ids(pkg, oracle, t, p, _rays(np.random.default_rng(12), 1_000_000, lo, hi), 100_000)


def _psnr_vs_libm(pkg, oracle, scene, opts, spp, env=None, variant=4, mode=2, fast=0):
    t = pkg.GpuPathTracer(0)
    if env is not None:
        t.set_environment(env)
    assert t.sync(scene, opts)
    t.set_tuning(mode=mode, trace_variant=variant, closest_walk=1, fast_shading=fast)
    assert t.tuning().closest_walk == 1 and t.tuning().fast_shading == fast
    t.refine(spp)
    img = t.image()
    cpu, _ = oracle.render(t.prepared(), spp, libm=True)
    ref = oracle.resolve(cpu, t.resolve_params(False), hdr=False, libm=True)
    return scenes.psnr_rgb8(img, ref)


@pytest.mark.parametrize("fast", [0, 1])
def test_cornell_256_16spp_psnr_at_least_60db(pkg, oracle, fast):
    opts = pkg.RenderOptions(width=256, height=256, path_trace=pkg.PathTraceOptions(samples_per_pixel=16,
                                                                                    max_bounces=8, rr_start=3,
                                                                                    seed=0))
    assert _psnr_vs_libm(pkg, oracle, pkg.Scene.cornell(), opts, 16, fast=fast) >= 60.0


@pytest.mark.parametrize("variant,fast", [(3, 0), (5, 0), (4, 1)])
@pytest.mark.parametrize("which", ["layered", "alpha", "materials"])
def test_scenes_psnr_at_least_60db(pkg, oracle, which, variant, fast):
    env = None
    if which == "layered":
        scene = pkg.Scene.icosphere(freq=24, seed=9, n_materials=16, n_textures=4, tex_size=128, n_punctual=4,
                                    n_emissive=32, material_mix=1)
        env = pkg.EnvironmentMap.sky(128, 64)
    elif which == "alpha":
        scene = scenes.alpha_scene(pkg)
    else:
        scene = scenes.materials_scene(pkg)
    opts = pkg.RenderOptions(width=64, height=48, path_trace=pkg.PathTraceOptions(samples_per_pixel=16,
                                                                                  max_bounces=10))
    assert _psnr_vs_libm(pkg, oracle, scene, opts, 16, env, variant, fast=fast) >= 60.0


def test_tolerance_plan_needs_the_short_stack_kernels(pkg):
    t = pkg.GpuPathTracer(0)
    with pytest.raises(pkg.InvalidOptionsError):
        t.set_tuning(trace_variant=0, closest_walk=1)


def test_fast_shading_needs_the_split_wavefront(pkg):
    t = pkg.GpuPathTracer(0)
    with pytest.raises(pkg.InvalidOptionsError):
        t.set_tuning(mode=1, fast_shading=1)
    t.set_tuning(mode=2, fast_shading=1)
    assert t.tuning().fast_shading == 1
