"""Behavioural invariants of the estimator, on the CPU oracle
(tests/pathtrace.rs:420-565 restated without a GPU)."""
from __future__ import annotations

import numpy as np
import pytest

import scenes


def _prep(pkg, scene, w, h, env=None, **pt):
    o = pkg.RenderOptions(width=w, height=h, path_trace=pkg.PathTraceOptions(**pt))
    return pkg.prepare(scene, o, env)


def test_deterministic_and_seed_sensitive(pkg, oracle):
    s = pkg.Scene.cornell()
    a, _ = oracle.render(_prep(pkg, s, 32, 32, max_bounces=8), 4)
    b, _ = oracle.render(_prep(pkg, s, 32, 32, max_bounces=8), 4)
    c, _ = oracle.render(_prep(pkg, s, 32, 32, max_bounces=8, seed=7), 4)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert not np.array_equal(a, c)


def test_refines_add_up_bitwise(pkg, oracle):
    """refine(3) + refine(5) == refine(8): the per-pixel sum is sequential
    in sample order whatever the dispatch split."""
    p = _prep(pkg, scenes.materials_scene(pkg), 40, 30)
    whole, _ = oracle.render(p, 8)
    split, _ = oracle.render(p, 3)
    oracle.dispatch(p, p.params, (3, 5, 0, 30), split)
    assert np.array_equal(whole.view(np.uint32), split.view(np.uint32))
    rows = np.zeros_like(whole)
    for y0 in range(0, 30, 7):
        oracle.dispatch(p, p.params, (0, 8, y0, min(7, 30 - y0)), rows)
    assert np.array_equal(whole.view(np.uint32), rows.view(np.uint32))


def test_thread_count_does_not_change_results(pkg, oracle):
    p = _prep(pkg, scenes.alpha_scene(pkg), 32, 24)
    a, ca = oracle.render(p, 4, threads=1)
    b, cb = oracle.render(p, 4, threads=8)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(ca, cb)


@pytest.mark.parametrize("which", ["cornell", "materials", "textured"])
def test_portable_math_vs_libm_psnr_at_least_60db(pkg, oracle, which):
    scene = {"cornell": lambda: pkg.Scene.cornell(), "materials": lambda: scenes.materials_scene(pkg),
             "textured": lambda: scenes.textured_scene(pkg)}[which]()
    p = _prep(pkg, scene, 48, 36)
    a, _ = oracle.render(p, 16, libm=False)
    b, _ = oracle.render(p, 16, libm=True)
    rp = pkg._native.ResolveParams((1, 3, 0, 0), (1.0, 16.0, 48.0, 0.0), (0.0, 0.0, 0.0, 1.0))
    ia = oracle.resolve(a, rp, hdr=False)
    ib = oracle.resolve(b, rp, hdr=False, libm=True)
    assert scenes.psnr_rgb8(ia, ib) >= 60.0


def test_background_bytes_round_trip_exactly(pkg, oracle):
    """An uncovered pixel keeps the background bytes for every byte value
    (sRGB decode, then encode, in resolve.wgsl:151-188)."""
    acc = np.zeros((1, 256, 4), np.float32)
    for a in (255, 180, 4):
        for v in range(256):
            rp = pkg._native.ResolveParams((1, 3, 0, 0), (1.0, 4.0, 256.0, 0.0), (v / 255.0, v / 255.0, v / 255.0,
                                                                                   a / 255.0))
            img = oracle.resolve(acc[:, :1], rp, hdr=False)
            assert img[0, 0].tolist() == [v, v, v, a], (v, a)


def test_partial_coverage_composites_over_background(pkg, oracle):
    acc = np.array([[[2.0, 1.0, 0.5, 2.0], [0.0, 0.0, 0.0, 0.0], [8.0, 8.0, 8.0, 4.0]]], np.float32)
    rp = pkg._native.ResolveParams((1, 3, 0, 1), (1.0, 4.0, 3.0, 0.0), (1.0, 0.0, 0.0, 0.5))
    hdr = oracle.resolve(acc, rp, hdr=True)
    # f = 0.5: alpha = 0.5 + 0.5 * 0.5 = 0.75, colour = (0.5 m + 0.25 bg) / 0.75.
    assert np.allclose(hdr[0, 0], [(0.5 * 1.0 + 0.25) / 0.75, 0.5 * 0.5 / 0.75, 0.5 * 0.25 / 0.75, 0.75], atol=1e-6)
    assert np.allclose(hdr[0, 1], [1.0, 0.0, 0.0, 0.5])
    assert np.allclose(hdr[0, 2], [2.0, 2.0, 2.0, 1.0])


def test_tone_maps(pkg, oracle):
    acc = np.array([[[0.5, 2.0, 8.0, 1.0]]], np.float32)
    for tm in (0, 1, 2):
        rp = pkg._native.ResolveParams((1, 3, tm, 0), (1.0, 1.0, 1.0, 0.0), (0.0, 0.0, 0.0, 1.0))
        img = oracle.resolve(acc, rp, hdr=False)[0, 0]
        assert img[3] == 255
        if tm == 0:
            assert img[1] == 255 and img[2] == 255 and 180 < img[0] < 200
        else:
            assert img[0] < img[1] <= img[2]


def test_empty_scene_all_uncovered(pkg, oracle):
    o = pkg.RenderOptions(width=16, height=12, scene_camera=None)
    p = pkg.prepare(pkg.Scene(), o)
    acc, cnt = oracle.render(p, 4)
    assert np.all(acc == 0) and cnt[0] == 16 * 12 * 4 and cnt[3] == 0
