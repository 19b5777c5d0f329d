"""Host-side preparation: the flat buffers follow the reference's layouts
(src/pathtrace.rs:970-1461) and this project's table rules."""
from __future__ import annotations

import numpy as np
import pytest

import scenes


def f32(words):
    return np.asarray(words, np.uint32).view(np.float32)


def _prep(pkg, scene, w=32, h=24, env=None, **pt):
    o = pkg.RenderOptions(width=w, height=h, path_trace=pkg.PathTraceOptions(**pt))
    return pkg.prepare(scene, o, env)


def test_bvh_is_a_valid_binary_tree_covering_every_triangle(pkg):
    s = pkg.Scene.icosphere(freq=20, seed=2, n_textures=0, n_punctual=0, n_emissive=4)
    p = _prep(pkg, s)
    nodes = p.geom[: p.node_count * 8].reshape(-1, 8)
    lo, hi = f32(nodes[:, 0:3]), f32(nodes[:, 4:7])
    first, count = nodes[:, 3], nodes[:, 7]
    tris = p.geom[p.node_count * 8:].reshape(-1, 12)
    assert tris.shape[0] == p.slot_count == s.triangle_count()
    pos = f32(tris[:, [0, 1, 2, 4, 5, 6, 8, 9, 10]]).reshape(-1, 3, 3)
    seen = np.zeros(p.slot_count, np.int32)
    stack, depth_max = [(0, 1)], 0
    while stack:
        n, d = stack.pop()
        depth_max = max(depth_max, d)
        if count[n] > 0:
            sl = slice(first[n], first[n] + count[n])
            seen[sl] += 1
            assert np.all(pos[sl].min(axis=1) >= lo[n] - 1e-6) and np.all(pos[sl].max(axis=1) <= hi[n] + 1e-6)
        else:
            l = first[n]
            assert l % 2 == 1 and l + 1 < p.node_count
            for c in (l, l + 1):
                assert np.all(lo[c] >= lo[n]) and np.all(hi[c] <= hi[n])
                stack.append((c, d + 1))
    assert np.all(seen == 1)
    assert depth_max == p.bvh_depth < 64
    # Global ids: a permutation; p0.w / p1.w / p2.w words.
    assert sorted(tris[:, 3].tolist()) == list(range(p.slot_count))
    assert np.all(count <= 8)


def test_cornell_tables_layout(pkg):
    p = _prep(pkg, pkg.Scene.cornell())
    P = p.params
    t = p.tables
    # Sobol' block first, then the 512-entry sheen LUT.
    assert P.offs0[0] == 0 and P.offs0[1] == 128
    dirs = t[:128].reshape(4, 32)
    assert np.all(dirs[0] == (1 << (31 - np.arange(32))).astype(np.uint32))
    assert dirs[1][0] == 1 << 31 and dirs[2][0] == 1 << 31 and dirs[3][0] == 1 << 31
    lut = f32(t[128:640]).reshape(16, 32)
    assert np.all((lut >= 0) & (lut <= 1)) and lut.max() > 0.05
    # No textures: materials start right after the LUT; 4 materials.
    assert P.offs0[2] == 640 and P.offs0[3] == 640 + 4 * 136
    mats = t[640:640 + 4 * 136].reshape(4, 136)
    red = f32(mats[1])
    assert np.allclose(red[0:4], [0.63, 0.065, 0.05, 1.0])
    assert red[8] == 0.0 and red[9] == 1.0 and red[13] == 0.0  # metallic, roughness, specular factor 0
    assert mats[1][7] == 0  # opaque, single-sided, lit, not emissive
    assert mats[3][7] == 16  # the emitter: emissive bit
    assert np.allclose(f32(mats[3])[4:7], [17, 12, 4])
    assert np.all(mats[:, 32::8][:, :13] == 0xFFFFFFFF)  # no texture slots
    # Emissive records: 2 triangles of equal area, cdf (0.5, 1), pmf 0.5.
    assert P.cfg[3] == 2 and P.cfg[2] == 0
    e = t[P.offs1[0]:P.offs1[0] + 8].reshape(2, 4)
    assert np.allclose(f32(e[:, 0]), [0.5, 1.0]) and np.allclose(f32(e[:, 1]), [0.5, 0.5])
    # Slot of each emissive record points at a triangle whose light word is the record index.
    tris = p.geom[p.node_count * 8:].reshape(-1, 12)
    for li in range(2):
        assert tris[e[li, 3], 7] == li and tris[e[li, 3], 3] == e[li, 2]
    # Params: dims, camera, no env, p_env 0.
    assert list(P.dims) == [32, 24, 0, 8] and P.cfg[0] == 3
    assert P.env[2] == 0 and P.fparams[2] == 0.0 and P.env[3] == p.node_count
    assert P.offs2[2] == 2 * p.node_count
    assert abs(P.up[3] - 2 * P.side[3] / 24) < 1e-7
    assert abs(P.forward[3] / P.side[3] - 32 / 24) < 1e-6


def test_material_words_extension_defaults_and_clamps(pkg):
    s = pkg.Scene()
    m0 = s.add_material(pkg.material())
    m1 = s.add_material(pkg.material(has_specular=1, specular=3.0, specular_color=(2.0, -1.0, float("nan")),
                                     has_transmission=1, transmission=0.4, has_volume=1, thickness=-2.0,
                                     attenuation_color=(0.5, 2.0, 0.1), attenuation_distance=float("inf"),
                                     has_clearcoat=1, clearcoat=0.7, clearcoat_roughness=1.5,
                                     has_sheen=1, sheen_color=(0.2, 0.3, 1.7), sheen_roughness=0.4,
                                     alpha_mode=1, alpha_cutoff=0.25, double_sided=1, unlit=1))
    s.add_mesh(scenes.quad_tris((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0)), m0)
    s.add_mesh(scenes.quad_tris((0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)), m1)
    p = _prep(pkg, s)
    o = p.params.offs0[2]
    w0, w1 = p.tables[o:o + 136], p.tables[o + 136:o + 272]
    a0, a1 = f32(w0), f32(w1)
    # Defaults (src/pathtrace.rs:1359-1416).
    assert a0[13] == 1.0 and np.all(a0[14:17] == 1.0) and a0[17] == 0.0 and a0[18] == 0.0
    assert np.all(a0[19:22] == 1.0) and a0[22] == -1.0 and a0[23] == 0 and a0[24] == 0 and a0[25] == 1.0
    assert np.all(a0[26:30] == 0.0) and w0[7] == 0 and a0[11] == 0.0
    # Clamps and finiteness fallbacks.
    assert a1[13] == 1.0 and list(a1[14:17]) == [2.0, 0.0, 1.0]
    assert a1[17] == pytest.approx(0.4) and a1[18] == 0.0 and list(a1[19:22]) == pytest.approx([0.5, 1.0, 0.1])
    assert a1[22] == -1.0 and a1[23] == pytest.approx(0.7) and a1[24] == 1.0
    assert list(a1[26:29]) == pytest.approx([0.2, 0.3, 1.0]) and a1[29] == pytest.approx(0.4)
    assert w1[7] == 1 | 4 | 8 and a1[11] == pytest.approx(0.25)


def test_texture_descriptors_and_atlas(pkg):
    s = scenes.textured_scene(pkg, min_filter=5)
    p = _prep(pkg, s)
    t = p.tables
    o = p.params.offs0[2]
    desc_floor = t[o + 32]  # base slot of material 0
    assert desc_floor != 0xFFFFFFFF
    levels, flags, w, h, skip, kept = t[desc_floor:desc_floor + 6]
    assert (w, h, levels, skip, kept) == (256, 256, 9, 0, 9)
    assert flags == 2 | 2 << 2 | 1 << 4 | 5 << 5
    side = p.atlas_side
    assert side == 256
    atlas = p.atlas.reshape(p.atlas_layers, side, side, 4)
    # Level 0 rect holds the decoded (sRGB -> linear) checker in f16.
    layer, x, y, wh = t[desc_floor + 8:desc_floor + 12]
    assert (wh & 0xFFFF, wh >> 16) == (256, 256)
    tex = atlas[layer, y:y + 256, x:x + 256].view(np.float16).astype(np.float32)
    src = scenes.checker(256, 16)
    lin = np.where(src[..., :3] <= 0.04045, src[..., :3] / 12.92, ((src[..., :3] + 0.055) / 1.055) ** 2.4)
    assert np.allclose(tex[..., :3], lin, atol=2e-3)
    # Every kept level's rect is in bounds, levels halve, rects do not overlap.
    seen = np.zeros((p.atlas_layers, side, side), np.int32)
    for dsc in sorted({int(t[o + 136 * m + 32 + 8 * k]) for m in range(2) for k in range(13)} - {0xFFFFFFFF}):
        kept = t[dsc + 5]
        for l in range(kept):
            layer, x, y, wh = t[dsc + 8 + 4 * l: dsc + 12 + 4 * l]
            ww, hh = wh & 0xFFFF, wh >> 16
            assert x + ww <= side and y + hh <= side and layer < p.atlas_layers
            seen[layer, y:y + hh, x:x + ww] += 1
    assert seen.max() == 1


def test_environment_cdfs(pkg):
    img = scenes.sky(64, 32)
    env = pkg.EnvironmentMap(img, 1.5)
    p = _prep(pkg, pkg.Scene.cornell(), env=env)
    P = p.params
    w, h = P.env[0], P.env[1]
    assert (w, h, P.env[2]) == (64, 32, 1) and P.fparams[2] == 0.5  # env + emitters
    t = p.tables
    marg = f32(t[P.offs1[2]:P.offs1[2] + h + 1])
    assert marg[0] == 0 and marg[-1] == 1 and np.all(np.diff(marg) >= 0)
    cond = f32(t[P.offs1[3]:P.offs1[3] + h * (w + 1)]).reshape(h, w + 1)
    assert np.all(cond[:, 0] == 0) and np.all(cond[:, -1] == 1) and np.all(np.diff(cond, axis=1) >= 0)
    mass = f32(t[P.offs2[0]:P.offs2[0] + w * h]).reshape(h, w)
    assert mass.sum() == pytest.approx(1.0, abs=1e-5)
    # mass = P(row) P(col | row).
    pr = np.diff(marg.astype(np.float64))
    pc = np.diff(cond.astype(np.float64), axis=1)
    assert np.allclose(mass, pr[:, None] * pc, atol=1e-6)
    rad = f32(t[P.offs2[1]:P.offs2[1] + 3 * w * h]).reshape(h, w, 3)
    assert np.allclose(rad, img[..., :3] * 1.5)
    # The 6-texel sun patch holds about a quarter of the mass.
    assert mass[6:8, 40:43].sum() > 0.2


def test_headlight_is_a_directional_punctual_light(pkg):
    s = pkg.Scene.cornell()
    o = pkg.RenderOptions(width=8, height=8, light_intensity=2.0)
    p = pkg.prepare(s, o)
    P = p.params
    assert P.cfg[2] == 1
    rec = p.tables[P.offs0[3]:P.offs0[3] + 16]
    assert rec[3] == 0 and np.allclose(f32(rec[8:11]), 2.0)


def test_empty_scene_prepares_to_an_empty_bvh(pkg):
    p = _prep(pkg, pkg.Scene())
    assert p.node_count == 0 and p.slot_count == 0 and p.params.env[3] == 0
    assert p.geom.size == 8 and p.attrs.size == 48


def test_attribute_flags_and_layout(pkg):
    s = scenes.textured_scene(pkg)
    p = _prep(pkg, s)
    a = p.attrs.reshape(-1, 12, 4)
    flags = a[:, 0, 3].view(np.uint32)
    # Floor: uv0 only (8). Sphere: normals, tangents, uv0 (1 | 2 | 8).
    assert set(np.unique(flags)) == {8, 11}
    sph = flags == 11
    assert np.allclose(np.linalg.norm(a[sph, 0:3, 0:3], axis=2), 1.0, atol=1e-5)
    assert np.all(a[sph, 3:6, 3] == 1.0)
    assert np.all(a[:, 9:12, :] == 1.0)  # absent colours are white
