"""Serving loop on the GPU: each request's result is the same alone and in
the mix.

Three resident scenes, a burst of 64 requests of different resolutions and
sample targets, 30% camera moves on open sessions; at least 32 complete
(some are superseded by a camera move on their session), camera-moved
sessions among them. The server advances all
admitted sessions together in batched ticks; afterwards every completed
request is rendered again alone (a fresh view, one plain refine to its
target) and its accumulator must match bit for bit. Views borrow the
owner's device scene and tables.
"""
from __future__ import annotations

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu


def _owners(pkg):
    out = []
    for scene in (pkg.Scene.cornell(), scenes.materials_scene(pkg),
                  pkg.Scene.icosphere(freq=10, seed=3, n_materials=8, n_textures=2, tex_size=64, n_punctual=4,
                                      n_emissive=8, material_mix=1)):
        t = pkg.GpuPathTracer(0)
        t.sync(scene, pkg.RenderOptions(width=32, height=32,
                                        path_trace=pkg.PathTraceOptions(samples_per_pixel=1, max_bounces=8)))
        t.prepared()
        out.append(t)
    return out


def _options(pkg):
    def f(r):
        return pkg.RenderOptions(width=r.width, height=r.height,
                                 path_trace=pkg.PathTraceOptions(samples_per_pixel=r.spp, max_bounces=8))
    return f


def _stream(serve, rng, n=64):
    reqs, opened, t = [], [], 0.0
    for rid in range(n):
        t += rng.exponential(0.004)
        if opened and rng.random() < 0.3:
            base = reqs[opened[int(rng.integers(len(opened)))]]
            key = base.session if base.session is not None else base.rid
            cam = ((float(rng.uniform(-0.5, 0.5)), 1.0, 3.5), (0.0, 0.4, 0.0))
            reqs.append(serve.Request(rid, t, base.scene, base.width, base.height, int(rng.choice([2, 5])), cam, key))
        else:
            w, h = [(48, 32), (64, 64), (40, 56)][int(rng.integers(3))]
            reqs.append(serve.Request(rid, t, int(rng.integers(3)), w, h, int(rng.choice([3, 6, 9]))))
            opened.append(rid)
    return reqs


def _alone(pkg, ex, r):
    v = ex.open(r)
    v.refine(r.spp)
    return v.read_accum()


@pytest.mark.parametrize("graphs", [0, 1])
def test_each_request_is_the_same_alone_and_in_the_mix(pkg, graphs):
    from oxideav_render_vulkan_b200 import serve
    owners = _owners(pkg)
    ex = serve.GpuExecutor(pkg, owners, _options(pkg), keep=lambda o: True)
    ex.exe.set_tuning(mode=2, graphs=graphs, wave_items=6000)
    reqs = _stream(serve, np.random.default_rng(3 + graphs))
    st = serve.Server(ex, budget=1 << 40, tick_paths=20000).run(reqs)
    done = st.completed()
    by = {r.rid: r for r in reqs}
    assert len(done) >= 32 and st.ticks > 1
    assert any(o.superseded for o in st.outcomes)
    assert sum(by[o.rid].camera is not None for o in done) >= 4  # camera-moved sessions among the checked
    for o in done:
        r = by[o.rid]
        got = ex.kept[o.rid]
        want = _alone(pkg, ex, r)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"request {o.rid} differs"


def test_views_borrow_the_owner_scene_and_tables(pkg):
    owner = _owners(pkg)[1]
    v = owner.view()
    v.sync_view(pkg.RenderOptions(width=20, height=10, path_trace=pkg.PathTraceOptions(samples_per_pixel=2)))
    v.refine(2)
    m_owner, m_view = owner.memory(), v.memory()
    assert m_owner["scene"] > 0 and m_view["scene"] == 0
    assert m_view["tables"] == 0  # the owner's resident tables
    assert m_view["images"] >= 20 * 10 * 16
    # a camera move resets, and equals a fresh view rendered at that camera
    v.set_camera(eye=(0.3, 1.0, 3.0), target=(0.0, 0.5, 0.0))
    assert v.samples() == 0
    v.refine(2)
    w = owner.view()
    w.sync_view(pkg.RenderOptions(width=20, height=10, path_trace=pkg.PathTraceOptions(samples_per_pixel=2)))
    w.set_camera(eye=(0.3, 1.0, 3.0), target=(0.0, 0.5, 0.0))
    w.refine(2)
    assert np.array_equal(v.read_accum().view(np.uint32), w.read_accum().view(np.uint32))
