"""Staged scene uploads (oxpt_stage_scene) against plain uploads.

A context alternates between two scenes through its second buffer set:
each refine after a stage traces the staged scene, bit for bit what a
context given the same scene by oxpt_upload_scene + oxpt_set_tables
traces; work queued before a stage keeps tracing the previous scene; the
classic upload after a stage replaces the staged scene.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu

W, H, SPP = 48, 32, 3


def _prepared(pkg, which):
    if which == "a":
        return pkg.prepare(scenes.materials_scene(pkg), pkg.RenderOptions(width=W, height=H))
    scene = pkg.Scene.icosphere(freq=12, seed=4, n_materials=6, n_textures=2, tex_size=64, n_punctual=2,
                                n_emissive=8, material_mix=1)
    return pkg.prepare(scene, pkg.RenderOptions(width=W, height=H, scene_camera=0),
                       pkg.EnvironmentMap.sky(64, 32))


def _desc(N, p):
    return N.SceneDesc(p.geom.ctypes.data, p.geom.size, p.attrs.ctypes.data, p.attrs.size, p.atlas.ctypes.data,
                       p.atlas_side, p.atlas_layers, p.node_count, p.slot_count)


class Ctx:
    def __init__(self, N):
        self.N, self.L = N, N.lib()
        h = C.c_void_p()
        assert self.L.oxpt_create(0, C.byref(h)) == 0
        self.h = h
        assert self.L.oxpt_resize(h, W, H) == 0

    def ok(self, st):
        assert st == 0, self.L.oxpt_last_error(self.h).decode()

    def upload(self, p):
        self.ok(self.L.oxpt_upload_scene(self.h, C.byref(_desc(self.N, p))))
        self.ok(self.L.oxpt_set_tables(self.h, p.tables.ctypes.data, p.tables.size))

    def stage(self, p):
        self.ok(self.L.oxpt_stage_scene(self.h, C.byref(_desc(self.N, p)), p.tables.ctypes.data, p.tables.size))

    def refine(self, p, first=0):
        params = p.params
        self.ok(self.L.oxpt_set_params(self.h, C.byref(params)))
        self.ok(self.L.oxpt_reset(self.h))
        self.ok(self.L.oxpt_refine(self.h, first, SPP))

    def accum(self):
        out = np.empty((H, W, 4), np.float32)
        self.ok(self.L.oxpt_read_accum(self.h, out.ctypes.data))
        self.ok(self.L.oxpt_finish(self.h))
        return out

    def close(self):
        self.L.oxpt_destroy(self.h)


@pytest.mark.parametrize("mode,graphs", [(2, 0), (2, 1), (0, 0)])
def test_staged_scenes_equal_plain_uploads(pkg, mode, graphs):
    N = pkg._native
    pa, pb = _prepared(pkg, "a"), _prepared(pkg, "b")
    want = {}
    for k, p in (("a", pa), ("b", pb)):
        c = Ctx(N)
        c.upload(p)
        c.refine(p)
        want[k] = c.accum()
        c.close()
    assert not np.array_equal(want["a"], want["b"])
    c = Ctx(N)
    t = N.Tuning()
    L = N.lib()
    L.oxpt_get_tuning(c.h, C.byref(t))
    t.mode, t.graphs = mode, graphs
    c.ok(L.oxpt_set_tuning(c.h, C.byref(t)))
    for k in "ababba":  # both buffer sets reused, a repeat stage replaces the pending one
        p = pa if k == "a" else pb
        c.stage(p)
        c.refine(p)
        got = c.accum()
        assert np.array_equal(got.view(np.uint32), want[k].view(np.uint32)), k
    c.close()


def test_queued_work_keeps_the_previous_scene(pkg):
    N = pkg._native
    pa, pb = _prepared(pkg, "a"), _prepared(pkg, "b")
    ref = Ctx(N)
    ref.upload(pa)
    ref.refine(pa)
    want_a = ref.accum()
    ref.close()
    c = Ctx(N)
    c.stage(pa)
    c.refine(pa)          # queued, not waited for
    c.stage(pb)           # the next scene goes up meanwhile
    got = c.accum()       # the queued refine traced scene a
    assert np.array_equal(got.view(np.uint32), want_a.view(np.uint32))
    c.refine(pb)
    c.upload(pa)          # a plain upload after a stage replaces the staged scene
    c.refine(pa)
    assert np.array_equal(c.accum().view(np.uint32), want_a.view(np.uint32))
    c.close()


def test_stage_rejects_bad_input(pkg):
    N = pkg._native
    L = N.lib()
    c = Ctx(N)
    pa = _prepared(pkg, "a")
    d = _desc(N, pa)
    assert L.oxpt_stage_scene(c.h, C.byref(d), None, 0) == N.E_INVALID
    d.geom_words = 4
    assert L.oxpt_stage_scene(c.h, C.byref(d), pa.tables.ctypes.data, pa.tables.size) == N.E_INVALID
    c.close()


def test_restaging_one_scene_reuses_both_step_graphs(pkg):
    """A renderer that re-stages the same scene every step alternates
    between the context's two buffer sets: each set keeps its own step
    graph, so after the first two steps nothing is captured again, and
    every step is the same frame."""
    N = pkg._native
    L = N.lib()
    pa = _prepared(pkg, "a")
    c = Ctx(N)
    t = N.Tuning()
    L.oxpt_get_tuning(c.h, C.byref(t))
    t.mode, t.graphs = 2, 1
    c.ok(L.oxpt_set_tuning(c.h, C.byref(t)))
    frames = []
    for _ in range(6):
        c.stage(pa)
        c.refine(pa)
        frames.append(c.accum())
    builds = C.c_uint64()
    c.ok(L.oxpt_diag_graph_builds(c.h, C.byref(builds)))
    assert builds.value == 2
    for f in frames[1:]:
        assert np.array_equal(f.view(np.uint32), frames[0].view(np.uint32))
    c.close()
