"""Scene preparation on the device (oxpt_build_scene) against the host
preparation: the same geom, attrs, atlas and tables word for word, the same
renders, on scenes with every optional attribute stream present and absent,
sRGB and linear textures of odd sizes, levels too large for a layer,
emissive triangles and several meshes; and the inputs the call rejects
before touching the device."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu


def _streams_scene(pkg):
    rng = np.random.default_rng(11)
    s = pkg.Scene()
    big = rng.random((3, 4100, 4), dtype=np.float32)      # level 0 wider than any layer: skipped
    t_big = s.add_texture(big.astype(np.float32), srgb_encoded=True)
    odd = rng.random((37, 5, 4), dtype=np.float32) * 1.5  # odd sides, values above 1
    t_odd = s.add_texture(odd.astype(np.float32), srgb_encoded=True, wrap=(1, 2), min_filter=3)
    lin = rng.random((16, 64, 4), dtype=np.float32)
    t_lin = s.add_texture(lin.astype(np.float32))
    m0 = pkg.material(base_color=(0.8, 0.7, 0.6, 1), metallic=0.0, roughness=0.5,
                      tex={scenes.SLOT_BASE: (t_odd, 0), scenes.SLOT_MR: (t_odd, 1)})
    m1 = pkg.material(base_color=(0.5, 0.6, 0.7, 1), metallic=0.2, roughness=0.3,
                      tex={scenes.SLOT_BASE: (t_big, 0), scenes.SLOT_NORMAL: (t_lin, 0)})
    m2 = pkg.material(base_color=(0, 0, 0, 1), metallic=0.0, emissive=(3.0, 2.0, 1.0))
    ids = [s.add_material(m) for m in (m0, m1, m2)]
    for k in range(6):
        n = int(rng.integers(1, 400))
        pos = (rng.normal(size=(n, 9)) + k).astype(np.float32)
        kw = {}
        if k & 1:
            kw["normals"] = rng.normal(size=(n, 9)).astype(np.float32)
        if k & 2:
            kw["tangents"] = rng.normal(size=(n, 12)).astype(np.float32)
        if k % 3 == 0:
            kw["uv0"] = rng.random((n, 6), dtype=np.float32)
        if k % 3 == 1:
            kw["uv1"] = rng.random((n, 6), dtype=np.float32)
        if k >= 4:
            kw["colors"] = rng.random((n, 12), dtype=np.float32)
        s.add_mesh(pos, ids[k % 3] if k != 5 else -1, **kw)   # mesh 5: the default material
    s.add_light(1, position=(2.0, 4.0, 2.0), intensity=20.0)
    return s


def _scenes(pkg):
    return {
        "materials": scenes.materials_scene(pkg),
        "textured": scenes.textured_scene(pkg),
        "streams": _streams_scene(pkg),
        "cornell": pkg.Scene.cornell(),
        "icosphere": pkg.Scene.icosphere(freq=40, seed=3, n_textures=3, tex_size=96, n_punctual=2, n_emissive=40),
        "boxes": pkg.Scene.box_field(500, seed=2),
    }


def _pair(pkg, scene, w=64, h=48, spp=2):
    opts = pkg.RenderOptions(width=w, height=h, path_trace=pkg.PathTraceOptions(samples_per_pixel=spp))
    a, b = pkg.GpuPathTracer(0), pkg.GpuPathTracer(0)
    a.set_gpu_prepare(False)  # the host preparation
    b.set_gpu_prepare(True)
    a.sync(scene, opts)
    b.sync(scene, opts)
    return a, b


@pytest.mark.parametrize("which", ["materials", "textured", "streams", "cornell", "icosphere", "boxes"])
def test_device_preparation_equals_the_host(pkg, which):
    a, b = _pair(pkg, _scenes(pkg)[which])
    pa, pb = a.prepared(), b.prepared()
    assert (pa.node_count, pa.slot_count, pa.bvh_depth) == (pb.node_count, pb.slot_count, pb.bvh_depth)
    assert (pa.atlas_side, pa.atlas_layers) == (pb.atlas_side, pb.atlas_layers)
    assert np.array_equal(pa.geom, pb.geom)
    assert np.array_equal(pa.attrs.view(np.uint32), pb.attrs.view(np.uint32))
    assert np.array_equal(pa.atlas, pb.atlas)
    assert np.array_equal(pa.tables, pb.tables)
    a.refine(2)
    b.refine(2)
    assert np.array_equal(a.read_accum().view(np.uint32), b.read_accum().view(np.uint32))


def test_device_prepared_scene_serves_views_and_reprepares(pkg):
    scene = scenes.textured_scene(pkg)
    a, b = _pair(pkg, scene)
    v = b.view()
    opts = pkg.RenderOptions(width=64, height=48, path_trace=pkg.PathTraceOptions(samples_per_pixel=2))
    v.sync_view(opts)
    v.refine(2)
    a.refine(2)
    assert np.array_equal(a.read_accum().view(np.uint32), v.read_accum().view(np.uint32))
    # switching back to the host preparation prepares again, same result
    b.set_gpu_prepare(False)
    b.sync(scene, opts)
    b.refine(2)
    assert np.array_equal(a.read_accum().view(np.uint32), b.read_accum().view(np.uint32))


class _Mesh(C.Structure):
    _fields_ = [("ntri", C.c_uint32), ("material", C.c_uint32), ("pos", C.c_void_p), ("nrm", C.c_void_p),
                ("tan", C.c_void_p), ("uv0", C.c_void_p), ("uv1", C.c_void_p), ("col", C.c_void_p)]


class _Chain(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("rgba", C.c_void_p), ("srgb_decode", C.c_uint32),
                ("skip", C.c_uint32), ("n_rects", C.c_uint32), ("rects", C.c_void_p)]


class _Src(C.Structure):
    _fields_ = [("meshes", C.c_void_p), ("n_meshes", C.c_uint32), ("light_tris", C.c_void_p),
                ("n_lights", C.c_uint32), ("chains", C.c_void_p), ("n_chains", C.c_uint32),
                ("atlas_side", C.c_uint32), ("atlas_layers", C.c_uint32)]


def test_invalid_sources_are_rejected(pkg):
    L = pkg._native.lib()
    t = pkg.GpuPathTracer(0)
    pos = np.random.default_rng(1).normal(size=(10, 9)).astype(np.float32)
    tex = np.ones((8, 8, 4), np.float32)
    mesh = _Mesh(10, 0, pos.ctypes.data, None, None, None, None, None)
    out = (C.c_uint32 * 3)()

    def run(rects, side=16, layers=1, lights=None, n_rects=None, skip=0):
        r = np.ascontiguousarray(np.array(rects, np.uint32).reshape(-1))
        ch = _Chain(8, 8, tex.ctypes.data, 0, skip, len(r) // 4 if n_rects is None else n_rects, r.ctypes.data)
        lt = np.array(lights or [], np.uint32)
        ls = np.zeros(max(1, lt.size), np.uint32)
        src = _Src(C.addressof(mesh), 1, lt.ctypes.data if lt.size else None, lt.size, C.addressof(ch), 1, side, layers)
        return L.oxpt_build_scene(t.ctx, C.byref(src), ls.ctypes.data, out)

    level_rects = [[0, 0, 0, 8 | 8 << 16], [0, 8, 0, 4 | 4 << 16], [0, 12, 0, 2 | 2 << 16], [0, 14, 0, 1 | 1 << 16]]
    assert run(level_rects) == 0
    assert list(out)[1] == 10
    assert run([[0, 9, 0, 8 | 8 << 16]], n_rects=1) == 4             # outside the layer
    assert run([[1, 0, 0, 8 | 8 << 16]], n_rects=1) == 4             # no such layer
    assert run([[0, 0, 0, 7 | 8 << 16]], n_rects=1) == 4             # not the level's size
    assert run(level_rects + [[0, 15, 0, 1 | 1 << 16]]) == 4         # more levels than the chain has
    assert run(level_rects, lights=[3, 3]) == 4                      # light ids must increase
    assert run(level_rects, lights=[10]) == 4                        # light id out of range
    assert run(level_rects, side=20000) == 3                         # layer side limit
    assert run(level_rects, lights=[2, 7]) == 0                      # and the context still works
