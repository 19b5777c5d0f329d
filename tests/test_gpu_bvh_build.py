"""GPU BVH build (csrc/bvh_build.cu) against the host builder
(host/bvh.cpp): the same node words, slot order, node count and depth on
real and adversarial triangle sets (coincident centroids, flat sets,
negative zeros, huge and tiny triangles). The tracer's device preparation
is covered by test_gpu_scene_prep.py."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest


pytestmark = pytest.mark.gpu


def _build(pkg, pos, on_gpu):
    L = pkg._native.lib()
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 9)
    n = pos.shape[0]
    words = np.zeros(max(1, 2 * n) * 8, np.uint32)
    slots = np.zeros(max(1, n), np.uint32)
    nc, dp = C.c_uint32(), C.c_uint32()
    st = L.oxpt_diag_bvh_build(0, pos.ctypes.data, n, int(on_gpu), words.ctypes.data, slots.ctypes.data,
                               C.byref(nc), C.byref(dp))
    assert st == 0
    return words[: nc.value * 8], slots[:n], nc.value, dp.value


def _scene_triangles(pkg, scene):
    p = pkg.prepare(scene, pkg.RenderOptions(width=8, height=8))
    tris = p.geom[p.node_count * 8:].reshape(-1, 12).view(np.float32)
    return tris[:, [0, 1, 2, 4, 5, 6, 8, 9, 10]].copy()


def _cases(pkg):
    rng = np.random.default_rng(5)
    rnd = rng.normal(size=(200_000, 9)).astype(np.float32)
    same = np.tile(rng.normal(size=(1, 9)).astype(np.float32), (300, 1))   # coincident centroids
    flat = rng.random((5000, 9)).astype(np.float32)
    flat[:, [2, 5, 8]] = -0.0                                                # a plane at z = -0
    mixed = np.concatenate([rnd[:20000] * 1e-6, rnd[20000:40000] * 1e4, same, flat])
    return {
        "icosphere": _scene_triangles(pkg, pkg.Scene.icosphere(freq=60, seed=2, n_textures=0, n_punctual=0,
                                                              n_emissive=0)),
        "boxes": _scene_triangles(pkg, pkg.Scene.box_field(4000, seed=3)),
        "cornell": _scene_triangles(pkg, pkg.Scene.cornell()),
        "random": rnd,
        "mixed": mixed,
        "one": rnd[:1],
        "two_same": same[:2],
    }


@pytest.mark.parametrize("which", ["icosphere", "boxes", "cornell", "random", "mixed", "one", "two_same"])
def test_gpu_build_matches_the_host_build(pkg, which):
    pos = _cases(pkg)[which]
    hw, hs, hn, hd = _build(pkg, pos, False)
    gw, gs, gn, gd = _build(pkg, pos, True)
    assert (gn, gd) == (hn, hd)
    assert np.array_equal(gs, hs)
    assert np.array_equal(gw, hw)
