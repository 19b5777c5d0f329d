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


def _widest_level(words, nodes):
    w = words.reshape(-1, 8)
    first, count = w[:, 3].astype(np.int64), w[:, 7].astype(np.int64)
    level, widest = np.array([0], np.int64), 1
    while level.size:
        widest = max(widest, level.size)
        inner = level[count[level] == 0]
        level = np.concatenate([first[inner], first[inner] + 1])
    return widest


def test_gpu_build_with_levels_wider_than_one_block_of_blocks(pkg):
    """A tree whose widest level holds more than 1024 x 1024 nodes (2.5 M
    tiny triangles spread through a cube: a leaf per triangle) takes the
    third scan level of the device build: the host's words, slots and depth;
    and the four-wide collapse of that tree matches the host collapse."""
    pos = np.random.default_rng(9).random((2_500_000, 9), dtype=np.float32)
    pos[:, 3:] = pos[:, :3].repeat(2, axis=0).reshape(-1, 6) + 1e-4 * pos[:, 3:]  # small triangles
    hw, hs, hn, hd = _build(pkg, pos, False)
    gw, gs, gn, gd = _build(pkg, pos, True)
    assert _widest_level(hw, hn) > 1024 * 1024
    assert (gn, gd) == (hn, hd)
    assert np.array_equal(gs, hs) and np.array_equal(gw, hw)
    L = pkg._native.lib()
    words, root, need = C.c_size_t(), C.c_uint32(), C.c_uint32()
    assert L.oxpt_diag_bvh4_build(hw.ctypes.data, hn, None, 0, C.byref(words), C.byref(root), C.byref(need)) == 0
    host4 = np.zeros(words.value, np.uint32)
    assert L.oxpt_diag_bvh4_build(hw.ctypes.data, hn, host4.ctypes.data, host4.size, C.byref(words), C.byref(root),
                                  C.byref(need)) == 0
    dev4 = np.zeros(words.value + 32, np.uint32)
    w2, r2, n2, d2, h2 = C.c_size_t(), C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
    assert L.oxpt_diag_bvh4_build_device(0, hw.ctypes.data, hn, dev4.ctypes.data, dev4.size, C.byref(w2),
                                         C.byref(r2), C.byref(n2), C.byref(d2), C.byref(h2)) == 0
    assert (w2.value, r2.value, n2.value) == (words.value, root.value, need.value)
    assert np.array_equal(dev4[: w2.value], host4)
    assert d2.value == h2.value == hd
