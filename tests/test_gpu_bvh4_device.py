"""The four-wide tree collapsed on the device (csrc/bvh4_build.cu) against
the host collapse (host/bvh4.cpp): the same words node for node, root
reference and stack bound, the same binary depth, on the trees of several
scenes; and the same refusals on trees the collapse cannot take exactly."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu


def _host(L, geom, nodes):
    words, root, need = C.c_size_t(), C.c_uint32(), C.c_uint32()
    st = L.oxpt_diag_bvh4_build(geom.ctypes.data, nodes, None, 0, C.byref(words), C.byref(root), C.byref(need))
    if st != 0:
        return st, None, None, None
    out = np.zeros(max(words.value, 1), np.uint32)
    st = L.oxpt_diag_bvh4_build(geom.ctypes.data, nodes, out.ctypes.data, out.size, C.byref(words), C.byref(root),
                                C.byref(need))
    return st, out[: words.value], root.value, need.value


def _device(L, geom, nodes):
    words, root, need, depth, hdepth = C.c_size_t(), C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
    cap = max(nodes * 16 + 32, 32)
    out = np.zeros(cap, np.uint32)
    st = L.oxpt_diag_bvh4_build_device(0, geom.ctypes.data, nodes, out.ctypes.data, cap, C.byref(words),
                                       C.byref(root), C.byref(need), C.byref(depth), C.byref(hdepth))
    return st, out[: words.value] if st == 0 else None, root.value, need.value, depth.value, hdepth.value


def _tree(pkg, scene):
    p = pkg.prepare(scene, pkg.RenderOptions(width=8, height=8))
    return np.ascontiguousarray(p.geom[: p.node_count * 8]), p.node_count, p.bvh_depth


def _random_tree(pkg, n, seed):
    L = pkg._native.lib()
    pos = np.random.default_rng(seed).normal(size=(n, 9)).astype(np.float32)
    words = np.zeros(2 * n * 8, np.uint32)
    slots = np.zeros(n, np.uint32)
    nc, dp = C.c_uint32(), C.c_uint32()
    assert L.oxpt_diag_bvh_build(0, pos.ctypes.data, n, 1, words.ctypes.data, slots.ctypes.data, C.byref(nc),
                                 C.byref(dp)) == 0
    return np.ascontiguousarray(words[: nc.value * 8]), nc.value, dp.value


@pytest.mark.parametrize("which", ["cornell", "materials", "textured", "icosphere", "boxes", "random", "one"])
def test_device_collapse_equals_the_host(pkg, which):
    L = pkg._native.lib()
    if which == "random":
        geom, nodes, depth = _random_tree(pkg, 300_000, 3)
    elif which == "one":
        geom, nodes, depth = _random_tree(pkg, 1, 4)
    else:
        scene = {"cornell": lambda: pkg.Scene.cornell(), "materials": lambda: scenes.materials_scene(pkg),
                 "textured": lambda: scenes.textured_scene(pkg),
                 "icosphere": lambda: pkg.Scene.icosphere(freq=80, seed=2, n_textures=0, n_punctual=0, n_emissive=0),
                 "boxes": lambda: pkg.Scene.box_field(3000, seed=5)}[which]()
        geom, nodes, depth = _tree(pkg, scene)
    hs, hw, hr, hn = _host(L, geom, nodes)
    ds, dw, dr, dn, dd, hd = _device(L, geom, nodes)
    assert hs == 0 and ds == 0
    assert (dr, dn) == (hr, hn)
    assert np.array_equal(dw, hw)
    assert dd == hd == depth


def test_device_collapse_refuses_what_the_host_refuses(pkg):
    L = pkg._native.lib()
    geom, nodes, _ = _tree(pkg, scenes.materials_scene(pkg))
    g = geom.reshape(-1, 8).view(np.float32).copy()
    # a child box that pokes out of its parent's
    bad = g.copy()
    inner = np.nonzero(geom.reshape(-1, 8)[:, 7] == 0)[0]
    child = int(geom.reshape(-1, 8)[inner[3], 3])
    bad[child, 4] = bad[inner[3], 4] + 1.0
    # a leaf of more than 16 triangles
    big = geom.reshape(-1, 8).copy()
    leaf = np.nonzero(big[:, 7] > 0)[0][5]
    big[leaf, 7] = 17
    # a child index past the end
    past = geom.reshape(-1, 8).copy()
    past[inner[-1], 3] = nodes - 1
    for t in (bad.view(np.uint32), big, past):
        t = np.ascontiguousarray(t.reshape(-1))
        hs = _host(L, t, nodes)[0]
        ds, _, _, _, dd, hd = _device(L, t, nodes)
        assert hs == 4 and ds == 4
        assert dd == hd
    assert _device(L, np.ascontiguousarray(past.reshape(-1)), nodes)[4] == 65
