"""The four-wide any-hit tree (host/bvh4.cpp) against the binary BVH it is
collapsed from.

Shadow rays in the wavefront plans walk a four-wide tree instead of the
reference's binary one (pathtrace.wgsl:646-735). The walk answers the same
occlusion when it tests the same leaves: with no stack overflow and no
t_max change before the first accepted hit, the binary any-hit walk tests
exactly the leaves whose box and every ancestor's box pass the slab test.
These CPU tests check, with the kernels' float32 slab arithmetic restated in
numpy, that the four-wide tree reaches the same leaves for every ray of a
mixed set (random, axis-aligned, origins on box planes, finite and infinite
t_max), that it holds every binary leaf exactly once, that its stack bound
holds, and that a tree it cannot collapse exactly is refused.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import scenes

F32 = np.float32
NONE = 0xFFFFFFFF


def _prep(pkg, scene):
    o = pkg.RenderOptions(width=16, height=16, path_trace=pkg.PathTraceOptions(samples_per_pixel=1))
    return pkg.prepare(scene, o)


def _collapse(pkg, geom, nodes):
    L = pkg._native.lib()
    words, root, need = C.c_size_t(), C.c_uint32(), C.c_uint32()
    st = L.oxpt_diag_bvh4_build(geom.ctypes.data, nodes, None, 0, C.byref(words), C.byref(root), C.byref(need))
    if st != 0:
        return st, None, None, None
    out = np.zeros(max(words.value, 1), np.uint32)
    st = L.oxpt_diag_bvh4_build(geom.ctypes.data, nodes, out.ctypes.data, out.size, C.byref(words), C.byref(root),
                                C.byref(need))
    assert st == 0
    return st, out[: words.value].reshape(-1, 32), root.value, need.value


def _slab(o, inv, lo, hi, tmax):
    """Pass mask (rays x boxes) of the kernels' slab test, in float32."""
    t0 = (lo[None, :, :] - o[:, None, :]) * inv[:, None, :]
    t1 = (hi[None, :, :] - o[:, None, :]) * inv[:, None, :]
    tn, tf = np.fmin(t0, t1), np.fmax(t0, t1)
    near = np.fmax(np.fmax(F32(0), tn[..., 0]), np.fmax(tn[..., 1], tn[..., 2]))
    far = np.fmin(tmax[:, None], np.fmin(tf[..., 0], np.fmin(tf[..., 1], tf[..., 2])) * F32(1.0000004))
    assert near.dtype == np.float32 and far.dtype == np.float32
    return near <= far


def _inv(d):
    small = np.abs(d) < F32(1e-30)
    sign = np.where(np.signbit(d), F32(-1), F32(1))
    with np.errstate(divide="ignore"):
        return np.where(small, sign * F32(1e30), F32(1) / d).astype(np.float32)


def _rays(p, rng, n):
    nodes = p.geom[: p.node_count * 8].reshape(-1, 8)
    lo, hi = nodes[:, 0:3].view(np.float32), nodes[:, 4:7].view(np.float32)
    slo, shi = lo[0], hi[0]
    ext = shi - slo
    o = (slo - 0.2 * ext + rng.random((n, 3)) * 1.4 * ext).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    q = n // 4
    # axis-aligned and axis-plane directions, with signed zeros
    d[:q] *= (rng.random((q, 3)) < 0.5)
    d[:q // 2] = np.where(d[:q // 2] == 0, F32(-0.0), d[:q // 2])
    d[:q][np.all(d[:q] == 0, axis=1)] = (1, 0, 0)
    # origins on the planes of random node boxes
    idx = rng.integers(0, nodes.shape[0], q)
    ax = rng.integers(0, 3, q)
    on = np.where(rng.random(q) < 0.5, lo[idx, ax], hi[idx, ax])
    o[q:2 * q, :] = (lo[idx] + (hi[idx] - lo[idx]) * rng.random((q, 3)).astype(np.float32))
    o[q + np.arange(q), ax] = on
    tmax = np.where(rng.random(n) < 0.5, F32(np.inf), (rng.random(n) * np.linalg.norm(ext)).astype(np.float32))
    return o, d, tmax.astype(np.float32)


def _binary_leaves(p, o, inv, tmax):
    nodes = p.geom[: p.node_count * 8].reshape(-1, 8)
    lo, hi = nodes[:, 0:3].view(np.float32), nodes[:, 4:7].view(np.float32)
    ok = _slab(o, inv, lo, hi, tmax)
    reach = {0: ok[:, 0]}
    leaves = {}
    order = [0]
    while order:
        n = order.pop()
        first, count = int(nodes[n, 3]), int(nodes[n, 7])
        if count > 0:
            leaves[(first, count)] = reach[n]
            continue
        for c in (first, first + 1):
            reach[c] = reach[n] & ok[:, c]
            order.append(c)
    return leaves


def _four_leaves(t4, root, o, inv, tmax):
    n = o.shape[0]
    leaves = {}
    if root & 0x80000000:
        leaves[(root & 0x07FFFFFF, ((root >> 27) & 15) + 1)] = np.ones(n, bool)
        return leaves
    f = t4[:, :24].view(np.float32)
    refs = t4[:, 24:28]
    lo = np.stack([f[:, 0:4], f[:, 4:8], f[:, 8:12]], axis=-1).reshape(-1, 3)
    hi = np.stack([f[:, 12:16], f[:, 16:20], f[:, 20:24]], axis=-1).reshape(-1, 3)
    ok = _slab(o, inv, lo, hi, tmax).reshape(n, -1, 4)
    reach = {root: np.ones(n, bool)}
    order = [root]
    while order:
        j = order.pop()
        for k in range(4):
            r = int(refs[j, k])
            if r == NONE:
                continue
            got = reach[j] & ok[:, j, k]
            if r & 0x80000000:
                key = (r & 0x07FFFFFF, ((r >> 27) & 15) + 1)
                assert key not in leaves, "leaf held twice"
                leaves[key] = got
            else:
                assert r not in reach, "node referenced twice"
                reach[r] = got
                order.append(r)
    return leaves


SCENES = {
    "cornell": lambda pkg: pkg.Scene.cornell(),
    "materials": lambda pkg: scenes.materials_scene(pkg),
    "icosphere": lambda pkg: pkg.Scene.icosphere(freq=12, seed=3, n_textures=0, n_punctual=2, n_emissive=8),
    "box_field": lambda pkg: pkg.Scene.box_field(300, seed=5),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_four_wide_tree_reaches_the_binary_walks_leaves(pkg, name):
    p = _prep(pkg, SCENES[name](pkg))
    st, t4, root, need = _collapse(pkg, p.geom, p.node_count)
    assert st == 0
    nodes = p.geom[: p.node_count * 8].reshape(-1, 8)
    n_leaves = int(np.count_nonzero(nodes[:, 7]))
    assert n_leaves <= 3 * t4.shape[0] + 1 and t4.shape[0] <= p.node_count
    assert 1 <= need <= 64
    rng = np.random.default_rng(len(name))
    o, d, tmax = _rays(p, rng, 4096)
    inv = _inv(d)
    want = _binary_leaves(p, o, inv, tmax)
    got = _four_leaves(t4, root, o, inv, tmax)
    assert set(got) == set(want) and len(want) == n_leaves
    hits = 0
    for key, mask in want.items():
        assert np.array_equal(got[key], mask), key
        hits += int(mask.sum())
    assert hits > 4096  # the rays do reach leaves


def test_stack_bound_covers_an_all_pass_walk(pkg):
    p = _prep(pkg, pkg.Scene.icosphere(freq=16, seed=7, n_textures=0, n_punctual=0, n_emissive=0))
    _, t4, root, need = _collapse(pkg, p.geom, p.node_count)
    refs = t4[:, 24:28]
    stack, cur, most = [], root, 0
    while True:
        if not cur & 0x80000000:
            kids = [int(r) for r in refs[cur] if r != NONE]
            stack.extend(kids[1:])
            most = max(most, len(stack))
            cur = kids[0]
            continue
        if not stack:
            break
        cur = stack.pop()
    assert most <= need <= 64


def test_tree_it_cannot_collapse_exactly_is_refused(pkg):
    p = _prep(pkg, scenes.materials_scene(pkg))
    geom = p.geom.copy()
    nodes = geom[: p.node_count * 8].reshape(-1, 8)
    assert _collapse(pkg, geom, p.node_count)[0] == 0
    # a child box reaching outside its parent's: the walks could differ
    child = int(nodes[0, 3])
    box = nodes[child].copy()
    hi = box[4:7].view(np.float32)
    hi[0] = np.nextafter(nodes[0, 4:7].view(np.float32)[0], F32(np.inf))
    nodes[child] = box
    assert _collapse(pkg, geom, p.node_count)[0] == pkg._native.E_INVALID
    # a leaf of more than 16 triangles does not fit the reference encoding
    geom = p.geom.copy()
    nodes = geom[: p.node_count * 8].reshape(-1, 8)
    leaf = int(np.flatnonzero(nodes[:, 7])[0])
    nodes[leaf, 7] = 17
    assert _collapse(pkg, geom, p.node_count)[0] == pkg._native.E_INVALID


def test_single_leaf_and_empty_trees(pkg):
    geom = np.zeros(8, np.uint32)
    geom[0:3] = np.array([0, 0, 0], np.float32).view(np.uint32)
    geom[4:7] = np.array([1, 1, 1], np.float32).view(np.uint32)
    geom[3], geom[7] = 0, 2
    st, t4, root, need = _collapse(pkg, geom, 1)
    assert st == 0 and t4.shape[0] == 0 and root == 0x80000000 | (1 << 27)
    st, t4, root, need = _collapse(pkg, geom, 0)
    assert st == 0 and t4.shape[0] == 0 and root == NONE
