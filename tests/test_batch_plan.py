"""Round planning of batched refinement (oxpt_diag_batch_plan; host/batch.cpp).

A batched refine traces many frames as one wavefront in rounds of at most
`cap` launch items. The plan must cover every (pixel, sample) of every
frame exactly once, keep each round within `cap`, and hand out each row
band's samples in increasing order across rounds, which is what keeps each
pixel's accumulation order that of the frame's own refine.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest


def _plan(pkg, frames, cap):
    L = pkg._native.lib()
    fr = np.ascontiguousarray(np.asarray(frames, np.uint32).reshape(-1, 5))
    n = C.c_size_t()
    assert L.oxpt_diag_batch_plan(fr.ctypes.data, fr.shape[0], cap, None, 0, C.byref(n)) == 0
    out = np.zeros((max(n.value, 1), 7), np.uint64)
    assert L.oxpt_diag_batch_plan(fr.ctypes.data, fr.shape[0], cap, out.ctypes.data, n.value, C.byref(n)) == 0
    return out[: n.value]


def _check(frames, pieces, cap):
    cover = [np.zeros((f[4], f[2]), np.int32) for f in frames]  # rows x samples
    last = {}
    by_round = {}
    for r, f, first, count, y0, rows, base in pieces.astype(np.int64):
        w, f_first, f_count, f_y0, f_rows = frames[f]
        assert f_first <= first and first + count <= f_first + f_count
        assert f_y0 <= y0 and y0 + rows <= f_y0 + f_rows
        cover[f][y0 - f_y0: y0 - f_y0 + rows, first - f_first: first - f_first + count] += 1
        band = (f, y0)
        assert last.get(band, (-1, -1))[0] < r, "a band appears twice in one round"
        assert last.get(band, (-1, f_first))[1] <= first, "samples out of order"
        last[band] = (r, first + count)
        by_round.setdefault(r, []).append((base, w * rows * count))
    for r, items in by_round.items():
        items.sort()
        end = 0
        for base, n in items:
            assert base == end, "items of a round are not contiguous"
            end += n
        assert end <= cap
    for c in cover:
        assert np.all(c == 1)


@pytest.mark.parametrize("seed", range(6))
def test_random_batches_cover_every_sample_once_in_order(pkg, seed):
    rng = np.random.default_rng(seed)
    cap = int(rng.choice([4096, 20000, 1 << 16]))
    frames = []
    for _ in range(int(rng.integers(1, 12))):
        w = int(rng.integers(1, 300))
        h = int(rng.integers(1, 300))
        y0 = int(rng.integers(0, h))
        rows = int(rng.integers(0, h - y0 + 1))
        frames.append((min(w, cap), int(rng.integers(0, 1000)), int(rng.integers(0, 40)), y0, rows))
    pieces = _plan(pkg, frames, cap)
    _check(frames, pieces, cap)


def test_frame_wider_than_a_round_is_cut_into_row_bands(pkg):
    frames = [(1920, 0, 64, 0, 1080), (256, 5, 3, 0, 256)]
    cap = 1 << 20
    pieces = _plan(pkg, frames, cap)
    _check(frames, pieces, cap)
    bands = {(int(p[1]), int(p[4])) for p in pieces if p[1] == 0}
    assert len(bands) == 2  # 1080 rows of 1920 pixels in bands of at most 546 rows
    # every round is full except the last ones
    totals = np.bincount(pieces[:, 0].astype(np.int64),
                         weights=[frames[int(p[1])][0] * int(p[5]) * int(p[3]) for p in pieces])
    assert totals[0] > 0.9 * cap


def test_empty_frames_and_rejects(pkg):
    assert _plan(pkg, [(10, 0, 0, 0, 5), (10, 0, 4, 2, 0)], 100).shape[0] == 0
    L = pkg._native.lib()
    n = C.c_size_t()
    fr = np.array([[200, 0, 1, 0, 1]], np.uint32)
    assert L.oxpt_diag_batch_plan(fr.ctypes.data, 1, 100, None, 0, C.byref(n)) == pkg._native.E_INVALID
