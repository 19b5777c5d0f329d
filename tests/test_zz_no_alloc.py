"""The allocation-free dispatch (oxpt_dispatch_noalloc) against the
context-based dispatch.

Some callers may not let this library allocate device memory (they own all
of it through their own allocator, or cannot take the synchronisation an
allocation can cause mid-frame). For them, oxpt_dispatch_noalloc traces into
the caller's own device buffers and keeps its scratch in a fixed array that
is part of the library's device image. This test gives it device buffers
allocated by the test (the caller) and checks, over two calls in a row,
that the caller's accumulator is bit-identical to the context path's.
The frame is larger than the fixed scratch, so the calls also exercise the
split into several launches and the reuse of the array between calls.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h", [(640, 480), (64, 32)])
def test_noalloc_dispatch_matches_the_context_path_on_two_calls(pkg, w, h):
    """640x480 (307,200 pixels) is more than the 2^18-path scratch per
    sample, so each sample runs as several row launches; 64x32 puts several
    consecutive samples into one launch."""
    import torch

    N = pkg._native
    L = N.lib()
    t = pkg.GpuPathTracer(0)
    opts = pkg.RenderOptions(width=w, height=h, path_trace=pkg.PathTraceOptions(samples_per_pixel=5))
    t.sync(scenes.materials_scene(pkg), opts)
    p = t.prepared()

    dev = torch.device("cuda", 0)
    geom = torch.from_numpy(p.geom.view(np.int32)).to(dev)
    attrs = torch.from_numpy(p.attrs).to(dev)
    tables = torch.from_numpy(p.tables.view(np.int32)).to(dev)
    atlas = torch.from_numpy(p.atlas.view(np.int16)).to(dev)
    accum = torch.zeros((h, w, 4), dtype=torch.float32, device=dev)
    scene = N.DeviceScene(geom.data_ptr(), p.geom.size, attrs.data_ptr(), p.attrs.size, tables.data_ptr(),
                          p.tables.size, atlas.data_ptr(), p.atlas_side, p.atlas_layers)
    params = p.params
    stream = torch.cuda.current_stream(dev)

    for first, count in ((0, 2), (2, 3)):
        frame = N.Frame(first, count, 0, h)
        st = L.oxpt_dispatch_noalloc(C.byref(scene), C.byref(params), C.byref(frame),
                                     C.c_void_p(accum.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert st == N.OK
        torch.cuda.synchronize(dev)
        t.refine(count)  # the context path: same samples, its own buffers
        want = t.read_accum()
        got = accum.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (first, count)
    assert t.samples() == 5


def test_noalloc_rejects_rows_wider_than_its_scratch(pkg):
    N = pkg._native
    L = N.lib()
    params = N.Params()
    params.dims[0] = N.NOALLOC_MAX_PATHS + 1
    params.dims[1] = 1
    one = (C.c_uint32 * 64)()
    scene = N.DeviceScene(C.addressof(one), 8, C.addressof(one), 48, C.addressof(one), 1, C.addressof(one), 1, 1)
    frame = N.Frame(0, 1, 0, 1)
    st = L.oxpt_dispatch_noalloc(C.byref(scene), C.byref(params), C.byref(frame), C.c_void_p(C.addressof(one)),
                                 None)
    assert st == N.E_LIMIT


def test_noalloc_empty_frame_is_a_no_op_anywhere(pkg):
    """A frame with no rows or no samples returns OK even when its first row
    lies outside the image, as oxpt_dispatch does (nothing is launched, so
    the dummy host pointers are never read)."""
    N = pkg._native
    L = N.lib()
    params = N.Params()
    params.dims[0] = 16
    params.dims[1] = 8
    one = (C.c_uint32 * 64)()
    scene = N.DeviceScene(C.addressof(one), 8, C.addressof(one), 48, C.addressof(one), 1, C.addressof(one), 1, 1)
    for frame in (N.Frame(0, 1, 9, 0), N.Frame(0, 0, 9, 3)):
        st = L.oxpt_dispatch_noalloc(C.byref(scene), C.byref(params), C.byref(frame),
                                     C.c_void_p(C.addressof(one)), None)
        assert st == N.OK
