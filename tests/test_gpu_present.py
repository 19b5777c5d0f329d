"""Present path (oxpt_resolve_async): image() as an asynchronous pinned
readback on a copy stream, overlapping the next refine.

The bytes must be those image() gives at the moment of the call, even
when a refine that changes the accumulator is enqueued right after it.
"""
from __future__ import annotations

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu


def test_async_image_is_the_image_at_the_call_despite_a_following_refine(pkg):
    t = pkg.GpuPathTracer(0)
    t.sync(scenes.materials_scene(pkg), pkg.RenderOptions(width=320, height=200,
                                                          path_trace=pkg.PathTraceOptions(samples_per_pixel=64)))
    t.refine(2)
    want = t.image()
    buf = t.image_async()
    t.refine(6)  # enqueued while the copy may still run
    got = buf.wait().copy()
    assert np.array_equal(got, want)
    later = t.image()
    assert not np.array_equal(later, want)  # the refine did change the accumulation
    # again, reusing the device image: the second call waits for the first copy
    b1 = t.image_async()
    b2 = t.image_async()
    assert np.array_equal(b1.wait(), later) and np.array_equal(b2.wait(), later)
