"""Radiance-cache network on the tensor cores against the FP64 model
(oracle/nrc.py): forward outputs, loss, gradients (the backward kernel),
one Adam step, and that online training drives the loss down.

Tolerances: the GPU multiplies BF16 operands with FP32 accumulation; the
model rounds the same operands to BF16 and sums in FP64, so the remaining
differences are summation order and the rare BF16 rounding that a last-bit
difference flips (2% relative on outputs, 3% on each layer's gradient).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle import nrc

pytestmark = pytest.mark.gpu


@pytest.fixture()
def cache(pkg):
    L = pkg._native.lib()
    t = pkg.GpuPathTracer(0)
    h = C.c_void_p()
    assert L.oxpt_nrc_create(t.ctx, 11, C.byref(h)) == 0
    yield L, h
    L.oxpt_nrc_destroy(h)


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 12), np.float32)
    x[:, :10] = rng.random((n, 10))
    return x


def _target(x):
    t = np.zeros((x.shape[0], 4), np.float32)
    t[:, 0] = 0.6 + 0.4 * np.sin(3.0 * x[:, 0]) * np.cos(2.0 * x[:, 3])
    t[:, 1] = 0.3 + 0.5 * x[:, 1] * x[:, 9]
    t[:, 2] = 1.0 + 0.5 * np.cos(5.0 * x[:, 2] + x[:, 6])
    return t


def _set(L, h, w):
    w = np.ascontiguousarray(w, np.float32)
    assert L.oxpt_nrc_set_weights(h, w.ctypes.data) == 0


def test_forward_matches_the_fp64_model(cache):
    L, h = cache
    w = nrc.init(7)
    _set(L, h, w)
    x = _inputs(1037, 1)  # not a multiple of the 128-sample tile
    out = np.zeros((x.shape[0], 4), np.float32)
    assert L.oxpt_nrc_infer(h, x.ctypes.data, x.shape[0], out.ctypes.data) == 0
    y, _ = nrc.forward(w, x, bf=True)
    ref = y[:, :3]
    err = np.abs(out[:, :3] - ref) / (np.abs(ref) + 0.05 * np.mean(np.abs(ref)))
    assert np.quantile(err, 0.999) < 0.02 and err.max() < 0.1, (np.quantile(err, 0.999), err.max())
    assert np.all(out[:, 3] == 0.0)


def test_loss_and_gradient_match_the_fp64_model(cache):
    L, h = cache
    w = nrc.init(9)
    _set(L, h, w)
    x = _inputs(1000, 2)
    t = _target(x)
    loss = C.c_float()
    g = np.zeros(nrc.PARAMS, np.float32)
    assert L.oxpt_nrc_train(h, x.ctypes.data, t.ctypes.data, x.shape[0], 0, C.byref(loss), g.ctypes.data) == 0
    want_loss, want_g = nrc.loss_grad(w, x, t, bf=True)
    assert abs(loss.value - want_loss) <= 2e-3 * want_loss
    for l in range(nrc.LAYERS):
        a, b = g[nrc.OFFS[l]:nrc.OFFS[l + 1]], want_g[nrc.OFFS[l]:nrc.OFFS[l + 1]]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert rel < 0.03, (l, rel)
    # weights unchanged without `apply`
    w2 = np.zeros(nrc.PARAMS, np.float32)
    assert L.oxpt_nrc_get_weights(h, w2.ctypes.data) == 0
    assert np.array_equal(w2, w)


def test_adam_step_on_the_device_gradient(cache):
    L, h = cache
    w = nrc.init(3)
    _set(L, h, w)
    x = _inputs(640, 3)
    t = _target(x)
    loss = C.c_float()
    g = np.zeros(nrc.PARAMS, np.float32)
    assert L.oxpt_nrc_train(h, x.ctypes.data, t.ctypes.data, x.shape[0], 1, C.byref(loss), g.ctypes.data) == 0
    w1 = np.zeros(nrc.PARAMS, np.float32)
    L.oxpt_nrc_get_weights(h, w1.ctypes.data)
    want, _, _ = nrc.adam(w.astype(np.float64), g.astype(np.float64), 0.0, 0.0, 1)
    assert np.allclose(w1, want, rtol=1e-5, atol=1e-6)


def test_online_training_reduces_the_loss(cache):
    L, h = cache
    rng = np.random.default_rng(4)
    losses = []
    for step in range(300):
        x = _inputs(4096, 100 + step)
        t = _target(x)
        loss = C.c_float()
        assert L.oxpt_nrc_train(h, x.ctypes.data, t.ctypes.data, x.shape[0], 1, C.byref(loss), None) == 0
        losses.append(loss.value)
    assert np.isfinite(losses).all()
    assert np.mean(losses[-20:]) < 0.2 * np.mean(losses[:5]), (losses[:5], losses[-5:])
    # and it generalises to unseen inputs
    x = _inputs(2048, 9999)
    out = np.zeros((x.shape[0], 4), np.float32)
    assert L.oxpt_nrc_infer(h, x.ctypes.data, x.shape[0], out.ctypes.data) == 0
    t = _target(x)
    rel = np.mean((out[:, :3] - t[:, :3]) ** 2 / (t[:, :3] ** 2 + 0.01))
    assert rel < 0.02, rel


# ---------------------------------------------------------------------
# Cache frames on the path tracer.
# ---------------------------------------------------------------------

import scenes  # noqa: E402


def _tracer(pkg, w=96, h=64, bounces=8, scene=None):
    t = pkg.GpuPathTracer(0)
    t.sync(scene or scenes.materials_scene(pkg),
           pkg.RenderOptions(width=w, height=h,
                             path_trace=pkg.PathTraceOptions(samples_per_pixel=64, max_bounces=bounces)))
    return t


def test_zero_cache_ends_paths_exactly_at_the_query_bounce(pkg, oracle):
    """With a cache that predicts zero and no training paths, a cache
    frame is the plain tracer cut after two bounces (keeping the emission
    of the vertex where it stops): bit for bit, against the oracle too."""
    from oxideav_render_vulkan_b200.nrc import RadianceCache
    t = _tracer(pkg)
    cache = RadianceCache(t)
    cache.set_weights(np.zeros(nrc.PARAMS, np.float32))
    cache.configure(train_one_in=1 << 31, train=0, spread=0)
    cache.refine(3)
    assert t.samples() == 3
    got = t.read_accum()
    cut = _tracer(pkg, bounces=2)
    cut.refine(3)
    assert np.array_equal(got.view(np.uint32), cut.read_accum().view(np.uint32))
    cpu, _ = oracle.render(cut.prepared(), 3)
    assert np.array_equal(got.view(np.uint32), cpu.view(np.uint32))
    q, s = cache.frame_counts()
    assert q > 0 and s == 0


@pytest.mark.parametrize("per_wave", [2, 3])
def test_frames_sharing_a_wavefront_are_the_same_frames(pkg, per_wave):
    """Frames traced as one wavefront (the next frame's paths refill the
    slots the previous frame's free) are the frames traced one by one: with
    a zero cache and no training, bit for bit the plain tracer cut after
    two bounces, for a refine whose frame count is not a multiple of the
    frames per wave too."""
    from oxideav_render_vulkan_b200.nrc import RadianceCache
    t = _tracer(pkg)
    cache = RadianceCache(t)
    cache.set_weights(np.zeros(nrc.PARAMS, np.float32))
    cache.configure(train_one_in=1 << 31, train=0, spread=0, frames_per_wave=per_wave)
    cache.refine(5)
    assert t.samples() == 5
    cut = _tracer(pkg, bounces=2)
    cut.refine(5)
    assert np.array_equal(t.read_accum().view(np.uint32), cut.read_accum().view(np.uint32))
    q, s = cache.frame_counts()
    assert q > 0 and s == 0


def test_frames_sharing_a_wavefront_train(pkg):
    """Online training with four frames per wavefront: one training step
    per wave moves the weights, losses stay finite, and the frames
    accumulate as frames."""
    from oxideav_render_vulkan_b200.nrc import RadianceCache
    t = _tracer(pkg, 64, 64, 8, pkg.Scene.cornell())
    cache = RadianceCache(t)
    cache.configure(frames_per_wave=4, max_train=8192)
    w0 = cache.weights()
    losses = [cache.refine(4, loss=True) for _ in range(12)]
    assert np.isfinite(losses).all() and min(losses) > 0.0, losses
    assert not np.array_equal(w0, cache.weights())
    q, s = cache.frame_counts()
    assert q > 0 and 0 < s
    assert t.samples() == 48
    assert np.isfinite(t.read_accum()).all()


def test_training_paths_are_the_plain_tracer(pkg):
    """When every path is a training path nothing is cut: the frames equal
    the plain tracer's, and the paths that reach the query vertex become
    training samples."""
    from oxideav_render_vulkan_b200.nrc import RadianceCache
    t = _tracer(pkg)
    cache = RadianceCache(t)
    cache.configure(train_one_in=1, train=0, max_train=1 << 20, train_suffix=0)
    cache.refine(2)
    plain = _tracer(pkg)
    plain.refine(2)
    assert np.array_equal(t.read_accum().view(np.uint32), plain.read_accum().view(np.uint32))
    q, s = cache.frame_counts()
    assert q == 0 and s > 100


def test_training_frames_helper_is_the_plain_tracer_and_restores_the_config(pkg):
    from oxideav_render_vulkan_b200.nrc import RadianceCache
    t = _tracer(pkg)
    cache = RadianceCache(t)
    cache.configure(train_one_in=4, train_suffix=4)
    cache.refine_training(2)
    plain = _tracer(pkg)
    plain.refine(2)
    assert np.array_equal(t.read_accum().view(np.uint32), plain.read_accum().view(np.uint32))
    assert (cache.cfg.train_one_in, cache.cfg.train_suffix) == (4, 4)


def test_path_spread_decides_where_paths_end(pkg):
    """The path-spread heuristic: a spread no path reaches ends no path
    (the frames are the plain tracer's, bit for bit); the default ends
    fewer paths at the first eligible bounce than the fixed cut does (the
    glossy ones go on) but still most of them."""
    from oxideav_render_vulkan_b200.nrc import RadianceCache

    def counts(spread):
        t = _tracer(pkg)
        cache = RadianceCache(t)
        cache.set_weights(np.zeros(nrc.PARAMS, np.float32))
        cache.configure(train_one_in=1 << 31, train=0, spread=spread)
        cache.refine(2)
        return t, cache.frame_counts()[0]

    never, q_never = counts(1e30)
    plain = _tracer(pkg)
    plain.refine(2)
    assert q_never == 0
    assert np.array_equal(never.read_accum().view(np.uint32), plain.read_accum().view(np.uint32))
    _, q_fixed = counts(0.0)
    _, q_default = counts(0.01)
    assert 0 < q_default <= q_fixed, (q_default, q_fixed)


def test_path_spread_training_paths_record_once(pkg):
    """With the default spread every training path records at most one
    vertex, and all-training frames are still the plain tracer's."""
    from oxideav_render_vulkan_b200.nrc import RadianceCache
    t = _tracer(pkg)
    cache = RadianceCache(t)
    cache.configure(train_one_in=1, train=0, max_train=1 << 20, train_suffix=0)
    cache.refine(1)
    q, samples = cache.frame_counts()
    plain = _tracer(pkg)
    plain.refine(1)
    assert q == 0 and 0 < samples <= 96 * 64
    assert np.array_equal(t.read_accum().view(np.uint32), plain.read_accum().view(np.uint32))


def _mean_image(t):
    a = t.read_accum()
    return a[..., :3] / np.maximum(a[..., 3:4], 1.0)


def _rel_mse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 0.01)))


def test_trained_cache_recovers_the_light_beyond_the_cut(pkg):
    """The ablation, in a closed room where much of the light takes more
    than two bounces: after online training, cache frames are much closer
    to a converged plain reference than the same frames with the cache
    switched off at the cut (zero prediction), which lose every light path
    longer than two bounces."""
    from oxideav_render_vulkan_b200.nrc import RadianceCache

    def _tracer(pkg, bounces=8):
        return globals()["_tracer"](pkg, 64, 64, bounces, pkg.Scene.cornell())
    ref_t = _tracer(pkg)
    ref_t.refine(1024)
    ref = _mean_image(ref_t)
    t = _tracer(pkg)
    cache = RadianceCache(t)
    losses = [cache.refine(1, loss=True) for _ in range(60)]  # warm-up training
    assert np.isfinite(losses).all()
    q, s = cache.frame_counts()
    assert q > 0 and 0 < s <= 65536
    t.reset()
    cache.refine(40)
    trained = _mean_image(t)
    cut_t = _tracer(pkg)
    cut = RadianceCache(cut_t)
    cut.set_weights(np.zeros(nrc.PARAMS, np.float32))
    cut.configure(train=0)
    cut.refine(40)
    zero = _mean_image(cut_t)
    e_trained, e_zero = _rel_mse(trained, ref), _rel_mse(zero, ref)
    assert np.isfinite(trained).all()
    assert e_trained < 0.5 * e_zero, (e_trained, e_zero)
