"""GPU parity: each stage of the CUDA path against the CPU oracle.

* portable transcendentals: bit-identical on device and host;
* Owen-scrambled Sobol' points: identical integers;
* closest-hit triangle ids on 10^6 random rays: identical except ties
  within 1e-6 relative t; any-hit occlusion identical;
* whole-path accumulators: bit-identical to the oracle at equal sample
  counts (so the >= 60 dB image bar holds with margin), and the images
  against the oracle's libm build >= 60 dB PSNR;
* traversal counters: identical (same nodes, leaves and triangles tested).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu


def _tracer(pkg, scene, opts, env=None):
    t = pkg.GpuPathTracer(0)
    if env is not None:
        t.set_environment(env)
    assert t.sync(scene, opts)
    return t


def _opts(pkg, w, h, spp, bounces=8, **kw):
    return pkg.RenderOptions(width=w, height=h, path_trace=pkg.PathTraceOptions(samples_per_pixel=spp,
                                                                                max_bounces=bounces, **kw))


@pytest.mark.parametrize("op", range(8))
def test_math_bit_exact(pkg, oracle, op):
    rng = np.random.default_rng(op)
    n = 1 << 20
    if op in (0, 1):
        a = rng.uniform(-20, 20, n)
    elif op == 2:
        a = np.concatenate([rng.uniform(-1, 1, n - 8), [-1, 1, 0, -0.0, 1.0000001, -2, 0.5, -0.5]])
    elif op == 3:
        a = rng.standard_normal(n) * np.exp(rng.uniform(-20, 20, n))
    elif op == 4:
        a = rng.uniform(-110, 95, n)
    else:
        a = np.exp(rng.uniform(-100, 100, n))
    b = rng.standard_normal(n) if op == 3 else rng.uniform(0.01, 600, n)
    a = a.astype(np.float32)
    b = b.astype(np.float32)
    t = pkg.GpuPathTracer(0)
    out = np.empty(n, np.float32)
    st = pkg._native.lib().oxpt_diag_math(t.ctx, op, n, a.ctypes.data, b.ctypes.data, out.ctypes.data)
    assert st == 0
    want = oracle.math(op, a, b, libm=False)
    same = (out.view(np.uint32) == want.view(np.uint32)) | (np.isnan(out) & np.isnan(want))
    assert same.all(), f"op {op}: {np.count_nonzero(~same)} of {n} differ"


def test_sobol_points_identical(pkg, oracle):
    rng = np.random.default_rng(5)
    n = 1 << 20
    x = rng.integers(0, 4096, n, dtype=np.uint32)
    y = rng.integers(0, 4096, n, dtype=np.uint32)
    idx = np.concatenate([np.arange(n // 2, dtype=np.uint32), rng.integers(0, 2**32, n - n // 2, dtype=np.uint32)])
    pat = rng.integers(0, 40, n, dtype=np.uint32)
    dirs = np.empty(128, np.uint32)
    L = pkg._native.lib()
    L.oxpt_sobol_directions(dirs.ctypes.data)
    t = pkg.GpuPathTracer(0)
    out = np.empty((n, 4), np.uint32)
    for seed in (0, 7, 0xDEADBEEF):
        st = L.oxpt_diag_sobol(t.ctx, dirs.ctypes.data, seed, n, x.ctypes.data, y.ctypes.data, idx.ctypes.data,
                               pat.ctypes.data, out.ctypes.data)
        assert st == 0
        want = oracle.sobol(dirs, seed, x, y, idx, pat)
        assert np.array_equal(out, want)
        # The floats the tracer uses: top 24 bits x 2^-24.
        f = (out >> 8).astype(np.float32) * np.float32(1.0 / 16777216.0)
        assert f.min() >= 0.0 and f.max() < 1.0


def _random_rays(rng, n, lo, hi):
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.standard_normal((n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 3.0e38
    rays[:, 4:7] = d
    rays[:, 7] = np.frombuffer(np.full(n, 0xFFFFFFFF, np.uint32).tobytes(), np.float32)
    return rays


@pytest.mark.parametrize("which", ["icosphere", "boxes", "cornell", "alpha"])
def test_closest_hit_ids_on_a_million_rays(pkg, oracle, which):
    if which == "icosphere":
        scene = pkg.Scene.icosphere(freq=64, seed=3, n_textures=0, n_punctual=0, n_emissive=16)
        lo, hi = -1.3, 1.3
    elif which == "boxes":
        scene = pkg.Scene.box_field(2000, seed=4, material_mix=0)
        lo, hi = -8.0, 8.0
    elif which == "alpha":
        scene = scenes.alpha_scene(pkg)
        lo, hi = -1.5, 1.5
    else:
        scene = pkg.Scene.cornell()
        lo, hi = 0.01, 0.99
    opts = _opts(pkg, 16, 16, 1)
    t = _tracer(pkg, scene, opts)
    p = t.prepared()
    rng = np.random.default_rng(11)
    n = 1_000_000
    rays = _random_rays(rng, n, lo, hi)
    rays[: n // 4, 3] = rng.uniform(0.0, 2.0 * (hi - lo), n // 4).astype(np.float32)  # finite t_max
    L = pkg._native.lib()
    info = (C.c_uint32 * 4)()
    assert L.oxpt_diag_bvh4(t.ctx, info) == 0 and info[0] == 1
    # bit 2: any-hit rays walk the four-wide tree; occlusion must not change
    for flags in (0, 1, 2, 3, 5, 7):
        slot = np.empty(n, np.uint32)
        gid = np.empty(n, np.uint32)
        tt = np.empty(n, np.float32)
        bary = np.empty((n, 3), np.float32)
        st = L.oxpt_diag_trace_rays(t.ctx, n, rays.ctypes.data, flags, slot.ctypes.data, gid.ctypes.data,
                                    tt.ctypes.data, bary.ctypes.data)
        assert st == 0
        oslot, ogid, ot, obary, _ = oracle.trace_rays(p, rays, flags & 3)
        if flags & 1:
            assert np.array_equal(slot == 0xFFFFFFFF, oslot == 0xFFFFFFFF)
            continue
        hit = ogid != 0xFFFFFFFF
        assert hit.sum() > n // 10
        diff = gid != ogid
        # Ties: another triangle at the same distance within 1e-6 relative t.
        if diff.any():
            rel = np.abs(tt[diff] - ot[diff]) / np.maximum(np.abs(ot[diff]), 1e-30)
            assert np.all(rel <= 1e-6), f"{diff.sum()} ids differ beyond ties"
        same = ~diff
        assert np.array_equal(tt[same].view(np.uint32), ot[same].view(np.uint32))
        assert np.array_equal(bary[same].view(np.uint32), obary[same].view(np.uint32))


def _accum_parity(pkg, oracle, scene, opts, spp, env_gpu=None):
    t = _tracer(pkg, scene, opts, env_gpu)
    t.refine(spp)
    t.finish()
    gpu = t.read_accum()
    p = t.prepared()
    cpu, cnt = oracle.render(p, spp)
    diff = gpu.view(np.uint32) != cpu.view(np.uint32)
    assert not diff.any(), f"{np.count_nonzero(diff.any(axis=2))} of {diff.shape[0] * diff.shape[1]} pixels differ"
    return t, p, cpu, cnt


def test_cornell_accumulator_bit_exact(pkg, oracle):
    _accum_parity(pkg, oracle, pkg.Scene.cornell(), _opts(pkg, 64, 48, 16), 16)


def test_materials_accumulator_bit_exact(pkg, oracle):
    _accum_parity(pkg, oracle, scenes.materials_scene(pkg), _opts(pkg, 64, 48, 8), 8)


@pytest.mark.parametrize("minf", [1, 3, 5])
def test_textured_accumulator_bit_exact(pkg, oracle, minf):
    _accum_parity(pkg, oracle, scenes.textured_scene(pkg, min_filter=minf), _opts(pkg, 64, 48, 4), 4)


def test_alpha_accumulator_bit_exact(pkg, oracle):
    _accum_parity(pkg, oracle, scenes.alpha_scene(pkg), _opts(pkg, 64, 48, 8), 8)


def test_environment_accumulator_bit_exact(pkg, oracle):
    env = pkg.EnvironmentMap(scenes.sky())
    _accum_parity(pkg, oracle, scenes.env_scene(pkg), _opts(pkg, 64, 48, 8, bounces=6), 8, env_gpu=env)


@pytest.mark.parametrize("strategy", [0, 1, 2])
def test_strategies_bit_exact(pkg, oracle, strategy):
    _accum_parity(pkg, oracle, scenes.materials_scene(pkg), _opts(pkg, 40, 30, 4, strategy=strategy), 4)


def test_layered_mix_with_env_and_lights_bit_exact(pkg, oracle):
    """Icosphere with the layered material mix, textures, punctual and
    emissive lights and the analytic sky (the batched/radiance-cache
    scenes' material model)."""
    scene = pkg.Scene.icosphere(freq=24, seed=9, n_materials=16, n_textures=4, tex_size=128, n_punctual=4,
                                n_emissive=32, material_mix=1)
    env = pkg.EnvironmentMap.sky(128, 64)
    _accum_parity(pkg, oracle, scene, _opts(pkg, 48, 32, 4, bounces=12), 4, env_gpu=env)


def test_images_vs_libm_oracle_psnr_at_least_60db(pkg, oracle):
    opts = _opts(pkg, 96, 96, 64)
    t = _tracer(pkg, pkg.Scene.cornell(), opts)
    t.refine(64)
    img = t.image()
    p = t.prepared()
    cpu, _ = oracle.render(p, 64, libm=True)
    ref = oracle.resolve(cpu, t.resolve_params(False), hdr=False, libm=True)
    psnr = scenes.psnr_rgb8(img, ref)
    assert psnr >= 60.0, psnr


@pytest.mark.parametrize("tv", [0, 4])
@pytest.mark.parametrize("mode,refill", [(0, 0), (1, 8), (2, 8), (1, 1), (2, 32), (2, 16)])
@pytest.mark.parametrize("which", ["materials", "layered", "alpha"])
def test_both_execution_modes_bit_exact(pkg, oracle, mode, refill, which, tv):
    """Megakernel and wavefront plans give the oracle's accumulator, also
    with few wavefront slots (path regeneration), split launches and every
    traversal refill policy (lanes taking new rays while others walk)."""
    if which == "materials":
        scene, env = scenes.materials_scene(pkg), None
    elif which == "alpha":
        scene, env = scenes.alpha_scene(pkg), None
    else:
        scene = pkg.Scene.icosphere(freq=16, seed=2, n_materials=12, n_textures=3, tex_size=64, n_punctual=3,
                                    n_emissive=16, material_mix=1)
        env = pkg.EnvironmentMap.sky(64, 32)
    t = _tracer(pkg, scene, _opts(pkg, 40, 28, 6, bounces=10), env)
    t.set_tuning(mode=mode, wave_slots=333, wave_items=2000, max_paths=2000, check_every=3, refill=refill,
                 trace_variant=tv)
    t.refine(6)
    gpu = t.read_accum()
    cpu, _ = oracle.render(t.prepared(), 6)
    assert np.array_equal(gpu.view(np.uint32), cpu.view(np.uint32))


@pytest.mark.parametrize("nee", [0, 2, 3, 4, 5])
@pytest.mark.parametrize("which", ["materials", "layered"])
def test_nee_kernel_orders_bit_exact(pkg, oracle, nee, which):
    """The split plan's NEE kernel job-major (0-2) or vertex-major (3-5):
    the same jobs in another order, the oracle's accumulator bit for bit."""
    if which == "materials":
        scene, env = scenes.materials_scene(pkg), None
    else:
        scene = pkg.Scene.icosphere(freq=16, seed=2, n_materials=12, n_textures=3, tex_size=64, n_punctual=3,
                                    n_emissive=16, material_mix=1)
        env = pkg.EnvironmentMap.sky(64, 32)
    t = _tracer(pkg, scene, _opts(pkg, 40, 28, 6, bounces=10), env)
    t.set_tuning(mode=2, nee_variant=nee, wave_slots=333, wave_items=2000)
    t.refine(6)
    cpu, _ = oracle.render(t.prepared(), 6)
    assert np.array_equal(t.read_accum().view(np.uint32), cpu.view(np.uint32))


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_traversal_counters_match_oracle(pkg, oracle, mode):
    opts = _opts(pkg, 48, 32, 4)
    t = _tracer(pkg, scenes.materials_scene(pkg), opts)
    t.set_tuning(mode=mode, shadow_walk=1)  # the reference's binary walk for every ray
    p = t.prepared()  # binds tables and params on the context
    out = (C.c_uint64 * 8)()
    st = pkg._native.lib().oxpt_diag_refine_counted(t.ctx, 0, 4, out)
    assert st == 0
    cpu, cnt = oracle.render(p, 4)
    assert list(out) == [int(c) for c in cnt]
    assert np.array_equal(t.read_accum().view(np.uint32), cpu.view(np.uint32))


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("which", ["materials", "alpha"])
def test_four_wide_shadow_walk_matches_the_binary_walk(pkg, oracle, mode, which):
    """Shadow rays through the four-wide tree: the accumulator is the
    oracle's bit for bit, the continuation rays' counters are the binary
    run's, and as many shadow rays are traced."""
    scene = scenes.materials_scene(pkg) if which == "materials" else scenes.alpha_scene(pkg)
    opts = _opts(pkg, 48, 32, 4)
    L = pkg._native.lib()
    runs = []
    for walk in (1, 0):
        t = _tracer(pkg, scene, opts)
        t.set_tuning(mode=mode, shadow_walk=walk)
        p = t.prepared()
        out = (C.c_uint64 * 8)()
        assert L.oxpt_diag_refine_counted(t.ctx, 0, 4, out) == 0
        split = (C.c_uint64 * 16)()
        assert L.oxpt_diag_counters_split(t.ctx, split) == 0
        runs.append((list(out), list(split), t.read_accum()))
    info = (C.c_uint32 * 4)()
    assert L.oxpt_diag_bvh4(t.ctx, info) == 0 and info[0] == 1 and 1 <= info[3] <= 64
    (tot_b, split_b, acc_b), (tot_f, split_f, acc_f) = runs
    cpu, cnt = oracle.render(p, 4)
    assert tot_b == [int(c) for c in cnt]
    assert np.array_equal(acc_f.view(np.uint32), cpu.view(np.uint32))
    assert np.array_equal(acc_b.view(np.uint32), cpu.view(np.uint32))
    assert split_f[:8] == split_b[:8]
    assert split_f[8 + 2] == split_b[8 + 2] > 0  # shadow rays


def test_full_size_scene_rows_bit_exact(pkg, oracle):
    """The 1920x1080 displaced-icosphere configuration (reduced triangle
    count): a full-frame GPU pass, then a few rows recomputed by the oracle
    must match bit for bit; every pixel is finite and counted once."""
    scene = pkg.Scene.icosphere(freq=96, seed=1, n_materials=64, n_textures=8, tex_size=512, n_punctual=16,
                                n_emissive=512)
    env = pkg.EnvironmentMap.sky(1024, 512)
    opts = _opts(pkg, 1920, 1080, 1, bounces=12)
    t = _tracer(pkg, scene, opts, env)
    t.refine(1)
    t.finish()
    gpu = t.read_accum()
    assert np.isfinite(gpu).all()
    assert set(np.unique(gpu[..., 3])) <= {0.0, 1.0}
    p = t.prepared()
    cpu = np.zeros_like(gpu)
    for y0 in (0, 540, 1077):
        oracle.dispatch(p, p.params, (0, 1, y0, 3), cpu)
        assert np.array_equal(gpu[y0:y0 + 3].view(np.uint32), cpu[y0:y0 + 3].view(np.uint32))
