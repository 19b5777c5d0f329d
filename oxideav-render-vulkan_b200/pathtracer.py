"""Python face of the B200 path tracer, mirroring the reference crate's API.

``GpuPathTracer`` has the reference's progressive surface
(src/pathtrace.rs:309-725): ``sync`` / ``refine`` / ``finish`` / ``image`` /
``hdr`` / ``draw_texture`` / ``reset`` / ``samples`` / ``is_converged`` /
``size`` / ``set_environment`` / ``invalidate_scene`` /
``set_texture_resolver``, plus the ``Renderer`` trait's ``render`` /
``render_hdr`` (:1250-1264). ``register_into`` registers it as
``"gpu-pathtrace"`` (src/lib.rs:117, 329-338). Everything below calls the
C++ host layer and the CUDA kernels in liboxpt.so.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from typing import Callable, Dict, Optional, Tuple

import numpy as np

from . import _native as N

PATHTRACE_BACKEND_NAME = "gpu-pathtrace"
CRATE_NAME = "oxideav-render-cuda"


class Error(Exception):
    """oxideav_render::Error."""


class BackendError(Error):
    """Error::Backend: device, memory or kernel failure."""


class InvalidOptionsError(Error):
    """Error::InvalidOptions: the options cannot be honoured."""


def _raise(status: int, msg: str):
    if status == N.OK:
        return
    if status == N.E_INVALID:
        raise InvalidOptionsError(msg)
    raise BackendError(f"[{status}] {msg}")


class ToneMap(enum.IntEnum):
    CLAMP = 0
    REINHARD = 1
    ACES_FITTED = 2


class LightStrategy(enum.IntEnum):
    MIS = 0
    LIGHT_ONLY = 1
    BSDF_ONLY = 2


@dataclass
class PathTraceOptions:
    samples_per_pixel: int = 16
    max_bounces: int = 8
    rr_start: int = 3
    seed: int = 0
    strategy: LightStrategy = LightStrategy.MIS
    clamp: float = 0.0


@dataclass
class RenderOptions:
    width: int = 256
    height: int = 256
    scene_camera: Optional[int] = 0
    background: Tuple[int, int, int, int] = (0, 0, 0, 255)
    exposure: float = 1.0
    tone_map: ToneMap = ToneMap.CLAMP
    ambient: float = 0.0
    light_intensity: float = 0.0
    path_trace: PathTraceOptions = field(default_factory=PathTraceOptions)

    def to_c(self) -> N.RenderOptions:
        o = N.RenderOptions()
        o.width, o.height = int(self.width), int(self.height)
        o.scene_camera = -1 if self.scene_camera is None else int(self.scene_camera)
        for k in range(4):
            o.background[k] = int(self.background[k])
        o.exposure = float(self.exposure)
        o.tone_map = int(self.tone_map)
        o.ambient = float(self.ambient)
        o.light_intensity = float(self.light_intensity)
        pt = self.path_trace
        o.samples_per_pixel = int(pt.samples_per_pixel)
        o.max_bounces = int(pt.max_bounces)
        o.rr_start = int(pt.rr_start)
        o.seed = int(pt.seed) & 0xFFFFFFFF
        o.strategy = int(pt.strategy)
        o.clamp = float(pt.clamp)
        return o


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def _f32(a) -> Optional[np.ndarray]:
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def material(**kw) -> N.Material:
    """A glTF material with the reference defaults, fields set from kw
    (scalars or sequences; ``tex`` = {slot: (texture, uv_set)})."""
    m = N.Material()
    N.lib().oxpt_material_default(C.byref(m))
    tex = kw.pop("tex", {})
    for k, v in kw.items():
        cur = getattr(m, k)
        if isinstance(cur, C.Array):
            for i, x in enumerate(v):
                cur[i] = x
        else:
            setattr(m, k, v)
    for slot, ref in tex.items():
        tid, uv = ref if isinstance(ref, tuple) else (ref, 0)
        m.tex[slot].texture = tid
        m.tex[slot].uv_set = uv
    return m


class Scene:
    """A scene (oxideav_mesh3d::Scene3D stand-in) owned by the C++ layer."""

    def __init__(self, handle=None):
        self._h = handle if handle is not None else N.lib().oxpt_scene_new()
        if not self._h:
            raise BackendError("scene allocation failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and N is not None:  # None while the interpreter shuts down
            N.lib().oxpt_scene_free(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    # ---- builders
    def add_material(self, m: N.Material) -> int:
        return N.lib().oxpt_scene_add_material(self._h, C.byref(m))

    def add_texture(self, rgba: np.ndarray, srgb_encoded: bool = False, wrap=(2, 2), mag_linear=True,
                    min_filter=5) -> int:
        a = np.ascontiguousarray(rgba, dtype=np.float32)
        h, w = a.shape[:2]
        smp = N.Sampler(wrap[0], wrap[1], int(mag_linear), min_filter)
        return N.lib().oxpt_scene_add_texture(self._h, w, h, a.ctypes.data, int(srgb_encoded), C.byref(smp))

    def add_mesh(self, positions, material: int = -1, normals=None, tangents=None, uv0=None, uv1=None,
                 colors=None) -> int:
        p = _f32(positions).reshape(-1, 9)
        arrs = [_f32(x) for x in (normals, tangents, uv0, uv1, colors)]
        return N.lib().oxpt_scene_add_mesh(self._h, p.shape[0], p.ctypes.data, *map(_ptr, arrs), material)

    def add_light(self, kind: int, position=(0, 0, 0), direction=(0, -1, 0), color=(1, 1, 1), intensity=1.0,
                  range=0.0, inner_cone=0.0, outer_cone=0.7853982) -> int:
        l = N.Light(kind, (N.f32 * 3)(*position), (N.f32 * 3)(*direction), (N.f32 * 3)(*color), intensity,
                    range, inner_cone, outer_cone)
        return N.lib().oxpt_scene_add_light(self._h, C.byref(l))

    def add_camera(self, eye, target, yfov, up=(0, 1, 0), orthographic=False, ymag=1.0) -> int:
        c = N.Camera((N.f32 * 3)(*eye), (N.f32 * 3)(*target), (N.f32 * 3)(*up), yfov, int(orthographic), ymag)
        return N.lib().oxpt_scene_add_camera(self._h, C.byref(c))

    def triangle_count(self) -> int:
        return int(N.lib().oxpt_scene_triangle_count(self._h))

    # ---- procedural scenes
    @classmethod
    def cornell(cls) -> "Scene":
        return cls(N.lib().oxpt_scene_cornell())

    @classmethod
    def icosphere(cls, freq=229, seed=1, n_materials=64, n_textures=8, tex_size=2048, n_punctual=16,
                  n_emissive=512, material_mix=0) -> "Scene":
        return cls(N.lib().oxpt_scene_icosphere(freq, seed, n_materials, n_textures, tex_size, n_punctual,
                                                 n_emissive, material_mix))

    @classmethod
    def box_field(cls, n: int, seed: int = 1, material_mix: int = 1) -> "Scene":
        return cls(N.lib().oxpt_scene_box_field(n, seed, material_mix))

    @classmethod
    def furnace(cls, rho: float = 0.5, le: float = 1.0) -> "Scene":
        return cls(N.lib().oxpt_scene_furnace(rho, le))


class EnvironmentMap:
    """oxideav_render::pathtrace::EnvironmentMap: an equirectangular RGBA
    float image times an intensity."""

    def __init__(self, rgba: Optional[np.ndarray] = None, intensity: float = 1.0, handle=None):
        if handle is None:
            a = np.ascontiguousarray(rgba, dtype=np.float32)
            h, w = a.shape[:2]
            handle = N.lib().oxpt_env_new(w, h, a.ctypes.data, intensity)
        if not handle:
            raise InvalidOptionsError("bad environment image")
        self._h = handle

    @classmethod
    def sky(cls, w=1024, h=512, sun_dir=(0.3, 0.8, -0.5), sun_radiance=2000.0) -> "EnvironmentMap":
        return cls(handle=N.lib().oxpt_env_sky(w, h, C.byref((N.f32 * 3)(*sun_dir)), sun_radiance))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and N is not None:  # None while the interpreter shuts down
            N.lib().oxpt_env_free(h)
            self._h = None

    @property
    def handle(self):
        return self._h


@dataclass
class Prepared:
    """Flat buffers + Params exactly as uploaded (what the reference binds)."""
    geom: np.ndarray
    attrs: np.ndarray
    tables: np.ndarray
    atlas: np.ndarray
    atlas_side: int
    atlas_layers: int
    node_count: int
    slot_count: int
    params: N.Params
    bvh_depth: int


def _copy_view(v: N.PreparedView) -> Prepared:
    def arr(ptr, n, ct, dt):
        if n == 0:
            return np.zeros(0, dtype=dt)
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(n,)).copy()

    atlas_n = v.atlas_side * v.atlas_side * v.atlas_layers * 4
    p = N.Params()
    C.memmove(C.byref(p), C.byref(v.params), C.sizeof(p))
    return Prepared(arr(v.geom, v.geom_words, N.u32, np.uint32), arr(v.attrs, v.attr_floats, N.f32, np.float32),
                    arr(v.tables, v.table_words, N.u32, np.uint32), arr(v.atlas, atlas_n, N.u16, np.uint16),
                    v.atlas_side, v.atlas_layers, v.node_count, v.slot_count, p, v.bvh_depth)


def prepare(scene: Scene, opts: RenderOptions, env: Optional[EnvironmentMap] = None) -> Prepared:
    """Scene preparation without a device (upload + ensure_binding)."""
    o = opts.to_c()
    h = N.lib().oxpt_prepare(scene.handle, C.byref(o), env.handle if env else None)
    try:
        v = N.PreparedView()
        N.lib().oxpt_prepared_view_of(h, C.byref(v))
        return _copy_view(v)
    finally:
        N.lib().oxpt_prepared_free(h)


@dataclass
class DeviceImage:
    """draw_texture's headless result: device pointer, size, format."""
    data: int
    width: int
    height: int
    pitch_bytes: int
    format: str


class PinnedImage:
    """Page-locked RGBA8 host image (oxpt_host_alloc) for the present path."""

    def __init__(self, h: int, w: int):
        n = max(1, h * w * 4)
        self.ptr = N.lib().oxpt_host_alloc(n)
        if not self.ptr:
            raise BackendError("cannot allocate pinned host memory")
        self.array = np.ctypeslib.as_array(C.cast(self.ptr, C.POINTER(C.c_uint8)), shape=(h, w, 4))
        self._tracer = None

    def wait(self) -> np.ndarray:
        if self._tracer is not None:
            self._tracer.present_wait()
        return self.array

    def __del__(self):
        p = getattr(self, "ptr", None)
        if p and N is not None:  # None while the interpreter shuts down
            if self._tracer is not None:
                N.lib().oxpt_tracer_present_wait(self._tracer._h)
            N.lib().oxpt_host_free(p)
            self.ptr = None


class GpuPathTracer:
    """Progressive CUDA path tracer with the reference's API and reset rules."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        st = N.lib().oxpt_tracer_new(device, C.byref(h))
        if st != N.OK:
            raise BackendError(f"no usable CUDA device {device} (status {st}); the path tracer needs sm_100")
        self._h = h.value
        self._env = None

    @classmethod
    def new(cls, device: int = 0) -> "GpuPathTracer":
        return cls(device)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and N is not None:  # None while the interpreter shuts down
            N.lib().oxpt_tracer_free(h)
            self._h = None

    def _check(self, st: int):
        if st != N.OK:
            _raise(st, N.lib().oxpt_tracer_last_error(self._h).decode())

    @property
    def ctx(self):
        return N.lib().oxpt_tracer_ctx(self._h)

    def tuning(self) -> N.Tuning:
        t = N.Tuning()
        N.lib().oxpt_get_tuning(self.ctx, C.byref(t))
        return t

    def set_tuning(self, **kw):
        """Change the execution plan (mode, launch shape); results are
        bit-identical under every plan."""
        t = self.tuning()
        for k, v in kw.items():
            setattr(t, k, v)
        st = N.lib().oxpt_set_tuning(self.ctx, C.byref(t))
        if st != N.OK:
            _raise(st, N.lib().oxpt_last_error(self.ctx).decode())

    def view(self) -> "GpuPathTracer":
        """A session on this tracer's scene (oxpt_serve.h): its own camera,
        resolution, options and accumulator, sharing the resident prepared
        scene and device buffers. Sync it with sync_view()."""
        h = C.c_void_p()
        st = N.lib().oxpt_tracer_new_view(self._h, C.byref(h))
        if st != N.OK:
            _raise(st, "cannot make a view: the owner must be a synced tracer, not a view")
        v = GpuPathTracer.__new__(GpuPathTracer)
        v._h = h.value
        v._env = self._env
        v._owner = self  # the owner's device buffers must outlive the view
        return v

    def sync_view(self, opts: "RenderOptions") -> bool:
        o = opts.to_c()
        r = C.c_int()
        self._check(N.lib().oxpt_tracer_view_sync(self._h, C.byref(o), C.byref(r)))
        return bool(r.value)

    def set_camera(self, eye=None, target=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0), yfov=0.7853982,
                   orthographic=False, ymag=1.0):
        """Camera override (None: the options' camera); resets the accumulation."""
        if eye is None:
            self._check(N.lib().oxpt_tracer_set_camera(self._h, None))
            return
        cam = N.Camera((N.f32 * 3)(*eye), (N.f32 * 3)(*target), (N.f32 * 3)(*up), yfov, int(orthographic), ymag)
        self._check(N.lib().oxpt_tracer_set_camera(self._h, C.cast(C.pointer(cam), C.c_void_p)))

    def memory(self) -> dict:
        """Device bytes held (oxpt_ctx_memory): scene, tables, images, working."""
        out = (N.u64 * 4)()
        N.lib().oxpt_ctx_memory(self.ctx, out)
        return {"scene": int(out[0]), "tables": int(out[1]), "images": int(out[2]), "working": int(out[3])}

    def adapter_summary(self) -> str:
        buf = C.create_string_buffer(256)
        N.lib().oxpt_device_summary(self.ctx, buf, 256)
        return buf.value.decode()

    def set_gpu_prepare(self, on: bool = True):
        """Prepare the scene on this tracer's GPU (the default): BVH,
        leaf-slot flattening and atlas texels, the host preparation's
        buffers word for word; False prepares on the host. Takes effect at
        the next sync."""
        N.lib().oxpt_tracer_set_gpu_prepare(self._h, int(bool(on)))

    def prepare_timing(self) -> dict:
        """Milliseconds of the last device preparation: device time of the
        source upload, BVH build, slot flattening and atlas (its own stream,
        overlapping the others), host wall time of the whole call and of the
        four-wide tree, and the kernels it launched."""
        ms = (C.c_float * 8)()
        st = N.lib().oxpt_diag_scene_build(self.ctx, ms)
        if st != N.OK:
            _raise(st, N.lib().oxpt_last_error(self.ctx).decode())
        return dict(zip(("upload", "bvh", "flatten", "atlas", "total", "tree4", "launches"), list(ms)))

    def set_texture_resolver(self, resolver=None):
        N.lib().oxpt_tracer_set_texture_resolver(self._h)

    def set_environment(self, env: Optional[EnvironmentMap]):
        self._env = env
        N.lib().oxpt_tracer_set_environment(self._h, env.handle if env else None)

    def invalidate_scene(self):
        N.lib().oxpt_tracer_invalidate_scene(self._h)

    def reset(self):
        self._check(N.lib().oxpt_tracer_reset(self._h))

    def samples(self) -> int:
        return int(N.lib().oxpt_tracer_samples(self._h))

    def is_converged(self) -> bool:
        return bool(N.lib().oxpt_tracer_is_converged(self._h))

    def size(self) -> Tuple[int, int]:
        w, h = N.u32(), N.u32()
        N.lib().oxpt_tracer_size(self._h, C.byref(w), C.byref(h))
        return w.value, h.value

    def sync(self, scene: Scene, opts: RenderOptions) -> bool:
        o = opts.to_c()
        r = C.c_int(0)
        self._check(N.lib().oxpt_tracer_sync(self._h, scene.handle, C.byref(o), C.byref(r)))
        return bool(r.value)

    def refine(self, samples: int):
        self._check(N.lib().oxpt_tracer_refine(self._h, int(samples)))

    def finish(self):
        self._check(N.lib().oxpt_tracer_finish(self._h))

    def image(self) -> np.ndarray:
        w, h = self.size()
        out = np.empty((h, w, 4), dtype=np.uint8)
        self._check(N.lib().oxpt_tracer_image(self._h, out.ctypes.data))
        return out

    def image_async(self) -> "PinnedImage":
        """image() without waiting: returns a pinned buffer that holds the
        RGBA8 image once .wait() returns; refines enqueued meanwhile overlap
        the copy."""
        w, h = self.size()
        buf = PinnedImage(h, w)
        self._check(N.lib().oxpt_tracer_image_async(self._h, buf.ptr))
        buf._tracer = self
        return buf

    def present_wait(self):
        self._check(N.lib().oxpt_tracer_present_wait(self._h))

    def hdr(self) -> np.ndarray:
        w, h = self.size()
        out = np.empty((h, w, 4), dtype=np.float32)
        self._check(N.lib().oxpt_tracer_hdr(self._h, out.ctypes.data))
        return out

    def draw_texture(self) -> DeviceImage:
        d = N.DevImage()
        self._check(N.lib().oxpt_tracer_draw_texture(self._h, C.byref(d)))
        return DeviceImage(d.data, d.width, d.height, d.pitch_bytes, "rgba8" if d.format == 0 else "rgba32f")

    def read_accum(self) -> np.ndarray:
        w, h = self.size()
        out = np.empty((h, w, 4), dtype=np.float32)
        self._check(N.lib().oxpt_tracer_read_accum(self._h, out.ctypes.data))
        return out

    def prepared(self) -> Prepared:
        v = N.PreparedView()
        self._check(N.lib().oxpt_tracer_prepared(self._h, C.byref(v)))
        return _copy_view(v)

    def resolve_params(self, hdr: bool) -> N.ResolveParams:
        rp = N.ResolveParams()
        self._check(N.lib().oxpt_tracer_resolve_params(self._h, int(hdr), C.byref(rp)))
        return rp

    # ---- Renderer trait (src/pathtrace.rs:1241-1264)
    def _run(self, scene: Scene, opts: RenderOptions):
        self.invalidate_scene()
        self.sync(scene, opts)
        self.refine(max(opts.path_trace.samples_per_pixel, 1))

    def render(self, scene: Scene, opts: RenderOptions) -> np.ndarray:
        self._run(scene, opts)
        return self.image()

    def render_hdr(self, scene: Scene, opts: RenderOptions) -> np.ndarray:
        self._run(scene, opts)
        return self.hdr()


def refine_batch(tracers, samples, executor: Optional["GpuPathTracer"] = None):
    """refine() of several tracers traced as one wavefront (oxpt_batch.h).

    `samples` is one count for all or one per tracer. Every tracer's
    accumulation ends bit-identical to its own refine(); the executor's
    (default: the first tracer's) stream and execution plan run the batch."""
    tracers = list(tracers)
    if not tracers:
        return
    counts = [int(samples)] * len(tracers) if np.isscalar(samples) else [int(x) for x in samples]
    if len(counts) != len(tracers):
        raise ValueError("one sample count per tracer")
    hs = (C.c_void_p * len(tracers))(*[t._h for t in tracers])
    ns = (N.u32 * len(tracers))(*counts)
    ex = executor.ctx if executor is not None else None
    st = N.lib().oxpt_tracers_refine_batch(hs, len(tracers), ns, ex)
    if st != N.OK:
        who = executor if executor is not None else tracers[0]
        _raise(st, N.lib().oxpt_last_error(who.ctx).decode())


class GpuMode(enum.Enum):
    """Which pipeline GpuRenderer renders with; only the path tracer exists
    here (the rasteriser is outside this build)."""
    PATH_TRACE = "path_trace"


class GpuRenderer:
    """GpuRenderer reduced to its path-trace mode (src/lib.rs:146-314)."""

    def __init__(self, device: int = 0):
        self._device = device
        self._pt: Optional[GpuPathTracer] = None
        self._mode = GpuMode.PATH_TRACE

    def set_mode(self, mode: GpuMode):
        if mode is not GpuMode.PATH_TRACE:
            raise InvalidOptionsError("only GpuMode.PATH_TRACE is available")
        self._mode = mode

    def mode(self) -> GpuMode:
        return self._mode

    def path_tracer(self) -> GpuPathTracer:
        if self._pt is None:
            self._pt = GpuPathTracer(self._device)
        return self._pt

    def render(self, scene: Scene, opts: RenderOptions) -> np.ndarray:
        return self.path_tracer().render(scene, opts)

    def render_hdr(self, scene: Scene, opts: RenderOptions) -> np.ndarray:
        return self.path_tracer().render_hdr(scene, opts)


class RenderRegistry:
    """oxideav_render::RenderRegistry: name -> factory."""

    def __init__(self):
        self._f: Dict[str, Callable[[], object]] = {}

    def register(self, name: str, factory: Callable[[], object]):
        self._f[name] = factory

    def names(self):
        return sorted(self._f)

    def make(self, name: str):
        if name not in self._f:
            raise InvalidOptionsError(f"no renderer named {name!r}")
        return self._f[name]()


def register_into(registry: RenderRegistry):
    """Register the path tracer under "gpu-pathtrace". The factory opens the
    device lazily, on each make() call."""
    registry.register(PATHTRACE_BACKEND_NAME, lambda: GpuPathTracer())
