"""ctypes bindings of liboxpt.so (include/oxpt.h, oxpt_batch.h, oxpt_serve.h, oxpt_host.h, oxpt_diag.h).

The library is built in-tree by ``build.py``. Loading fails loudly when it
is missing: there is no CPU fallback on this path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboxpt.so"
HOST_LIB_PATH = HERE / "liboxpt_host.so"  # scene building and preparation only, no CUDA

u8, u16, u32, u64, i32, f32 = C.c_uint8, C.c_uint16, C.c_uint32, C.c_uint64, C.c_int32, C.c_float
vp, sz, cint = C.c_void_p, C.c_size_t, C.c_int

# Status codes (oxpt_status).
OK, E_NODEV, E_NOMEM, E_LIMIT, E_INVALID, E_TIMEOUT, E_CUDA = range(7)


class Params(C.Structure):
    _fields_ = [("eye", f32 * 4), ("forward", f32 * 4), ("side", f32 * 4), ("up", f32 * 4),
                ("dims", u32 * 4), ("cfg", u32 * 4), ("env", u32 * 4), ("offs0", u32 * 4),
                ("offs1", u32 * 4), ("offs2", u32 * 4), ("fparams", f32 * 4)]


class Frame(C.Structure):
    _fields_ = [("first", u32), ("count", u32), ("y0", u32), ("rows", u32)]


class ResolveParams(C.Structure):
    _fields_ = [("cfg", u32 * 4), ("exposure", f32 * 4), ("background", f32 * 4)]


class SceneDesc(C.Structure):
    _fields_ = [("geom", vp), ("geom_words", sz), ("attrs", vp), ("attr_floats", sz),
                ("atlas", vp), ("atlas_side", u32), ("atlas_layers", u32),
                ("node_count", u32), ("slot_count", u32)]


class DeviceScene(C.Structure):
    _fields_ = [("geom", vp), ("geom_words", sz), ("attrs", vp), ("attr_floats", sz), ("tables", vp),
                ("table_words", sz), ("atlas", vp), ("atlas_side", u32), ("atlas_layers", u32)]


NOALLOC_MAX_PATHS = 1 << 18
NRC_PARAMS = 29696
NRC_INPUTS = 12


class BatchFrame(C.Structure):
    _fields_ = [("ctx", vp), ("first", u32), ("count", u32), ("y0", u32), ("rows", u32)]


class NrcConfig(C.Structure):
    _fields_ = [("enabled", u32), ("query_bounce", u32), ("train_one_in", u32), ("max_train", u32),
                ("train", u32), ("train_suffix", u32), ("spread", C.c_float), ("frames_per_wave", u32)]


class DevImage(C.Structure):
    _fields_ = [("data", vp), ("width", u32), ("height", u32), ("pitch_bytes", u32), ("format", u32)]


class Sampler(C.Structure):
    _fields_ = [("wrap_s", u32), ("wrap_t", u32), ("mag_linear", u32), ("min_filter", u32)]


class TexRef(C.Structure):
    _fields_ = [("texture", i32), ("uv_set", u32), ("transform", f32 * 6)]


class Material(C.Structure):
    _fields_ = [("base_color", f32 * 4), ("emissive", f32 * 3), ("metallic", f32), ("roughness", f32),
                ("normal_scale", f32), ("alpha_mode", u32), ("alpha_cutoff", f32),
                ("double_sided", u32), ("unlit", u32), ("ior", f32),
                ("has_specular", u32), ("specular", f32), ("specular_color", f32 * 3),
                ("has_transmission", u32), ("transmission", f32),
                ("has_volume", u32), ("thickness", f32), ("attenuation_color", f32 * 3),
                ("attenuation_distance", f32),
                ("has_clearcoat", u32), ("clearcoat", f32), ("clearcoat_roughness", f32),
                ("clearcoat_normal_scale", f32),
                ("has_sheen", u32), ("sheen_color", f32 * 3), ("sheen_roughness", f32),
                ("tex", TexRef * 13)]


class Light(C.Structure):
    _fields_ = [("kind", u32), ("position", f32 * 3), ("direction", f32 * 3), ("color", f32 * 3),
                ("intensity", f32), ("range", f32), ("inner_cone", f32), ("outer_cone", f32)]


class Camera(C.Structure):
    _fields_ = [("eye", f32 * 3), ("target", f32 * 3), ("up", f32 * 3), ("yfov", f32),
                ("orthographic", u32), ("ymag", f32)]


class RenderOptions(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("scene_camera", i32), ("background", u8 * 4),
                ("exposure", f32), ("tone_map", u32), ("ambient", f32), ("light_intensity", f32),
                ("samples_per_pixel", u32), ("max_bounces", u32), ("rr_start", u32), ("seed", u32),
                ("strategy", u32), ("clamp", f32)]


class PreparedView(C.Structure):
    _fields_ = [("geom", vp), ("geom_words", sz), ("attrs", vp), ("attr_floats", sz),
                ("tables", vp), ("table_words", sz), ("atlas", vp), ("atlas_side", u32),
                ("atlas_layers", u32), ("node_count", u32), ("slot_count", u32),
                ("params", Params), ("bvh_depth", u32)]


class Tuning(C.Structure):
    _fields_ = [("mode", u32), ("threads", u32), ("blocks_per_sm", u32), ("wave_slots", u32),
                ("max_paths", u64), ("wave_items", u64), ("check_every", u32), ("shade_variant", u32),
                ("trace_variant", u32), ("stack", u32), ("nee_variant", u32), ("shadow_walk", u32),
                ("graphs", u32), ("refill", u32), ("closest_walk", u32), ("fast_shading", u32)]


MODE_MEGAKERNEL, MODE_WAVEFRONT, MODE_WAVEFRONT_SPLIT = 0, 1, 2

assert C.sizeof(Params) == 176
assert C.sizeof(ResolveParams) == 48
assert C.sizeof(Tuning) == 72

_SIGS = {
    # oxpt.h
    "oxpt_abi_version": (u32, []),
    "oxpt_create": (cint, [cint, C.POINTER(vp)]),
    "oxpt_destroy": (cint, [vp]),
    "oxpt_last_error": (C.c_char_p, [vp]),
    "oxpt_set_stream": (cint, [vp, vp]),
    "oxpt_get_stream": (vp, [vp]),
    "oxpt_device_summary": (cint, [vp, C.c_char_p, sz]),
    "oxpt_upload_scene": (cint, [vp, C.POINTER(SceneDesc)]),
    "oxpt_set_tables": (cint, [vp, vp, sz]),
    "oxpt_stage_scene": (cint, [vp, C.POINTER(SceneDesc), vp, sz]),
    "oxpt_share_scene": (cint, [vp, vp]),
    "oxpt_share_tables": (cint, [vp, vp]),
    "oxpt_set_params": (cint, [vp, C.POINTER(Params)]),
    "oxpt_resize": (cint, [vp, u32, u32]),
    "oxpt_reset": (cint, [vp]),
    "oxpt_dispatch": (cint, [vp, C.POINTER(Frame)]),
    "oxpt_refine": (cint, [vp, u32, u32]),
    "oxpt_finish": (cint, [vp]),
    "oxpt_resolve": (cint, [vp, C.POINTER(ResolveParams), cint, vp, C.POINTER(DevImage)]),
    "oxpt_read_accum": (cint, [vp, vp]),
    "oxpt_resolve_async": (cint, [vp, C.POINTER(ResolveParams), cint, vp]),
    "oxpt_resolve_wait": (cint, [vp]),
    "oxpt_host_alloc": (vp, [sz]),
    "oxpt_host_free": (None, [vp]),
    "oxpt_accum_view": (cint, [vp, C.POINTER(DevImage)]),
    "oxpt_dispatch_noalloc": (cint, [C.c_void_p, C.POINTER(Params), C.POINTER(Frame), vp, vp]),
    # oxpt_batch.h
    "oxpt_refine_batch": (cint, [vp, C.POINTER(BatchFrame), u32]),
    "oxpt_diag_batch_plan": (cint, [vp, u32, u64, vp, sz, C.POINTER(sz)]),
    # oxpt_diag.h
    "oxpt_diag_sobol": (cint, [vp, vp, u32, sz, vp, vp, vp, vp, vp]),
    "oxpt_diag_trace_rays": (cint, [vp, sz, vp, u32, vp, vp, vp, vp]),
    "oxpt_diag_math": (cint, [vp, cint, sz, vp, vp, vp]),
    "oxpt_diag_refine_counted": (cint, [vp, u32, u32, vp]),
    "oxpt_diag_set_launch": (cint, [vp, u32, u32, u64]),
    "oxpt_diag_set_walk": (cint, [vp, u32, u32]),
    "oxpt_diag_get_walk": (cint, [vp, C.POINTER(u32)]),
    "oxpt_diag_set_nee_mask": (cint, [vp, cint]),
    "oxpt_diag_set_shadow_postpone": (cint, [vp, cint]),
    "oxpt_diag_set_ray_order": (cint, [vp, cint]),
    "oxpt_diag_set_l2_window": (cint, [vp, cint, C.POINTER(u64)]),
    "oxpt_diag_launch_count": (cint, [vp, C.POINTER(u64)]),
    "oxpt_diag_set_timing": (cint, [vp, cint]),
    "oxpt_set_tuning": (cint, [vp, C.POINTER(Tuning)]),
    "oxpt_get_tuning": (cint, [vp, C.POINTER(Tuning)]),
    "oxpt_diag_wave_iterations": (cint, [vp, C.POINTER(u64)]),
    "oxpt_diag_bvh4": (cint, [vp, C.POINTER(u32 * 4)]),
    "oxpt_diag_bvh_build": (cint, [cint, vp, u32, cint, vp, vp, C.POINTER(u32), C.POINTER(u32)]),
    "oxpt_diag_graph_builds": (cint, [vp, C.POINTER(u64)]),
    "oxpt_diag_bvh4_build": (cint, [vp, u32, vp, sz, C.POINTER(sz), C.POINTER(u32), C.POINTER(u32)]),
    "oxpt_diag_timing_kinds": (cint, [vp, vp, vp]),
    "oxpt_diag_counters_split": (cint, [vp, vp]),
    "oxpt_diag_timing": (cint, [vp, C.POINTER(C.c_double), C.POINTER(u64), C.POINTER(C.c_double), C.POINTER(u64)]),
    # oxpt_nrc.h
    "oxpt_nrc_create": (cint, [vp, u64, C.POINTER(vp)]),
    "oxpt_nrc_destroy": (None, [vp]),
    "oxpt_nrc_last_error": (C.c_char_p, [vp]),
    "oxpt_nrc_get_weights": (cint, [vp, vp]),
    "oxpt_nrc_set_weights": (cint, [vp, vp]),
    "oxpt_nrc_set_adam": (cint, [vp, f32, f32, f32, f32]),
    "oxpt_nrc_infer": (cint, [vp, vp, u32, vp]),
    "oxpt_nrc_train": (cint, [vp, vp, vp, u32, cint, C.POINTER(f32), vp]),
    "oxpt_nrc_config_default": (None, [C.c_void_p]),
    "oxpt_nrc_refine": (cint, [vp, vp, u32, u32, C.c_void_p, C.POINTER(f32)]),
    "oxpt_nrc_frame_counts": (cint, [vp, C.POINTER(u32), C.POINTER(u32)]),
    "oxpt_tracer_refine_nrc": (cint, [vp, vp, u32, C.c_void_p, C.POINTER(f32)]),
    # oxpt_serve.h
    "oxpt_ctx_device": (cint, [vp]),
    "oxpt_mark": (cint, [vp, C.POINTER(u64)]),
    "oxpt_wait_mark": (cint, [vp, u64]),
    "oxpt_ctx_memory": (cint, [vp, C.POINTER(u64 * 4)]),
    "oxpt_tracer_new_view": (cint, [vp, C.POINTER(vp)]),
    "oxpt_tracer_view_sync": (cint, [vp, C.POINTER(RenderOptions), C.POINTER(cint)]),
    "oxpt_tracer_set_camera": (cint, [vp, C.c_void_p]),
    # oxpt_host.h
    "oxpt_material_default": (None, [C.POINTER(Material)]),
    "oxpt_scene_new": (vp, []),
    "oxpt_scene_free": (None, [vp]),
    "oxpt_scene_add_material": (i32, [vp, C.POINTER(Material)]),
    "oxpt_scene_add_texture": (i32, [vp, u32, u32, vp, u32, C.POINTER(Sampler)]),
    "oxpt_scene_add_mesh": (i32, [vp, u32, vp, vp, vp, vp, vp, vp, i32]),
    "oxpt_scene_add_light": (i32, [vp, C.POINTER(Light)]),
    "oxpt_scene_add_camera": (i32, [vp, C.POINTER(Camera)]),
    "oxpt_scene_triangle_count": (u64, [vp]),
    "oxpt_scene_cornell": (vp, []),
    "oxpt_scene_icosphere": (vp, [u32, u64, u32, u32, u32, u32, u32, u32]),
    "oxpt_scene_box_field": (vp, [u32, u64, u32]),
    "oxpt_scene_furnace": (vp, [f32, f32]),
    "oxpt_env_new": (vp, [u32, u32, vp, f32]),
    "oxpt_env_sky": (vp, [u32, u32, C.POINTER(f32 * 3), f32]),
    "oxpt_env_free": (None, [vp]),
    "oxpt_render_options_default": (None, [C.POINTER(RenderOptions)]),
    "oxpt_prepare": (vp, [vp, C.POINTER(RenderOptions), vp]),
    "oxpt_prepared_view_of": (None, [vp, C.POINTER(PreparedView)]),
    "oxpt_prepared_free": (None, [vp]),
    "oxpt_tracer_new": (cint, [cint, C.POINTER(vp)]),
    "oxpt_tracer_free": (None, [vp]),
    "oxpt_tracer_last_error": (C.c_char_p, [vp]),
    "oxpt_tracer_ctx": (vp, [vp]),
    "oxpt_tracer_set_environment": (None, [vp, vp]),
    "oxpt_tracer_invalidate_scene": (None, [vp]),
    "oxpt_tracer_set_texture_resolver": (None, [vp]),
    "oxpt_tracer_reset": (cint, [vp]),
    "oxpt_tracer_samples": (u32, [vp]),
    "oxpt_tracer_is_converged": (cint, [vp]),
    "oxpt_tracer_size": (None, [vp, C.POINTER(u32), C.POINTER(u32)]),
    "oxpt_tracer_sync": (cint, [vp, vp, C.POINTER(RenderOptions), C.POINTER(cint)]),
    "oxpt_tracer_refine": (cint, [vp, u32]),
    "oxpt_tracer_set_gpu_prepare": (None, [vp, cint]),
    "oxpt_build_scene": (cint, [vp, vp, vp, vp]),
    "oxpt_read_scene": (cint, [vp, vp, vp, vp]),
    "oxpt_diag_scene_build": (cint, [vp, vp]),
    "oxpt_diag_bvh4_build_device": (cint, [cint, vp, C.c_uint32, vp, sz, vp, vp, vp, vp, vp]),
    "oxpt_tracer_refine_rows": (cint, [vp, u32, u32, u32]),
    "oxpt_tracers_refine_batch": (cint, [C.POINTER(vp), u32, C.POINTER(u32), vp]),
    "oxpt_tracer_finish": (cint, [vp]),
    "oxpt_tracer_image": (cint, [vp, vp]),
    "oxpt_tracer_hdr": (cint, [vp, vp]),
    "oxpt_tracer_image_async": (cint, [vp, vp]),
    "oxpt_tracer_present_wait": (cint, [vp]),
    "oxpt_tracer_draw_texture": (cint, [vp, C.POINTER(DevImage)]),
    "oxpt_tracer_read_accum": (cint, [vp, vp]),
    "oxpt_tracer_prepared": (cint, [vp, C.POINTER(PreparedView)]),
    "oxpt_tracer_resolve_params": (cint, [vp, cint, C.POINTER(ResolveParams)]),
    "oxpt_f32_to_f16": (u16, [f32]),
    "oxpt_sobol_directions": (None, [vp]),
    "oxpt_sheen_albedo_table": (None, [vp]),
}

_lib = None
_host_only = False


def select_host_only():
    """Make lib() load liboxpt_host.so instead: scene building and
    preparation on the CPU, with no CUDA library mapped into the process.
    Tracer calls are then unavailable (their symbols are absent). Must be
    called before the first lib()."""
    global _host_only
    if _lib is not None and not _host_only:
        raise RuntimeError("liboxpt.so is already loaded in this process")
    _host_only = True


def lib() -> C.CDLL:
    """The loaded liboxpt.so (raises if it has not been built), or
    liboxpt_host.so after select_host_only()."""
    global _lib
    if _lib is None:
        path = HOST_LIB_PATH if _host_only else LIB_PATH
        if not path.exists():
            raise RuntimeError(
                f"{path} is missing: build it with oxideav-render-vulkan_b200/build.py "
                "(there is no CPU fallback for the path tracer)")
        L = C.CDLL(str(path))
        for name, (res, args) in _SIGS.items():
            if _host_only and not hasattr(L, name):
                continue
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)
