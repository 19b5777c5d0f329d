"""B200-native drop-in for the `gpu-pathtrace` path of OxideAV/oxideav-render-vulkan.

The package directory name contains hyphens, so it is loaded by path (see
``load_package`` in ``__graft_entry__.py``) under the module name
``oxideav_render_vulkan_b200``.
"""
from .pathtracer import (  # noqa: F401
    PATHTRACE_BACKEND_NAME, BackendError, DeviceImage, EnvironmentMap, Error, GpuMode, GpuPathTracer,
    GpuRenderer, InvalidOptionsError, LightStrategy, PathTraceOptions, Prepared, RenderOptions,
    RenderRegistry, Scene, ToneMap, material, prepare, refine_batch, register_into,
)
from . import _native  # noqa: F401
