"""CPU oracle bindings — TEST INFRASTRUCTURE ONLY.

Used by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
bench.py as the checker; never by the product path. See oracle.h for what
the oracle restates (pathtrace.wgsl + fs_resolve_pt) and how far its parity
with the reference is pinned.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import build as _build

HERE = Path(__file__).resolve().parent
vp, sz, u32, u64, cint, f32 = C.c_void_p, C.c_size_t, C.c_uint32, C.c_uint64, C.c_int, C.c_float


class _Scene(C.Structure):
    _fields_ = [("geom", vp), ("geom_words", sz), ("attrs", vp), ("attr_floats", sz), ("tables", vp),
                ("table_words", sz), ("atlas", vp), ("atlas_side", u32), ("atlas_layers", u32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(str(path))
        L.oxo_dispatch.argtypes = [C.POINTER(_Scene), vp, vp, vp, cint, cint, vp]
        L.oxo_dispatch.restype = cint
        L.oxo_resolve.argtypes = [vp, u32, u32, vp, cint, cint, vp]
        L.oxo_resolve.restype = None
        L.oxo_sobol.argtypes = [vp, u32, sz, vp, vp, vp, vp, vp]
        L.oxo_sobol.restype = None
        L.oxo_trace_rays.argtypes = [C.POINTER(_Scene), vp, sz, vp, u32, vp, vp, vp, vp, cint, vp]
        L.oxo_trace_rays.restype = None
        L.oxo_f32_to_f16.argtypes = [f32]
        L.oxo_f32_to_f16.restype = C.c_uint16
        L.oxo_math.argtypes = [cint, sz, vp, vp, vp, cint]
        L.oxo_math.restype = None
        _lib = L
    return _lib


def _scene(p):
    """p: a Prepared (geom, attrs, tables, atlas numpy arrays + sizes)."""
    s = _Scene(p.geom.ctypes.data, p.geom.size, p.attrs.ctypes.data, p.attrs.size, p.tables.ctypes.data,
               p.tables.size, p.atlas.ctypes.data, p.atlas_side, p.atlas_layers)
    return s


def dispatch(p, params, frame, accum: np.ndarray, threads: int = 0, libm: bool = False):
    """One trace_main dispatch; accum (h, w, 4) float32 updated in place.
    Returns the 8 counters (paths, path rays, shadow rays, AABBs tested,
    leaves, triangle tests, shaded hits, stack pops)."""
    assert accum.dtype == np.float32 and accum.flags.c_contiguous
    s = _scene(p)
    fr = (u32 * 4)(*frame)
    cnt = np.zeros(8, dtype=np.uint64)
    lib().oxo_dispatch(C.byref(s), C.byref(params), fr, accum.ctypes.data, threads, int(libm), cnt.ctypes.data)
    return cnt


def render(p, spp: int, first: int = 0, threads: int = 0, libm: bool = False, accum=None):
    """All rows, samples [first, first + spp): the accumulator (h, w, 4)."""
    w, h = p.params.dims[0], p.params.dims[1]
    if accum is None:
        accum = np.zeros((h, w, 4), dtype=np.float32)
    cnt = dispatch(p, p.params, (first, spp, 0, h), accum, threads, libm)
    return accum, cnt


def resolve(accum: np.ndarray, rparams, hdr: bool, libm: bool = False) -> np.ndarray:
    h, w = accum.shape[:2]
    a = np.ascontiguousarray(accum, dtype=np.float32)
    out = np.empty((h, w, 4), dtype=np.float32 if hdr else np.uint8)
    lib().oxo_resolve(a.ctypes.data, w, h, C.byref(rparams), int(hdr), int(libm), out.ctypes.data)
    return out


def sobol(dirs: np.ndarray, seed: int, x, y, index, pattern_id) -> np.ndarray:
    arrs = [np.ascontiguousarray(a, dtype=np.uint32) for a in (x, y, index, pattern_id)]
    n = arrs[0].size
    out = np.empty((n, 4), dtype=np.uint32)
    d = np.ascontiguousarray(dirs, dtype=np.uint32)
    lib().oxo_sobol(d.ctypes.data, seed, n, *[a.ctypes.data for a in arrs], out.ctypes.data)
    return out


def trace_rays(p, rays: np.ndarray, flags: int, threads: int = 0):
    r = np.ascontiguousarray(rays, dtype=np.float32)
    n = r.shape[0]
    slot = np.empty(n, np.uint32)
    gid = np.empty(n, np.uint32)
    t = np.empty(n, np.float32)
    bary = np.empty((n, 3), np.float32)
    cnt = np.zeros(8, dtype=np.uint64)
    s = _scene(p)
    lib().oxo_trace_rays(C.byref(s), C.byref(p.params), n, r.ctypes.data, flags, slot.ctypes.data,
                         gid.ctypes.data, t.ctypes.data, bary.ctypes.data, threads, cnt.ctypes.data)
    return slot, gid, t, bary, cnt


def f32_to_f16(v: float) -> int:
    return int(lib().oxo_f32_to_f16(v))


def math(op: int, a: np.ndarray, b=None, libm: bool = False) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    bb = None if b is None else np.ascontiguousarray(b, dtype=np.float32)
    out = np.empty_like(a)
    lib().oxo_math(op, a.size, a.ctypes.data, None if bb is None else bb.ctypes.data, out.ctypes.data, int(libm))
    return out
