"""The C-ABI library loads and exports every function include/*.h declares
(no compute calls: these tests run without a GPU)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(oxpt_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_the_boundary():
    names = declared_functions()
    for core in ("oxpt_create", "oxpt_destroy", "oxpt_upload_scene", "oxpt_set_tables", "oxpt_set_params",
                 "oxpt_resize", "oxpt_reset", "oxpt_dispatch", "oxpt_refine", "oxpt_finish", "oxpt_resolve",
                 "oxpt_tracer_sync", "oxpt_tracer_refine", "oxpt_tracer_image", "oxpt_tracer_hdr",
                 "oxpt_tracer_draw_texture"):
        assert core in names, core


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg._native.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # And the dynamic symbol table has them as C (unmangled) names.
    out = subprocess.run(["nm", "-D", "--defined-only", str(pkg._native.LIB_PATH)], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r"\b(oxpt_\w+)\b", out))
    assert set(declared_functions()) <= exported


def test_python_bindings_cover_the_headers(pkg):
    bound = set(pkg._native.exported_symbols())
    assert set(declared_functions()) <= bound, sorted(set(declared_functions()) - bound)


def test_abi_version_and_struct_sizes(pkg):
    lib = pkg._native.lib()
    assert lib.oxpt_abi_version() == 2  # 2: oxpt_tuning gained closest_walk
    N = pkg._native
    assert C.sizeof(N.Tuning) == 72
    assert C.sizeof(N.Params) == 176  # src/pathtrace.rs:100-114
    assert C.sizeof(N.Frame) == 16  # src/pathtrace.rs:116-123
    assert C.sizeof(N.ResolveParams) == 48  # src/pathtrace.rs:125-131


def test_create_reports_no_device_without_a_gpu(pkg):
    import torch
    if torch.cuda.is_available():
        return
    h = C.c_void_p()
    st = pkg._native.lib().oxpt_create(0, C.byref(h))
    assert st == pkg._native.E_NODEV and not h.value
    try:
        pkg.GpuPathTracer(0)
    except pkg.BackendError:
        pass
    else:
        raise AssertionError("GpuPathTracer must fail loudly without a CUDA device")


def test_host_only_library_prepares_without_cuda(pkg):
    """liboxpt_host.so (scene building and preparation, no CUDA) prepares
    the same buffers as liboxpt.so, and a process that selects it maps
    neither liboxpt.so nor the CUDA runtime (the CPU reference arm)."""
    import sys
    import tempfile

    import numpy as np
    root = ROOT
    code = (
        "import sys, os, numpy as np; sys.path.insert(0, %r)\n"
        "import __graft_entry__ as g\n"
        "pkg = g.load_package(); pkg._native.select_host_only()\n"
        "p = pkg.prepare(pkg.Scene.cornell(), pkg.RenderOptions(width=32, height=32))\n"
        "np.save(sys.argv[1], p.geom)\n"
        "m = open('/proc/%%d/maps' %% os.getpid()).read()\n"
        "print('liboxpt.so' in m, 'liboxpt_host.so' in m, 'cudart' in m)\n" % str(root))
    with tempfile.TemporaryDirectory() as d:
        out = Path(d) / "geom.npy"
        r = subprocess.run([sys.executable, "-c", code, str(out)], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        assert r.stdout.split() == ["False", "True", "False"]
        want = pkg.prepare(pkg.Scene.cornell(), pkg.RenderOptions(width=32, height=32)).geom
        assert np.array_equal(np.load(out), want)
