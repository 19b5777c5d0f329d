"""Build recipe for liboxpt.so (CUDA kernels for sm_100a + the C ABI + the
C++ host layer), written in-tree next to this file.

Device code is compiled without FMA contraction (``--fmad=false``) and with
IEEE division and square root, because the estimator's per-sample results
must match the CPU restatement bit for bit; host code likewise uses
``-ffp-contract=off``. The one exception is a second build of the split
wavefront's shading kernels with fast math, which only the tolerance plan
runs (``FAST_SOURCES``). Objects go to ``_build/`` and are rebuilt only when
a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
LIB = HERE / "liboxpt.so"
# Scene building and preparation alone (no CUDA): what a process that only
# prepares scenes on the CPU loads (the benchmark's CPU reference arm).
HOST_LIB = HERE / "liboxpt_host.so"
HOST_ONLY = ("prepare", "scene", "bvh", "bvh4", "batch")
BUILD = ROOT / "_build" / "oxpt"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-ftz=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-Xptxas", "-warn-spills",
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function"]
# Sources built a second time for the tolerance plan: FMA contraction,
# approximate division and square root, the CUDA library's transcendentals
# (launchers in oxd::fast; its results are held to image PSNR, not bits).
FAST_SOURCES = ("wave_split.cu",)
FAST_FLAGS = [f for f in NVCC_FLAGS if f not in ("--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false")] \
    + ["-use_fast_math", "-DOXPT_FAST"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build liboxpt.so")


def _sources():
    cu = sorted((HERE / "csrc").glob("*.cu"))
    cpp = sorted((HERE / "host").glob("*.cpp"))
    headers = sorted((HERE / "csrc").glob("*.h")) + sorted((HERE / "csrc").glob("*.cuh")) + \
        sorted((HERE / "host").glob("*.hpp")) + \
        sorted((ROOT / "include").glob("*.h"))
    return cu, cpp, headers


def _stale(obj: Path, src: Path, headers) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in headers)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile and link liboxpt.so; returns its path."""
    cu, cpp, headers = _sources()
    BUILD.mkdir(parents=True, exist_ok=True)
    nv = nvcc()
    inc = ["-I", str(ROOT / "include")] + os.environ.get("OXPT_NVCC_DEFINES", "").split()
    jobs_list = []
    objs = []
    for src in cu:
        obj = BUILD / (src.stem + ".cu.o")
        objs.append(obj)
        if _stale(obj, src, headers):
            jobs_list.append([nv, *ARCH, *NVCC_FLAGS, *inc, "-Xptxas", "-v", "-c", str(src), "-o", str(obj)])
        if src.name in FAST_SOURCES:
            fobj = BUILD / (src.stem + ".fast.cu.o")
            objs.append(fobj)
            if _stale(fobj, src, headers):
                jobs_list.append([nv, *ARCH, *FAST_FLAGS, *inc, "-Xptxas", "-v", "-c", str(src), "-o", str(fobj)])
    for src in cpp:
        obj = BUILD / (src.stem + ".cpp.o")
        objs.append(obj)
        if _stale(obj, src, headers):
            jobs_list.append(["g++", *CXX_FLAGS, *inc, "-c", str(src), "-o", str(obj)])
    logs = []
    if jobs_list:
        with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            logs = list(ex.map(_run, jobs_list))
    relink = not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs)
    if relink:
        tmp = LIB.with_suffix(".so.tmp")
        _run([nv, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lpthread"])
        os.replace(tmp, LIB)
    host_objs = [BUILD / (n + ".cpp.o") for n in HOST_ONLY]
    if not HOST_LIB.exists() or any(o.stat().st_mtime > HOST_LIB.stat().st_mtime for o in host_objs):
        tmp = HOST_LIB.with_suffix(".so.tmp")
        _run(["g++", "-shared", "-o", str(tmp), *map(str, host_objs), "-lpthread"])
        os.replace(tmp, HOST_LIB)
    if verbose:
        for log in logs:
            if log.strip():
                print(log, file=sys.stderr)
    (BUILD / "ptxas.log").write_text("\n".join(logs))
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
