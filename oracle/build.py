"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/oracle.cpp into oracle/liboxpt_oracle.so with
``-ffp-contract=off`` so that no multiply-add is fused. The reference's own
CPU tracer (oxideav_render::PathTracer, Rust, external crate) cannot be
built here: there is no Rust toolchain and the crate is not in the
reference tree, so there is no oracle/_ref build.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboxpt_oracle.so"
SRC = HERE / "oracle.cpp"
DEPS = [SRC, HERE / "oracle.h", HERE.parent / "oxideav-render-vulkan_b200" / "csrc" / "fmath.h"]


def build() -> Path:
    if LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in DEPS):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-Wall",
           str(SRC), "-o", str(tmp), "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build())
