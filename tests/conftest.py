"""Test configuration: the `gpu` marker, package loading and builds.

CPU tests (`-m "not gpu"`) cover the CPU oracle against the reference's
golden vectors, the host-side preparation logic, the portable math and the
C ABI's exported symbols. GPU tests (`-m gpu`) are the parity tests proper:
they drive the CUDA path through the C ABI and compare with the oracle.
"""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(ROOT / "tests") not in sys.path:
    sys.path.insert(0, str(ROOT / "tests"))

import __graft_entry__  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


_built = False


def _ensure_built():
    global _built
    if not _built:
        __graft_entry__.build()
        _built = True


@pytest.fixture(scope="session")
def pkg():
    _ensure_built()
    return __graft_entry__.load_package()


@pytest.fixture(scope="session")
def oracle(pkg):
    import oracle as o
    o.lib()
    return o


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_tracer_factory(pkg):
    if not _has_gpu():
        pytest.fail("GPU test collected on a machine without a CUDA device")

    def make():
        return pkg.GpuPathTracer(0)
    return make
