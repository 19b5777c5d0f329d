"""One frame across several GPUs: contiguous row tiles, one process per GPU.

The reference tracer is single-device; its only partitioning is row tiles
x runs of consecutive samples per dispatch (src/pathtrace.rs:592-615).
Here each rank traces every sample of its own contiguous row tile, so each
pixel's accumulation is done entirely by one GPU in sample order and the
result is bit-identical to a single-GPU render. The only exchange is one
all-gather of the accumulator's row tiles (w x rows x 16 bytes per rank)
before a resolve: NCCL over NVLink between GPUs, or gloo between CPU
processes in the tests.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import _native as N


def row_tile(height: int, rank: int, world: int) -> Tuple[int, int]:
    """(y0, rows) of `rank`'s tile: contiguous, sizes differing by at most
    one row, covering [0, height) exactly once over all ranks."""
    if not (0 <= rank < world):
        raise ValueError("rank outside the world")
    base, extra = divmod(height, world)
    y0 = rank * base + min(rank, extra)
    return y0, base + (1 if rank < extra else 0)


def gather_row_tiles(accum, height: int, group=None):
    """All-gather the row tiles of an (h, w, 4) float32 torch tensor in
    place: on entry each rank holds valid rows only in its own tile; on
    return every rank holds the whole accumulator."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    h, w = accum.shape[0], accum.shape[1]
    assert h == height
    max_rows = -(-height // world)
    y0, rows = row_tile(height, rank, world)
    send = torch.zeros((max_rows, w, 4), dtype=accum.dtype, device=accum.device)
    send[:rows] = accum[y0:y0 + rows]
    recv = torch.empty((world * max_rows, w, 4), dtype=accum.dtype, device=accum.device)
    dist.all_gather_into_tensor(recv, send, group=group)
    for r in range(world):
        ry0, rrows = row_tile(height, r, world)
        if r != rank and rrows:
            accum[ry0:ry0 + rrows] = recv[r * max_rows:r * max_rows + rrows]
    return accum


class _CudaArray:
    """__cuda_array_interface__ view of a device buffer (zero copy)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def accumulator_tensor(tracer, device: int):
    """The tracer's device accumulator as an (h, w, 4) float32 torch tensor
    (zero copy, read-write)."""
    import torch
    d = N.DevImage()
    tracer._check(N.lib().oxpt_accum_view(tracer.ctx, C.byref(d)))
    return torch.as_tensor(_CudaArray(d.data, (d.height, d.width, 4), "<f4"), device=f"cuda:{device}")


class ShardedPathTracer:
    """GpuPathTracer over the GPUs of a torch.distributed (NCCL) group: each
    rank refines its row tile; image() / hdr() first all-gather the
    accumulator tiles, so every rank resolves the full frame."""

    def __init__(self, device: int, group=None):
        import torch.distributed as dist
        from .pathtracer import GpuPathTracer
        self.pt = GpuPathTracer(device)
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.device = device

    def sync(self, scene, opts) -> bool:
        return self.pt.sync(scene, opts)

    def tile(self) -> Tuple[int, int]:
        return row_tile(self.pt.size()[1], self.rank, self.world)

    def refine(self, samples: int):
        y0, rows = self.tile()
        st = N.lib().oxpt_tracer_refine_rows(self.pt._h, int(samples), y0, rows)
        self.pt._check(st)

    def samples(self) -> int:
        return self.pt.samples()

    def accumulator(self):
        return accumulator_tensor(self.pt, self.device)

    def gather(self):
        import torch
        acc = self.accumulator()
        # The tracer's kernels run on its own stream: wait for them first.
        self.pt.finish()
        gather_row_tiles(acc, acc.shape[0], self.group)
        torch.cuda.synchronize(self.device)

    def image(self) -> np.ndarray:
        self.gather()
        return self.pt.image()

    def hdr(self) -> np.ndarray:
        self.gather()
        return self.pt.hdr()
