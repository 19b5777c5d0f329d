"""Row-tile split of one frame over 2 ranks (gloo, CPU): each rank renders
its tile with the oracle, the tiles are all-gathered, and the result equals
the single-process render bit for bit. Exercises the host logic of the
multi-GPU path (tile assignment and gather) without a GPU."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    import __graft_entry__ as g
    import oracle
    import scenes

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pkg = g.load_package()
        from oxideav_render_vulkan_b200 import shard
        p = pkg.prepare(scenes.materials_scene(pkg), pkg.RenderOptions(width=37, height=29))
        y0, rows = shard.row_tile(29, rank, world)
        acc = np.zeros((29, 37, 4), np.float32)
        oracle.dispatch(p, p.params, (0, 4, y0, rows), acc, threads=2)
        t = torch.from_numpy(acc)
        shard.gather_row_tiles(t, 29)
        np.save(Path(out_dir) / f"rank{rank}.npy", t.numpy())
    finally:
        dist.destroy_process_group()


def test_row_tiles_cover_the_frame_once():
    import importlib
    import __graft_entry__ as g
    g.load_package()
    shard = importlib.import_module("oxideav_render_vulkan_b200.shard")
    for h in (1, 7, 29, 1080):
        for world in (1, 2, 3, 8):
            tiles = [shard.row_tile(h, r, world) for r in range(world)]
            covered = np.zeros(h, np.int32)
            for y0, rows in tiles:
                covered[y0:y0 + rows] += 1
            assert np.all(covered == 1)
            assert max(t[1] for t in tiles) - min(t[1] for t in tiles) <= 1
    with pytest.raises(ValueError):
        shard.row_tile(10, 2, 2)


def test_two_rank_gloo_row_split_is_bit_exact(tmp_path, pkg, oracle):
    import torch.multiprocessing as mp
    import scenes
    world = 2
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    p = pkg.prepare(scenes.materials_scene(pkg), pkg.RenderOptions(width=37, height=29))
    whole, _ = oracle.render(p, 4)
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npy")
        assert np.array_equal(got.view(np.uint32), whole.view(np.uint32))
