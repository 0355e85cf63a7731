"""Row-sharded rendering across ranks: host logic on gloo (CPU, world size 2)
and the one-GPU identity of the sharded film with the whole-film render."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from tinypt_b200 import multigpu
from tinypt_b200.scene import RenderConfig


def test_shards_cover_every_row_once():
    for height in (1, 2, 5, 135, 1080):
        for world in (1, 2, 3, 8):
            if world > height:
                with pytest.raises(ValueError):
                    multigpu.shard_config(RenderConfig(width=4, height=height), 0, world)
                continue
            seen = []
            for rank in range(world):
                cfg = multigpu.shard_config(RenderConfig(width=4, height=height), rank, world)
                rows = multigpu.shard_rows(height, rank, world)
                assert cfg.film_rows == len(rows)
                assert all(r == cfg.row_begin + k * max(cfg.row_step, 1) for k, r in enumerate(rows))
                seen += rows
            assert sorted(seen) == list(range(height))


def test_assemble_rows_inverts_the_split():
    import torch

    height, width, world = 7, 3, 3
    full = torch.arange(height * width * 2, dtype=torch.float64).view(height, width, 2)
    max_rows = -(-height // world)
    parts = torch.full((world, max_rows, width, 2), -1.0, dtype=torch.float64)
    for r in range(world):
        rows = full[r::world]
        parts[r, : rows.shape[0]] = rows
    assert torch.equal(multigpu.assemble_rows(parts, height, world), full)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_worker(rank, world, port, height, width, out_dir):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # a fake shard film: value = 1000 * image row + column, channel 1 = rank
        rows = multigpu.shard_rows(height, rank, world)
        local = torch.zeros((len(rows), width, 2), dtype=torch.float64)
        for k, y in enumerate(rows):
            local[k, :, 0] = 1000.0 * y + torch.arange(width, dtype=torch.float64)
            local[k, :, 1] = rank
        full = multigpu.gather_film(local, height, world)
        grad = torch.full((8,), float(rank + 1), dtype=torch.float64)
        multigpu.allreduce_gradient(grad)
        torch.save({"full": full, "grad": grad}, os.path.join(out_dir, f"r{rank}.pt"))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("height", [5, 8])
def test_gather_and_allreduce_on_gloo(tmp_path, height):
    """Two gloo ranks: every rank ends with the whole film in image-row order
    and with the summed gradient."""
    import torch
    import torch.multiprocessing as mp

    world, width = 2, 3
    mp.start_processes(_gloo_worker, args=(world, _free_port(), height, width, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    for rank in range(world):
        d = torch.load(tmp_path / f"r{rank}.pt")
        full = d["full"]
        assert full.shape == (height, width, 2)
        for y in range(height):
            assert torch.equal(full[y, :, 0], 1000.0 * y + torch.arange(width, dtype=torch.float64))
            assert torch.all(full[y, :, 1] == y % world)
        assert torch.all(d["grad"] == 3.0)


# ---- one GPU: the shards of a film equal the whole-film render -------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["plain", "wavefront"])
def test_row_shards_equal_whole_film(gpu, mode):
    import torch

    from tinypt_b200 import _abi, scenes
    from tinypt_b200.render import DeviceScene

    m = _abi.TPT_MODE_PLAIN_F64 if mode == "plain" else _abi.TPT_MODE_WAVEFRONT_FP32
    cfg = RenderConfig(width=48, height=27, spp=24, max_bounces=8, rr_start=3, seed=5, mode=m)
    scene = scenes.sphere_scene(cfg.width, cfg.height)
    world = 3
    with DeviceScene(scene) as ds:
        n = cfg.width * cfg.height
        acc = torch.empty(3 * n, dtype=torch.float64, device="cuda")
        acc_w = torch.empty(n, dtype=torch.float64, device="cuda")
        ds.render_device(cfg, acc.data_ptr(), acc_w.data_ptr())
        whole = torch.cat([acc.view(cfg.height, cfg.width, 3), acc_w.view(cfg.height, cfg.width, 1)], 2)
        max_rows = -(-cfg.height // world)
        parts = torch.zeros((world, max_rows, cfg.width, 4), dtype=torch.float64, device="cuda")
        for r in range(world):
            sc = multigpu.shard_config(cfg, r, world)
            k = sc.film_pixels
            a = torch.empty(3 * k, dtype=torch.float64, device="cuda")
            w = torch.empty(k, dtype=torch.float64, device="cuda")
            ds.render_device(sc, a.data_ptr(), w.data_ptr())
            parts[r, : sc.film_rows, :, :3] = a.view(sc.film_rows, cfg.width, 3)
            parts[r, : sc.film_rows, :, 3] = w.view(sc.film_rows, cfg.width)
        assembled = multigpu.assemble_rows(parts, cfg.height, world)
    assert torch.equal(assembled, whole)


@pytest.mark.gpu
def test_adjoint_row_shards_sum_to_whole(gpu):
    """The adjoint of a film equals the sum of the adjoints of its row shards
    (up to the order of the f64 accumulation)."""
    import torch

    from tinypt_b200 import _abi, scenes
    from tinypt_b200.render import DeviceScene

    scene = scenes.gradcheck_scene(32, 24)
    cfg = RenderConfig(width=32, height=24, spp=8, max_bounces=6, rr_start=3, seed=3,
                       mode=_abi.TPT_MODE_WAVEFRONT_FP32)
    dimg = torch.tensor(np.random.default_rng(0).standard_normal((24, 32, 3)).astype(np.float32), device="cuda")
    world = 2
    with DeviceScene(scene) as ds:
        g = torch.empty(4 * ds.n_materials, dtype=torch.float64, device="cuda")
        ds.render_backward(cfg, dimg.contiguous().data_ptr(), g.data_ptr())
        total = torch.zeros_like(g)
        for r in range(world):
            sc = multigpu.shard_config(cfg, r, world)
            part = dimg[r::world].contiguous()
            gr = torch.empty_like(g)
            ds.render_backward(sc, part.data_ptr(), gr.data_ptr())
            total += gr
    assert torch.allclose(total, g, rtol=1e-6, atol=1e-9)
