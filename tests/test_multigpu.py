"""Sharded rendering across ranks: film rows of one frame and jobs of a
batch.  Host logic on gloo (CPU, world size 2); on one GPU, the shards'
films equal the whole render."""
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


def _bench_step_worker(rank, world, port, height, width, out_dir):
    """The exchange of bench.py's multi-GPU step with the render stubbed: a
    rank's shard rows hold a known function of (image row, column)."""
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rows = multigpu.shard_rows(height, rank, world)
        s_acc = torch.zeros((len(rows), width, 3), dtype=torch.float64)
        s_w = torch.zeros((len(rows), width), dtype=torch.float64)
        for k, y in enumerate(rows):
            for c in range(3):
                s_acc[k, :, c] = 1000.0 * y + 10.0 * torch.arange(width, dtype=torch.float64) + c
            s_w[k] = y + 0.5
        g = multigpu.ShardGather(width, height, rank, world)
        acc = torch.empty(height * width * 3, dtype=torch.float64)
        acc_w = torch.empty(height * width, dtype=torch.float64)
        for _ in range(2):  # the buffers are reused step after step
            acc.fill_(-1.0)
            acc_w.fill_(-1.0)
            g.gather(s_acc.reshape(-1), s_w.reshape(-1), acc, acc_w)
        torch.save({"acc": acc, "acc_w": acc_w}, os.path.join(out_dir, f"b{rank}.pt"))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("height", [7, 8])
def test_bench_step_exchange_on_gloo(tmp_path, height):
    """bench.py's multi-GPU step (multigpu.ShardGather): two gloo ranks each
    contribute their interleaved rows; both end with the whole flat film in
    image order, on two steps in a row."""
    import torch
    import torch.multiprocessing as mp

    world, width = 2, 5
    mp.start_processes(_bench_step_worker, args=(world, _free_port(), height, width, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    for rank in range(world):
        d = torch.load(tmp_path / f"b{rank}.pt")
        acc = d["acc"].view(height, width, 3)
        for y in range(height):
            for c in range(3):
                assert torch.equal(acc[y, :, c], 1000.0 * y + 10.0 * torch.arange(width, dtype=torch.float64) + c)
        assert torch.equal(d["acc_w"].view(height, width),
                           (torch.arange(height, dtype=torch.float64) + 0.5)[:, None].expand(height, width))


def test_shard_gather_on_one_rank_copies_the_film():
    import torch

    g = multigpu.ShardGather(4, 3, 0, 1)
    s_acc = torch.arange(36, dtype=torch.float64)
    s_w = torch.arange(12, dtype=torch.float64)
    acc, acc_w = torch.empty(36, dtype=torch.float64), torch.empty(12, dtype=torch.float64)
    g.gather(s_acc, s_w, acc, acc_w)
    assert torch.equal(acc, s_acc) and torch.equal(acc_w, s_w)


# ---- batch jobs sharded by scene -----------------------------------------------------------------
def _best_makespan(costs, world):
    import itertools

    best = float("inf")
    for a in itertools.product(range(world), repeat=len(costs)):
        load = [0.0] * world
        for j, r in enumerate(a):
            load[r] += costs[j]
        best = min(best, max(load))
    return best


def test_shard_jobs_covers_every_job_once_within_the_lpt_bound():
    rng = np.random.default_rng(4)
    for world in (1, 2, 3, 4):
        for n in (0, 1, 3, 7, 9):
            costs = [float(c) for c in rng.integers(1, 100, n)]
            a = multigpu.shard_jobs(costs, world)
            assert len(a) == world and a == multigpu.shard_jobs(costs, world)
            assert sorted(j for r in a for j in r) == list(range(n))
            assert all(r == sorted(r) for r in a)
            loads = [sum(costs[j] for j in r) for r in a]
            if n and world <= 3 and n <= 7:
                assert max(loads) <= 4.0 / 3.0 * _best_makespan(costs, world) + 1e-9
            if n:
                assert max(loads) - min(loads) <= max(costs)
    with pytest.raises(ValueError):
        multigpu.shard_jobs([1.0], 0)


def _gloo_jobs_worker(rank, world, port, sizes, out_dir):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assignment = multigpu.shard_jobs([float(s) for s in sizes], world)
        local = {j: 1000.0 * j + torch.arange(sizes[j], dtype=torch.float64) for j in assignment[rank]}
        full = multigpu.gather_job_films(local, assignment, sizes)
        torch.save({j: t.clone() for j, t in full.items()}, os.path.join(out_dir, f"j{rank}.pt"))
    finally:
        dist.destroy_process_group()


def test_gather_job_films_on_gloo(tmp_path):
    """Two gloo ranks holding films of uneven size: every rank ends with
    every job's film."""
    import torch
    import torch.multiprocessing as mp

    sizes = [12, 40, 4, 28, 8]
    mp.start_processes(_gloo_jobs_worker, args=(2, _free_port(), sizes, str(tmp_path)), nprocs=2,
                       start_method="spawn", join=True)
    for rank in range(2):
        got = torch.load(tmp_path / f"j{rank}.pt")
        assert sorted(got) == list(range(len(sizes)))
        for j, n in enumerate(sizes):
            assert torch.equal(got[j], 1000.0 * j + torch.arange(n, dtype=torch.float64))


@pytest.mark.gpu
def test_batch_job_shards_equal_the_whole_batch(gpu):
    """Each of 3 emulated ranks renders its shard_jobs share over just the
    scenes it uses: every film equals the whole batch's film bit for bit."""
    import torch

    from tinypt_b200 import _abi, scenes
    from tinypt_b200.render import BatchScenes

    w = _abi.TPT_MODE_WAVEFRONT_FP32
    scs = [scenes.sphere_scene(32, 24), scenes.gradcheck_scene(24, 24), scenes.sphere_scene(40, 20)]
    jobs = [(0, RenderConfig(width=32, height=24, spp=8, max_bounces=6, seed=1, mode=w)),
            (1, RenderConfig(width=24, height=24, spp=16, max_bounces=6, seed=2, mode=w)),
            (2, RenderConfig(width=40, height=20, spp=4, max_bounces=6, seed=3, mode=w)),
            (0, RenderConfig(width=32, height=24, spp=12, max_bounces=6, seed=4, mode=w))]
    whole = {j: torch.empty(4 * c.film_pixels, dtype=torch.float64, device="cuda") for j, (_, c) in enumerate(jobs)}
    with BatchScenes(scs) as bs:
        bs.render([(s, c, whole[j].data_ptr(), whole[j].data_ptr() + 24 * c.film_pixels)
                   for j, (s, c) in enumerate(jobs)])
    assignment = multigpu.shard_jobs(multigpu.job_costs(jobs), 3)
    seen = []
    for mine in assignment:
        films, st = multigpu.render_jobs(scs, jobs, mine)
        assert (st is None) == (not mine)
        for j, f in films.items():
            assert torch.equal(f, whole[j]), f"job {j}"
            seen.append(j)
    assert sorted(seen) == list(range(len(jobs)))
    films, _ = multigpu.render_batch_sharded(scs, jobs)        # no process group: one rank
    for j, (acc, acc_w) in enumerate(films):
        n = jobs[j][1].film_pixels
        assert torch.equal(acc.reshape(-1), whole[j][: 3 * n]) and torch.equal(acc_w, whole[j][3 * n:])


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
