"""One frame on several GPUs: row shards, film gather, gradient all-reduce;
and batches of many scenes sharded by job.

The reference splits one render over CPU worker threads that pull tiles of
the film (src/render.rs:116-206).  Across GPUs (one process per GPU,
``torch.distributed``) the units are interleaved film rows: rank r of N
renders rows r, r + N, r + 2N, ... (``RenderConfig.row_begin`` /
``row_step``), each pixel with the same RNG stream as in a one-GPU render,
so the assembled film equals the one-GPU film and the load of cheap (sky)
and expensive rows spreads evenly.  The only exchange of a render is one
gather of the f64 film rows; the adjoint's gradient (4 f64 per material)
is summed with one all-reduce.  A batch of many scenes (``BatchScenes``)
shards by job instead: each rank renders the jobs ``shard_jobs`` gives it
over just the scenes they use, and one all-gather assembles the films.
Works with any ``torch.distributed`` backend: NCCL between GPUs, gloo for
the CPU tests.
"""
from __future__ import annotations

import dataclasses
from typing import Optional

from .scene import RenderConfig


def shard_config(config: RenderConfig, rank: int, world: int) -> RenderConfig:
    """The rows of ``config``'s film that ``rank`` of ``world`` renders."""
    if world <= 1:
        return dataclasses.replace(config, row_begin=0, row_step=0)
    if world > config.height:
        raise ValueError(f"{world} ranks for a film of {config.height} rows")
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside 0..{world - 1}")
    return dataclasses.replace(config, row_begin=rank, row_step=world)


def shard_rows(height: int, rank: int, world: int) -> list:
    """Image rows of a shard, in film order."""
    return list(range(rank, height, world)) if world > 1 else list(range(height))


def assemble_rows(parts, height: int, world: int):
    """parts: (world, max_rows, width, C) tensor of padded shard films ->
    (height, width, C) film with image row y = shard y % world, row y // world."""
    import torch

    width, ch = parts.shape[2], parts.shape[3]
    out = torch.empty((height, width, ch), dtype=parts.dtype, device=parts.device)
    for r in range(world):
        n = len(range(r, height, world))
        out[r::world] = parts[r, :n]
    return out


def gather_film(local, height: int, world: int, group=None):
    """local: this rank's (n_rows, width, C) film rows.  Returns the whole
    (height, width, C) film on every rank (one all-gather of padded rows)."""
    import torch
    import torch.distributed as dist

    if world <= 1:
        return local
    max_rows = -(-height // world)
    pad = torch.zeros((max_rows,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return assemble_rows(torch.stack(parts), height, world)


class ShardGather:
    """The film exchange of a row-sharded frame, with its buffers allocated
    once (a render loop gathers every step): this rank's rows -- acc (rows *
    width * 3 f64) and acc_w (rows * width f64) -- are packed into padded
    (max_rows, width, 4) rows, one all-gather brings every rank's, and the
    whole film is written in image-row order into the caller's flat acc
    (height * width * 3) and acc_w (height * width) tensors."""

    def __init__(self, width: int, height: int, rank: int, world: int, device=None):
        import torch

        self.width, self.height, self.world = width, height, world
        self.rows = len(shard_rows(height, rank, world))
        max_rows = -(-height // world)
        self.pad = torch.zeros((max_rows, width, 4), dtype=torch.float64, device=device)
        self.parts = [torch.empty_like(self.pad) for _ in range(world)]

    def gather(self, s_acc, s_w, acc, acc_w, group=None):
        import torch
        import torch.distributed as dist

        rows, width = self.rows, self.width
        self.pad[:rows, :, :3] = s_acc.view(rows, width, 3)
        self.pad[:rows, :, 3] = s_w.view(rows, width)
        if self.world > 1:
            dist.all_gather(self.parts, self.pad, group=group)
            film = assemble_rows(torch.stack(self.parts), self.height, self.world)
        else:
            film = self.pad[:rows]
        acc.copy_(film[..., :3].reshape(-1))
        acc_w.copy_(film[..., 3].reshape(-1))


def allreduce_gradient(grad, group=None):
    """Sums a gradient (f64 tensor) over the ranks in place."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
    return grad


def _world(group=None):
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def render_sharded(ds, config: RenderConfig, group=None):
    """Renders this rank's rows with ``ds`` (a DeviceScene on this rank's
    GPU) and gathers the film: returns (acc (H, W, 3), acc_w (H, W)) f64 CUDA
    tensors holding the whole film, on every rank."""
    import torch

    rank, world = _world(group)
    cfg = shard_config(config, rank, world)
    rows, w = cfg.film_rows, cfg.width
    film = torch.zeros((rows, w, 4), dtype=torch.float64, device="cuda")
    acc = torch.empty((rows * w * 3,), dtype=torch.float64, device="cuda")
    acc_w = torch.empty((rows * w,), dtype=torch.float64, device="cuda")
    ds.render_device(cfg, acc.data_ptr(), acc_w.data_ptr())
    film[..., :3] = acc.view(rows, w, 3)
    film[..., 3] = acc_w.view(rows, w)
    full = gather_film(film, config.height, world, group)
    return full[..., :3].contiguous(), full[..., 3].contiguous()


def backward_sharded(ds, config: RenderConfig, dimage, group=None, n_materials: Optional[int] = None):
    """Adjoint render of a whole-film dL/dimage ((H, W, 3) float32 CUDA
    tensor) split by rows: each rank differentiates its rows, and the
    gradients (4 f64 per material) are summed over the ranks."""
    import torch

    rank, world = _world(group)
    cfg = shard_config(config, rank, world)
    local = dimage[rank::world].contiguous() if world > 1 else dimage.contiguous()
    n = n_materials if n_materials is not None else ds.n_materials
    grad = torch.empty(4 * n, dtype=torch.float64, device="cuda")
    ds.render_backward(cfg, local.data_ptr(), grad.data_ptr())
    return allreduce_gradient(grad, group)


# ---- batch renders: jobs sharded by scene (no counterpart in the reference) -----------------------
def shard_jobs(costs, world: int) -> list:
    """Assigns batch jobs to ``world`` ranks: longest job first, each to the
    least-loaded rank (ties to the lower rank) -- Graham's LPT rule, whose
    largest load is at most 4/3 of the best possible.  ``costs`` are the
    jobs' paths (film pixels x spp).  Returns, per rank, its job indices in
    ascending order; deterministic, so every rank computes the same split."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for j in sorted(range(len(costs)), key=lambda j: (-costs[j], j)):
        r = min(range(world), key=lambda r: (load[r], r))
        out[r].append(j)
        load[r] += costs[j]
    return [sorted(o) for o in out]


def job_costs(jobs) -> list:
    """Paths of each (scene index, RenderConfig) job."""
    return [c.film_pixels * c.spp for _, c in jobs]


def render_jobs(scenes, jobs, mine, tuning=None):
    """Renders the jobs ``mine`` (indices into ``jobs``, a list of (scene
    index, RenderConfig)) in one batch over just the scenes they use.
    Returns ({job: flat f64 CUDA tensor of 4 * pixels: acc rgb, then
    acc_w}, RenderStats or None when ``mine`` is empty)."""
    import torch

    from .render import BatchScenes

    if not mine:
        return {}, None
    used = sorted({jobs[j][0] for j in mine})
    slot = {s: k for k, s in enumerate(used)}
    films = {j: torch.empty(4 * jobs[j][1].film_pixels, dtype=torch.float64, device="cuda") for j in mine}
    batch = [(slot[jobs[j][0]], jobs[j][1], films[j].data_ptr(),
              films[j].data_ptr() + 8 * 3 * jobs[j][1].film_pixels) for j in mine]
    with BatchScenes([scenes[s] for s in used]) as bs:
        stats = bs.render(batch, tuning=tuning)
    return films, stats


def gather_job_films(local, assignment, sizes, group=None):
    """local: this rank's {job: flat tensor of sizes[job] values};
    assignment: shard_jobs' split.  One all-gather of per-rank buffers
    padded to the longest gives every rank {job: flat tensor} for all jobs
    (on the GPU under NCCL, on the host under gloo)."""
    import torch
    import torch.distributed as dist

    rank, world = _world(group)
    if world <= 1:
        return {j: t.reshape(-1) for j, t in local.items()}
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    n = max(1, max(sum(sizes[j] for j in a) for a in assignment))
    buf = torch.zeros(n, dtype=torch.float64, device=dev)
    off = 0
    for j in assignment[rank]:
        buf[off:off + sizes[j]] = local[j].reshape(-1).to(dev)
        off += sizes[j]
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = {}
    for r, a in enumerate(assignment):
        off = 0
        for j in a:
            out[j] = parts[r][off:off + sizes[j]]
            off += sizes[j]
    return out


def render_batch_sharded(scenes, jobs, group=None, tuning=None):
    """A batch of (scene index, RenderConfig) jobs over the ranks: each
    rank renders its shard_jobs share (scenes replicated only where a rank
    has jobs on them) and one all-gather assembles every film on every rank.
    Returns ([(acc (pixels, 3), acc_w (pixels,)) per job], this rank's
    RenderStats or None).  Every job's film equals its one-GPU render."""
    rank, world = _world(group)
    assignment = shard_jobs(job_costs(jobs), world)
    local, stats = render_jobs(scenes, jobs, assignment[rank], tuning)
    sizes = [4 * c.film_pixels for _, c in jobs]
    full = gather_job_films(local, assignment, sizes, group)
    films = []
    for j, (_, c) in enumerate(jobs):
        f = full[j]
        films.append((f[: 3 * c.film_pixels].view(-1, 3), f[3 * c.film_pixels:]))
    return films, stats
