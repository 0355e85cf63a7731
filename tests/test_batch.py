"""Batch renders: many scenes, films of uneven size and spp, one wavefront
loop.  Each job's film must equal the single-scene render of that scene and
config (the per-pixel RNG streams do not depend on the batch)."""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from tinypt_b200 import scenes


def small_workload():
    return scenes.batch_workload(5, seed=3, tri_range=(500, 30_000), res_range=(24, 80), spp_range=(4, 40),
                                 max_depth=8)


def test_batch_workload_is_seeded_and_in_range():
    a = scenes.batch_workload(4, seed=9, tri_range=(1_000, 50_000), res_range=(32, 128), spp_range=(16, 64))
    b = scenes.batch_workload(4, seed=9, tri_range=(1_000, 50_000), res_range=(32, 128), spp_range=(16, 64))
    for (sa, ca), (sb, cb) in zip(a, b):
        assert ca == cb
        assert [m.n_tris for m in sa.world.meshes] == [m.n_tris for m in sb.world.meshes]
        assert 32 <= ca.width <= 128 and ca.width == ca.height and ca.width % 8 == 0
        assert 16 <= ca.spp <= 64 and ca.max_bounces == 12
        lights = [m for m in sa.mats if m.emitted() is not None]
        assert len(lights) == 1 and 5.0 <= lights[0].rgb[0] <= 50.0


@pytest.mark.gpu
def test_batch_films_equal_single_renders(gpu, monkeypatch):
    """Each job's film equals tpt_render_device of its scene and config at
    the same task length (a batch's default is 8 samples per task; a single
    render picks its own unless TPT_TASK_SPP says), bit for bit."""
    import torch

    from tinypt_b200.render import BatchScenes, DeviceScene

    monkeypatch.setenv("TPT_TASK_SPP", "8")

    work = small_workload()
    jobs_cfg = [(k, cfg) for k, (_, cfg) in enumerate(work)]
    # a second job on scene 0 with another film size, seed and a row shard
    c0 = work[0][1]
    jobs_cfg.append((0, dataclasses.replace(c0, width=40, height=30, spp=20, seed=99, row_begin=1, row_step=2)))
    films = []
    for _, cfg in jobs_cfg:
        n = cfg.film_pixels
        films.append((torch.full((3 * n,), -1.0, dtype=torch.float64, device="cuda"),
                      torch.full((n,), -1.0, dtype=torch.float64, device="cuda")))
    with BatchScenes([s for s, _ in work]) as bs:
        st = bs.render([(k, cfg, a.data_ptr(), w.data_ptr()) for (k, cfg), (a, w) in zip(jobs_cfg, films)])
        assert st.device_flags == 0
        assert st.paths == sum(cfg.film_pixels * cfg.spp for _, cfg in jobs_cfg)
    for (k, cfg), (a, w) in zip(jobs_cfg, films):
        with DeviceScene(work[k][0]) as ds:
            n = cfg.film_pixels
            ra = torch.empty(3 * n, dtype=torch.float64, device="cuda")
            rw = torch.empty(n, dtype=torch.float64, device="cuda")
            ds.render_device(cfg, ra.data_ptr(), rw.data_ptr())
        assert torch.equal(w, rw), f"job on scene {k}: sample counts differ"
        assert torch.equal(a, ra), f"job on scene {k}: film differs"


@pytest.mark.gpu
@pytest.mark.parametrize("alone_paths", [1, 21_000])
def test_large_jobs_render_alone(gpu, monkeypatch, alone_paths):
    """Jobs of at least TPT_BATCH_ALONE_PATHS paths render one after another
    with the single render's schedule (its own task length, pool and shading
    variant) on the batch's merged arrays; the others share one loop. With
    no task length forced, every alone job's film equals tpt_render_device
    of its scene and config bit for bit. The threshold 21,000 sends three of
    the five jobs alone, 1 sends all five."""
    import torch

    from tinypt_b200.render import BatchScenes, DeviceScene

    monkeypatch.delenv("TPT_TASK_SPP", raising=False)
    monkeypatch.setenv("TPT_BATCH_ALONE_PATHS", str(alone_paths))
    work = small_workload()
    films = [(torch.full((3 * c.film_pixels,), -1.0, dtype=torch.float64, device="cuda"),
              torch.full((c.film_pixels,), -1.0, dtype=torch.float64, device="cuda")) for _, c in work]
    with BatchScenes([s for s, _ in work]) as bs:
        st = bs.render([(k, c, a.data_ptr(), w.data_ptr()) for k, ((_, c), (a, w)) in enumerate(zip(work, films))],
                       tuning=(0, 8, 0, 0))
    assert st.device_flags == 0
    assert st.paths == sum(c.film_pixels * c.spp for _, c in work)
    alone = [c.film_pixels * c.spp >= alone_paths for _, c in work]
    assert sum(alone) == (5 if alone_paths == 1 else 3)
    for k, ((s, c), (a, w)) in enumerate(zip(work, films)):
        with DeviceScene(s) as ds:
            ra = torch.empty(3 * c.film_pixels, dtype=torch.float64, device="cuda")
            rw = torch.empty(c.film_pixels, dtype=torch.float64, device="cuda")
            ds.render_device(c, ra.data_ptr(), rw.data_ptr())
        assert torch.equal(w, rw), f"job {k}: sample counts differ"
        if alone[k]:
            # (a job of the shared loop runs its 8-sample tasks; the single
            # render of so small a film picks 1-sample tasks)
            assert torch.equal(a, ra), f"job {k}: film differs"


@pytest.mark.gpu
def test_batch_culling_changes_no_film(gpu, monkeypatch):
    """Camera culling in a multi-job render works per job.

    * The batch's pixels are classified job by job, against each job's
      camera and top-level tree.
    * The pool fetches only the other pixels' tasks, job after job.
    * A coherent kernel renders the culled tasks.

    With culling on and off, every job's film and sample counts agree bit
    for bit. The batch scenes' black backgrounds leave open pixels, so
    something is culled. One job through a thin lens keeps all its pixels
    in the pool."""
    import torch

    from tinypt_b200.render import BatchScenes

    work = small_workload()
    jobs_cfg = [(k, cfg) for k, (_, cfg) in enumerate(work)]
    c0 = work[0][1]
    jobs_cfg.append((0, dataclasses.replace(c0, width=40, height=30, spp=20, seed=99, row_begin=1, row_step=2)))
    lens_scene = dataclasses.replace(work[1][0])
    cam = lens_scene.cam
    lens_scene.cam = scenes.Camera.look_at_dof(cam.eye, cam.target, cam.up, cam.fov_y_deg, cam.aspect, 6.0, 0.2)
    scenes_list = [s for s, _ in work] + [lens_scene]
    jobs_cfg.append((len(work), work[1][1]))

    def render(cull):
        monkeypatch.setenv("TPT_SKY_CULL", "1" if cull else "0")
        films = []
        for _, cfg in jobs_cfg:
            n = cfg.film_pixels
            films.append((torch.full((3 * n,), -1.0, dtype=torch.float64, device="cuda"),
                          torch.full((n,), -1.0, dtype=torch.float64, device="cuda")))
        with BatchScenes(scenes_list) as bs:
            st = bs.render([(k, cfg, a.data_ptr(), w.data_ptr()) for (k, cfg), (a, w) in zip(jobs_cfg, films)],
                           tuning=(0, 4, 0, 0))
        assert st.device_flags == 0
        return films, st

    on, st_on = render(True)
    off, st_off = render(False)
    print(f"batch: culled samples {st_on.sky_samples / st_on.paths:.3f} of {st_on.paths}")
    assert st_on.paths == st_off.paths == sum(cfg.film_pixels * cfg.spp for _, cfg in jobs_cfg)
    assert st_off.sky_samples == 0 < st_on.sky_samples
    lens_samples = work[1][1].film_pixels * work[1][1].spp
    assert st_on.sky_samples <= st_on.paths - lens_samples
    for (k, _), (a1, w1), (a0, w0) in zip(jobs_cfg, on, off):
        assert torch.equal(w1, w0), f"job on scene {k}: sample counts differ with culling"
        assert torch.equal(a1, a0), f"job on scene {k}: film differs with culling"


@pytest.mark.gpu
def test_batch_autotune(gpu):
    import torch

    from tinypt_b200.render import BatchScenes

    work = small_workload()
    films = [(torch.empty(3 * c.film_pixels, dtype=torch.float64, device="cuda"),
              torch.empty(c.film_pixels, dtype=torch.float64, device="cuda")) for _, c in work]
    jobs = [(k, c, a.data_ptr(), w.data_ptr()) for k, ((_, c), (a, w)) in enumerate(zip(work, films))]
    with BatchScenes([s for s, _ in work]) as bs:
        (pool, task_spp, chunk, ctas), trials = bs.autotune(jobs)
        assert pool >= 1 and task_spp in (4, 8, 16, 32) and chunk in (2, 4, 8, 16) and ctas in (4, 8)
        # warm-up + default, then each coordinate's other values, its starting
        # value skipped: 2 + at most 4 pools + 3 task lengths + 3 chunks + 1
        # shading variant
        assert 9 <= len(trials) <= 13 and all(t > 0 for t in trials)
        st = bs.render(jobs, tuning=(pool, task_spp, chunk, ctas))
        assert st.device_flags == 0
        assert st.paths == sum(c.film_pixels * c.spp for _, c in work)
        for (_, c), (_, w) in zip(work, films):
            assert torch.all(w == c.spp)


@pytest.mark.gpu
def test_batch_shading_variants_agree(gpu):
    """The batch shading kernel compiled for 4 and for 8 resident blocks per
    SM gives the same films bit for bit (the FP32 units are built without
    automatic FMA contraction)."""
    import torch

    from tinypt_b200.render import BatchScenes

    work = small_workload()
    out = []
    with BatchScenes([s for s, _ in work]) as bs:
        for ctas in (4, 8):
            films = [(torch.empty(3 * c.film_pixels, dtype=torch.float64, device="cuda"),
                      torch.empty(c.film_pixels, dtype=torch.float64, device="cuda")) for _, c in work]
            jobs = [(k, c, a.data_ptr(), w.data_ptr()) for k, ((_, c), (a, w)) in enumerate(zip(work, films))]
            st = bs.render(jobs, tuning=(0, 0, 0, ctas))
            assert st.device_flags == 0
            torch.cuda.synchronize()
            out.append([(a.cpu(), w.cpu()) for a, w in films])
    for (a4, w4), (a8, w8) in zip(out[0], out[1]):
        assert torch.equal(a4, a8) and torch.equal(w4, w8)
