"""The oracle's sample-chunked task schedule and an analytic known answer.

The FP32 wavefront form cuts each pixel's samples into tasks of 8, each a
reference Task { sample_start, sample_end } seeded from
seed_for(x, y, sample_start) ^ seed (src/render.rs:142, src/task.rs:11-27)
and merged in task order (src/render.rs:226-241).  The oracle renders the
same schedule (``OracleScene.render(..., sample_chunk=k)``) so the GPU
parity tests can compare that schedule with it; these tests pin the
oracle's schedule to per-sample calls of the oracle's own integrator.

The furnace test is a known answer the reference's arithmetic implies: a
convex Lambert sphere of albedo 1 under a constant environment, with Russian
roulette off, has every pixel's expected radiance equal to the environment's.
"""
import math

import numpy as np

from tinypt_b200 import _abi, scenes
from tinypt_b200.scene import Camera, EnvMap, Material, RenderConfig, Scene, Sphere, World

PLAIN = _abi.TPT_MODE_PLAIN_F64


def _cfg(w, h, spp, depth=8, seed=1, rr=3):
    return RenderConfig(width=w, height=h, spp=spp, max_bounces=depth, rr_start=rr, seed=seed, mode=PLAIN)


def test_chunk_as_long_as_spp_is_the_reference_schedule(oracle_mod):
    scene = scenes.sphere_scene(24, 16)
    c = _cfg(24, 16, 12)
    with oracle_mod.OracleScene(scene) as o:
        a = o.render(c, want_sq=True)
        for k in (12, 50):
            b = o.render(c, want_sq=True, sample_chunk=k)
            assert all(np.array_equal(x, y) for x, y in zip(a[:3], b[:3]))


def test_chunked_film_does_not_depend_on_threads(oracle_mod):
    scene = scenes.sphere_scene(24, 16)
    c = _cfg(24, 16, 20)
    with oracle_mod.OracleScene(scene) as o:
        a = o.render(c, want_sq=True, sample_chunk=8, threads=1)
        b = o.render(c, want_sq=True, sample_chunk=8, threads=7)
    assert all(np.array_equal(x, y) for x, y in zip(a[:3], b[:3]))
    assert np.all(a[1] == 20)


def test_chunked_pixels_are_task_sums_in_task_order(oracle_mod):
    """A pixel of a 20-spp render in 8-sample tasks is
    ((0 + sum of samples 0..7) + sum of 8..15) + sum of 16..19, each task's
    samples drawn from Rng::new(seed_for(x, y, sample_start) ^ seed) and
    summed from zero in sample order (render.rs:142-191, 226-241)."""
    scene = scenes.sphere_scene(24, 16)
    c = _cfg(24, 16, 20, seed=5)
    with oracle_mod.OracleScene(scene) as o:
        acc, acc_w, _, _ = o.render(c, sample_chunk=8)
    for x, y in ((0, 0), (11, 9), (23, 15), (5, 12)):
        film = np.zeros(3)
        for start, end in ((0, 8), (8, 16), (16, 20)):
            state = oracle_mod.seed_for(x, y, start) ^ c.seed
            task = np.zeros(3)
            for _ in range(start, end):
                rgb, state = oracle_mod.radiance_sample(scene, c, x, y, state)
                task = task + rgb
            film = film + task
        i = y * c.width + x
        assert np.array_equal(acc[i], film), (x, y)
        assert acc_w[i] == 20


def test_first_chunk_is_the_reference_stream(oracle_mod):
    """Chunk 0 of every pixel starts the reference's own per-pixel stream:
    an 8-spp film equals the first task of the chunked render."""
    scene = scenes.sphere_scene(24, 16)
    with oracle_mod.OracleScene(scene) as o:
        full8, _, _, _ = o.render(_cfg(24, 16, 8, seed=3))
        one_task, _, _, _ = o.render(_cfg(24, 16, 8, seed=3), sample_chunk=8)
    assert np.array_equal(full8, one_task)


def furnace_scene(w=32, h=32, env=(0.25, 0.5, 0.75), kind="lambert"):
    """A unit sphere of albedo 1 filling part of the view under a constant
    environment.  Lambert: white furnace; Metal albedo 1: a perfect mirror."""
    mat = Material.lambert((1.0, 1.0, 1.0)) if kind == "lambert" else Material.metal((1.0, 1.0, 1.0))
    cam = Camera.look_at((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 40.0, w / h)
    return Scene(cam, World(spheres=[Sphere((0.0, 0.0, 0.0), 1.0, 0)]), [mat], EnvMap.constant(env))


def test_white_furnace_returns_the_environment(oracle_mod):
    """Convex albedo-1 Lambert sphere, constant env (0.25, 0.5, 0.75), RR
    off: env NEE + BSDF sampling with the power heuristic (integrator.rs:
    108-121, 148-172) is unbiased, so every pixel's mean is the env value.
    The image mean over 32x32 pixels x 256 spp is within 5 standard errors
    of it; pixels that miss the sphere are exactly the env value."""
    env = np.array([0.25, 0.5, 0.75])
    c = _cfg(32, 32, 256, depth=4, rr=1000)
    with oracle_mod.OracleScene(furnace_scene(env=tuple(env))) as o:
        acc, w, sq, _ = o.render(c, want_sq=True)
    mean_px = acc / w[:, None]
    var_px = np.maximum(sq / w[:, None] - mean_px * mean_px, 0.0)
    miss = np.all(var_px == 0.0, axis=1)
    assert miss.any() and (~miss).any()
    assert np.all(mean_px[miss] == env)
    n = w.sum()
    mean = acc.sum(axis=0) / n
    se = np.sqrt(var_px.sum(axis=0) * w[0] / n / n)
    z = (mean - env) / se
    print(f"furnace mean {mean}, z {z}")
    assert np.all(np.abs(z) < 5.0), z


def test_mirror_furnace_is_exact(oracle_mod):
    """A Metal sphere of albedo 1 reflects every camera ray once into the
    constant env: each sample is the env value (weight 1, integrator.rs:
    123-130), so the film is exact."""
    env = (0.25, 0.5, 0.75)
    c = _cfg(24, 24, 16, depth=4, rr=1000)
    with oracle_mod.OracleScene(furnace_scene(24, 24, env, kind="metal")) as o:
        acc, w, _, _ = o.render(c)
    assert np.allclose(acc / w[:, None], np.array(env)[None, :], rtol=1e-12, atol=0)


# ---- per-pixel loop with task-boundary streams (the adaptive rounds' schedule) ----------------
def test_reseed_beyond_spp_is_the_reference_stream(oracle_mod):
    scene = scenes.sphere_scene(24, 16)
    c = _cfg(24, 16, 12)
    with oracle_mod.OracleScene(scene) as o:
        a = o.render(c, want_sq=True)
        b = o.render(c, want_sq=True, reseed=64)
    assert all(np.array_equal(x, y) for x, y in zip(a[:3], b[:3]))


def _pixel_samples(O, scene, c, x, y, n, reseed):
    out, state = [], None
    for s in range(n):
        if s % reseed == 0:
            state = O.seed_for(x, y, s) ^ c.seed
        rgb, state = O.radiance_sample(scene, c, x, y, state)
        out.append(rgb)
    return out


def test_reseeded_pixels_sum_in_sample_order(oracle_mod):
    """reseed=8, 20 spp: one loop over the pixel's samples (c = c + sample,
    render.rs:181-191) whose RNG restarts at samples 0, 8 and 16."""
    scene = scenes.sphere_scene(24, 16)
    c = _cfg(24, 16, 20, seed=4)
    with oracle_mod.OracleScene(scene) as o:
        acc, acc_w, _, _ = o.render(c, reseed=8)
    for x, y in ((0, 0), (11, 9), (23, 15)):
        film = np.zeros(3)
        for rgb in _pixel_samples(oracle_mod, scene, c, x, y, 20, 8):
            film = film + rgb
        i = y * c.width + x
        assert np.array_equal(acc[i], film) and acc_w[i] == 20


def test_reseeded_adaptive_stops_where_the_rule_says(oracle_mod):
    """Adaptive, reseed=8: each pixel's sample count is where the reference's
    rule (render.rs:143-180: Welford on luminance, stop after min_spp when
    sqrt(m2/(n-1))/max(|mean|, 1e-4) < threshold) stops on its sample
    sequence, and its sum is the sum of those samples in order."""
    scene = scenes.sphere_scene(24, 16)
    c = _cfg(24, 16, 48, seed=6)
    c.adaptive_enabled, c.adaptive_min_spp, c.adaptive_threshold = True, 8, 0.5
    with oracle_mod.OracleScene(scene) as o:
        acc, acc_w, _, _ = o.render(c, reseed=8)
    assert 8 <= acc_w.min() and acc_w.max() <= 48 and len(set(acc_w.tolist())) > 2
    for x, y in ((0, 0), (11, 9), (23, 15), (7, 3), (16, 12)):
        film, n, mean, m2 = np.zeros(3), 0, 0.0, 0.0
        for rgb in _pixel_samples(oracle_mod, scene, c, x, y, 48, 8):
            film = film + rgb
            n += 1
            lum = 0.2126 * rgb[0] + 0.7152 * rgb[1] + 0.0722 * rgb[2]
            delta = lum - mean
            mean += delta / n
            m2 += delta * (lum - mean)
            if n >= 8:
                var = m2 / (n - 1) if n > 1 else float("inf")
                if math.sqrt(var) / max(abs(mean), 1e-4) < 0.5:
                    break
        i = y * c.width + x
        assert acc_w[i] == n, (x, y)
        assert np.array_equal(acc[i], film), (x, y)
