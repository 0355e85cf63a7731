"""GPU parity: the f64 and FP32 kernels against the oracle, through the C ABI.

Bars (each test states its own):
  * plain f64 kernel -- same RNG stream, same f64 arithmetic; pixels match
    the oracle to 1e-9 relative except where a last-bit difference between
    CUDA's and glibc's transcendentals flips a branch and the stream diverges
    (a small fraction, bounded below);
  * FP32 wavefront -- same RNG stream at FP32 precision; per-pixel Welch test
    per channel against the oracle at equal seed/spp: at most 1% of
    pixel-channels beyond |z| > 4 (independent streams would give 0.006%),
    image-mean relative difference below 1%;
  * sample counts (acc_w) exact in both forms.
"""
import numpy as np
import pytest

from tinypt_b200 import _abi, scenes
from tinypt_b200.render import DeviceScene
from tests.parity_util import cfg, relative_rms, small_mesh_env_scene, welch_z

pytestmark = pytest.mark.gpu

PLAIN, WF = _abi.TPT_MODE_PLAIN_F64, _abi.TPT_MODE_WAVEFRONT_FP32


def gpu_render(ds: DeviceScene, c, want_sq=True):
    import torch

    n = c.width * c.height
    acc = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    acc_w = torch.zeros(n, dtype=torch.float64, device="cuda")
    acc_sq = torch.zeros(3 * n, dtype=torch.float64, device="cuda") if want_sq else None
    st = ds.render_device(c, acc.data_ptr(), acc_w.data_ptr(), acc_sq.data_ptr() if want_sq else 0)
    torch.cuda.synchronize()
    out = (acc.cpu().numpy().reshape(n, 3), acc_w.cpu().numpy(), acc_sq.cpu().numpy().reshape(n, 3) if want_sq else None)
    return out, st


def oracle_render(O, scene, c):
    with O.OracleScene(scene) as s:
        acc, w, sq, _ = s.render(c, want_sq=True)
    return acc, w, sq


SCENES = {
    "spheres": lambda: (scenes.sphere_scene(64, 48), 8, 8),
    "builtin_sky": lambda: (scenes.build_scene(64, 36), 8, 8),
    "mesh_env": lambda: (small_mesh_env_scene(), 4, 16),
}


@pytest.mark.parametrize("name", list(SCENES))
def test_plain_f64_matches_oracle(gpu, oracle_mod, name):
    scene, spp, depth = SCENES[name]()
    w_, h_ = _wh(scene)
    c = cfg(w_, h_, spp, depth, PLAIN)
    want = oracle_render(oracle_mod, scene, c)
    with DeviceScene(scene) as ds:
        (acc, w, sq), st = gpu_render(ds, c)
    assert np.array_equal(w, want[1])
    assert st.paths == c.width * c.height * spp
    rel = np.abs(acc - want[0]) / np.maximum(np.abs(want[0]), 1e-12)
    exact = np.all(rel <= 1e-9, axis=1)
    frac = float(exact.mean())
    print(f"{name}: {frac:.4f} of pixels within 1e-9, image rel rms {relative_rms(acc, want[0]):.2e}")
    assert frac >= 0.97, frac
    assert relative_rms(acc, want[0]) < 0.05


def _wh(scene):
    a = scene.cam.aspect
    # The test scenes are built at these sizes (aspect identifies them).
    for w, h in ((64, 48), (64, 36), (96, 54)):
        if abs(w / h - a) < 1e-12:
            return w, h
    raise AssertionError("unknown test scene size")


@pytest.mark.parametrize("name", list(SCENES))
def test_wavefront_fp32_welch_vs_oracle(gpu, oracle_mod, name, monkeypatch):
    # One task per pixel: the FP32 form then draws each pixel's reference
    # stream, like the oracle, and the two images differ only where an FP32
    # decision flips a path -- so the image means agree far inside 1%, not
    # just within the Monte Carlo noise of two independent renders.
    scene, spp, depth = SCENES[name]()
    spp = 32
    monkeypatch.setenv("TPT_TASK_SPP", str(spp))
    w_, h_ = _wh(scene)
    c_o = cfg(w_, h_, spp, depth, PLAIN)
    want = oracle_render(oracle_mod, scene, c_o)
    with DeviceScene(scene) as ds:
        (acc, w, sq), st = gpu_render(ds, cfg(w_, h_, spp, depth, WF))
    assert np.all(w == spp)
    assert st.paths == w_ * h_ * spp
    z = welch_z(acc, sq, w, want[0], want[2], want[1])
    frac = float(np.mean(np.abs(z) > 4.0))
    mean_rel = abs(acc.sum() - want[0].sum()) / max(abs(want[0].sum()), 1e-30)
    print(f"{name}: |z|>4 fraction {frac:.5f}, image-mean rel diff {mean_rel:.2e}")
    assert frac <= 0.01, frac
    assert mean_rel < 0.01, mean_rel


def test_wavefront_is_deterministic(gpu):
    scene = scenes.sphere_scene(64, 48)
    c = cfg(64, 48, 16, 8, WF)
    with DeviceScene(scene) as ds:
        a, _ = gpu_render(ds, c)
        b, _ = gpu_render(ds, c)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_shading_kernel_variants_agree(gpu, monkeypatch):
    """The shading kernel is compiled for 8 and for 4 resident blocks per SM
    (single renders pick by render kind): the FP32 units are built without
    automatic FMA contraction, so both give the same film bit for bit."""
    scene = scenes.mesh_env_scene(64, 48, subdiv=4, n_spheres=30, env_w=64, env_h=32)
    c = cfg(64, 48, 16, 8, WF)
    films = []
    with DeviceScene(scene) as ds:
        for ctas in ("8", "4"):
            monkeypatch.setenv("TPT_SHADE_CTAS", ctas)
            films.append(gpu_render(ds, c)[0])
    assert np.array_equal(films[0][0], films[1][0]) and np.array_equal(films[0][1], films[1][1])


def test_camera_miss_fast_path_gives_the_same_film(gpu, monkeypatch):
    """Camera rays that leave the scene finish inside the closest-hit kernel
    (TPT_CAMERA_FAST=1, the default) with the same arithmetic and draws as
    the shading kernel's path (=0): same film, counts and second moments."""
    scene = small_mesh_env_scene()
    c = cfg(96, 54, 24, 16, WF)
    monkeypatch.setenv("TPT_TASK_SPP", "8")
    out = []
    with DeviceScene(scene) as ds:
        for fast in ("1", "0"):
            monkeypatch.setenv("TPT_CAMERA_FAST", fast)
            film, st = gpu_render(ds, c)
            assert st.paths == c.width * c.height * c.spp
            out.append(film)
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_chunk_batches_give_the_same_film(gpu, monkeypatch):
    """A render whose per-task sums exceed TPT_MAX_PART_TASKS runs its sample
    chunks in batches and merges each onto the film in task order: the film,
    its sample counts and second moments equal the one-batch render bit for
    bit (3 chunks of 8 samples: batches of 1 and of 2 chunks)."""
    scene = scenes.mesh_env_scene(48, 32, subdiv=4, n_spheres=20, env_w=64, env_h=32)
    c = cfg(48, 32, 24, 8, WF)
    n = c.width * c.height
    monkeypatch.setenv("TPT_TASK_SPP", "8")
    out = []
    with DeviceScene(scene) as ds:
        for limit in (None, n, 2 * n):
            if limit is None:
                monkeypatch.delenv("TPT_MAX_PART_TASKS", raising=False)
            else:
                monkeypatch.setenv("TPT_MAX_PART_TASKS", str(limit))
            film, st = gpu_render(ds, c)
            assert st.paths == n * c.spp and st.device_flags == 0
            out.append(film)
    for film in out[1:]:
        for a, b in zip(film, out[0]):
            assert np.array_equal(a, b)


def test_host_and_device_outputs_agree(gpu):
    scene = scenes.sphere_scene(64, 48)
    for mode in (PLAIN, WF):
        c = cfg(64, 48, 4, 8, mode)
        with DeviceScene(scene) as ds:
            (acc, w, _), _ = gpu_render(ds, c, want_sq=False)
            host = ds.render(c)
        assert np.array_equal(host.acc, acc) and np.array_equal(host.acc_w, w)


def test_plain_adaptive_matches_oracle(gpu, oracle_mod):
    scene = scenes.sphere_scene(64, 48)
    c = cfg(64, 48, 64, 8, PLAIN, adaptive_enabled=True, adaptive_min_spp=8, adaptive_threshold=0.5)
    want = oracle_render(oracle_mod, scene, c)
    with DeviceScene(scene) as ds:
        (acc, w, _), _ = gpu_render(ds, c)
    same_w = float(np.mean(w == want[1]))
    assert 8 <= w.min() and w.max() <= 64
    assert same_w >= 0.97, same_w


def test_wavefront_adaptive_stops_between_bounds(gpu, oracle_mod):
    scene = scenes.sphere_scene(64, 48)
    c = cfg(64, 48, 64, 8, WF, adaptive_enabled=True, adaptive_min_spp=8, adaptive_threshold=0.5)
    want = oracle_render(oracle_mod, scene, cfg(64, 48, 64, 8, PLAIN, adaptive_enabled=True, adaptive_min_spp=8,
                                                 adaptive_threshold=0.5))
    with DeviceScene(scene) as ds:
        (acc, w, _), st = gpu_render(ds, c)
    assert 8 <= w.min() and w.max() <= 64
    assert st.paths == int(w.sum())
    # average sample count within 5% of the reference's
    assert abs(w.mean() - want[1].mean()) / want[1].mean() < 0.05


def test_empty_scene_weights(gpu):
    """render.rs:335-364 on the GPU: an empty 2x2 scene gives acc_w == spp."""
    from tinypt_b200.scene import Camera, Scene, World

    scene = Scene(Camera.look_at((0.0, 0.0, 1.5), (0, 0, 0), (0, 1, 0), 45.0, 1.0), World(), [], None)
    for mode in (PLAIN, WF):
        c = cfg(2, 2, 1, 8, mode, seed=0)
        c.tile = 1
        with DeviceScene(scene) as ds:
            out = ds.render(c)
        assert np.all(out.acc_w == 1) and np.all(np.isfinite(out.acc))


def test_full_size_mesh_env_properties(gpu):
    """The 1920x1080 / 1.31M-triangle workload at 1 spp: size-independent
    properties (every pixel one sample, finite non-negative radiance, both
    forms agree on the image mean within noise)."""
    scene = scenes.mesh_env_scene()
    assert scene.n_triangles() == 1_310_720 and len(scene.world.spheres) == 200
    with DeviceScene(scene) as ds:
        outs = {}
        for mode in (PLAIN, WF):
            c = cfg(1920, 1080, 1, 16, mode)
            (acc, w, _), st = gpu_render(ds, c, want_sq=False)
            assert np.all(w == 1)
            assert np.all(np.isfinite(acc)) and acc.min() >= 0.0
            assert st.paths == 1920 * 1080
            outs[mode] = acc
    m_plain, m_wf = outs[PLAIN].mean(), outs[WF].mean()
    assert abs(m_plain - m_wf) / m_plain < 0.02


# ---- precision against the 65536-spp f64 ground truth (240x135 mesh+env) -----
@pytest.mark.gpu
def test_precision_vs_ground_truth(gpu):
    """The FP32 wavefront form converges to the f64 ground truth: at 4096 spp
    its relative RMSE is small and its image mean matches; at 256 spp its
    error is comparable to the plain f64 form's at the same spp."""
    import torch

    from tinypt_b200 import precision, scenes
    from tinypt_b200.scene import RenderConfig

    truth, meta = precision.load_truth()
    assert meta["spp"] == 65536
    w, h = precision.TRUTH_WIDTH, precision.TRUTH_HEIGHT
    n = w * h
    acc = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    acc_w = torch.zeros(n, dtype=torch.float64, device="cuda")
    with DeviceScene(scenes.mesh_env_scene(w, h)) as ds:
        def err(mode, spp, seed):
            cfg = RenderConfig(width=w, height=h, spp=spp, max_bounces=16, rr_start=3, seed=seed, mode=mode)
            st = ds.render_device(cfg, acc.data_ptr(), acc_w.data_ptr())
            assert st.device_flags == 0
            img = (acc.view(n, 3) / acc_w.clamp(min=1.0)[:, None]).cpu().numpy()
            return precision.image_error(img, truth), img

        e_hi, img_hi = err(_abi.TPT_MODE_WAVEFRONT_FP32, 4096, 41)
        mean_rel = abs(img_hi.mean() - truth.mean()) / truth.mean()
        print(f"wavefront 4096 spp: rel_rmse {e_hi['rel_rmse']:.4f}, mean_rel_err {e_hi['mean_rel_err']:.4f}, "
              f"image-mean diff {mean_rel:.2e}")
        assert e_hi["rel_rmse"] < 0.04
        assert mean_rel < 5e-3
        mse_wf = np.mean([err(_abi.TPT_MODE_WAVEFRONT_FP32, 256, s)[0]["mse"] for s in (51, 52, 53, 54)])
        mse_pl = np.mean([err(_abi.TPT_MODE_PLAIN_F64, 256, s)[0]["mse"] for s in (61, 62, 63, 64)])
        print(f"256 spp MSE: wavefront {mse_wf:.3e}, plain {mse_pl:.3e}")
        assert mse_wf < 2.0 * mse_pl


# ---- adaptive sampling on the Cornell scene against its 65536-spp f64 ground truth ------------
@pytest.mark.gpu
def test_cornell_adaptive_vs_ground_truth(gpu):
    """The adaptive FP32 render (rel. sample std < 0.01 after 8, at most 1024
    spp) of the 160x90 Cornell film: every pixel between 8 and 1024 samples,
    black background pixels stop at 8.  The reference's rule also stops any
    pixel whose first 8 samples are equal -- all zero in a dim corner, or
    the light seen directly -- so those pixels are exact or 0 by design.
    Against the f64 ground truth, the other pixels' means are within their
    own standard errors (|z| > 4 on at most 5% of pixel-channels: the glass
    sphere's caustics make the tail heavy) and the image mean within 2%."""
    import dataclasses

    import torch

    from tinypt_b200 import precision

    truth, meta = precision.load_truth(precision.CORNELL_TRUTH_FILE)
    assert meta["spp"] == 65536 and meta["max_bounces"] == 32
    w, h = precision.CORNELL_WIDTH, precision.CORNELL_HEIGHT
    cfg = dataclasses.replace(scenes.cornell_config(w, h, spp=1024), seed=11)
    with DeviceScene(scenes.cornell_scene(w, h)) as ds:
        n = w * h
        acc = torch.empty(3 * n, dtype=torch.float64, device="cuda")
        aw = torch.empty(n, dtype=torch.float64, device="cuda")
        asq = torch.empty(3 * n, dtype=torch.float64, device="cuda")
        st = ds.render_device(cfg, acc.data_ptr(), aw.data_ptr(), asq.data_ptr())
        assert st.device_flags == 0
        spp = aw.cpu().numpy()
        s1 = acc.view(n, 3).cpu().numpy()
        s2 = asq.view(n, 3).cpu().numpy()
    assert spp.min() >= 8 and spp.max() <= 1024
    dark = truth.max(axis=1) == 0.0
    assert dark.any() and np.all(spp[dark] == 8)
    nn = spp[:, None]
    mean = s1 / nn
    var = np.maximum(s2 - s1 * s1 / nn, 0.0) / np.maximum(nn - 1.0, 1.0)
    se = np.sqrt(var / nn)
    live = se > 0
    z = np.abs(mean - truth)[live] / se[live]
    frac = float((z > 4.0).mean())
    mean_rel = abs(mean.mean() - truth.mean()) / truth.mean()
    e = precision.image_error(mean, truth)
    zero_stop = (spp == 8) & (mean.max(axis=1) == 0.0) & ~dark
    print(f"cornell adaptive 1024: mean spp {spp.mean():.1f}, |z|>4 fraction {frac:.4f}, rel_rmse {e['rel_rmse']:.4f}, "
          f"image-mean diff {mean_rel:.2e}, pixels stopped on 8 zero samples {int(zero_stop.sum())}")
    assert frac < 0.05
    assert mean_rel < 0.02
    # zero-variance pixels saw 8 equal samples: black, or the light's emission
    const = ~live.any(axis=1)
    emit = np.array([17.0, 12.0, 4.0])
    ok = (mean.max(axis=1) == 0.0) | np.isclose(mean, emit[None, :], rtol=1e-6).all(axis=1)
    assert np.all(ok[const])
