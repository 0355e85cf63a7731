"""Edge cases of the FP32 wavefront's camera culling and drain handover.

* A scene with no geometry has every pixel culled, so no task reaches the
  path pool. The film must still be the reference's: every sample sees
  the sky (src/integrator.rs:71-83). The test compares it with the oracle
  and with the render that has culling and the handover off.
* max_bounces = 0 makes radiance() return 0 for every sample
  (src/integrator.rs:67), so nothing is culled and the film is black.
* 1x1 films, spp below the task length and an odd spp give the same film
  with culling and the handover on and off.
"""
import numpy as np
import pytest

from tinypt_b200 import _abi, scenes
from tinypt_b200.render import DeviceScene
from tinypt_b200.scene import Camera, Scene, World
from tests.parity_util import cfg, small_mesh_env_scene

pytestmark = pytest.mark.gpu

WF = _abi.TPT_MODE_WAVEFRONT_FP32
PLAIN = _abi.TPT_MODE_PLAIN_F64


@pytest.fixture(autouse=True)
def default_schedule(monkeypatch):
    for k in ("TPT_TASK_SPP", "TPT_POOL", "TPT_CAMERA_FAST", "TPT_SHADE_CTAS", "TPT_MAX_PART_TASKS",
              "TPT_WAVEFRONT_HOST_LOOP", "TPT_QUEUE_ORDER", "TPT_QUEUE_DIV", "TPT_SKY_CULL", "TPT_TAIL_SLOTS"):
        monkeypatch.delenv(k, raising=False)


def _film(ds, c, monkeypatch, cull=True, tail=None):
    import torch

    monkeypatch.setenv("TPT_SKY_CULL", "1" if cull else "0")
    if tail is None:
        monkeypatch.delenv("TPT_TAIL_SLOTS", raising=False)
    else:
        monkeypatch.setenv("TPT_TAIL_SLOTS", str(tail))
    n = c.film_pixels
    acc = torch.full((3 * n,), -1.0, dtype=torch.float64, device="cuda")
    acc_w = torch.full((n,), -1.0, dtype=torch.float64, device="cuda")
    st = ds.render_device(c, acc.data_ptr(), acc_w.data_ptr())
    torch.cuda.synchronize()
    return acc.cpu().numpy().reshape(n, 3), acc_w.cpu().numpy(), st


def _same_all_ways(ds, c, monkeypatch):
    ref = _film(ds, c, monkeypatch, cull=False, tail=0)
    for cull, tail in ((True, None), (True, 1 << 30), (False, 1 << 30)):
        got = _film(ds, c, monkeypatch, cull, tail)
        assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1]), (cull, tail)
        assert got[2].paths == ref[2].paths
    return ref


@pytest.mark.parametrize("env", [False, True])
def test_empty_scene_is_all_sky(gpu, oracle_mod, monkeypatch, env):
    """No geometry: every pixel is culled (no pool task at all); the film
    is the sky's, the oracle's within FP32 rounding of the camera rays."""
    w, h, spp = 24, 16, 8
    sky = scenes.sky_env(32, 16, 3) if env else None
    scene = Scene(Camera.look_at((0.0, 0.3, 2.0), (0, 0, 0), (0, 1, 0), 50.0, w / h), World(), [], sky)
    c = cfg(w, h, spp, 8, WF)
    with DeviceScene(scene) as ds:
        acc, acc_w, st = _same_all_ways(ds, c, monkeypatch)
        _, _, st_on = _film(ds, c, monkeypatch)
    assert st_on.sky_samples == st_on.paths == w * h * spp
    assert np.all(acc_w == spp)
    with oracle_mod.OracleScene(scene) as o:
        o_acc, o_w, _, _ = o.render(cfg(w, h, spp, 8, PLAIN), want_sq=True, sample_chunk=st_on.task_spp)
    assert np.array_equal(o_w, acc_w)
    mean, o_mean = acc / acc_w[:, None], o_acc / o_w[:, None]
    rel = np.abs(mean - o_mean) / np.maximum(np.abs(o_mean), 1e-6)
    print(f"empty scene (env {env}): max relative difference to the oracle {rel.max():.2e}")
    assert rel.max() < (1e-4 if env else 1e-6)  # measured 2.1e-6 / 4.2e-8


def test_zero_bounces_is_black(gpu, monkeypatch):
    """max_bounces = 0: radiance() returns 0 before any ray (integrator.rs:67),
    so no pixel is culled and the film is black with spp samples each."""
    scene = small_mesh_env_scene(32, 18)
    c = cfg(32, 18, 4, 0, WF)
    with DeviceScene(scene) as ds:
        acc, acc_w, _ = _same_all_ways(ds, c, monkeypatch)
        _, _, st = _film(ds, c, monkeypatch)
    assert st.sky_samples == 0
    assert np.all(acc == 0.0) and np.all(acc_w == 4)


@pytest.mark.parametrize("w,h,spp,task", [(1, 1, 5, None), (1, 1, 16, 8), (7, 3, 3, 8), (33, 17, 13, 4)])
def test_small_films_and_odd_counts(gpu, monkeypatch, w, h, spp, task):
    """A 1x1 film, spp below the task length, an odd spp: the same film with
    culling and the handover on and off, spp samples in every pixel."""
    if task is not None:
        monkeypatch.setenv("TPT_TASK_SPP", str(task))
    scene = small_mesh_env_scene(w, h)
    c = cfg(w, h, spp, 8, WF)
    with DeviceScene(scene) as ds:
        _, acc_w, _ = _same_all_ways(ds, c, monkeypatch)
    assert np.all(acc_w == spp)
