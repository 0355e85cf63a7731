"""Camera culling of the FP32 wavefront form.

Some film pixels send every camera ray out of the scene. The test for this
is a conservative f64 frustum test of the pixel's footprint against the
top-level tree's leaf boxes, with margins above the FP32 error of the camera
rays and of the slab tests. Such pixels are rendered by a coherent kernel
that draws their samples exactly as the path pool would:

* the same streams (src/render.rs:142-158);
* the same camera rays (src/ray.rs:91-108);
* the same background lookups at bounce 0 (src/integrator.rs:71-83);
* the same f64 sums in sample order.

So the film with culling on (the default) equals the film with
TPT_SKY_CULL=0 bit for bit. The tests check this on the following:

* scenes with an env map, with the sky gradient and with instances,
  including a scene whose top-level tree is a single instance leaf;
* a far, narrow camera, which has the largest FP32 direction error per pixel;
* the 1080p benchmark frame at full size;
* row shards, chunk batches, one-task-per-pixel schedules and the host-driven
  loop.
"""
import numpy as np
import pytest

from tinypt_b200 import _abi, scenes
from tinypt_b200.render import DeviceScene
from tinypt_b200.scene import Camera
from tests.parity_util import cfg, small_mesh_env_scene

pytestmark = pytest.mark.gpu

WF = _abi.TPT_MODE_WAVEFRONT_FP32


@pytest.fixture(autouse=True)
def default_schedule(monkeypatch):
    for k in ("TPT_TASK_SPP", "TPT_POOL", "TPT_CAMERA_FAST", "TPT_SHADE_CTAS", "TPT_MAX_PART_TASKS",
              "TPT_WAVEFRONT_HOST_LOOP", "TPT_QUEUE_ORDER", "TPT_QUEUE_DIV", "TPT_SKY_CULL", "TPT_TAIL_SLOTS"):
        monkeypatch.delenv(k, raising=False)


def _film(ds, c, monkeypatch, cull):
    import torch

    monkeypatch.setenv("TPT_SKY_CULL", "1" if cull else "0")
    n = c.film_pixels
    acc = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    acc_w = torch.zeros(n, dtype=torch.float64, device="cuda")
    acc_sq = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    st = ds.render_device(c, acc.data_ptr(), acc_w.data_ptr(), acc_sq.data_ptr())
    torch.cuda.synchronize()
    return (acc.cpu().numpy(), acc_w.cpu().numpy(), acc_sq.cpu().numpy()), st


def _same_film(ds, c, monkeypatch, what):
    on, st_on = _film(ds, c, monkeypatch, True)
    off, st_off = _film(ds, c, monkeypatch, False)
    share = st_on.sky_samples / max(st_on.paths, 1)
    print(f"{what}: culled samples {share:.3f} of {st_on.paths}")
    for a, b, name in zip(on, off, ("acc", "acc_w", "acc_sq")):
        assert np.array_equal(a, b), f"{what}: {name} differs with culling"
    assert st_on.paths == st_off.paths == c.film_pixels * c.spp
    assert st_off.sky_samples == 0
    return share


def _far_camera_scene(w, h):
    s = small_mesh_env_scene(w, h)
    s.cam = Camera.look_at((3.0, 40.0, 400.0), (0.0, 0.4, 0.0), (0.0, 1.0, 0.0), 1.6, w / h)
    return s


SCENES = {
    "mesh_env": lambda: (small_mesh_env_scene(96, 54), 96, 54, 16, 0.2),
    "builtin_sky": lambda: (scenes.build_scene(64, 36), 64, 36, 8, 0.0),
    "spheres": lambda: (scenes.sphere_scene(64, 48), 64, 48, 8, 0.0),
    "far_camera": lambda: (_far_camera_scene(96, 54), 96, 54, 8, 0.2),
    # one mesh instance and nothing else: the top-level root is a leaf
    "one_instance": lambda: (scenes.inverse_scene(96, 96, nx=32, nz=64, env_w=64, env_h=32), 96, 96, 8, 0.1),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_culled_film_equals_traced_film(gpu, monkeypatch, name):
    """Culling changes no bit of the film, its weights or its second
    moments. It takes the expected share of samples where the scene leaves
    sky in view."""
    scene, w, h, spp, min_share = SCENES[name]()
    with DeviceScene(scene) as ds:
        share = _same_film(ds, cfg(w, h, spp, 8, WF), monkeypatch, name)
    assert share >= min_share


@pytest.mark.parametrize("schedule", ["one_task", "task8", "long_tasks", "chunk_batches", "row_shard", "host_loop"])
def test_culling_under_every_schedule(gpu, monkeypatch, schedule):
    """The same equality under each schedule:

    * one task per pixel (the reference's streams; the film written directly);
    * 8-sample tasks;
    * 48-sample tasks;
    * chunk batches (TPT_MAX_PART_TASKS: several pool drains, each merged in
      task order);
    * a row shard (rows 1, 4, 7, ...);
    * the host-driven loop.
    """
    scene = small_mesh_env_scene(96, 54)
    c = cfg(96, 54, 16, 8, WF)
    if schedule == "one_task":
        monkeypatch.setenv("TPT_TASK_SPP", "16")
    elif schedule == "task8":
        monkeypatch.setenv("TPT_TASK_SPP", "8")
    elif schedule == "long_tasks":
        c = cfg(96, 54, 96, 8, WF)
        monkeypatch.setenv("TPT_TASK_SPP", "48")
    elif schedule == "chunk_batches":
        monkeypatch.setenv("TPT_TASK_SPP", "4")
        monkeypatch.setenv("TPT_MAX_PART_TASKS", str(96 * 54))
    elif schedule == "row_shard":
        c = cfg(96, 54, 16, 8, WF, row_begin=1, row_step=3)
    else:
        monkeypatch.setenv("TPT_WAVEFRONT_HOST_LOOP", "1")
    with DeviceScene(scene) as ds:
        share = _same_film(ds, c, monkeypatch, schedule)
    assert share >= 0.2


def test_culling_on_the_benchmark_frame(gpu, monkeypatch):
    """The 1080p benchmark scene: 1,310,720 triangles, 200 spheres and a
    1024x512 env. It is rendered at full size, 2 spp, depth 16. Every
    culled pixel's samples equal the traced ones. Over a third of the
    frame's samples are culled."""
    scene = scenes.mesh_env_scene(1920, 1080)
    c = cfg(1920, 1080, 2, 16, WF)
    with DeviceScene(scene) as ds:
        share = _same_film(ds, c, monkeypatch, "mesh_env 1080p")
    assert share >= 0.35


def test_no_culling_through_a_lens(gpu, monkeypatch):
    """A thin-lens camera moves the ray origin over the lens. The pinhole
    frustum would not bound its rays, so no pixel is culled."""
    w, h = 64, 48
    s = scenes.sphere_scene(w, h)
    s.cam = Camera.look_at_dof((0.0, 1.2, 4.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 40.0, w / h, 4.0, 0.3)
    with DeviceScene(s) as ds:
        _, st = _film(ds, cfg(w, h, 4, 8, WF), monkeypatch, True)
    assert st.sky_samples == 0 and st.paths == w * h * 4


def test_kernel_launch_count(gpu, monkeypatch):
    """tpt_stats.kernel_launches counts the following launches:

    * 8 per iteration of the bounce loop: trace, shade, shadow trace,
      completion, three compaction kernels and the loop step;
    * the pool start;
    * the merge of the task sums;
    * with culling, the classification and its compactions (7) and the
      sky kernel;
    * with the drain's handover, the tail kernel.
    """
    scene = small_mesh_env_scene(96, 54)
    c = cfg(96, 54, 16, 8, WF)
    monkeypatch.setenv("TPT_TASK_SPP", "4")
    monkeypatch.setenv("TPT_TAIL_SLOTS", "0")
    with DeviceScene(scene) as ds:
        _, on = _film(ds, c, monkeypatch, True)
        _, off = _film(ds, c, monkeypatch, False)
        monkeypatch.setenv("TPT_TAIL_SLOTS", "1024")
        _, tail = _film(ds, c, monkeypatch, True)
    assert off.kernel_launches == 8 * off.iterations + 1 + 1
    assert on.kernel_launches == 8 * on.iterations + 1 + 1 + 7 + 1
    assert tail.kernel_launches == 8 * tail.iterations + 1 + 1 + 7 + 1 + 1
