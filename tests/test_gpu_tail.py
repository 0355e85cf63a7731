"""The drain of the FP32 wavefront's bounce loop.

Once every task has been taken and at most TPT_TAIL_SLOTS slots are still
live, the loop stops. k_tail then runs each live slot to the end of its
task, one thread per slot, with the wavefront kernels' own per-slot steps
in their order:
* the closest hit;
* the shading visit;
* the shadow rays;
* the completion of a path that ended with shadow rays pending.

So the film is bit for bit that of the loop run to the end. The tests check
this in single, batch and adaptive-round renders, and for three thresholds:
* a threshold the drain crosses late;
* one the drain crosses early;
* one so large that k_tail takes over right after the first iteration and
  renders nearly everything itself.
"""
import numpy as np
import pytest

from tinypt_b200 import _abi, scenes
from tinypt_b200.render import DeviceScene
from tests.parity_util import cfg, small_mesh_env_scene

pytestmark = pytest.mark.gpu

WF = _abi.TPT_MODE_WAVEFRONT_FP32


@pytest.fixture(autouse=True)
def default_schedule(monkeypatch):
    for k in ("TPT_TASK_SPP", "TPT_POOL", "TPT_CAMERA_FAST", "TPT_SHADE_CTAS", "TPT_MAX_PART_TASKS",
              "TPT_WAVEFRONT_HOST_LOOP", "TPT_QUEUE_ORDER", "TPT_QUEUE_DIV", "TPT_SKY_CULL", "TPT_TAIL_SLOTS"):
        monkeypatch.delenv(k, raising=False)


def _film(ds, c, monkeypatch, tail):
    import torch

    monkeypatch.setenv("TPT_TAIL_SLOTS", str(tail))
    n = c.film_pixels
    acc = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    acc_w = torch.zeros(n, dtype=torch.float64, device="cuda")
    acc_sq = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    st = ds.render_device(c, acc.data_ptr(), acc_w.data_ptr(), acc_sq.data_ptr())
    torch.cuda.synchronize()
    return (acc.cpu().numpy(), acc_w.cpu().numpy(), acc_sq.cpu().numpy()), st


SCENES = {
    "mesh_env": lambda: (small_mesh_env_scene(96, 54), cfg(96, 54, 16, 16, WF)),
    "spheres": lambda: (scenes.sphere_scene(64, 48), cfg(64, 48, 16, 8, WF)),
}


@pytest.mark.parametrize("tail", [64, 2048, 1 << 30])
@pytest.mark.parametrize("name", sorted(SCENES))
@pytest.mark.parametrize("schedule", ["auto", "task4", "host_loop"])
def test_tail_kernel_changes_no_film(gpu, monkeypatch, name, tail, schedule):
    scene, c = SCENES[name]()
    if schedule == "task4":
        monkeypatch.setenv("TPT_TASK_SPP", "4")
        monkeypatch.setenv("TPT_POOL", "4096")  # more tasks than slots: the pool refills before the drain
    elif schedule == "host_loop":
        monkeypatch.setenv("TPT_WAVEFRONT_HOST_LOOP", "1")
    with DeviceScene(scene) as ds:
        off, st_off = _film(ds, c, monkeypatch, 0)
        on, st_on = _film(ds, c, monkeypatch, tail)
    print(f"{name} {schedule} tail {tail}: iterations {st_off.iterations} -> {st_on.iterations}")
    for a, b, what in zip(on, off, ("acc", "acc_w", "acc_sq")):
        assert np.array_equal(a, b), f"{what} differs with the tail kernel"
    assert st_on.paths == st_off.paths == c.film_pixels * c.spp
    assert st_on.rays_closest == st_off.rays_closest
    assert st_on.rays_shadow == st_off.rays_shadow
    assert st_on.iterations <= st_off.iterations


def test_tail_kernel_in_batch_renders(gpu, monkeypatch):
    """A multi-job render hands its drain over the same way, each slot under
    its job's view: every job's film is the same with the handover off
    and with it taking over early."""
    import torch

    from tinypt_b200.render import BatchScenes

    work = scenes.batch_workload(4, seed=3, tri_range=(500, 20_000), res_range=(24, 64), spp_range=(4, 24),
                                 max_depth=8)

    def render(tail):
        monkeypatch.setenv("TPT_TAIL_SLOTS", str(tail))
        films = [(torch.zeros(3 * c.film_pixels, dtype=torch.float64, device="cuda"),
                  torch.zeros(c.film_pixels, dtype=torch.float64, device="cuda")) for _, c in work]
        with BatchScenes([s for s, _ in work]) as bs:
            st = bs.render([(k, c, a.data_ptr(), w.data_ptr()) for k, ((_, c), (a, w)) in enumerate(zip(work, films))])
        assert st.device_flags == 0
        return films, st

    off, st_off = render(0)
    on, st_on = render(1 << 30)
    print(f"batch: iterations {st_off.iterations} -> {st_on.iterations}")
    assert st_on.paths == st_off.paths
    for (a1, w1), (a0, w0) in zip(on, off):
        assert torch.equal(w1, w0) and torch.equal(a1, a0)


def test_tail_kernel_in_adaptive_rounds(gpu, monkeypatch):
    """An adaptive render in rounds hands each round's drain over. The
    round's sample records, and with them the stopping rule, the sample
    counts and the film, are the same with the handover off and on."""
    scene = scenes.sphere_scene(48, 32)
    c = cfg(48, 32, 64, 8, WF, adaptive_enabled=1, adaptive_min_spp=8, adaptive_threshold=0.05)
    with DeviceScene(scene) as ds:
        off, st_off = _film(ds, c, monkeypatch, 0)
        on, st_on = _film(ds, c, monkeypatch, 1 << 30)
    print(f"adaptive rounds: iterations {st_off.iterations} -> {st_on.iterations}, mean spp {off[1].mean():.1f}")
    assert st_on.paths == st_off.paths
    for a, b, what in zip(on, off, ("acc", "acc_w", "acc_sq")):
        assert np.array_equal(a, b), f"{what} differs with the tail kernel"
