"""The allocation-free render entry point, tpt_render_device_noalloc.

It exists for callers that must not allocate device memory while they
render: a process whose own allocator reserves the GPU at start-up, or a
frame loop that cannot take the device-wide synchronisation that
cudaMalloc/cudaFree cause.  It keeps its scratch in a fixed device array
inside the library and so only serves films up to 16384 pixels.

This file is named to run last: it checks the entry point against the
regular device entry point (tpt_render_device, same FP32 wavefront kernels)
on two calls in a row, and as the first render of a new handle, whether it
runs alone in a fresh process or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from tinypt_b200 import _abi, scenes
from tinypt_b200.render import DeviceScene
from tests.parity_util import cfg, small_mesh_env_scene

pytestmark = pytest.mark.gpu


def _buffers(n):
    import torch

    # The caller allocates its outputs up front; the entry point allocates nothing.
    return (torch.zeros(3 * n, dtype=torch.float64, device="cuda"),
            torch.zeros(n, dtype=torch.float64, device="cuda"))


def _noalloc(ds: DeviceScene, c, acc, acc_w):
    conf = c.to_c()
    st = _abi.tpt_stats()
    rc = _abi.lib().tpt_render_device_noalloc(ds._handle, C.byref(conf), C.c_void_p(acc.data_ptr()),
                                               C.c_void_p(acc_w.data_ptr()), C.byref(st))
    return rc, st


def test_noalloc_as_the_first_render_of_a_handle(gpu, monkeypatch):
    """The allocation-free entry point called before any other render on a
    new scene handle (run alone in a fresh process, it is also the first
    wavefront render of the process, so its first-call set-up runs here),
    then the regular entry point: same film."""
    import torch

    scene, c = scenes.sphere_scene(48, 32), cfg(48, 32, 8, 8, _abi.TPT_MODE_WAVEFRONT_FP32, seed=9)
    n = c.width * c.height
    monkeypatch.setenv("TPT_TASK_SPP", str(c.spp))
    with DeviceScene(scene) as ds:
        acc, acc_w = _buffers(n)
        rc, st = _noalloc(ds, c, acc, acc_w)
        assert rc == _abi.TPT_OK, _abi.lib().tpt_last_error()
        torch.cuda.synchronize()
        got_acc, got_w = acc.cpu().numpy(), acc_w.cpu().numpy()
        ref_acc, ref_w = _buffers(n)
        ds.render_device(c, ref_acc.data_ptr(), ref_w.data_ptr())
        torch.cuda.synchronize()
    assert np.array_equal(got_w, ref_w.cpu().numpy())
    want = ref_acc.cpu().numpy()
    assert np.max(np.abs(got_acc - want) / np.maximum(np.abs(want), 1e-12)) <= 1e-12
    assert st.paths == n * c.spp


@pytest.mark.parametrize("which", ["spheres", "mesh_env"])
def test_noalloc_matches_device_entry_point_twice(gpu, which, monkeypatch):
    import torch

    if which == "spheres":
        scene, c = scenes.sphere_scene(64, 48), cfg(64, 48, 16, 8, _abi.TPT_MODE_WAVEFRONT_FP32)
    else:
        scene, c = small_mesh_env_scene(), cfg(96, 54, 8, 16, _abi.TPT_MODE_WAVEFRONT_FP32)
    n = c.width * c.height
    # The allocation-free entry point runs one task per pixel; ask the regular
    # one for the same schedule, so both draw each pixel's samples from one
    # stream.
    monkeypatch.setenv("TPT_TASK_SPP", str(c.spp))
    with DeviceScene(scene) as ds:
        ref_acc, ref_w = _buffers(n)
        ds.render_device(c, ref_acc.data_ptr(), ref_w.data_ptr())
        torch.cuda.synchronize()
        want_acc, want_w = ref_acc.cpu().numpy(), ref_w.cpu().numpy()
        acc, acc_w = _buffers(n)
        for call in range(2):
            acc.fill_(-1.0)
            acc_w.fill_(-1.0)
            torch.cuda.synchronize()
            rc, st = _noalloc(ds, c, acc, acc_w)
            assert rc == _abi.TPT_OK, _abi.lib().tpt_last_error()
            torch.cuda.synchronize()
            got_acc, got_w = acc.cpu().numpy(), acc_w.cpu().numpy()
            # Same kernels and RNG streams: the regular entry point's tolerance
            # (exact agreement, as in the determinism test) applies.
            assert np.array_equal(got_w, want_w), f"call {call}: sample counts differ"
            rel = np.max(np.abs(got_acc - want_acc) / np.maximum(np.abs(want_acc), 1e-12))
            assert rel <= 1e-12, f"call {call}: radiance differs by {rel}"
            assert st.paths == n * c.spp


def test_noalloc_rejects_films_beyond_its_limit(gpu):
    scene = scenes.sphere_scene(256, 256)
    c = cfg(256, 256, 1, 8, _abi.TPT_MODE_WAVEFRONT_FP32)
    with DeviceScene(scene) as ds:
        acc, acc_w = _buffers(256 * 256)
        rc, _ = _noalloc(ds, c, acc, acc_w)
    assert rc == _abi.TPT_ERR_INVALID
    assert b"allocation-free limit" in _abi.lib().tpt_last_error()
