"""render() through the C ABI (src/render.rs:42 and src/output.rs:96-102)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _abi
from .scene import RenderConfig, Scene, SceneDesc


@dataclass
class RenderStats:
    render_ms: float
    paths: int
    rays_closest: int
    rays_shadow: int
    iterations: int
    device_flags: int
    # profiling pass only (profile=True): per-stage device time and launch
    # counts (extend, shade, shadow, regen) and traversal work counters
    # ([closest-hit, occlusion]).
    stage_ms: tuple = ()
    stage_launches: tuple = ()
    nodes_visited: tuple = ()
    tris_tested: tuple = ()
    spheres_tested: tuple = ()
    instances_tested: tuple = ()
    # adjoint renders: sum of dL/dimage . image over the adjoint's own paths
    adjoint_linear: float = 0.0
    # profiling pass only: warp-wide node-loop steps per trace kind, and
    # samples finished by the closest-hit kernel's camera-miss fast path
    node_steps: tuple = ()
    camera_fast: int = 0
    leaf_visits: tuple = ()
    leaf_steps: tuple = ()
    fast_steps: int = 0
    # wavefront renders: samples per pool task, and the path slots in flight
    task_spp: int = 0
    pool_slots: int = 0
    # wavefront renders: samples of camera-culled pixels (rendered without a
    # trace; counted in paths), and the kernels the render launched
    sky_samples: int = 0
    kernel_launches: int = 0

    @staticmethod
    def from_c(s: _abi.tpt_stats) -> "RenderStats":
        return RenderStats(s.render_ms, s.paths, s.rays_closest, s.rays_shadow, s.iterations, s.device_flags,
                           tuple(s.stage_ms), tuple(s.stage_launches), tuple(s.nodes_visited), tuple(s.tris_tested),
                           tuple(s.spheres_tested), tuple(s.instances_tested), s.adjoint_linear,
                           tuple(s.node_steps), s.camera_fast, tuple(s.leaf_visits), tuple(s.leaf_steps),
                           s.fast_steps, s.task_spp, s.pool_slots, s.sky_samples, s.kernel_launches)

    @property
    def rays(self) -> int:
        return self.rays_closest + self.rays_shadow


@dataclass
class RenderOutput:
    """RenderOutput (src/render.rs:34-39): per-pixel radiance sums and weights."""

    acc: np.ndarray    # (h*w, 3) f64
    acc_w: np.ndarray  # (h*w,) f64
    stats: Optional[RenderStats] = None


class DeviceScene:
    """A Scene uploaded to the current CUDA device (tpt_scene_create)."""

    def __init__(self, scene: Scene):
        self._desc = SceneDesc(scene)
        self._handle = C.c_void_p()
        _abi.check(_abi.lib().tpt_scene_create(self._desc.ptr(), C.byref(self._handle)))

    def close(self) -> None:
        if self._handle:
            _abi.lib().tpt_scene_destroy(self._handle)
            self._handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, config: RenderConfig, acc: Optional[np.ndarray] = None,
               acc_w: Optional[np.ndarray] = None, profile: bool = False) -> RenderOutput:
        """Renders into host arrays (allocated if not given)."""
        n = config.film_pixels
        if acc is None:
            acc = np.empty((n, 3), dtype=np.float64)
        if acc_w is None:
            acc_w = np.empty((n,), dtype=np.float64)
        _check_film(acc, 3 * n, "acc")
        _check_film(acc_w, n, "acc_w")
        cfg = config.to_c()
        st = _abi.tpt_stats()
        st.profile = int(profile)
        _abi.check(
            _abi.lib().tpt_render(
                self._handle,
                C.byref(cfg),
                acc.ctypes.data_as(C.POINTER(C.c_double)),
                acc_w.ctypes.data_as(C.POINTER(C.c_double)),
                C.byref(st),
            )
        )
        return RenderOutput(acc, acc_w, RenderStats.from_c(st))

    def render_resume(self, config: RenderConfig, ckpt_path: str, scene_hash: int) -> RenderOutput:
        """render() with a checkpoint file (tpt_render_resume): tiles before
        the file's next_id come from it, the others from this render; the
        final checkpoint is left at ckpt_path."""
        n = config.width * config.height
        acc = np.empty((n, 3), dtype=np.float64)
        acc_w = np.empty((n,), dtype=np.float64)
        st = _abi.tpt_stats()
        _abi.check(_abi.lib().tpt_render_resume(self._handle, C.byref(config.to_c()), str(ckpt_path).encode(),
                                                scene_hash, acc.ctypes.data_as(C.POINTER(C.c_double)),
                                                acc_w.ctypes.data_as(C.POINTER(C.c_double)), C.byref(st)))
        return RenderOutput(acc, acc_w, RenderStats.from_c(st))

    def render_device(self, config: RenderConfig, acc_ptr: int, acc_w_ptr: int, acc_sq_ptr: int = 0,
                      profile: bool = False) -> RenderStats:
        """Renders into device buffers given as raw pointers (e.g.
        ``tensor.data_ptr()`` of CUDA float64 tensors of 3*w*h and w*h).
        profile=True runs the instrumented wavefront loop (per-stage event
        timing and traversal counters; slower)."""
        cfg = config.to_c()
        st = _abi.tpt_stats()
        st.profile = int(profile)
        _abi.check(
            _abi.lib().tpt_render_device(
                self._handle, C.byref(cfg), C.c_void_p(acc_ptr), C.c_void_p(acc_w_ptr),
                C.c_void_p(acc_sq_ptr) if acc_sq_ptr else None, C.byref(st)
            )
        )
        return RenderStats.from_c(st)


    # ---- differentiation (no counterpart in the reference) ------------------------------------------------
    @property
    def n_materials(self) -> int:
        return int(_abi.lib().tpt_scene_material_count(self._handle))

    def set_materials(self, materials, sampling_materials=None) -> None:
        """Replaces the scene's materials (same count and kinds).  Sampling
        follows ``sampling_materials`` when given (detached sampling; see
        tpt_scene_set_materials)."""
        n = len(materials)
        arr = _materials_c(materials)
        sarr = _materials_c(sampling_materials) if sampling_materials is not None else None
        if sarr is not None and len(sampling_materials) != n:
            raise ValueError("sampling_materials must have one entry per material")
        _abi.check(_abi.lib().tpt_scene_set_materials(self._handle, arr, sarr, n))

    def render_forward(self, config: RenderConfig, image_ptr: int) -> RenderStats:
        """Resolved float image (width*height*3, DEVICE pointer)."""
        st = _abi.tpt_stats()
        _abi.check(_abi.lib().tpt_render_forward_device(self._handle, C.byref(config.to_c()), C.c_void_p(image_ptr),
                                                        C.byref(st)))
        return RenderStats.from_c(st)

    def render_backward(self, config: RenderConfig, dimage_ptr: int, grad_ptr: int) -> RenderStats:
        """Writes dL/dparams (4 f64 per material, DEVICE pointer) for a
        dL/dimage (width*height*3 float, DEVICE pointer)."""
        st = _abi.tpt_stats()
        _abi.check(_abi.lib().tpt_render_backward_device(self._handle, C.byref(config.to_c()),
                                                         C.c_void_p(dimage_ptr), C.c_void_p(grad_ptr), C.byref(st)))
        return RenderStats.from_c(st)

    def render_backward_host(self, config: RenderConfig, dimage: np.ndarray) -> tuple:
        """Host-array form of render_backward: returns (grad (n_materials, 4), stats)."""
        d = np.ascontiguousarray(dimage, dtype=np.float32).reshape(-1)
        if d.size != 3 * config.film_pixels:
            raise ValueError(f"dimage has {d.size} values; the film needs {3 * config.film_pixels}")
        g = np.zeros(4 * self.n_materials, dtype=np.float64)
        st = _abi.tpt_stats()
        _abi.check(_abi.lib().tpt_render_backward(self._handle, C.byref(config.to_c()),
                                                  d.ctypes.data_as(C.POINTER(C.c_float)),
                                                  g.ctypes.data_as(C.POINTER(C.c_double)), C.byref(st)))
        return g.reshape(-1, 4), RenderStats.from_c(st)


def _check_film(a: np.ndarray, size: int, name: str) -> None:
    if a.dtype != np.float64 or not a.flags.c_contiguous or a.size != size:
        raise ValueError(f"{name} must be a C-contiguous float64 array of {size} values "
                         f"(got {a.dtype}, {a.size} values, contiguous={a.flags.c_contiguous})")


def _materials_c(materials):
    arr = (_abi.tpt_material * max(len(materials), 1))()
    for i, m in enumerate(materials):
        arr[i] = _abi.tpt_material(int(m.kind), 0, _abi.D3(*m.rgb), float(m.param))
    return arr


def render(scene: Scene, config: RenderConfig) -> RenderOutput:
    """render(scene, config) (src/render.rs:42) on the current CUDA device."""
    with DeviceScene(scene) as ds:
        return ds.render(config)


def resolve_pixels(w: int, h: int, acc: np.ndarray, acc_w: np.ndarray) -> np.ndarray:
    """acc / max(acc_w, 1) per pixel (src/output.rs:96-102); returns (h*w, 3)."""
    acc = np.asarray(acc, dtype=np.float64).reshape(w * h, 3)
    wts = np.maximum(np.asarray(acc_w, dtype=np.float64).reshape(w * h), 1.0)
    return acc / wts[:, None]


# ---- batch renders (no counterpart in the reference) --------------------------------------------
class BatchScenes:
    """Several scenes merged on the current CUDA device (tpt_batch_create);
    ``render`` draws any number of (scene index, config, film) jobs in one
    wavefront loop."""

    def __init__(self, scenes):
        self._descs = [SceneDesc(s) for s in scenes]
        arr = (_abi.tpt_scene_desc * len(self._descs))(*[d.desc for d in self._descs])
        self._handle = C.c_void_p()
        _abi.check(_abi.lib().tpt_batch_create(arr, len(self._descs), C.byref(self._handle)))
        self.n_scenes = len(self._descs)

    def close(self) -> None:
        if self._handle:
            _abi.lib().tpt_batch_destroy(self._handle)
            self._handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _jobs(jobs):
        """jobs: sequence of (scene index, RenderConfig, acc_ptr, acc_w_ptr)."""
        arr = (_abi.tpt_batch_job * len(jobs))()
        for k, (scene, cfg, acc, acc_w) in enumerate(jobs):
            arr[k] = _abi.tpt_batch_job(int(scene), 0, cfg.to_c(), C.c_void_p(acc), C.c_void_p(acc_w))
        return arr

    def render(self, jobs, tuning=None) -> RenderStats:
        """Renders every job into its DEVICE film; tuning = (pool_slots,
        task_spp, trace_chunk[, shade_ctas]) or None for the defaults."""
        arr = self._jobs(jobs)
        t = _abi.tpt_tuning(*(tuple(tuning) + (0,) * (4 - len(tuning)))) if tuning is not None else None
        st = _abi.tpt_stats()
        _abi.check(_abi.lib().tpt_batch_render_device(self._handle, arr, len(jobs),
                                                      C.byref(t) if t is not None else None, C.byref(st)))
        return RenderStats.from_c(st)

    def autotune(self, jobs, max_trials: int = 32):
        """Returns ((pool_slots, task_spp, trace_chunk, shade_ctas), [trial ms, ...])."""
        arr = self._jobs(jobs)
        best = _abi.tpt_tuning()
        ms = (C.c_double * max_trials)()
        n = _abi.lib().tpt_batch_autotune(self._handle, arr, len(jobs), C.byref(best), ms, max_trials)
        if n < 0:
            _abi.check(n)
        return (best.pool_slots, best.task_spp, best.trace_chunk, best.shade_ctas), list(ms[: min(n, max_trials)])
