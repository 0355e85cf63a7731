"""ORACLE -- test infrastructure only.

ctypes binding of the CPU f64 restatement of tinypt's path integrator
(oracle/ref_model.hpp, oracle/ref_impl.cpp).  Imported only by tests/, by
``__graft_entry__.smoke()`` and by the CPU-baseline leg of ``bench.py``; the
product (``tinypt_b200``) never imports it.

Parity status: the reference cannot be built here (no Rust toolchain), so
this oracle is pinned by the reference's own unit-test assertions (restated in
tests/test_oracle_kats.py) and by an independent pure-Python restatement of
the integer paths (tests/golden/make_golden.py).  Image-level parity with the
Rust binary is unpinned.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from tinypt_b200 import _abi
from tinypt_b200.scene import RenderConfig, Scene, SceneDesc

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"


class oracle_counts(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("world_hits", "node_pops", "node_box_tests", "tri_tests", "sphere_tests")]


_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        srcs = [HERE / n for n in ("ref_impl.cpp", "oracle_abi.cpp", "ref_model.hpp", "oracle.h")]
        if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < max(p.stat().st_mtime for p in srcs):
            build()
        L = C.CDLL(str(LIB_PATH))
        P = C.POINTER
        dp = P(C.c_double)
        L.oracle_scene_create.argtypes = [P(_abi.tpt_scene_desc), P(C.c_void_p)]
        L.oracle_scene_create.restype = C.c_int
        L.oracle_scene_destroy.argtypes = [C.c_void_p]
        L.oracle_scene_destroy.restype = None
        L.oracle_scene_set_materials.argtypes = [C.c_void_p, P(_abi.tpt_material), P(_abi.tpt_material), C.c_int64]
        L.oracle_scene_set_materials.restype = C.c_int
        L.oracle_scene_render.argtypes = [C.c_void_p, P(_abi.tpt_render_config), P(C.c_int32), dp, dp, dp, C.c_int,
                                          P(oracle_counts)]
        L.oracle_scene_render.restype = C.c_int
        L.oracle_scene_render_tasks.argtypes = [C.c_void_p, P(_abi.tpt_render_config), P(C.c_int32), C.c_int, dp,
                                                dp, dp, C.c_int, P(oracle_counts)]
        L.oracle_scene_render_tasks.restype = C.c_int
        L.oracle_scene_render_streams.argtypes = [C.c_void_p, P(_abi.tpt_render_config), P(C.c_int32), C.c_int,
                                                  C.c_int, dp, dp, dp, C.c_int, P(oracle_counts)]
        L.oracle_scene_render_streams.restype = C.c_int
        L.oracle_resolve_pixels.argtypes = [C.c_int64, dp, dp, dp]
        L.oracle_resolve_pixels.restype = None
        L.oracle_render.argtypes = [P(_abi.tpt_scene_desc), P(_abi.tpt_render_config), dp, dp, dp, C.c_int,
                                    P(oracle_counts)]
        L.oracle_render.restype = C.c_int
        L.oracle_rng_u32.argtypes = [C.c_uint64, C.c_int, P(C.c_uint32)]
        L.oracle_rng_u32.restype = None
        L.oracle_rng_f64.argtypes = [C.c_uint64, C.c_int, dp]
        L.oracle_rng_f64.restype = None
        L.oracle_seed_for.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        L.oracle_seed_for.restype = C.c_uint64
        L.oracle_interleave_bits.argtypes = [C.c_uint64]
        L.oracle_interleave_bits.restype = C.c_uint64
        L.oracle_tile_order.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_int32)]
        L.oracle_tile_order.restype = C.c_int
        L.oracle_bvh_build.argtypes = [P(_abi.tpt_mesh_desc), dp, P(C.c_int32), P(C.c_uint32), P(C.c_int64)]
        L.oracle_bvh_build.restype = C.c_int64
        L.oracle_material_sample.argtypes = [P(_abi.tpt_material), dp, dp, C.c_double, C.c_double, dp, dp,
                                             P(C.c_uint64), dp]
        L.oracle_material_sample.restype = C.c_int
        L.oracle_material_eval.argtypes = [P(_abi.tpt_material), dp, dp, dp, dp]
        L.oracle_material_eval.restype = None
        L.oracle_material_eval_n.argtypes = [P(_abi.tpt_material), dp, dp, dp, C.c_int64, dp]
        L.oracle_material_eval_n.restype = None
        L.oracle_material_classify.argtypes = [P(_abi.tpt_material), P(C.c_int32)]
        L.oracle_material_classify.restype = None
        L.oracle_transform.argtypes = [C.c_int, P(C.c_int32), dp, C.c_int, dp, dp, dp]
        L.oracle_transform.restype = None
        L.oracle_sample_light.argtypes = [P(_abi.tpt_scene_desc), P(C.c_uint64), C.c_double, dp, dp, dp,
                                          P(C.c_int64)]
        L.oracle_sample_light.restype = C.c_int
        L.oracle_camera_ray.argtypes = [P(_abi.tpt_camera_desc), C.c_double, C.c_double, P(C.c_uint64), dp]
        L.oracle_camera_ray.restype = None
        L.oracle_env_eval.argtypes = [P(_abi.tpt_env_desc), dp, dp]
        L.oracle_env_eval.restype = C.c_int
        L.oracle_env_sample_dir.argtypes = [P(_abi.tpt_env_desc), P(C.c_uint64), dp]
        L.oracle_env_sample_dir.restype = C.c_int
        L.oracle_radiance.argtypes = [P(_abi.tpt_scene_desc), P(_abi.tpt_render_config), C.c_int, C.c_int,
                                      P(C.c_uint64), dp]
        L.oracle_radiance.restype = C.c_int
        L.oracle_last_error.argtypes = []
        L.oracle_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def _ok(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(f"oracle error {rc}: {lib().oracle_last_error().decode()}")


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class OracleScene:
    """The reference Scene built once on the CPU (BVHs, lights, env CDF)."""

    def __init__(self, scene: Scene):
        self._desc = SceneDesc(scene)
        self._h = C.c_void_p()
        _ok(lib().oracle_scene_create(self._desc.ptr(), C.byref(self._h)))

    def set_materials(self, materials, sampling_materials=None):
        """Replaces the materials; sampling follows sampling_materials when
        given (detached sampling, for finite-difference checks)."""
        def arr(ms):
            a = (_abi.tpt_material * max(len(ms), 1))()
            for i, m in enumerate(ms):
                a[i] = _abi.tpt_material(int(m.kind), 0, _abi.D3(*m.rgb), float(m.param))
            return a

        sa = arr(sampling_materials) if sampling_materials is not None else None
        _ok(lib().oracle_scene_set_materials(self._h, arr(materials), sa, len(materials)))

    def close(self):
        if self._h:
            lib().oracle_scene_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, cfg: RenderConfig, rect=None, threads: int = 0, want_sq: bool = False, counts: bool = False,
               sample_chunk: int = 0, reseed: int = 0):
        """Returns (acc (n,3), acc_w (n,), acc_sq or None, counts or None);
        rect = (x0, y0, x1, y1) renders that sub-rectangle only.
        sample_chunk > 0 cuts each pixel's samples into tasks of that many
        samples, each seeded from seed_for(x, y, sample_start) and merged in
        task order (the reference worker's Task { sample_start, sample_end },
        render.rs:142, 226-241); 0 is the reference's own task list.
        reseed > 0 keeps the reference's loop over each pixel's samples (sums
        in sample order, one Welford statistic) but restarts the pixel's RNG
        from seed_for(x, y, s) ^ seed at every sample s that is a multiple of
        reseed: the schedule of the wavefront form's adaptive rounds."""
        threads = threads or os.cpu_count() or 1
        if rect is None:
            n = cfg.width * cfg.height
            rp = None
        else:
            x0, y0, x1, y1 = rect
            n = (x1 - x0) * (y1 - y0)
            r = (C.c_int32 * 4)(x0, y0, x1, y1)
            rp = r
        acc = np.zeros((n, 3))
        acc_w = np.zeros(n)
        acc_sq = np.zeros((n, 3)) if want_sq else None
        cnt = oracle_counts() if counts else None
        c = cfg.to_c()
        _ok(lib().oracle_scene_render_streams(self._h, C.byref(c), rp, int(sample_chunk), int(reseed), _dp(acc),
                                              _dp(acc_w), _dp(acc_sq) if want_sq else None, threads,
                                              C.byref(cnt) if counts else None))
        return acc, acc_w, acc_sq, cnt


def resolve_pixels(acc: np.ndarray, acc_w: np.ndarray) -> np.ndarray:
    """output.rs:96-102: acc / max(acc_w, 1) per pixel, in f64."""
    a = np.ascontiguousarray(acc, dtype=np.float64).reshape(-1, 3)
    w = np.ascontiguousarray(acc_w, dtype=np.float64).reshape(-1)
    out = np.zeros_like(a)
    lib().oracle_resolve_pixels(len(w), _dp(a), _dp(w), _dp(out))
    return out


def rng_u32(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.uint32)
    lib().oracle_rng_u32(seed, n, out.ctypes.data_as(C.POINTER(C.c_uint32)))
    return out


def rng_f64(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n)
    lib().oracle_rng_f64(seed, n, _dp(out))
    return out


def seed_for(px: int, py: int, s: int) -> int:
    return int(lib().oracle_seed_for(px, py, s))


def interleave_bits(v: int) -> int:
    return int(lib().oracle_interleave_bits(v))


def tile_order(w: int, h: int, tile: int, morton: bool) -> np.ndarray:
    n = lib().oracle_tile_order(w, h, tile, int(morton), None)
    out = np.zeros((n, 4), dtype=np.int32)
    lib().oracle_tile_order(w, h, tile, int(morton), out.ctypes.data_as(C.POINTER(C.c_int32)))
    return out


def bvh_build(mesh_desc: _abi.tpt_mesh_desc, n_tris: int):
    n = lib().oracle_bvh_build(C.byref(mesh_desc), None, None, None, None)
    if n < 0:
        raise RuntimeError(lib().oracle_last_error().decode())
    bbox = np.zeros((n, 6))
    lr = np.zeros((n, 2), dtype=np.int32)
    sc = np.zeros((n, 2), dtype=np.uint32)
    idx = np.zeros(n_tris, dtype=np.int64)
    lib().oracle_bvh_build(C.byref(mesh_desc), _dp(bbox), lr.ctypes.data_as(C.POINTER(C.c_int32)),
                           sc.ctypes.data_as(C.POINTER(C.c_uint32)), idx.ctypes.data_as(C.POINTER(C.c_int64)))
    return bbox, lr, sc, idx


def material_sample(mat, ray_o, ray_d, time, hit_t, hit_p, hit_n, rng_state: int):
    m = _abi.tpt_material(mat.kind, 0, _abi.D3(*mat.rgb), float(mat.param))
    st = C.c_uint64(rng_state)
    out = np.zeros(11)
    arr = lambda v: np.ascontiguousarray(v, dtype=np.float64)
    o, d, p, nn = arr(ray_o), arr(ray_d), arr(hit_p), arr(hit_n)
    ok = lib().oracle_material_sample(C.byref(m), _dp(o), _dp(d), time, hit_t, _dp(p), _dp(nn), C.byref(st), _dp(out))
    return (out if ok else None), int(st.value)


def material_eval(mat, wo, wi, n):
    m = _abi.tpt_material(mat.kind, 0, _abi.D3(*mat.rgb), float(mat.param))
    arr = lambda v: np.ascontiguousarray(v, dtype=np.float64)
    a, b, c = arr(wo), arr(wi), arr(n)
    out = np.zeros(4)
    lib().oracle_material_eval(C.byref(m), _dp(a), _dp(b), _dp(c), _dp(out))
    return out[:3], out[3]


def material_eval_n(mat, wo, wi, n):
    """eval() of every row of wi (k x 3): returns (f (k x 3), pdf (k,))."""
    m = _abi.tpt_material(mat.kind, 0, _abi.D3(*mat.rgb), float(mat.param))
    arr = lambda v: np.ascontiguousarray(v, dtype=np.float64)
    a, b, c = arr(wo), arr(wi).reshape(-1, 3), arr(n)
    out = np.zeros((len(b), 4))
    lib().oracle_material_eval_n(C.byref(m), _dp(a), _dp(b), _dp(c), len(b), _dp(out))
    return out[:, :3], out[:, 3]


def material_classify(mat):
    """(is_delta(), emitted().is_some()) of material.rs."""
    m = _abi.tpt_material(mat.kind, 0, _abi.D3(*mat.rgb), float(mat.param))
    out = (C.c_int32 * 2)()
    lib().oracle_material_classify(C.byref(m), out)
    return bool(out[0]), bool(out[1])


def radiance_sample(scene: Scene, cfg: RenderConfig, x: int, y: int, rng_state: int):
    """One sample of pixel (x, y) from the RNG state given: jitter, camera
    ray and radiance() (render.rs:151-158); returns (rgb, the RNG state after)."""
    d = SceneDesc(scene)
    c = cfg.to_c()
    st = C.c_uint64(rng_state)
    out = np.zeros(3)
    _ok(lib().oracle_radiance(d.ptr(), C.byref(c), x, y, C.byref(st), _dp(out)))
    return out, int(st.value)


def transform(ops, mode: int, p):
    """ops: list of (kind, params[5]); kinds 0 translate, 1 scale, 2 rotate, 3 new."""
    kinds = np.array([k for k, _ in ops], dtype=np.int32)
    params = np.array([list(q) + [0.0] * (5 - len(q)) for _, q in ops], dtype=np.float64).reshape(-1)
    pp = np.ascontiguousarray(p, dtype=np.float64)
    out = np.zeros(3)
    at = np.zeros(12)
    lib().oracle_transform(len(ops), kinds.ctypes.data_as(C.POINTER(C.c_int32)), _dp(params), mode, _dp(pp),
                           _dp(out), _dp(at))
    return out, at


def sample_light(scene: Scene, rng_state: int, time: float, p):
    d = SceneDesc(scene)
    st = C.c_uint64(rng_state)
    pp = np.ascontiguousarray(p, dtype=np.float64)
    out = np.zeros(10)
    total = C.c_double()
    nl = C.c_int64()
    ok = lib().oracle_sample_light(d.ptr(), C.byref(st), time, _dp(pp), _dp(out), C.byref(total), C.byref(nl))
    if ok < 0:
        raise RuntimeError(lib().oracle_last_error().decode())
    return (out if ok == 1 else None), int(st.value), total.value, nl.value


def camera_ray(cam, sx: float, sy: float, rng_state: int):
    c = _abi.tpt_camera_desc(cam.kind, 0, _abi.D3(*cam.eye), _abi.D3(*cam.target), _abi.D3(*cam.up), cam.fov_y_deg,
                             cam.aspect, cam.focus_dist, cam.aperture)
    st = C.c_uint64(rng_state)
    out = np.zeros(7)
    lib().oracle_camera_ray(C.byref(c), sx, sy, C.byref(st), _dp(out))
    return out, int(st.value)


def _env_desc(env):
    px = np.ascontiguousarray(env.data, dtype=np.float64)
    return _abi.tpt_env_desc(_abi.TPT_ENV_MAP, env.width, env.height, 0, _dp(px)), px


def env_eval(env, direction):
    d, keep = _env_desc(env)
    dd = np.ascontiguousarray(direction, dtype=np.float64)
    out = np.zeros(4)
    _ok(lib().oracle_env_eval(C.byref(d), _dp(dd), _dp(out)))
    return out[:3], out[3]


def env_sample_dir(env, rng_state: int):
    d, keep = _env_desc(env)
    st = C.c_uint64(rng_state)
    out = np.zeros(7)
    _ok(lib().oracle_env_sample_dir(C.byref(d), C.byref(st), _dp(out)))
    return out, int(st.value)
