"""Scene files and image files through the C ABI (host only, no GPU).

Mirrors the reference's ingestion and output: ``load_scene`` (Mitsuba XML
subset with OBJ meshes and .hdr env maps, src/mitsuba.rs:137-595),
``build_scene`` (src/scene.rs:26-95), ``OutputFormat::write``
(src/output.rs:59-132) and ``read_hdr`` (src/hdr.rs:20-60).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import List, Optional, Tuple

import numpy as np

from . import _abi
from .scene import Camera, EnvMap, Instance, Material, Mesh, RenderConfig, Scene, Sphere, Transform, World


class LoadedScene:
    """A scene description built by the library's loaders (owns the arrays)."""

    def __init__(self, handle: C.c_void_p):
        self._handle = handle

    @staticmethod
    def from_xml(path: str, config: RenderConfig) -> Tuple["LoadedScene", RenderConfig]:
        """Loads a Mitsuba XML scene; returns it and the config with the
        file's film / sampler / integrator values applied."""
        c = config.to_c()
        h = C.c_void_p()
        _abi.check(_abi.lib().tpt_scene_load_xml(str(path).encode(), C.byref(c), C.byref(h)))
        cfg = dataclasses.replace(config, width=c.width, height=c.height, spp=c.spp, max_bounces=c.max_bounces,
                                  rr_start=c.rr_start)
        return LoadedScene(h), cfg

    @staticmethod
    def default(config: RenderConfig, env_path: Optional[str] = None) -> "LoadedScene":
        """The built-in scene for the config's aspect (procedural sky unless
        env_path names a .hdr env map)."""
        h = C.c_void_p()
        _abi.check(_abi.lib().tpt_scene_default(C.byref(config.to_c()), env_path.encode() if env_path else None,
                                                C.byref(h)))
        return LoadedScene(h)

    @property
    def desc(self) -> _abi.tpt_scene_desc:
        return _abi.lib().tpt_loaded_desc(self._handle).contents

    @property
    def warnings(self) -> List[str]:
        L = _abi.lib()
        return [L.tpt_loaded_warning(self._handle, k).decode() for k in range(L.tpt_loaded_warning_count(self._handle))]

    def to_scene(self) -> Scene:
        """The description as a ``Scene`` (arrays copied)."""
        d = self.desc
        c = d.camera
        cam = Camera(c.kind, tuple(c.eye), tuple(c.target), tuple(c.up), c.fov_y_deg, c.aspect, c.focus_dist,
                     c.aperture)
        mats = [Material(m.kind, tuple(m.rgb), m.param) for m in d.materials[: d.n_materials]]
        w = World()
        w.spheres = [Sphere(tuple(s.center), s.radius, int(s.mat_id)) for s in d.spheres[: d.n_spheres]]
        for md in d.meshes[: d.n_meshes]:
            pos = np.ctypeslib.as_array(md.positions, shape=(md.n_vertices * 3,)).copy() if md.n_vertices else []
            idx = np.ctypeslib.as_array(md.indices, shape=(md.n_tris * 3,)).copy() if md.n_tris else []
            mid = np.ctypeslib.as_array(md.mat_ids, shape=(md.n_tris,)).copy() if md.n_tris else []
            w.meshes.append(Mesh.from_arrays(np.asarray(pos, dtype=np.float64), np.asarray(idx, dtype=np.int32),
                                             np.asarray(mid, dtype=np.int32)))
        for x in d.instances[: d.n_instances]:
            a = [[x.linear[3 * r + k] for k in range(3)] for r in range(3)]
            ov = None if x.mat_override < 0 else int(x.mat_override)
            w.instances.append(Instance(int(x.mesh_id), Transform.from_affine(a, list(x.translation)), ov))
        env = None
        if d.env.kind == _abi.TPT_ENV_MAP:
            n = d.env.width * d.env.height * 3
            env = EnvMap.from_pixels(d.env.width, d.env.height, np.ctypeslib.as_array(d.env.pixels, shape=(n,)).copy())
        return Scene(cam, w, mats, env)

    def close(self) -> None:
        if self._handle:
            _abi.lib().tpt_loaded_destroy(self._handle)
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


def load_obj_via_xml(path: str) -> Mesh:
    """An OBJ file's mesh as the loader reads it (one obj shape)."""
    import os
    import tempfile

    with tempfile.TemporaryDirectory() as d:
        x = os.path.join(d, "s.xml")
        with open(x, "w") as f:
            f.write(f'<scene><shape type="obj"><string name="filename" value="{os.path.abspath(path)}"/>'
                    f'<bsdf type="diffuse"/></shape></scene>')
        ls, _ = LoadedScene.from_xml(x, RenderConfig(width=16, height=9))
        with ls:
            return ls.to_scene().world.meshes[0]


def write_image(path: str, rgb: np.ndarray, exposure: float = 0.0, tonemap: str = "aces") -> None:
    """rgb: (h, w, 3) linear; the format follows the extension."""
    a = np.ascontiguousarray(rgb, dtype=np.float64)
    h, w = a.shape[:2]
    tm = {"none": 0, "aces": 1}[tonemap]
    _abi.check(_abi.lib().tpt_write_image(str(path).encode(), w, h, a.ctypes.data_as(C.POINTER(C.c_double)),
                                          float(exposure), tm))


def read_hdr(path: str) -> np.ndarray:
    """(h, w, 3) linear RGB of a Radiance .hdr file, row 0 at the top."""
    w, h = C.c_int32(0), C.c_int32(0)
    L = _abi.lib()
    _abi.check(L.tpt_read_hdr(str(path).encode(), C.byref(w), C.byref(h), None))
    out = np.empty((h.value, w.value, 3), dtype=np.float64)
    _abi.check(L.tpt_read_hdr(str(path).encode(), C.byref(w), C.byref(h), out.ctypes.data_as(C.POINTER(C.c_double))))
    return out


# ---- checkpoints (src/checkpoint.rs, HYPCKPT v1) ------------------------------------------------
def film_tiles(width: int, height: int, tile: int = 16, morton: bool = True) -> np.ndarray:
    """(n, 4) x0, y0, x1, y1 of the film's tiles in task order."""
    L = _abi.lib()
    n = L.tpt_film_tiles(width, height, tile, int(morton), None)
    if n < 0:
        _abi.check(int(n))
    out = np.zeros((n, 4), dtype=np.int32)
    L.tpt_film_tiles(width, height, tile, int(morton), out.ctypes.data_as(C.POINTER(C.c_int32)))
    return out


def save_checkpoint(path: str, scene_hash: int, width: int, height: int, next_id: int, acc, acc_w) -> None:
    a = np.ascontiguousarray(acc, dtype=np.float64).reshape(-1)
    w = np.ascontiguousarray(acc_w, dtype=np.float64).reshape(-1)
    if a.size != 3 * width * height or w.size != width * height:
        raise ValueError(f"film of {a.size // 3} / {w.size} pixels for a {width}x{height} checkpoint")
    _abi.check(_abi.lib().tpt_checkpoint_save(str(path).encode(), scene_hash, width, height, next_id,
                                              a.ctypes.data_as(C.POINTER(C.c_double)),
                                              w.ctypes.data_as(C.POINTER(C.c_double))))


def load_checkpoint(path: str, scene_hash: int, width: int, height: int):
    """(next_id, acc (n, 3), acc_w (n,)) or None when absent or not matching."""
    n = width * height
    a = np.empty(3 * n)
    w = np.empty(n)
    nid = C.c_uint64(0)
    rc = _abi.lib().tpt_checkpoint_load(str(path).encode(), scene_hash, width, height, C.byref(nid),
                                        a.ctypes.data_as(C.POINTER(C.c_double)),
                                        w.ctypes.data_as(C.POINTER(C.c_double)))
    if rc < 0:
        _abi.check(rc)
    return (int(nid.value), a.reshape(n, 3), w) if rc == 1 else None
