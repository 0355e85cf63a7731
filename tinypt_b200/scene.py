"""Scene model of the reference renderer, mirrored for the C ABI.

The names and argument meanings follow tinypt's Rust API:

* ``Material`` -- src/material.rs:30-43 (``lambert``, ``metal``, ``dielectric``,
  ``ggx``, ``subsurface``, ``diffuse_light``);
* ``Camera.look_at`` / ``Camera.look_at_dof`` -- src/ray.rs:36-86;
* ``Transform`` -- src/transform.rs (affine ``p' = A p + t`` with Mitsuba-order
  composition);
* ``Sphere``, ``Mesh``, ``Instance``, ``World`` -- src/geometry.rs, src/world.rs;
* ``EnvMap`` -- src/env.rs (``from_pixels``, ``constant``, ``scaled``);
* ``Scene`` -- src/scene.rs:14-23;
* ``RenderConfig`` -- src/config.rs:5-92 (hot-path fields, same defaults);
* ``render(scene, config) -> RenderOutput(acc, acc_w)`` -- src/render.rs:42.

Host-side f64 arithmetic here (sRGB decode, transform composition) uses the
reference's operation order so the values handed to the library are the
ones the reference would build.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _abi

Vec = Sequence[float]


# ---- src/math.rs:176-191 ---------------------------------------------------------
def srgb_to_linear(c: float) -> float:
    if c <= 0.04045:
        return c / 12.92
    return ((c + 0.055) / 1.055) ** 2.4


def linear_to_srgb(c: float) -> float:
    if c <= 0.0031308:
        return 12.92 * c
    return 1.055 * c ** (1.0 / 2.4) - 0.055


def color_from_srgb(r: float, g: float, b: float):
    return (srgb_to_linear(r), srgb_to_linear(g), srgb_to_linear(b))


def luminance(c) -> float:
    return 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2]


# ---- src/material.rs:30-43 -----------------------------------------------------------
@dataclass(frozen=True)
class Material:
    kind: int
    rgb: tuple
    param: float = 0.0

    @staticmethod
    def lambert(albedo: Vec) -> "Material":
        return Material(_abi.TPT_MAT_LAMBERT, tuple(map(float, albedo)))

    @staticmethod
    def metal(albedo: Vec) -> "Material":
        return Material(_abi.TPT_MAT_METAL, tuple(map(float, albedo)))

    @staticmethod
    def dielectric(ior: float, absorption: Vec = (0.0, 0.0, 0.0)) -> "Material":
        return Material(_abi.TPT_MAT_DIELECTRIC, tuple(map(float, absorption)), float(ior))

    @staticmethod
    def ggx(albedo: Vec, alpha: float) -> "Material":
        return Material(_abi.TPT_MAT_GGX, tuple(map(float, albedo)), float(alpha))

    @staticmethod
    def subsurface(albedo: Vec, scatter_dist: float) -> "Material":
        return Material(_abi.TPT_MAT_SUBSURFACE, tuple(map(float, albedo)), float(scatter_dist))

    @staticmethod
    def diffuse_light(emit: Vec) -> "Material":
        return Material(_abi.TPT_MAT_DIFFUSE_LIGHT, tuple(map(float, emit)))

    def is_delta(self) -> bool:  # material.rs:70-72
        return self.kind in (_abi.TPT_MAT_METAL, _abi.TPT_MAT_DIELECTRIC)

    def emitted(self):  # material.rs:62-67
        return self.rgb if self.kind == _abi.TPT_MAT_DIFFUSE_LIGHT else None


# ---- src/ray.rs:36-86 -------------------------------------------------------------------
@dataclass(frozen=True)
class Camera:
    kind: int
    eye: tuple
    target: tuple
    up: tuple
    fov_y_deg: float
    aspect: float
    focus_dist: float = 0.0
    aperture: float = 0.0

    @staticmethod
    def look_at(eye: Vec, target: Vec, up: Vec, fov_deg: float, aspect: float) -> "Camera":
        return Camera(_abi.TPT_CAMERA_LOOK_AT, tuple(eye), tuple(target), tuple(up), float(fov_deg), float(aspect))

    @staticmethod
    def look_at_dof(eye, target, up, fov_deg, aspect, focus_dist, aperture) -> "Camera":
        return Camera(
            _abi.TPT_CAMERA_LOOK_AT_DOF,
            tuple(eye),
            tuple(target),
            tuple(up),
            float(fov_deg),
            float(aspect),
            float(focus_dist),
            float(aperture),
        )


# ---- src/transform.rs ----------------------------------------------------------------
def _mat_mul(a, b):  # math.rs:117-127
    return [[a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j] for j in range(3)] for i in range(3)]


def _mat_vec(a, v):  # math.rs:130-136
    return [a[i][0] * v[0] + a[i][1] * v[1] + a[i][2] * v[2] for i in range(3)]


def _norm(v):  # math.rs:69-72
    l = max(math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]), 1e-30)
    return [v[0] / l, v[1] / l, v[2] / l]


def _rotation(axis, deg):  # transform.rs:101-111
    k = _norm(axis)
    rad = deg * (math.pi / 180.0)
    s, c = math.sin(rad), math.cos(rad)
    one_c = 1.0 - c
    x, y, z = k
    return [
        [c + x * x * one_c, x * y * one_c - z * s, x * z * one_c + y * s],
        [y * x * one_c + z * s, c + y * y * one_c, y * z * one_c - x * s],
        [z * x * one_c - y * s, z * y * one_c + x * s, c + z * z * one_c],
    ]


@dataclass
class Transform:
    """Object-to-world affine transform p' = A p + t (transform.rs:11-21)."""

    a: list
    t: list

    @staticmethod
    def identity() -> "Transform":
        return Transform([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]], [0.0, 0.0, 0.0])

    @staticmethod
    def from_affine(a, t) -> "Transform":
        return Transform([list(map(float, r)) for r in a], list(map(float, t)))

    @staticmethod
    def translate(t: Vec) -> "Transform":
        return Transform.from_affine([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]], t)

    @staticmethod
    def rotate(axis: Vec, deg: float) -> "Transform":
        return Transform.from_affine(_rotation(axis, deg), [0.0, 0.0, 0.0])

    @staticmethod
    def scale(s: Vec) -> "Transform":
        return Transform.from_affine([[s[0], 0.0, 0.0], [0.0, s[1], 0.0], [0.0, 0.0, s[2]]], [0.0, 0.0, 0.0])

    @staticmethod
    def new(t: Vec, rot_y_deg: float, s: float) -> "Transform":  # transform.rs:38-40
        return Transform.from_affine(
            _mat_mul(_rotation([0.0, 1.0, 0.0], rot_y_deg), [[s, 0.0, 0.0], [0.0, s, 0.0], [0.0, 0.0, s]]), t
        )

    @staticmethod
    def from_matrix4(m) -> "Transform":  # transform.rs:61-67
        return Transform.from_affine([row[:3] for row in m[:3]], [m[0][3], m[1][3], m[2][3]])

    def compose(self, inner: "Transform") -> "Transform":  # transform.rs:70-72
        at = _mat_vec(self.a, inner.t)
        return Transform.from_affine(_mat_mul(self.a, inner.a), [at[0] + self.t[0], at[1] + self.t[1], at[2] + self.t[2]])

    def apply_point(self, p: Vec):  # transform.rs:75-77
        r = _mat_vec(self.a, p)
        return [r[0] + self.t[0], r[1] + self.t[1], r[2] + self.t[2]]


# ---- src/geometry.rs, src/world.rs ---------------------------------------------------------
@dataclass
class Sphere:
    c: tuple
    r: float
    mat_id: int


@dataclass
class Mesh:
    """Static triangle mesh: f64 positions (V,3), int32 indices (T,3) and a
    per-triangle material id (T,) -- Mesh::new over Triangle::new_static."""

    positions: np.ndarray
    indices: np.ndarray
    mat_ids: np.ndarray

    @staticmethod
    def from_arrays(positions, indices, mat_ids) -> "Mesh":
        p = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        i = np.ascontiguousarray(indices, dtype=np.int32).reshape(-1, 3)
        m = np.ascontiguousarray(np.broadcast_to(np.asarray(mat_ids, dtype=np.int32), (len(i),)))
        return Mesh(p, i, m)

    @property
    def n_tris(self) -> int:
        return int(self.indices.shape[0])


@dataclass
class Instance:
    mesh_id: int
    xform: Transform
    mat_override: Optional[int] = None


@dataclass
class World:
    spheres: List[Sphere] = field(default_factory=list)
    meshes: List[Mesh] = field(default_factory=list)
    instances: List[Instance] = field(default_factory=list)


# ---- src/env.rs -----------------------------------------------------------------------
@dataclass
class EnvMap:
    width: int
    height: int
    data: np.ndarray  # (h, w, 3) f64 linear RGB, row 0 = theta 0

    @staticmethod
    def from_pixels(w: int, h: int, data) -> "EnvMap":
        d = np.ascontiguousarray(np.asarray(data, dtype=np.float64).reshape(h, w, 3))
        return EnvMap(w, h, d)

    @staticmethod
    def constant(color: Vec) -> "EnvMap":
        return EnvMap.from_pixels(1, 1, np.array(color, dtype=np.float64))

    def scaled(self, factor: float) -> "EnvMap":
        if factor == 1.0:
            return self
        return EnvMap.from_pixels(self.width, self.height, self.data * factor)


@dataclass
class Scene:
    cam: Camera
    world: World
    mats: List[Material]
    env: Optional[EnvMap] = None

    def n_triangles(self) -> int:
        return sum(m.n_tris for m in self.world.meshes)


# ---- src/config.rs:5-92 -------------------------------------------------------------------
@dataclass
class RenderConfig:
    width: int = 1920
    height: int = 1080
    spp: int = 512
    max_bounces: int = 8
    rr_start: int = 3
    tile: int = 16
    adaptive_enabled: bool = False
    adaptive_min_spp: int = 8
    adaptive_threshold: float = 0.02
    morton_enabled: bool = True
    seed: int = 0
    mode: int = _abi.TPT_MODE_WAVEFRONT_FP32
    # row sharding (no counterpart in the reference): rows row_begin,
    # row_begin + row_step, ... of the film; row_step <= 0 = the whole film
    row_begin: int = 0
    row_step: int = 0

    def to_c(self) -> _abi.tpt_render_config:
        return _abi.tpt_render_config(
            int(self.width),
            int(self.height),
            int(self.spp),
            int(self.max_bounces),
            int(self.rr_start),
            int(self.tile),
            int(bool(self.adaptive_enabled)),
            int(self.adaptive_min_spp),
            float(self.adaptive_threshold),
            int(bool(self.morton_enabled)),
            int(self.mode),
            int(self.seed) & 0xFFFFFFFFFFFFFFFF,
            int(self.row_begin),
            int(self.row_step),
        )

    @property
    def film_rows(self) -> int:
        """Rows of the output film (all rows, or this shard's rows)."""
        if self.row_step <= 0:
            return self.height
        return max(0, -(-(self.height - self.row_begin) // self.row_step))

    @property
    def film_pixels(self) -> int:
        return self.width * self.film_rows


# ---- flattening ----------------------------------------------------------------------------------
class SceneDesc:
    """tpt_scene_desc for a Scene; keeps the backing arrays alive."""

    def __init__(self, scene: Scene):
        self._keep = []
        d = _abi.tpt_scene_desc()
        c = scene.cam
        d.camera = _abi.tpt_camera_desc(
            c.kind, 0, _abi.D3(*c.eye), _abi.D3(*c.target), _abi.D3(*c.up), c.fov_y_deg, c.aspect, c.focus_dist, c.aperture
        )
        w = scene.world
        sph = (_abi.tpt_sphere * max(len(w.spheres), 1))()
        for i, s in enumerate(w.spheres):
            sph[i] = _abi.tpt_sphere(_abi.D3(*s.c), float(s.r), int(s.mat_id))
        d.spheres, d.n_spheres = sph, len(w.spheres)
        meshes = (_abi.tpt_mesh_desc * max(len(w.meshes), 1))()
        for i, m in enumerate(w.meshes):
            self._keep += [m.positions, m.indices, m.mat_ids]
            meshes[i] = _abi.tpt_mesh_desc(
                m.positions.ctypes.data_as(C.POINTER(C.c_double)),
                m.positions.shape[0],
                m.indices.ctypes.data_as(C.POINTER(C.c_int32)),
                m.mat_ids.ctypes.data_as(C.POINTER(C.c_int32)),
                m.indices.shape[0],
            )
        d.meshes, d.n_meshes = meshes, len(w.meshes)
        inst = (_abi.tpt_instance_desc * max(len(w.instances), 1))()
        for i, x in enumerate(w.instances):
            a = [v for row in x.xform.a for v in row]
            inst[i] = _abi.tpt_instance_desc(
                int(x.mesh_id),
                (C.c_double * 9)(*a),
                _abi.D3(*x.xform.t),
                -1 if x.mat_override is None else int(x.mat_override),
            )
        d.instances, d.n_instances = inst, len(w.instances)
        mats = (_abi.tpt_material * max(len(scene.mats), 1))()
        for i, m in enumerate(scene.mats):
            mats[i] = _abi.tpt_material(m.kind, 0, _abi.D3(*m.rgb), float(m.param))
        d.materials, d.n_materials = mats, len(scene.mats)
        if scene.env is None:
            d.env = _abi.tpt_env_desc(_abi.TPT_ENV_NONE, 0, 0, 0, None)
        else:
            px = np.ascontiguousarray(scene.env.data, dtype=np.float64)
            self._keep.append(px)
            d.env = _abi.tpt_env_desc(
                _abi.TPT_ENV_MAP, scene.env.width, scene.env.height, 0, px.ctypes.data_as(C.POINTER(C.c_double))
            )
        self._keep += [sph, meshes, inst, mats]
        self.desc = d

    def ptr(self):
        return C.byref(self.desc)
