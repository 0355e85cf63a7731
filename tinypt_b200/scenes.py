"""Scene builders: the reference's built-in scene, Mitsuba canonical shapes,
and seeded synthetic scenes for the benchmark workloads.

* ``build_scene`` -- the reference's default scene (src/scene.rs:26-95).
* ``unit_rectangle`` / ``unit_cube`` / ``unit_disk`` -- Mitsuba canonical
  shapes as the reference's XML loader generates them (src/mitsuba.rs:414-469).
* ``sphere_scene`` -- five spheres on a ground sphere under a 1x1 area light,
  black background (256x256, 64 spp, depth 8).
* ``mesh_env_scene`` -- a displaced icosphere (subdivision 8 = 1,310,720
  triangles) with 200 random spheres under a 1024x512 sky+sun env map
  (1920x1080, 256 spp, depth 16).

The synthetic generators are deterministic for a given seed (numpy PCG64 and
fixed integer hashing); no external data is used.
"""
from __future__ import annotations

import math

import numpy as np

from .scene import (
    Camera,
    EnvMap,
    Instance,
    Material,
    Mesh,
    RenderConfig,
    Scene,
    Sphere,
    Transform,
    World,
    color_from_srgb,
)
from . import _abi


# ---- Mitsuba canonical shapes (src/mitsuba.rs:414-469) --------------------------------
def unit_rectangle(mat_id: int) -> Mesh:
    p = [(-1.0, -1.0, 0.0), (1.0, -1.0, 0.0), (1.0, 1.0, 0.0), (-1.0, 1.0, 0.0)]
    return Mesh.from_arrays(p, [(0, 1, 2), (0, 2, 3)], mat_id)


def unit_cube(mat_id: int) -> Mesh:
    v = [(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1), (-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)]
    quads = [(0, 1, 2, 3), (4, 7, 6, 5), (0, 4, 5, 1), (1, 5, 6, 2), (2, 6, 7, 3), (3, 7, 4, 0)]
    tris = []
    for q in quads:
        tris.append((q[0], q[1], q[2]))
        tris.append((q[0], q[2], q[3]))
    return Mesh.from_arrays(np.array(v, dtype=np.float64), tris, mat_id)


def unit_disk(mat_id: int, n: int = 64) -> Mesh:
    pos = [(0.0, 0.0, 0.0)]
    tris = []
    for i in range(n):
        a0 = math.tau * i / n
        a1 = math.tau * (i + 1) / n
        pos.append((math.cos(a0), math.sin(a0), 0.0))
        pos.append((math.cos(a1), math.sin(a1), 0.0))
        tris.append((0, len(pos) - 2, len(pos) - 1))
    return Mesh.from_arrays(pos, tris, mat_id)


def add_mesh_instance(scene: Scene, mesh: Mesh, xform: Transform, mat_override=None) -> int:
    mesh_id = len(scene.world.meshes)
    scene.world.meshes.append(mesh)
    scene.world.instances.append(Instance(mesh_id, xform, mat_override))
    return mesh_id


# ---- src/scene.rs:26-95 ---------------------------------------------------------------
def build_scene(width: int = 1920, height: int = 1080) -> Scene:
    """The reference's built-in default scene (procedural sky, no env map)."""
    eye, target = (0.0, 1.2, 4.0), (0.0, 0.5, 0.0)
    focus = math.sqrt(sum((a - b) * (a - b) for a, b in zip(eye, target)))
    cam = Camera.look_at_dof(eye, target, (0.0, 1.0, 0.0), 40.0, width / height, focus, 0.0)
    mats = [
        Material.lambert(color_from_srgb(0.5, 0.5, 0.5)),
        Material.lambert(color_from_srgb(0.8, 0.3, 0.3)),
        Material.metal(color_from_srgb(0.8, 0.8, 0.8)),
        Material.ggx(color_from_srgb(0.95, 0.78, 0.35), 0.25),
        Material.dielectric(1.5, (0.02, 0.05, 0.02)),
        Material.diffuse_light((8.0, 7.0, 5.0)),
    ]
    w = World()
    w.spheres = [
        Sphere((0.0, -1000.0, 0.0), 1000.0, 0),
        Sphere((-1.8, 0.5, 0.0), 0.5, 1),
        Sphere((-0.6, 0.5, 0.0), 0.5, 2),
        Sphere((0.6, 0.5, 0.0), 0.5, 3),
        Sphere((1.8, 0.5, 0.0), 0.5, 4),
        Sphere((0.0, 3.0, -1.0), 0.8, 5),
    ]
    return Scene(cam, w, mats, None)


# ---- sphere scene: 256x256, 64 spp, depth 8 ----------------------------------------------
def sphere_scene(width: int = 256, height: int = 256) -> Scene:
    """Ground sphere + Lambert/Metal/GGX/Dielectric/Subsurface spheres under a
    1x1 downward-facing area light at y=3; black background (a constant black
    env map, as the reference's XML loader installs)."""
    cam = Camera.look_at((0.0, 1.2, 4.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 40.0, width / height)
    mats = [
        Material.lambert((0.5, 0.5, 0.5)),
        Material.lambert((0.8, 0.3, 0.3)),
        Material.metal((0.9, 0.9, 0.9)),
        Material.ggx((0.95, 0.78, 0.35), 0.25),
        Material.dielectric(1.5, (0.0, 0.0, 0.0)),
        Material.subsurface((0.9, 0.6, 0.5), 0.1),
        Material.diffuse_light((10.0, 10.0, 10.0)),
    ]
    w = World()
    w.spheres.append(Sphere((0.0, -1000.0, 0.0), 1000.0, 0))
    for i, x in enumerate((-2.0, -1.0, 0.0, 1.0, 2.0)):
        w.spheres.append(Sphere((x, 0.5, 0.0), 0.5, 1 + i))
    scene = Scene(cam, w, mats, EnvMap.constant((0.0, 0.0, 0.0)))
    # 1x1 rectangle at y=3 facing down: translate . rotate(x, 90) . scale(0.5)
    xf = (
        Transform.identity()
        .compose(Transform.translate((0.0, 3.0, 0.0)))
        .compose(Transform.rotate((1.0, 0.0, 0.0), 90.0))
        .compose(Transform.scale((0.5, 0.5, 1.0)))
    )
    add_mesh_instance(scene, unit_rectangle(6), xf)
    return scene


def sphere_scene_config(width: int = 256, height: int = 256, spp: int = 64) -> RenderConfig:
    return RenderConfig(width=width, height=height, spp=spp, max_bounces=8, rr_start=3, seed=1)


# ---- icosphere + fBm ---------------------------------------------------------------------------
def icosphere(subdiv: int):
    """Unit icosphere: 20 * 4**subdiv triangles (edge midpoints re-projected)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array(
        [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
         [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]],
        dtype=np.float64,
    )
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(
        [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
         [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11],
         [6, 2, 10], [8, 6, 7], [9, 8, 1]],
        dtype=np.int64,
    )
    for _ in range(subdiv):
        nf = len(f)
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        lo, hi = np.minimum(e[:, 0], e[:, 1]), np.maximum(e[:, 0], e[:, 1])
        key = lo * len(v) + hi
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // len(v), uniq % len(v)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        m01, m12, m20 = base + inv[:nf], base + inv[nf:2 * nf], base + inv[2 * nf:]
        f = np.concatenate(
            [
                np.stack([f[:, 0], m01, m20], 1),
                np.stack([f[:, 1], m12, m01], 1),
                np.stack([f[:, 2], m20, m12], 1),
                np.stack([m01, m12, m20], 1),
            ]
        )
    return v, f.astype(np.int32)


def _hash3(ix, iy, iz, seed: int) -> np.ndarray:
    """Integer lattice hash -> float in [-1, 1] (uint64 wrap-around mixing)."""
    with np.errstate(over="ignore"):
        h = (ix.astype(np.uint64) * np.uint64(0x9E3779B185EBCA87)
             ^ iy.astype(np.uint64) * np.uint64(0xC2B2AE3D27D4EB4F)
             ^ iz.astype(np.uint64) * np.uint64(0x165667B19E3779F9)
             ^ np.uint64(seed & 0xFFFFFFFFFFFFFFFF) * np.uint64(0xD6E8FEB86659FD93))
        h ^= h >> np.uint64(32)
        h *= np.uint64(0xD6E8FEB86659FD93)
        h ^= h >> np.uint64(32)
    return (h >> np.uint64(11)).astype(np.float64) * (2.0 / 9007199254740992.0) - 1.0


def value_noise3(p: np.ndarray, seed: int) -> np.ndarray:
    """Trilinear value noise with smoothstep weights, range [-1, 1]."""
    pf = np.floor(p)
    pi = pf.astype(np.int64)
    f = p - pf
    u = f * f * (3.0 - 2.0 * f)
    out = np.zeros(len(p))
    for dx in (0, 1):
        wx = u[:, 0] if dx else 1.0 - u[:, 0]
        for dy in (0, 1):
            wy = u[:, 1] if dy else 1.0 - u[:, 1]
            for dz in (0, 1):
                wz = u[:, 2] if dz else 1.0 - u[:, 2]
                out += wx * wy * wz * _hash3(pi[:, 0] + dx, pi[:, 1] + dy, pi[:, 2] + dz, seed)
    return out


def fbm(p: np.ndarray, octaves: int, seed: int, base_freq: float = 2.0) -> np.ndarray:
    total = np.zeros(len(p))
    norm = 0.0
    amp, freq = 1.0, base_freq
    for o in range(octaves):
        total += amp * value_noise3(p * freq, seed + 7919 * o)
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def displaced_icosphere(subdiv: int, amplitude: float, octaves: int, seed: int):
    v, f = icosphere(subdiv)
    r = 1.0 + amplitude * fbm(v, octaves, seed)
    return v * r[:, None], f


# ---- env map: gradient sky, lognormal noise, Gaussian sun lobe ------------------------------
def sky_env(width: int = 1024, height: int = 512, seed: int = 0, sigma: float = 0.5, sun_peak: float = 1e4,
            sun_width_deg: float = 0.5, sun_elev_deg: float = 35.0, sun_azim_deg: float = 60.0) -> EnvMap:
    """Equirect float32 RGB env map in the reference's layout (row 0 is theta=0,
    u = phi / 2pi with dir = (cos phi sin theta, cos theta, sin phi sin theta))."""
    rng = np.random.default_rng(seed)
    theta = math.pi * (np.arange(height) + 0.5) / height
    phi = math.tau * (np.arange(width) + 0.5) / width
    th, ph = np.meshgrid(theta, phi, indexing="ij")
    elev = math.pi / 2 - th
    up = np.clip(elev / (math.pi / 2), 0.0, 1.0) ** 0.5
    zen, hor, gnd = np.array([0.25, 0.45, 1.0]), np.array([1.0, 0.9, 0.8]), np.array([0.3, 0.26, 0.22])
    sky = (1.0 - up)[..., None] * hor + up[..., None] * zen
    ground = gnd * (0.6 + 0.4 * np.clip(1.0 + elev / (math.pi / 2), 0.0, 1.0))[..., None]
    img = np.where((elev > 0)[..., None], sky, ground)
    img = img * np.exp(sigma * rng.standard_normal((height, width))[..., None] - 0.5 * sigma * sigma)
    se, sa = math.radians(sun_elev_deg), math.radians(sun_azim_deg)
    s = np.array([math.cos(sa) * math.cos(se), math.sin(se), math.sin(sa) * math.cos(se)])
    d = np.stack([np.cos(ph) * np.sin(th), np.cos(th), np.sin(ph) * np.sin(th)], -1)
    ang = np.arccos(np.clip(d @ s, -1.0, 1.0))
    w = math.radians(sun_width_deg)
    img = img + sun_peak * np.exp(-0.5 * (ang / w) ** 2)[..., None] * np.array([1.0, 0.95, 0.9])
    img32 = img.astype(np.float32)
    return EnvMap.from_pixels(width, height, img32.astype(np.float64))


# ---- mesh + env scene: 1080p, 1.31M triangles + 200 spheres, 256 spp, depth 16 --------------
def mesh_env_scene(width: int = 1920, height: int = 1080, subdiv: int = 8, n_spheres: int = 200,
                   env_w: int = 1024, env_h: int = 512, seed: int = 2024) -> Scene:
    cam = Camera.look_at((0.0, 1.6, 6.5), (0.0, 0.4, 0.0), (0.0, 1.0, 0.0), 40.0, width / height)
    mats = [Material.ggx((0.95, 0.64, 0.54), 0.3)]
    rng = np.random.default_rng(seed)
    w = World()
    for _ in range(n_spheres):
        r = float(rng.uniform(0.05, 0.2))
        c = (float(rng.uniform(-4, 4)), float(rng.uniform(0, 1)), float(rng.uniform(-4, 4)))
        kind = int(rng.integers(0, 3))
        albedo = tuple(float(x) for x in rng.uniform(0.1, 0.9, 3))
        alpha = float(rng.uniform(0.05, 0.5))
        if kind == 0:
            mats.append(Material.lambert(albedo))
        elif kind == 1:
            mats.append(Material.ggx(albedo, alpha))
        else:
            mats.append(Material.dielectric(1.5, (0.0, 0.0, 0.0)))
        w.spheres.append(Sphere(c, r, len(mats) - 1))
    scene = Scene(cam, w, mats, sky_env(env_w, env_h, seed + 1))
    v, f = displaced_icosphere(subdiv, 0.05, 5, seed + 2)
    add_mesh_instance(scene, Mesh.from_arrays(v, f, 0), Transform.identity())
    return scene


def mesh_env_config(width: int = 1920, height: int = 1080, spp: int = 256) -> RenderConfig:
    return RenderConfig(width=width, height=height, spp=spp, max_bounces=16, rr_start=3, seed=1)


# ---- inverse-rendering scene: 262,144-triangle heightfield in 16 GGX material groups -------
def heightfield(nx: int, nz: int, extent: float, amplitude: float, seed: int):
    """(nx x nz quads, 2 triangles each) fBm heightfield over [-extent, extent]^2
    at y = height; returns vertices, faces and each face's (ix, iz) quad."""
    xs = np.linspace(-extent, extent, nx + 1)
    zs = np.linspace(-extent, extent, nz + 1)
    X, Z = np.meshgrid(xs, zs, indexing="ij")
    p = np.stack([X.ravel(), np.zeros(X.size), Z.ravel()], 1)
    y = amplitude * fbm(p * 0.5, 5, seed)
    v = np.stack([X.ravel(), y, Z.ravel()], 1)
    ix, iz = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    a = (ix * (nz + 1) + iz).ravel()
    b = a + (nz + 1)
    f = np.concatenate([np.stack([a, a + 1, b], 1), np.stack([b, a + 1, b + 1], 1)])
    quad = np.concatenate([np.stack([ix.ravel(), iz.ravel()], 1)] * 2)
    return v, f.astype(np.int32), quad


def inverse_params(seed: int = 5, n_groups: int = 16) -> np.ndarray:
    """Seeded ground-truth parameters, (n_groups, 4): GGX albedo rgb, alpha."""
    rng = np.random.default_rng(seed)
    return np.concatenate([rng.uniform(0.2, 0.9, (n_groups, 3)), rng.uniform(0.1, 0.6, (n_groups, 1))], 1)


def inverse_scene(width: int = 512, height: int = 512, nx: int = 256, nz: int = 512, params=None,
                  env_w: int = 512, env_h: int = 256, seed: int = 11) -> Scene:
    """Heightfield of nx*nz*2 triangles (262,144 by default) split into a 4 x 4
    grid of material groups, one GGX material each (albedo rgb + alpha from
    `params`, default inverse_params()), under a 512x256 float32 sky."""
    params = inverse_params() if params is None else np.asarray(params, dtype=np.float64)
    n_groups = len(params)
    side = int(round(math.sqrt(n_groups)))
    if side * side != n_groups:
        raise ValueError(f"{n_groups} material groups do not form a square grid")
    mats = [Material.ggx(tuple(p[:3]), float(p[3])) for p in params]
    cam = Camera.look_at((0.0, 3.2, 4.2), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 45.0, width / height)
    scene = Scene(cam, World(), mats, sky_env(env_w, env_h, seed, sun_peak=200.0, sun_width_deg=3.0))
    v, f, quad = heightfield(nx, nz, 2.0, 0.35, seed + 1)
    group = (quad[:, 0] * side // nx) * side + (quad[:, 1] * side // nz)
    add_mesh_instance(scene, Mesh.from_arrays(v, f, group), Transform.identity())
    return scene


def gradcheck_scene(width: int = 64, height: int = 64, seed: int = 3) -> Scene:
    """Small scene with every differentiable parameter in play: Lambert
    ground, GGX / Metal / absorbing Dielectric / Subsurface / Lambert spheres,
    a 1.5 x 1.5 downward-facing area light (DiffuseLight) and a sky env map
    with a soft sun (env NEE, MIS on misses)."""
    cam = Camera.look_at((0.0, 1.4, 4.2), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 45.0, width / height)
    mats = [
        Material.lambert((0.6, 0.55, 0.5)),
        Material.ggx((0.9, 0.7, 0.4), 0.3),
        Material.metal((0.8, 0.85, 0.9)),
        Material.dielectric(1.5, (0.3, 0.1, 0.05)),
        Material.subsurface((0.8, 0.5, 0.4), 0.05),
        Material.lambert((0.3, 0.6, 0.3)),
        Material.diffuse_light((6.0, 5.0, 4.0)),
    ]
    w = World()
    w.spheres.append(Sphere((0.0, -1000.0, 0.0), 1000.0, 0))
    for i, x in enumerate((-2.2, -1.1, 0.0, 1.1, 2.2)):
        w.spheres.append(Sphere((x, 0.5, 0.0), 0.5, 1 + i))
    scene = Scene(cam, w, mats, sky_env(128, 64, seed, sun_peak=20.0, sun_width_deg=5.0))
    xf = (
        Transform.identity()
        .compose(Transform.translate((0.0, 3.0, 0.5)))
        .compose(Transform.rotate((1.0, 0.0, 0.0), 90.0))
        .compose(Transform.scale((0.75, 0.75, 1.0)))
    )
    add_mesh_instance(scene, unit_rectangle(6), xf)
    return scene


# ---- batch workload: 64 scenes of uneven size --------------------------------------------------
def _log_uniform(rng, lo: float, hi: float) -> float:
    return float(math.exp(rng.uniform(math.log(lo), math.log(hi))))


def batch_scene(seed: int, n_tris: int, width: int, height: int) -> Scene:
    """One scene of the batch workload: about n_tris triangles of displaced
    icospheres and boxes on a ground box, a random material mix, one
    rectangular area light (emit uniform 5-50) and a black background."""
    rng = np.random.default_rng(seed)
    mats = [Material.lambert(tuple(rng.uniform(0.3, 0.8, 3)))]          # ground
    light = float(rng.uniform(5.0, 50.0))
    mats.append(Material.diffuse_light((light, light * 0.95, light * 0.9)))
    for _ in range(6):
        k = int(rng.integers(0, 4))
        albedo = tuple(float(x) for x in rng.uniform(0.15, 0.9, 3))
        if k == 0:
            mats.append(Material.lambert(albedo))
        elif k == 1:
            mats.append(Material.ggx(albedo, float(rng.uniform(0.05, 0.5))))
        elif k == 2:
            mats.append(Material.metal(albedo))
        else:
            mats.append(Material.dielectric(1.5, tuple(float(x) for x in rng.uniform(0.0, 0.3, 3))))
    az = float(rng.uniform(0.0, math.tau))
    eye = (6.0 * math.cos(az), 2.5, 6.0 * math.sin(az))
    cam = Camera.look_at(eye, (0.0, 0.6, 0.0), (0.0, 1.0, 0.0), 40.0, width / height)
    scene = Scene(cam, World(), mats, EnvMap.constant((0.0, 0.0, 0.0)))
    ground = (Transform.identity().compose(Transform.translate((0.0, -0.05, 0.0)))
              .compose(Transform.scale((5.0, 0.05, 5.0))))
    add_mesh_instance(scene, unit_cube(0), ground)
    budget = max(int(n_tris) - 12, 20)
    n_obj = int(rng.integers(1, 5))
    for o in range(n_obj):
        share = budget // n_obj
        sub = int(min(max(round(math.log(max(share / 20.0, 1.0), 4)), 0), 7))
        v, f = displaced_icosphere(sub, 0.08, 4, seed * 31 + o)
        r = float(rng.uniform(0.3, 1.0))
        c = (float(rng.uniform(-2.5, 2.5)), r, float(rng.uniform(-2.5, 2.5)))
        xf = Transform.identity().compose(Transform.translate(c)).compose(Transform.scale((r, r, r)))
        add_mesh_instance(scene, Mesh.from_arrays(v, f, 2 + int(rng.integers(0, 6))), xf)
    for b in range(int(rng.integers(1, 4))):
        s = float(rng.uniform(0.2, 0.6))
        c = (float(rng.uniform(-3.0, 3.0)), s, float(rng.uniform(-3.0, 3.0)))
        xf = (Transform.identity().compose(Transform.translate(c))
              .compose(Transform.rotate((0.0, 1.0, 0.0), float(rng.uniform(0, 90))))
              .compose(Transform.scale((s, s, s))))
        add_mesh_instance(scene, unit_cube(2 + int(rng.integers(0, 6))), xf)
    lx = (Transform.identity().compose(Transform.translate((0.0, 4.0, 0.0)))
          .compose(Transform.rotate((1.0, 0.0, 0.0), 90.0)).compose(Transform.scale((1.2, 1.2, 1.0))))
    add_mesh_instance(scene, unit_rectangle(1), lx)
    return scene


def batch_workload(n_scenes: int = 64, seed: int = 77, tri_range=(1_000, 500_000), res_range=(128, 1024),
                   spp_range=(16, 256), max_depth: int = 12):
    """[(scene, RenderConfig)]: triangle counts, square resolutions and spp
    log-uniform over the given ranges (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_scenes):
        n_tris = int(_log_uniform(rng, *tri_range))
        res = int(round(_log_uniform(rng, *res_range) / 8.0)) * 8
        res = max(res, 8)
        spp = int(round(_log_uniform(rng, *spp_range)))
        scene = batch_scene(seed * 1000 + k, n_tris, res, res)
        cfg = RenderConfig(width=res, height=res, spp=spp, max_bounces=max_depth, rr_start=3, seed=k + 1,
                           mode=_abi.TPT_MODE_WAVEFRONT_FP32)
        out.append((scene, cfg))
    return out


# ---- adaptive-sampling scene: Cornell box + 262,144-triangle GGX mesh + absorbing glass ----------
def uv_sphere(n_lat: int, n_lon: int):
    """Latitude-longitude sphere of 2 * n_lat * n_lon triangles (the pole rows
    keep their degenerate triangles, so the count is exact)."""
    th = np.linspace(0.0, math.pi, n_lat + 1)
    ph = np.linspace(0.0, math.tau, n_lon + 1)
    T, P = np.meshgrid(th, ph, indexing="ij")
    v = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], -1).reshape(-1, 3)
    i, j = np.meshgrid(np.arange(n_lat), np.arange(n_lon), indexing="ij")
    a = (i * (n_lon + 1) + j).ravel()
    b = a + (n_lon + 1)
    f = np.concatenate([np.stack([a, b, a + 1], 1), np.stack([a + 1, b, b + 1], 1)])
    return v, f.astype(np.int32)


def cornell_scene(width: int = 1920, height: int = 1080, n_lat: int = 256, n_lon: int = 512, seed: int = 17) -> Scene:
    """Cornell box of 6 rectangles (Lambert red / green / white walls), a
    0.5 x 0.5 ceiling light emitting (17, 12, 4) and 2 white cubes, plus a
    displaced GGX mesh of 2 * n_lat * n_lon triangles (262,144 by default,
    alpha 0.1) and a Dielectric sphere (ior 1.5, absorption (0.2, 0.05, 0.05));
    black background.  The box spans [-1, 1]^3."""
    red, green, white = (0.63, 0.065, 0.05), (0.14, 0.45, 0.09), (0.725, 0.71, 0.68)
    mats = [Material.lambert(red), Material.lambert(green), Material.lambert(white),
            Material.diffuse_light((17.0, 12.0, 4.0)), Material.ggx((0.9, 0.75, 0.45), 0.1),
            Material.dielectric(1.5, (0.2, 0.05, 0.05))]
    cam = Camera.look_at((0.0, 0.0, 3.9), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 40.0, width / height)
    scene = Scene(cam, World(), mats, EnvMap.constant((0.0, 0.0, 0.0)))

    def wall(mat, t, axis, deg, sx=1.0, sy=1.0):
        xf = Transform.identity().compose(Transform.translate(t))
        if axis is not None:
            xf = xf.compose(Transform.rotate(axis, deg))
        add_mesh_instance(scene, unit_rectangle(mat), xf.compose(Transform.scale((sx, sy, 1.0))))

    wall(2, (0.0, 0.0, -1.0), None, 0.0)                       # back (normal +z)
    wall(2, (0.0, -1.0, 0.0), (1.0, 0.0, 0.0), -90.0)          # floor (normal +y)
    wall(2, (0.0, 1.0, 0.0), (1.0, 0.0, 0.0), 90.0)            # ceiling (normal -y)
    wall(0, (-1.0, 0.0, 0.0), (0.0, 1.0, 0.0), 90.0)           # left, red (normal +x)
    wall(1, (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), -90.0)           # right, green (normal -x)
    wall(3, (0.0, 0.999, 0.0), (1.0, 0.0, 0.0), 90.0, 0.25, 0.25)  # light, 0.5 x 0.5 facing down
    for c, s, yaw in (((-0.45, -0.7, -0.35), 0.3, 18.0), ((0.5, -0.75, 0.45), 0.25, -20.0)):
        xf = (Transform.identity().compose(Transform.translate(c))
              .compose(Transform.rotate((0.0, 1.0, 0.0), yaw)).compose(Transform.scale((s, s, s))))
        add_mesh_instance(scene, unit_cube(2), xf)
    v, f = uv_sphere(n_lat, n_lon)
    v = v * (1.0 + 0.06 * fbm(v, 5, seed))[:, None]
    xf = Transform.identity().compose(Transform.translate((-0.45, -0.05, -0.35))).compose(
        Transform.scale((0.3, 0.3, 0.3)))
    add_mesh_instance(scene, Mesh.from_arrays(v, f, 4), xf)
    scene.world.spheres.append(Sphere((0.45, -0.2, 0.45), 0.25, 5))
    return scene


def cornell_config(width: int = 1920, height: int = 1080, spp: int = 4096) -> RenderConfig:
    """Adaptive sampling: up to spp samples, stop when the relative standard
    deviation of the samples' luminance is below 0.01 (after 8), depth 32."""
    return RenderConfig(width=width, height=height, spp=spp, max_bounces=32, rr_start=3, seed=1,
                        adaptive_enabled=True, adaptive_min_spp=8, adaptive_threshold=0.01,
                        mode=_abi.TPT_MODE_WAVEFRONT_FP32)
