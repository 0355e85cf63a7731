"""Device BVH builder (tpt_bvh_build_device): the same tree as the host
builder -- node boxes bit for bit, children, leaf ranges, leaf order -- on
the reference's golden meshes, on edge-case meshes (flat, coincident
centroids, lopsided SAH splits, tiny) and on the benchmark meshes; and scene
creation through it renders the same film as through the host builder."""
import ctypes as C
import json
import time
from pathlib import Path

import numpy as np
import pytest

from tinypt_b200 import _abi, bvh, scenes
from tinypt_b200.scene import Mesh

GOLD = json.loads((Path(__file__).parent / "golden" / "golden_vectors.json").read_text())


def _same(a: bvh.MeshBvh, b: bvh.MeshBvh) -> None:
    assert a.n_nodes == b.n_nodes
    assert a.bbox.tobytes() == b.bbox.tobytes()
    assert np.array_equal(a.left_right, b.left_right)
    assert np.array_equal(a.start_count, b.start_count)
    assert np.array_equal(a.indices, b.indices)


def _lopsided(n: int, base: float) -> Mesh:
    """Triangles at x = base**i: every SAH split peels a few off the top."""
    x = base ** np.arange(n, dtype=np.float64)
    s = 1e-3 * x
    p = np.stack([np.stack([x, 0 * x, 0 * x], 1), np.stack([x + s, 0 * x, 0 * x], 1),
                  np.stack([x, s, 0 * x], 1)], 1).reshape(-1, 3)
    return Mesh.from_arrays(p, np.arange(3 * n).reshape(-1, 3), 0)


def _outlier_chains(ratio: float = 2.0, cluster: int = 1100) -> Mesh:
    """A cluster of tiny triangles at the origin and, on each axis, a chain of
    triangles at 1e-6 * ratio**j up to 1e148: each SAH split peels the one
    outermost triangle, giving about 385 levels of nodes above the
    one-thread node size (areas stay finite, so every split is a SAH split)."""
    rng = np.random.default_rng(3)
    pts = [(rng.uniform(-1e-10, 1e-10, (cluster, 1, 3)) + rng.uniform(-1e-10, 1e-10, (cluster, 3, 3))).reshape(-1, 3)]
    vals = 1e-6 * ratio ** np.arange(int(np.log(1e148 / 1e-6) / np.log(ratio)) + 1)
    for a in range(3):
        for v in vals:
            t = np.zeros((3, 3))
            t[:, a] = v
            t[1, a] += 1e-3 * v
            t[2, (a + 1) % 3] += 1e-3 * v
            pts.append(t)
    p = np.concatenate(pts)
    return Mesh.from_arrays(p, np.arange(len(p)).reshape(-1, 3), 0)


def _edge_meshes():
    rng = np.random.default_rng(11)
    out = {}
    out["one_tri"] = Mesh.from_arrays([[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 1, 2]], 0)
    out["five_tris"] = Mesh.from_arrays(rng.uniform(0, 1, (15, 3)), np.arange(15).reshape(-1, 3), 0)
    out["seventeen"] = Mesh.from_arrays(rng.uniform(0, 1, (51, 3)), np.arange(51).reshape(-1, 3), 0)
    # coincident centroids above and below the one-thread node size
    for n in (120, 5000):
        q = np.tile(np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0]]), (n, 1))
        out[f"same_centroid_{n}"] = Mesh.from_arrays(q, np.arange(3 * n).reshape(-1, 3), 0)
    # a flat grid (zero extent on one axis), 80,000 triangles
    v, f, _ = scenes.heightfield(200, 200, 4.0, 0.0, 1)
    out["flat_grid_80k"] = Mesh.from_arrays(v, f, 0)
    # triangle soup, log-uniform sizes over six decades
    n = 100_000
    c = rng.uniform(-5, 5, (n, 1, 3))
    size = np.exp(rng.uniform(np.log(1e-4), np.log(1e2), (n, 1, 1)))
    out["soup_100k"] = Mesh.from_arrays((c + size * rng.normal(size=(n, 3, 3))).reshape(-1, 3),
                                        np.arange(3 * n).reshape(-1, 3), 0)
    # about 190 levels of lopsided splits above the one-thread node size
    out["lopsided_20k"] = _lopsided(20_000, 1.02)
    out["outlier_chains"] = _outlier_chains()
    return out


EDGE = _edge_meshes()


def _golden_mesh(entry):
    pos = np.array([[float.fromhex(x) for x in p] for p in entry["positions"]])
    return Mesh.from_arrays(pos, np.array(entry["tris"], dtype=np.int32), 0)


def _has_cuda() -> bool:
    import torch

    return torch.cuda.is_available()


@pytest.mark.skipif(_has_cuda(), reason="checks the no-device error path")
def test_device_builder_without_a_device_reports_a_cuda_error():
    m = EDGE["seventeen"]
    rc = _abi.lib().tpt_bvh_build_device(C.byref(bvh.mesh_desc(m)), None, None, None, None)
    assert rc == _abi.TPT_ERR_CUDA
    assert b"device BVH build" in _abi.lib().tpt_last_error()


def test_device_builder_rejects_bad_meshes_before_the_device():
    m = Mesh.from_arrays([[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 1, 7]], 0)
    rc = _abi.lib().tpt_bvh_build_device(C.byref(bvh.mesh_desc(m)), None, None, None, None)
    assert rc == _abi.TPT_ERR_INVALID
    assert b"out of range" in _abi.lib().tpt_last_error()
    assert _abi.lib().tpt_bvh_build_device(None, None, None, None, None) == _abi.TPT_ERR_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cube", "ico1", "ico2"])
def test_device_bvh_matches_golden_vectors(gpu, name):
    e = GOLD["bvh"][name]
    b = bvh.build(_golden_mesh(e), device=True)
    assert [[x.hex() for x in row] for row in b.bbox.tolist()] == e["bbox"]
    assert b.left_right.tolist() == e["left_right"]
    assert b.start_count.tolist() == e["start_count"]
    assert b.indices.tolist() == e["indices"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(EDGE.keys()))
def test_device_bvh_equals_host_bvh(gpu, name):
    m = EDGE[name]
    _same(bvh.build(m, device=True), bvh.build(m, device=False))


@pytest.mark.gpu
def test_device_bvh_empty_mesh(gpu):
    m = Mesh.from_arrays(np.zeros((0, 3)), np.zeros((0, 3), dtype=np.int32), 0)
    assert bvh.build(m, device=True).n_nodes == 0


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["displaced_ico8", "heightfield_256x512"])
def test_device_bvh_equals_host_bvh_on_benchmark_meshes(gpu, which):
    if which == "displaced_ico8":
        v, f = scenes.displaced_icosphere(8, 0.05, 5, 2026)  # the 1,310,720-triangle mesh+env mesh
    else:
        v, f, _ = scenes.heightfield(256, 512, 3.0, 0.35, 9)
    m = Mesh.from_arrays(v, f, 0)
    t0 = time.perf_counter()
    dev = bvh.build(m, device=True)
    t1 = time.perf_counter()
    host = bvh.build(m, device=False)
    t2 = time.perf_counter()
    _same(dev, host)
    print(f"{which}: {m.n_tris} tris, {dev.n_nodes} nodes, device {1e3 * (t1 - t0):.1f} ms, "
          f"host {1e3 * (t2 - t1):.1f} ms")


@pytest.mark.gpu
def test_scene_renders_identically_with_either_builder(gpu, monkeypatch):
    """The mesh+env scene (81,920-triangle mesh) through the device builder
    (the default at this size) and through TPT_BVH_BUILD=host: bit-identical
    FP32 films."""
    from tinypt_b200.render import render

    scene = scenes.mesh_env_scene(96, 64, subdiv=6, n_spheres=20, env_w=64, env_h=32)
    cfg = scenes.mesh_env_config(96, 64, spp=4)
    monkeypatch.delenv("TPT_BVH_BUILD", raising=False)
    a = render(scene, cfg)
    monkeypatch.setenv("TPT_BVH_BUILD", "host")
    b = render(scene, cfg)
    assert np.array_equal(a.acc, b.acc) and np.array_equal(a.acc_w, b.acc_w)
