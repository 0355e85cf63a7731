"""The C-ABI library without a GPU: symbols, host BVH builder, error paths."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from tinypt_b200 import _abi, scenes
from tinypt_b200.scene import Mesh

HEADER = Path(__file__).resolve().parent.parent / "include" / "tinypt_cuda.h"


def _declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tpt_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _abi.lib()
    declared = _declared_symbols()
    assert "tpt_render" in declared and "tpt_scene_create" in declared
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_abi.SIGNATURES), "ctypes signatures must cover exactly the header"


def test_version_string():
    assert b"sm_100a" in _abi.lib().tpt_version()


def _desc(m: Mesh):
    return _abi.tpt_mesh_desc(
        m.positions.ctypes.data_as(C.POINTER(C.c_double)), m.positions.shape[0],
        m.indices.ctypes.data_as(C.POINTER(C.c_int32)), m.mat_ids.ctypes.data_as(C.POINTER(C.c_int32)), m.n_tris)


def _product_bvh(m: Mesh):
    d = _desc(m)
    L = _abi.lib()
    n = L.tpt_bvh_build_host(C.byref(d), None, None, None, None)
    assert n >= 0, L.tpt_last_error()
    bbox = np.zeros((n, 6))
    lr = np.zeros((n, 2), dtype=np.int32)
    sc = np.zeros((n, 2), dtype=np.uint32)
    idx = np.zeros(m.n_tris, dtype=np.int64)
    L.tpt_bvh_build_host(C.byref(d), bbox.ctypes.data_as(C.POINTER(C.c_double)),
                         lr.ctypes.data_as(C.POINTER(C.c_int32)), sc.ctypes.data_as(C.POINTER(C.c_uint32)),
                         idx.ctypes.data_as(C.POINTER(C.c_int64)))
    return bbox, lr, sc, idx


def _meshes():
    rng = np.random.default_rng(5)
    out = {}
    v, f = scenes.displaced_icosphere(4, 0.05, 5, 3)
    out["displaced_ico4"] = Mesh.from_arrays(v, f, 0)
    # triangle soup with random sizes
    p = rng.uniform(-3, 3, (3 * 700, 3)) + np.repeat(rng.uniform(-1, 1, (700, 1, 3)), 3, 1).reshape(-1, 3)
    out["soup"] = Mesh.from_arrays(p, np.arange(3 * 700).reshape(-1, 3), 0)
    # every centroid identical: SAH must fall back to n/2 splits
    q = np.tile(np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0]]), (40, 1))
    out["same_centroid"] = Mesh.from_arrays(q, np.arange(120).reshape(-1, 3), 0)
    # flat: all triangles in the plane z = 0 (zero extent on one axis)
    g = np.stack(np.meshgrid(np.arange(9.0), np.arange(9.0), indexing="ij"), -1).reshape(-1, 2)
    pts = np.concatenate([g, np.zeros((len(g), 1))], 1)
    tris = []
    for i in range(8):
        for j in range(8):
            a = i * 9 + j
            tris += [(a, a + 9, a + 1), (a + 1, a + 9, a + 10)]
    out["flat_grid"] = Mesh.from_arrays(pts, tris, 0)
    out["one_tri"] = Mesh.from_arrays([[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 1, 2]], 0)
    out["five_tris"] = Mesh.from_arrays(rng.uniform(0, 1, (15, 3)), np.arange(15).reshape(-1, 3), 0)
    out["seventeen"] = Mesh.from_arrays(rng.uniform(0, 1, (51, 3)), np.arange(51).reshape(-1, 3), 0)
    return out


@pytest.mark.parametrize("name", list(_meshes().keys()))
def test_product_bvh_matches_oracle_bit_for_bit(oracle_mod, name):
    m = _meshes()[name]
    got = _product_bvh(m)
    want = oracle_mod.bvh_build(_desc(m), m.n_tris)
    assert got[0].tobytes() == want[0].tobytes()
    for a, b in zip(got[1:], want[1:]):
        assert np.array_equal(a, b)


def test_empty_mesh_has_no_nodes():
    m = Mesh.from_arrays(np.zeros((0, 3)), np.zeros((0, 3), dtype=np.int32), 0)
    assert _abi.lib().tpt_bvh_build_host(C.byref(_desc(m)), None, None, None, None) == 0


def test_bad_index_is_rejected():
    m = Mesh.from_arrays([[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 1, 7]], 0)
    rc = _abi.lib().tpt_bvh_build_host(C.byref(_desc(m)), None, None, None, None)
    assert rc == _abi.TPT_ERR_INVALID
    assert b"out of range" in _abi.lib().tpt_last_error()


def test_scene_create_rejects_bad_material_before_touching_the_device():
    from tinypt_b200.scene import Camera, Material, Scene, SceneDesc, Sphere, World

    scene = Scene(Camera.look_at((0, 0, 3), (0, 0, 0), (0, 1, 0), 40, 1.0), World(spheres=[Sphere((0, 0, 0), 1, 5)]),
                  [Material.lambert((0.5, 0.5, 0.5))])
    d = SceneDesc(scene)
    h = C.c_void_p()
    rc = _abi.lib().tpt_scene_create(d.ptr(), C.byref(h))
    assert rc == _abi.TPT_ERR_INVALID and not h
    assert b"mat_id" in _abi.lib().tpt_last_error()
