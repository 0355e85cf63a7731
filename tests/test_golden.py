"""Pins the oracle (and the product's host BVH builder) to the golden vectors of
tests/golden/make_golden.py, an independent pure-Python restatement of the
reference's RNG, seed, Morton tile order and BVH build."""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from tinypt_b200 import _abi
from tinypt_b200.scene import Mesh

GOLD = json.loads((Path(__file__).parent / "golden" / "golden_vectors.json").read_text())


def _mesh(entry):
    pos = np.array([[float.fromhex(x) for x in p] for p in entry["positions"]])
    return Mesh.from_arrays(pos, np.array(entry["tris"], dtype=np.int32), 0)


def _desc(m: Mesh):
    return _abi.tpt_mesh_desc(
        m.positions.ctypes.data_as(C.POINTER(C.c_double)), m.positions.shape[0],
        m.indices.ctypes.data_as(C.POINTER(C.c_int32)), m.mat_ids.ctypes.data_as(C.POINTER(C.c_int32)), m.n_tris)


@pytest.mark.parametrize("seed", list(GOLD["rng_u32"].keys()))
def test_rng_u32(oracle_mod, seed):
    got = oracle_mod.rng_u32(int(seed), 16)
    assert got.tolist() == GOLD["rng_u32"][seed]


@pytest.mark.parametrize("seed", list(GOLD["rng_f64"].keys()))
def test_rng_f64(oracle_mod, seed):
    got = oracle_mod.rng_f64(int(seed), 8)
    assert [float(x).hex() for x in got] == GOLD["rng_f64"][seed]


def test_seed_for(oracle_mod):
    for a, b, c, want in GOLD["seed_for"]:
        assert oracle_mod.seed_for(a, b, c) == want


def test_interleave_bits(oracle_mod):
    for v, want in GOLD["interleave_bits"]:
        assert oracle_mod.interleave_bits(v) == want


def test_tile_order(oracle_mod):
    for e in GOLD["tile_order"]:
        got = oracle_mod.tile_order(e["w"], e["h"], e["tile"], e["morton"])
        assert got.tolist() == [list(t) for t in e["tasks"]]


@pytest.mark.parametrize("name", ["cube", "ico1", "ico2"])
def test_bvh_oracle(oracle_mod, name):
    e = GOLD["bvh"][name]
    m = _mesh(e)
    bbox, lr, sc, idx = oracle_mod.bvh_build(_desc(m), m.n_tris)
    assert [[x.hex() for x in row] for row in bbox.tolist()] == e["bbox"]
    assert lr.tolist() == e["left_right"]
    assert sc.tolist() == e["start_count"]
    assert idx.tolist() == e["indices"]


@pytest.mark.parametrize("name", ["cube", "ico1", "ico2"])
def test_bvh_product_host_builder(name):
    e = GOLD["bvh"][name]
    m = _mesh(e)
    d = _desc(m)
    L = _abi.lib()
    n = L.tpt_bvh_build_host(C.byref(d), None, None, None, None)
    assert n == len(e["bbox"])
    bbox = np.zeros((n, 6))
    lr = np.zeros((n, 2), dtype=np.int32)
    sc = np.zeros((n, 2), dtype=np.uint32)
    idx = np.zeros(m.n_tris, dtype=np.int64)
    L.tpt_bvh_build_host(C.byref(d), bbox.ctypes.data_as(C.POINTER(C.c_double)),
                         lr.ctypes.data_as(C.POINTER(C.c_int32)), sc.ctypes.data_as(C.POINTER(C.c_uint32)),
                         idx.ctypes.data_as(C.POINTER(C.c_int64)))
    assert [[x.hex() for x in row] for row in bbox.tolist()] == e["bbox"]
    assert lr.tolist() == e["left_right"]
    assert sc.tolist() == e["start_count"]
    assert idx.tolist() == e["indices"]


def test_ground_truth_fixture():
    """The committed 65536-spp f64 ground truth of the 240x135 mesh+env film
    (made by tests/golden/make_mesh_env_truth.py) is complete and finite, and
    the error helpers behave on it."""
    from tinypt_b200 import precision

    img, meta = precision.load_truth()
    assert img.shape == (precision.TRUTH_WIDTH * precision.TRUTH_HEIGHT, 3)
    assert meta["spp"] == 65536 and meta["mode"] == "plain_f64" and meta["max_bounces"] == 16
    assert np.isfinite(img).all() and (img >= 0).all()
    e = precision.image_error(img, img)
    assert e["rmse"] == 0.0 and e["mean_rel_err"] == 0.0
    e2 = precision.image_error(img * 1.01, img)
    assert abs(e2["rel_rmse"] - 0.01 * np.sqrt(np.mean(img * img)) / img.mean()) < 1e-9
    assert precision.equal_rmse_speedup(20.0, 1.0, 1.0, 0.5) == 10.0


def test_cornell_ground_truth_fixture():
    """The committed 65536-spp f64 ground truth of the 160x90 Cornell film
    (made by tests/golden/make_cornell_truth.py): complete, finite, with
    black background pixels and the light's emission visible."""
    from tinypt_b200 import precision

    img, meta = precision.load_truth(precision.CORNELL_TRUTH_FILE)
    assert img.shape == (precision.CORNELL_WIDTH * precision.CORNELL_HEIGHT, 3)
    assert meta["spp"] == 65536 and meta["max_bounces"] == 32
    assert np.isfinite(img).all() and (img >= 0).all()
    assert (img.max(axis=1) == 0).any()
    assert img.max() <= 17.0 + 1e-6 and img.max() > 5.0
