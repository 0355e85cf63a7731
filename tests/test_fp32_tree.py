"""The FP32 forms' mesh tree (tpt_bvh_build_fp32, host; no GPU).

The plain f64 form walks the reference's tree (src/bvh.rs:51-242), and
tests/test_host_lib.py and tests/test_golden.py pin that tree. The FP32 forms
walk a binned-SAH tree of their own over the same triangles. The closest
hit does not depend on the tree, so these tests check what a traversal
relies on:

* every triangle sits in exactly one leaf, and a leaf holds 1 to 6 of them
  (the leaf code's count field);
* a leaf's box is exactly the union of its triangles' padded boxes (the
  reference's Aabb::from_points pad of 1e-9, geometry.rs:70-80), and an
  interior node's box is exactly the union of its children's;
* nodes are numbered in preorder, the left child right after its parent;
* the depth fits the 64-entry traversal stack;
* the tree does not depend on the build's threads (two builds agree);
* it asks for fewer triangle tests than the reference's tree (surface-area
  estimate).
"""
import numpy as np
import pytest

from tinypt_b200 import bvh, scenes
from tinypt_b200.scene import Mesh


def _padded_boxes(m: Mesh):
    p = m.positions[m.indices]  # (T, 3, 3)
    return p.min(axis=1) - 1e-9, p.max(axis=1) + 1e-9


def _check_tree(m: Mesh, t) -> int:
    n_nodes = t.bbox.shape[0]
    leaf = (t.left_right[:, 0] == -1) & (t.left_right[:, 1] == -1)
    assert np.all((t.left_right[:, 0] == -1) == (t.left_right[:, 1] == -1))
    assert sorted(t.indices.tolist()) == list(range(m.n_tris))
    lo, hi = _padded_boxes(m)
    covered = np.zeros(m.n_tris, dtype=np.int64)
    depth = np.zeros(n_nodes, dtype=np.int64)
    depth[0] = 1
    for i in range(n_nodes):
        box = t.bbox[i]
        if leaf[i]:
            s, c = int(t.start_count[i, 0]), int(t.start_count[i, 1])
            assert 1 <= c <= 6
            tris = t.indices[s:s + c]
            covered[s:s + c] += 1
            assert np.array_equal(box[:3], lo[tris].min(axis=0))
            assert np.array_equal(box[3:], hi[tris].max(axis=0))
        else:
            l, r = int(t.left_right[i, 0]), int(t.left_right[i, 1])
            assert l == i + 1 and r > l and r < n_nodes
            depth[l] = depth[r] = depth[i] + 1
            both = t.bbox[[l, r]]
            assert np.array_equal(box[:3], both[:, :3].min(axis=0))
            assert np.array_equal(box[3:], both[:, 3:].max(axis=0))
    assert np.all(covered == 1)
    assert depth.max() <= 64
    return int(depth.max())


def _half_area(b):
    e = np.maximum(b[:, 3:] - b[:, :3], 0.0)
    return e[:, 0] * e[:, 1] + e[:, 1] * e[:, 2] + e[:, 2] * e[:, 0]


def _expected_tri_tests(t) -> float:
    """Triangle tests of a random line through the root box: the leaves'
    areas times their counts over the root's area."""
    leaf = t.left_right[:, 0] == -1
    a = _half_area(t.bbox)
    return float((a[leaf] * t.start_count[leaf, 1]).sum() / a[0])


MESHES = {
    # 81,920 triangles: above the size at which subtrees build on threads
    "icosphere_6": lambda: Mesh.from_arrays(*scenes.displaced_icosphere(6, 0.05, 5, 7), 0),
    "icosphere_2": lambda: Mesh.from_arrays(*scenes.displaced_icosphere(2, 0.05, 5, 7), 0),
    "one": lambda: Mesh.from_arrays(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float), np.array([[0, 1, 2]]), 0),
    "seven": lambda: Mesh.from_arrays(np.random.default_rng(3).normal(size=(21, 3)), np.arange(21).reshape(7, 3), 0),
    # every centroid the same point: ranges are halved until leaves fit
    "stacked": lambda: Mesh.from_arrays(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float),
                                        np.tile(np.array([[0, 1, 2]]), (100, 1)), 0),
}


@pytest.mark.parametrize("name", sorted(MESHES))
def test_fp32_tree_is_a_valid_tree(name):
    m = MESHES[name]()
    a = bvh.build(m, fp32=True)
    depth = _check_tree(m, a)
    b = bvh.build(m, fp32=True)
    for x, y in zip((a.bbox, a.left_right, a.start_count, a.indices), (b.bbox, b.left_right, b.start_count, b.indices)):
        assert np.array_equal(x, y)
    print(f"{name}: {a.bbox.shape[0]} nodes, depth {depth}")


def test_fp32_tree_tests_fewer_triangles_than_the_reference_tree():
    m = MESHES["icosphere_6"]()
    own, ref = bvh.build(m, fp32=True), bvh.build(m)
    assert ref.bbox.shape[0] == ref.left_right.shape[0]
    ratio = _expected_tri_tests(own) / _expected_tri_tests(ref)
    print(f"expected triangle tests: {ratio:.3f} of the reference tree's")
    assert ratio < 0.9


def test_fp32_tree_of_an_empty_mesh():
    m = Mesh.from_arrays(np.zeros((0, 3)), np.zeros((0, 3), dtype=np.int32), 0)
    t = bvh.build(m, fp32=True)
    assert t.bbox.shape[0] == 0 and t.indices.shape[0] == 0
