"""Mesh BVHs in the reference layout, built on the host or on the device.

Both builders follow Bvh::build (src/bvh.rs:51-242): 8 SAH bins on the
largest centroid axis (nodes of 16 or more triangles with a centroid extent
above 1e-12), a stable reorder of the node's triangles by bin, leaves of at
most 4 triangles, nodes numbered in preorder.  The device builder returns
the host builder's tree node for node (boxes bit for bit).
"""
from __future__ import annotations

import ctypes as C
from typing import NamedTuple

import numpy as np

from . import _abi
from .scene import Mesh


class MeshBvh(NamedTuple):
    bbox: np.ndarray         # (n, 6) f64: min xyz, max xyz
    left_right: np.ndarray   # (n, 2) i32: children, -1 for leaves
    start_count: np.ndarray  # (n, 2) u32: leaf triangle range
    indices: np.ndarray      # (n_tris,) i64: triangles in leaf order

    @property
    def n_nodes(self) -> int:
        return self.bbox.shape[0]


def mesh_desc(m: Mesh) -> _abi.tpt_mesh_desc:
    """The C description of a mesh (borrows the mesh's arrays)."""
    return _abi.tpt_mesh_desc(
        m.positions.ctypes.data_as(C.POINTER(C.c_double)), m.positions.shape[0],
        m.indices.ctypes.data_as(C.POINTER(C.c_int32)), m.mat_ids.ctypes.data_as(C.POINTER(C.c_int32)), m.n_tris)


def build(mesh: Mesh, device: bool = False, fp32: bool = False) -> MeshBvh:
    """The mesh's BVH from tpt_bvh_build_host, or tpt_bvh_build_device on
    the current CUDA device; with fp32=True the FP32 forms' own tree
    (tpt_bvh_build_fp32, host).  Raises TinyptError on failure."""
    L = _abi.lib()
    fn = L.tpt_bvh_build_fp32 if fp32 else (L.tpt_bvh_build_device if device else L.tpt_bvh_build_host)
    d = mesh_desc(mesh)
    # A tree over n triangles has at most 2n - 1 nodes; pages past the
    # node count are never touched.
    cap = 2 * max(mesh.n_tris, 1)
    bbox = np.empty((cap, 6))
    lr = np.empty((cap, 2), dtype=np.int32)
    sc = np.empty((cap, 2), dtype=np.uint32)
    idx = np.empty(mesh.n_tris, dtype=np.int64)
    n = fn(C.byref(d), bbox.ctypes.data_as(C.POINTER(C.c_double)), lr.ctypes.data_as(C.POINTER(C.c_int32)),
           sc.ctypes.data_as(C.POINTER(C.c_uint32)), idx.ctypes.data_as(C.POINTER(C.c_int64)))
    if n < 0:
        _abi.check(int(n))
    return MeshBvh(bbox[:n], lr[:n], sc[:n], idx)
