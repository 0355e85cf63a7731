// GPU build of a mesh BVH with the reference's rules and node order.
#pragma once

#include <cstdint>
#include <functional>
#include <string>

#include "host_scene.hpp"

namespace tpt {

enum : int {
    kGpuBvhOk = 0,
    kGpuBvhUseHost = 1,     // a small node overflowed its thread's stack (a guard)
    kGpuBvhNoMemory = 2,    // a device allocation failed (nothing is left allocated)
    kGpuBvhCudaError = -1,  // another CUDA call failed (*err says which)
};

// Where a device build writes its tree (host memory; a NULL array is skipped).
struct GpuBvhSink {
    double* bbox;           // 6 per node
    int32_t* left_right;    // 2 per node
    uint32_t* start_count;  // 2 per node
    int64_t* indices;       // n_tris
};

// Builds the same BVH as build_mesh_bvh (src/bvh.rs:51-242) on the current
// CUDA device: identical node boxes, children, leaf ranges, leaf order and
// preorder numbering.  `sink` is called once with the node count and returns
// the arrays to fill; the maximum depth (root = 1) is reported when the sink
// returns at least one array.  Returns kGpuBvhOk, kGpuBvhUseHost (then
// build_mesh_bvh builds the tree; *err says why), kGpuBvhNoMemory (the
// device had no room: build_mesh_bvh can) or kGpuBvhCudaError.
// Throws std::runtime_error on a malformed mesh, like build_mesh_bvh.
int build_mesh_bvh_gpu(const double* positions, int64_t n_vertices, const int32_t* tri_idx, int64_t n_tris,
                       const std::function<GpuBvhSink(int64_t n_nodes)>& sink, int* max_depth,
                       int64_t* n_nodes, std::string* err);

// The same into a HostBvh.
int build_mesh_bvh_gpu(const double* positions, int64_t n_vertices, const int32_t* tri_idx, int64_t n_tris,
                       HostBvh& out, std::string* err);

// Meshes with at least this many triangles are built on the device when a
// scene is created (env TPT_BVH_BUILD=host|device overrides the choice).
constexpr int64_t kGpuBvhMinTris = 1 << 15;

}  // namespace tpt
