// Host-side scene model of the B200 path integrator.
//
// tpt_scene_desc (include/tinypt_cuda.h) is turned into:
//   * the f64 quantities the reference computes once per scene -- camera basis
//     (src/ray.rs:36-86), instance transforms with inverse and inverse-
//     transpose (src/transform.rs:24-27), per-mesh binned-SAH BVHs in the
//     reference's node order (src/bvh.rs:51-242), the light table and CDF
//     (src/world.rs:127-167) and the env-map CDFs (src/env.rs:61-89) -- which
//     must equal the reference bit for bit, because the f64 kernel reproduces
//     the reference's per-pixel RNG stream;
//   * the device layouts both kernels read (f64 arrays for the plain kernel;
//     32-byte-aligned FP32 BVH2 nodes, precomputed-edge triangles and float4
//     env texels for the wavefront kernels).
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "../../include/tinypt_cuda.h"
#include "device_types.h"

namespace tpt {

struct HVec { double x = 0, y = 0, z = 0; };

// One mesh BVH in the reference layout: node bbox (min xyz, max xyz), child
// indices (-1 for leaves), leaf triangle range, leaf order of triangles.
struct HostBvh {
    std::vector<double> bbox;          // 6 per node
    std::vector<int32_t> left_right;   // 2 per node
    std::vector<uint32_t> start_count; // 2 per node
    std::vector<int64_t> indices;      // leaf order
    int max_depth = 0;                 // root = depth 1
};

// Builds the reference BVH of one mesh (src/bvh.rs:51-242): same splits,
// same stable reordering, same preorder node numbering.
HostBvh build_mesh_bvh(const double* positions, int64_t n_vertices, const int32_t* indices, int64_t n_tris);

// Builds the mesh tree of the FP32 forms (fp32_tree.cpp): binned SAH over
// three axes, leaves of up to 6 triangles chosen by cost, in the same
// layout as build_mesh_bvh's.
HostBvh build_fp32_mesh_bvh(const double* positions, int64_t n_vertices, const int32_t* indices, int64_t n_tris);

struct HostLight {
    int32_t is_sphere;
    int64_t sphere;                      // sphere index
    int64_t mesh, tri, inst;             // triangle light
    int64_t mat;                         // emitter material
    double emit[3];
    double weight;
};

// Everything derived from a tpt_scene_desc on the host.
struct HostScene {
    CameraF64 cam;
    std::vector<tpt_material> mats;
    // Materials the samplers see (GGX alpha of the VNDF sampler and of the
    // pdfs used in weights and MIS, light-selection weights).  Equal to mats
    // unless set apart by set_materials, which detaches sampling from
    // evaluation for derivative checks.
    std::vector<tpt_material> smats;
    std::vector<tpt_sphere> spheres;
    struct Mesh {
        std::vector<double> pos;       // n_vertices*3
        std::vector<int32_t> idx;      // n_tris*3
        std::vector<int32_t> mat;      // n_tris
        HostBvh bvh;
    };
    std::vector<Mesh> meshes;
    std::vector<InstanceF64> instances;
    std::vector<HostLight> lights;
    std::vector<double> light_cdf;
    double light_total = 0;
    // env map
    int32_t env_kind = TPT_ENV_NONE;
    int32_t env_w = 0, env_h = 0;
    std::vector<double> env_data, env_row_cdf, env_col_cdf;
    double env_total = 0;
};

// Builds one (validated) mesh's BVH; the result must equal build_mesh_bvh's.
using MeshBvhBuilder = std::function<HostBvh(const tpt_mesh_desc& mesh)>;

// Throws std::runtime_error on a malformed description.  Mesh BVHs come from
// `bvh` when given, else from build_mesh_bvh.
void build_host_scene(const tpt_scene_desc& desc, HostScene& out, const MeshBvhBuilder& bvh = nullptr);

// World::build_lights (src/world.rs:127-167) over hs.smats (which primitives
// are lights and their selection weights) with the emission of hs.mats.
void build_lights(HostScene& hs);

// Replaces the materials (same count and kinds); sampling = nullptr means
// sampling follows evaluation.  Rebuilds the light table.
void set_materials(HostScene& hs, const tpt_material* mats, const tpt_material* sampling, size_t n);

// FP32 material and light tables of flatten_fp32, alone (for set_materials).
void flatten_fp32_materials(const HostScene& hs, std::vector<MaterialF32>& mats, std::vector<LightF32>& lights,
                            std::vector<float>& light_cdf);
// f64 material and light tables of flatten_plain, alone.
void flatten_plain_materials(const HostScene& hs, std::vector<MaterialF64>& mats, std::vector<LightF64>& lights);

// ---- flattened device images (host copies, uploaded by the C ABI) -------
struct PlainImage {      // f64 layout for the plain kernel
    std::vector<NodeF64> nodes;
    std::vector<TriF64> tris;                // leaf order, per mesh contiguous
    std::vector<MeshF64> meshes;
    std::vector<InstanceF64> instances;
    std::vector<SphereF64> spheres;
    std::vector<MaterialF64> mats;
    std::vector<LightF64> lights;
    std::vector<double> light_cdf;
    std::vector<double> env_data, env_row_cdf, env_col_cdf;
};
void flatten_plain(const HostScene& hs, PlainImage& img);

struct Fp32Image {       // FP32 layout for the wavefront kernels
    std::vector<BvhNode2> nodes;             // interior nodes, all meshes, then the sphere BVH
    std::vector<TriF32> tris;                // leaf order, all meshes
    std::vector<MeshF32> meshes;
    std::vector<InstanceF32> instances;
    std::vector<SphereF32> spheres;          // sphere-BVH leaf order
    int32_t top_root = TPT_REF_NONE;         // top-level BVH (spheres + instances)
    int32_t top_node_begin = 0;              // first node of the top-level tree
    std::vector<MaterialF32> mats;
    std::vector<LightF32> lights;
    std::vector<float> light_cdf;            // normalised, reference quirk kept
    std::vector<float4> env_texels;          // rgb + nearest-texel pdf_uv
    std::vector<float> env_row_cdf;          // normalised by the total
    std::vector<float> env_col_cdf;          // normalised per row
    int max_stack = 0;
};
void flatten_fp32(const HostScene& hs, Fp32Image& img);

// Several scenes in one set of device arrays for batch renders: the FP32
// images and the f64 light/instance/sphere tables of each scene appended,
// every index rebased (BVH node and leaf references, material ids, mesh
// ids, light records).  Each scene keeps its own top-level root, camera,
// env map and light range.
struct BatchScene {
    int32_t top_root;
    CameraF32 cam;
    int32_t env_kind, env_w, env_h, env_has_cdf;
    size_t env_tex_off, env_row_off, env_col_off;   // element offsets
    int32_t light_begin, n_lights;
    int32_t n_mats, mat_begin;
};
struct BatchImage {
    Fp32Image fp;                            // combined FP32 arrays (env/lights concatenated)
    std::vector<LightF64> lights64;
    std::vector<InstanceF64> inst64;
    std::vector<SphereF64> spheres64;
    std::vector<BatchScene> scenes;
};
void merge_scenes(const std::vector<const HostScene*>& scenes, BatchImage& out);

}  // namespace tpt
