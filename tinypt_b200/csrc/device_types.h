// Device data layouts shared by the host flattening code and the kernels.
// All structs are plain data; sizes and alignments are checked below.
#pragma once

#include <cstdint>
#include <vector_types.h>

namespace tpt {

// ---------------------------------------------------------------- f64 ----
// Camera basis as the reference stores it (src/ray.rs:22-33).
struct CameraF64 {
    double o[3], u[3], v[3], w[3];
    double half_h, half_w, lens_radius, focus_dist, shutter_open, shutter_close;
};

// Reference BvhNode (src/bvh.rs:24-35): bbox + child indices + leaf range.
struct alignas(16) NodeF64 {
    double bmin[3], bmax[3];
    int32_t left, right;
    uint32_t start, count;
};
static_assert(sizeof(NodeF64) == 64, "NodeF64 is 64 B");

// Static triangle (Triangle::new_static, src/geometry.rs:199-210); stored in
// BVH leaf order so leaves address a contiguous range.
struct alignas(16) TriF64 {
    double v0[3], v1[3], v2[3];
    int32_t mat;
    int32_t orig;   // index in the mesh's input order
};
static_assert(sizeof(TriF64) == 80, "TriF64 is 80 B");

struct MeshF64 { int32_t node_offset, n_nodes, tri_offset, n_tris; };

// Transform (src/transform.rs:11-21) + Instance (src/world.rs:39-46).
struct InstanceF64 {
    double a[9], t[3], a_inv[9], nmat[9];
    int32_t mesh_id, mat_override;   // -1 = None
};

struct SphereF64 { double c[3], r; int32_t mat, pad; };

struct MaterialF64 { int32_t kind, pad; double c[3]; double p; };

// LightInfo (src/world.rs:296-300) with Light (src/world.rs:218-221).
// The triangle's object-space vertices are copied in; the kernel applies
// vertices_at(time) and the instance transform like tri_world_verts
// (src/world.rs:276-292).
struct LightF64 {
    int32_t is_sphere, sphere, inst, pad;
    double v[9];
    double emit[3], weight;
};

// ---------------------------------------------------------------- FP32 ---
// Child reference in a BVH2 node: >= 0 interior node index; < 0 a leaf with
// ~ref = (first primitive << 3) | count; TPT_REF_NONE = no child.
constexpr int32_t TPT_REF_NONE = INT32_MIN;
__host__ __device__ inline int32_t make_leaf_ref(uint32_t start, uint32_t count) {
    return ~(int32_t)((start << 3) | count);
}

// Interior node of the flattened BVH2: the boxes of both children, so one
// 64-byte visit (four 16-byte loads) decides the traversal order.
//   lx = (c0.min.x, c0.max.x, c0.min.y, c0.max.y)
//   rx = (c1.min.x, c1.max.x, c1.min.y, c1.max.y)
//   zz = (c0.min.z, c0.max.z, c1.min.z, c1.max.z)
//   refs.x = child 0 ref, refs.y = child 1 ref
struct alignas(32) BvhNode2 {
    float4 lx, rx, zz;
    int4 refs;
};
static_assert(sizeof(BvhNode2) == 64, "BvhNode2 is 64 B");

// Triangle with precomputed Moeller-Trumbore edges, 48 B.
struct alignas(16) TriF32 {
    float4 v0;   // xyz, w = material id (int bits)
    float4 e1;   // xyz, w = index in the mesh input order (int bits)
    float4 e2;   // xyz, w = unused
};
static_assert(sizeof(TriF32) == 48, "TriF32 is 48 B");

struct MeshF32 {
    int32_t root_ref;      // node index or leaf ref of the root
    int32_t tri_offset;    // first triangle of this mesh in the global array
    int32_t n_tris, pad;
};

// w2o/o2w rows: (r0, r1, r2) with the translation in .w.
struct alignas(16) InstanceF32 {
    float4 w2o[3];         // p_obj = A^-1 (p - t)  ->  rows of A^-1, w = -(A^-1 t)
    float4 nrm[3];         // inverse transpose (normal transform), w unused
    float4 wbox_min;       // world-space box of the instance, w = mesh id and flags (int bits, below)
    float4 wbox_max;       // w = material override (int bits, -1 = none)
};
// InstanceF32::wbox_min.w: the mesh id in bits 0-29; bit 30 set when w2o is
// exactly the identity in FP32 (the traversal then walks the mesh tree with
// the world ray as it is).
constexpr int32_t kInstMeshMask = 0x3fffffff, kInstIdentity = 0x40000000;

struct alignas(16) SphereF32 {
    float4 cr;             // centre xyz, radius
    int32_t mat, orig, pad0, pad1;
};

struct alignas(16) MaterialF32 {
    float4 c;              // rgb, w = param (ior | alpha | scatter_dist)
    int32_t kind;
    float s_param;         // GGX alpha of the sampler and its pdf (= c.w unless
                           // sampling is detached from evaluation)
    int32_t pad1, pad2;
};

struct alignas(16) LightF32 {
    float4 p0;             // sphere: centre xyz + radius; triangle: v0 xyz
    float4 p1;             // triangle: v1 xyz
    float4 p2;             // triangle: v2 xyz
    float4 emit;           // rgb, w = pdf_select (weight / total)
    int32_t is_sphere;
    int32_t mat;           // material of the emitter
    int32_t pad1, pad2;
};

// Camera basis in FP32.
struct CameraF32 {
    float3 o, u, v, w;
    float half_h, half_w, lens_radius, focus_dist;
};

}  // namespace tpt
