// Device view of the f64 scene image and the plain kernel's launch: one
// thread per pixel runs the reference's render worker (src/render.rs:129-205)
// and radiance() (src/integrator.rs:53-135) in f64 over the reference's own
// node, triangle, sphere and instance layouts.
#pragma once

#include "device_common.cuh"
#include "../../include/tinypt_cuda.h"

namespace tpt {

struct PlainScene {
    const NodeF64* nodes;
    const TriF64* tris;
    const MeshF64* meshes;
    const InstanceF64* instances;
    int n_instances;
    const SphereF64* spheres;
    int n_spheres;
    const MaterialF64* mats;
    const LightF64* lights;
    const double* light_cdf;
    int n_lights;
    double light_total;
    int env_kind, env_w, env_h;
    const double* env_data;
    const double* env_row_cdf;
    const double* env_col_cdf;
    double env_total;
    CameraF64 cam;
};

struct PlainParams {
    int width, height, spp, max_bounces, rr_start;
    int adaptive, adaptive_min_spp;
    double adaptive_threshold;
    uint64_t seed;
    int row_begin, row_step, n_rows;  // film row k is image row row_begin + k * row_step
};

// counters[0] = samples, [1] = closest-hit rays, [2] = shadow rays.
cudaError_t launch_plain(const PlainScene& S, const PlainParams& P, double* acc, double* acc_w, double* acc_sq,
                         unsigned long long* counters, int* flags, cudaStream_t stream);

}  // namespace tpt
