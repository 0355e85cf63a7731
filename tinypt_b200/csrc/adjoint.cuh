// Adjoint of the FP32 path integrator: path-replay backpropagation of an
// image loss to the material parameters, and the film resolve.
#pragma once

#include <cuda_runtime.h>

#include "wavefront.cuh"

namespace tpt {

struct AdjParams {
    int width, height, spp, max_bounces, rr_start;
    uint64_t seed;
    int n_pixels;              // width * film rows
    int row_begin, row_step;   // film row k is image row row_begin + k * row_step
    int task_spp;              // samples per thread task
    int n_chunks;              // ceil(spp / task_spp)
    long long n_tasks;         // n_pixels * n_chunks
    int n_mats;                // 4 parameters per material
    int trace_chunk;           // wavefront form: leaf visits between lane refills
    FastDiv px_div, w_div;     // n_pixels and width as multiply-shift divisors (tasks < 2^31)
    int queue_div;             // slot selection of the wavefront adjoint (use_ext_queue)
    int ordered_queue;         // the extension queue rebuilt in slot order every iteration
    // camera culling (wavefront adjoint): sky_cull = 1 lets the render
    // classify its pixels; the pool then fetches, chunk by chunk, only the
    // tasks of the n_geo pixels listed in geo_map (null: every pixel), and
    // k_adj_sky replays the others
    int sky_cull;
    const int* geo_map;
    int n_geo;
    FastDiv geo_div;
};

// Extra per-slot state of the wavefront adjoint (device arrays).
struct AdjWfState {
    float4* acc;     // per slot: sum of the sample's a_k so far (xyz), w = sample time
    float4* vg;      // [bounce * n_slots + slot]: dlog w of that bounce's BSDF sample (rgb, alpha)
    float4* vc;      // [bounce * n_slots + slot]: C_j (xyz), w = its material (int bits, -1: none)
    float4* sh_gm;   // per shadow record: a * dlog f of the shading material (rgb, alpha)
    float4* sh_gl;   // per shadow record (area lights): a / emission (rgb), w = light material (int bits)
    int* sh_mat;     // per shadow record: the shading material
};
struct AdjBuffers {
    size_t slots = 0, bounces = 0, params = 0;
    void* block = nullptr;
    AdjWfState st{};
    double* gtot = nullptr;  // f64 totals: gradients, then the linearised loss
};
cudaError_t adj_reserve(AdjBuffers& b, size_t slots, int max_bounces, int n_params);
void adj_release(AdjBuffers& b);

// d_grad[4*m + k] (f64, overwritten) = sum over pixels p and channels c of
// d_dimg[3p+c] * dI[p][c]/dtheta, theta = material m's rgb[k] (k < 3) or its
// param (k = 3), where I is the image this config renders in expectation.
// counters[0] receives the number of paths replayed, counters[1] (as an f64)
// the linearised loss sum_p d_dimg[p] . I[p] of the adjoint's own paths;
// *flags the TPT_FLAG_* bits.  elapsed_ms (nullable) receives the kernel time.
cudaError_t adj_render_backward(const WfScene& S, const AdjParams& P, const float* d_dimg, double* d_grad, int* d_flags,
                                unsigned long long* d_counters, cudaStream_t s, int sm_count, float* elapsed_ms);

// The same quantity, computed on the forward form's wavefront machinery in
// one pass per sample (a pool of at most `pool` slots; B holds the path
// state, AB the adjoint's own).  culled_samples (nullable) receives the
// samples of pixels camera culling took out of the pool.
cudaError_t adj_render_backward_wf(const WfScene& S, const AdjParams& P, WfBuffers& B, AdjBuffers& AB,
                                   long long pool, const float* d_dimg, double* d_grad, int* d_flags,
                                   unsigned long long* d_counters, cudaStream_t s, int sm_count, bool use_graph_loop,
                                   float* elapsed_ms, unsigned long long* culled_samples = nullptr);

// img[3i+c] = acc[3i+c] / max(acc_w[i], 1) as float (src/output.rs:96-102).
cudaError_t resolve_film(const double* acc, const double* acc_w, float* img, int n_pixels, cudaStream_t s);

}  // namespace tpt
