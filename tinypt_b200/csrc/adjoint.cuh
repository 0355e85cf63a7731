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
};

// d_grad[4*m + k] (f64, overwritten) = sum over pixels p and channels c of
// d_dimg[3p+c] * dI[p][c]/dtheta, theta = material m's rgb[k] (k < 3) or its
// param (k = 3), where I is the image this config renders in expectation.
// counters[0] receives the number of paths replayed, counters[1] (as an f64)
// the linearised loss sum_p d_dimg[p] . I[p] of the adjoint's own paths;
// *flags the TPT_FLAG_* bits.  elapsed_ms (nullable) receives the kernel time.
cudaError_t adj_render_backward(const WfScene& S, const AdjParams& P, const float* d_dimg, double* d_grad, int* d_flags,
                                unsigned long long* d_counters, cudaStream_t s, int sm_count, float* elapsed_ms);

// img[3i+c] = acc[3i+c] / max(acc_w[i], 1) as float (src/output.rs:96-102).
cudaError_t resolve_film(const double* acc, const double* acc_w, float* img, int n_pixels, cudaStream_t s);

}  // namespace tpt
