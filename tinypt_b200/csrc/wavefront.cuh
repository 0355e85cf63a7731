// FP32 wavefront form: device views, state buffers and the host driver.
// The bounce loop of radiance() (src/integrator.rs:53-135) is split into
// closest-hit, shading, occlusion and completion kernels over a pool of path
// slots; tasks are the reference's Task { sample_start } (src/task.rs:42-45)
// per pixel, with per-pixel PCG32 streams seeded as in src/render.rs:142.
#pragma once

#include <functional>

#include "device_common.cuh"
#include "../../include/tinypt_cuda.h"

namespace tpt {

// Division by a divisor fixed for a whole render (pixels of the film, film
// width), as a multiply and shift (Granlund and Montgomery, "Division by
// invariant integers using multiplication", PLDI 1994, fig. 4.1, with the
// dividend below 2^31 so the sum cannot overflow): the task -> pixel and
// pixel -> (x, y) mappings run for every sample, and a 64-bit or 32-bit
// integer division there is a long instruction sequence.  Exact for every
// dividend n < 2^31 and divisor 1 <= d < 2^31.
struct FastDiv {
    uint32_t d, m, l;
};
__host__ __device__ inline FastDiv make_fastdiv(uint32_t d) {
    if (d == 0) d = 1;
    uint32_t l = 0;
    while ((1ull << l) < d) ++l;
    const uint64_t m = ((uint64_t(1) << 32) * ((uint64_t(1) << l) - d)) / d + 1;
    return FastDiv{d, (uint32_t)m, l};
}
__device__ __forceinline__ uint32_t fdiv(const FastDiv& f, uint32_t n) { return (__umulhi(n, f.m) + n) >> f.l; }

struct WfScene {
    const BvhNode2* nodes;
    const TriF32* tris;
    const MeshF32* meshes;
    const InstanceF32* inst;
    int n_inst;
    const SphereF32* spheres;
    int n_spheres;
    int top_root;              // top-level BVH over spheres and instances
    const MaterialF32* mats;
    const LightF32* lights;
    const float* light_cdf;
    int n_lights;
    int env_kind, env_w, env_h, env_has_cdf;
    const float4* env_tex;     // rgb + nearest-texel pdf_uv
    const float* env_row;      // h+1, normalised
    const float* env_col;      // h*(w+1), normalised per row
    CameraF32 cam;
    // f64 light data for the reference's self-occlusion test of area-light
    // shadow rays (shared with the plain kernel's scene image)
    const LightF64* lights64;
    const InstanceF64* inst64;
    const SphereF64* spheres64;
    int max_stack;             // deepest traversal stack the scene can need
};

// One job of a batch render: its scene's view into the combined arrays
// (top-level root, camera, env map, light range) and its film.
struct WfJob {
    CameraF32 cam;
    int top_root;
    int env_kind, env_w, env_h, env_has_cdf;
    const float4* env_tex;
    const float* env_row;
    const float* env_col;
    const LightF32* lights;
    const float* light_cdf;
    const LightF64* lights64;
    int n_lights;
    int width, height, spp, max_bounces, rr_start;
    uint64_t seed;
    int n_pixels, task_spp, n_chunks, row_begin, row_step;
    long long task_begin, n_tasks, pixel_begin;
    double* acc;
    double* acc_w;
    FastDiv px_div, w_div;     // by n_pixels, by width
    // Camera culling (filled on the device inside wf_render): the job's
    // stretch of the batch-wide "may hit" and "open" pixel lists, the first
    // pool fetch id and the first sky task of the job (n_chunks * n_geo of
    // the one, n_chunks * n_sky of the other).
    long long fetch_begin, sky_task_begin;
    int geo_begin, n_geo, sky_begin, n_sky;
    FastDiv geo_div, sky_div;  // by n_geo, by n_sky
};

struct WfParams {
    int width, height, spp, max_bounces, rr_start;
    int adaptive, adaptive_min_spp;
    double adaptive_threshold;
    uint64_t seed;
    int n_slots;               // path pool size (paths in flight)
    int n_pixels;              // width * film rows
    int row_begin, row_step;   // film row k is image row row_begin + k * row_step
    long long n_tasks;         // n_pixels * n_chunks (inside wf_render: end of the current chunk batch)
    long long task_first;      // inside wf_render: first task of the current chunk batch
    long long max_part_tasks;  // per-task partial sums held at once (single renders render chunk batches)
    int task_spp;              // samples per task (the last chunk may be shorter)
    int n_chunks;              // sample chunks per pixel = ceil(spp / task_spp)
    long long max_iters;       // iteration bound of the bounce loop
    int trace_chunk;           // leaf visits between lane refills in the trace kernels
    int shade_sort;            // 1: classify + per-material shading kernels; 0: one shading kernel
    int camera_fast;           // nonzero: the closest-hit kernel finishes camera-ray misses in place (not
                               // adaptive); 2 = on unless camera culling found open pixels (wf_render)
    int shade_ctas;            // shading kernel compiled for 4, 6 or 8 resident blocks per SM (batch renders: 4 or 8)
    int ext_queue;             // 1: below 1/queue_div of the pool live, the kernels take the active slots
                               // from WfState::q_ext (use_ext_queue); 0: always sweep the act bytes
    int queue_div;             // TPT_QUEUE_DIV, default 8
    int tail_live;             // > 0: once no tasks are left and at most this many slots are live, the
                               // bounce loop stops and k_tail runs each of them to the end (single,
                               // batch and adaptive-round renders; 0 = the loop drains the pool; -1 =
                               // the default, 262,144 but at most a sixteenth of the pool)
    int ordered_queue;         // 1: the extension queue is rebuilt in slot order after every iteration
                               // (wf_launch_compact) and the kernels always take it
    // batch renders: the jobs (device memory); the other per-render fields
    // above are then those of the whole batch (n_tasks, n_slots, ...)
    const WfJob* jobs;
    int n_jobs;
    long long total_pixels;
    // A round of an adaptive render (wf_render_adaptive): the tasks cover
    // samples [sample_base, sample_end) of the n_pixels film pixels listed
    // in px_map (task-space pixel j -> film pixel px_map[j]), and every
    // sample's radiance goes to WfState::rsamp at j * round_len + (sample -
    // sample_base).  Outside rounds: px_map null, sample_base 0, sample_end
    // 0 (= spp).
    const int* px_map;
    int sample_base, sample_end;
    int round_len;
    // n_pixels and width as multiply-shift divisors (set with them: wf_set_divisors)
    FastDiv px_div, w_div;
    // Camera culling (single forward renders with a pinhole camera): 1 = the
    // pixels whose every camera ray leaves the scene are rendered by
    // k_sky_tasks, and the pool's task cursor runs over the other pixels'
    // tasks only -- geo_map lists those n_geo film pixels (set inside
    // wf_render; null = every task goes through the pool).
    int sky_cull;
    const int* geo_map;
    int n_geo;
    FastDiv geo_div;           // by n_geo
    // batch renders with culling: the pool fetches ids [0, n_fetch), mapped
    // through each job's stretch of geo_map (batch-wide pixel ids)
    long long n_fetch;
};
inline void wf_set_divisors(WfParams& p) {
    p.px_div = make_fastdiv((uint32_t)(p.n_pixels > 0 ? p.n_pixels : 1));
    p.w_div = make_fastdiv((uint32_t)(p.width > 0 ? p.width : 1));
}

// Queue counters and statistics, one per render (device memory).
struct WfCounters {
    int n_ext[2];              // active slots this / next iteration (ping-pong)
    int n_sh;                  // shadow records this iteration
    int n_term;                // samples finishing in k_regen this iteration
    int n_done_in_shade;       // samples finished inside the shading kernels this iteration
    int n_mat[5];              // surface-hit queue lengths per material kind
    int fetch_ext, fetch_sh;   // dynamic work-fetch cursors of the trace kernels
    int flags;                 // TPT_FLAG_*
    int tail;                  // 1: the bounce loop handed its last live slots to k_tail
    long long iters;
    long long next_task;       // task pool cursor
    unsigned long long rays_closest, rays_shadow, samples;
    // profiling variant only: [0] closest hit, [1] occlusion
    unsigned long long cnt_nodes[2], cnt_tris[2], cnt_spheres[2], cnt_inst[2];
    unsigned long long cnt_node_steps[2];  // warp-wide node-loop steps
    unsigned long long cnt_fast;           // samples finished by the camera-miss fast path
    unsigned long long cnt_leaves[2], cnt_leaf_steps[2];  // leaf visits, their warp-wide steps
    unsigned long long cnt_fast_steps;     // warp-wide steps of the fast path
    unsigned long long sky_samples;        // samples of culled pixels (k_sky_tasks, which counts them only
                                           // here: it runs beside k_step; the host adds them to samples and
                                           // rays_closest)
    int pool_slots;                        // host side: the path slots the render ran with
    long long launches;                    // host side: kernels the render launched
};

// The packed path record (WfState::path, 16 B): x, y = the PCG32 state's
// low and high 32 bits (it continues the task's stream), z = task id, w =
// samples done in the task (bits 0-18), bounce (bits 19-26) and path flags
// (bits 27-31).  Hence the wavefront forms' limits on a task's samples and
// on max_bounces (the host rejects configs beyond them).
constexpr int kPathDoneBits = 19, kPathBounceBits = 8;
constexpr int kMaxTaskSamples = (1 << kPathDoneBits) - 1;   // 524,287
constexpr int kMaxWavefrontBounces = (1 << kPathBounceBits) - 1;  // 255

// Per-slot path state (structure of arrays) and the queues.
struct WfState {
    int4* path;                // PCG32 state, task, samples done, bounce, flags (packed, above)
    float4* ray_o;             // origin, w = self primitive (int bits)
    float4* ray_d;             // direction, w = self instance (int bits)
    float4* beta;              // throughput, w = last BSDF pdf
    float4* rad;               // radiance of the current sample
    float4* hit;               // t, prim (int bits), instance (int bits)
    float4* sh_o;              // 2 per slot: origin, w = tmax
    float4* sh_d;              // direction, w = self prim
    float4* sh_c;              // contribution, w = self inst -> visibility
    double2* welford;          // adaptive sampling: mean, m2 of luminance
    int* job;                  // batch renders: job of the slot's task
    double4* sacc;             // per slot: f64 sums of the current task (rgb, n)
    double4* ssq;              // per slot: f64 sums of squares (optional)
    double4* part;             // per task sums when a pixel has several tasks
    double4* part_sq;
    float4* surf_p;            // surface hit: position, w = t
    float4* surf_n;            // surface hit: geometric normal, w = material id (int bits)
    int* q_mat;                // 5 queues (one per material kind) of n_slots entries
    uint8_t* act;              // 1 = the slot has a ray to extend this iteration (adjoint renders)
    int* q_ext[2];             // forward renders: the slots with a ray to extend, this / next iteration
                               // (ping-pong; lengths WfCounters::n_ext[2])
    int* cmp_counts;           // ordered queue: live slots per 4096-slot span, then their offsets
    int* q_sh;
    int* q_term;
    WfCounters* ctr;
    double* acc;               // film (f64 sums), acc_w, acc_sq (optional)
    double* acc_w;
    double* acc_sq;
    float4* rsamp;             // adaptive rounds: radiance of every sample of the round (null otherwise)
};

// Allocated per handle and grown on demand.
struct WfBuffers {
    size_t slots = 0;
    size_t part_tasks = 0;
    void* block = nullptr;     // one device allocation for all state arrays
    WfState st{};
    // adaptive rounds: per film pixel the Welford state (n, mean, m2, done),
    // two active-pixel lists, and the round's sample radiance
    size_t round_pixels = 0, round_samples = 0;
    void* round_block = nullptr;
    double4* wstate = nullptr;
    int* active[2] = {nullptr, nullptr};
    int* n_active = nullptr;
    float4* rsamp = nullptr;
    // camera culling: per film pixel a "may hit" and an "open" byte, the two
    // compacted pixel lists, the compaction's span counts and the list lengths
    size_t cull_pixels = 0;
    void* cull_block = nullptr;
    uint8_t* cull_flag[2] = {nullptr, nullptr};
    int* cull_map[2] = {nullptr, nullptr};
    int* cull_counts[2] = {nullptr, nullptr};
    int* cull_n = nullptr;
    // the culled pixels' kernel runs on a side stream beside the bounce loop
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

cudaError_t wf_reserve(WfBuffers& b, size_t slots, size_t part_tasks);
void wf_release(WfBuffers& b);

// Renders one frame into st.acc / st.acc_w / st.acc_sq (device pointers).
// use_graph_loop: device-side WHILE conditional graph (one launch); else a
// host loop of graph launches.  Returns the CUDA error, and fills the
// counters' host copy.
// profile: host loop with CUDA events around every stage launch and the
// counting variants of the trace kernels; stage_ms/stage_launches (4 each:
// extend, shade, shadow, regen) receive the per-stage totals.
cudaError_t wf_render(const WfScene& S, const WfParams& P, WfBuffers& B, double* acc, double* acc_w,
                      double* acc_sq, cudaStream_t stream, int sm_count, bool use_graph_loop,
                      WfCounters* host_counters, float* ms, bool profile = false, double* stage_ms = nullptr,
                      unsigned long long* stage_launches = nullptr);

// Adaptive render with several tasks per pixel (P.adaptive, P.n_chunks > 1
// or forced): rounds of the ordinary wavefront loop over the pixels still
// sampling, each followed by a merge that replays the reference's stopping
// rule (src/render.rs:143-180) over the round's samples in sample order.
// round_bytes bounds the per-round sample buffer (16 B per sample).
cudaError_t wf_render_adaptive(const WfScene& S, const WfParams& P, WfBuffers& B, double* acc, double* acc_w,
                               double* acc_sq, cudaStream_t stream, int sm_count, bool use_graph_loop,
                               WfCounters* host_counters, float* ms, size_t round_bytes, int* rounds_out);

// Building blocks for other wavefront loops over the same path state (the
// adjoint render): the trace kernels, the end-of-iteration kernel and the
// device-driven loop.
//   wf_trace_grids: persistent grid sizes of the closest-hit / occlusion kernels;
//   wf_launch_trace: closest hit of every active slot (any = false) or
//     occlusion of the shadow-record queue (any = true); uses P.jobs,
//     P.n_slots and P.trace_chunk;
//   wf_launch_step: statistics, queue reset and the loop condition (k_step);
//   wf_run_loop: runs `enqueue` (two iterations, each ending in
//     wf_launch_step with the given conditional handle) until no slot is
//     active: inside one CUDA graph with a WHILE node when use_graph_loop,
//     else (or when that graph cannot be built) as relaunched graphs.
using WfEnqueue = std::function<void(cudaStream_t, cudaGraphConditionalHandle, int)>;
void wf_trace_grids(int sm_count, int* extend, int* shadow);
void wf_launch_trace(bool any, int grid, cudaStream_t s, const WfScene& S, const WfParams& P, const WfState& st,
                     int cur);
void wf_launch_step(cudaStream_t s, const WfState& st, int cur, long long max_iters, cudaGraphConditionalHandle h,
                    int use_cond);
//   wf_launch_compact: rebuilds the next iteration's extension queue from the
//     act bytes of n_slots slots, in slot order (three launches);
//   wf_compact_spans: the size of WfState::cmp_counts it needs.
void wf_launch_compact(cudaStream_t s, const WfState& st, int cur, int n_slots);
//   wf_cull_pixels: camera culling of a single render's film (P: n_pixels,
//   width, height, row_begin, row_step, w_div, max_bounces; pinhole cameras
//   only): B.cull_map[0] = the n_may pixels a camera ray may reach geometry
//   from, B.cull_map[1] = the n_open others, both in film order.
cudaError_t wf_cull_pixels(const WfScene& S, const WfParams& P, WfBuffers& B, cudaStream_t s, int* n_may,
                           int* n_open);
size_t wf_compact_spans(size_t n_slots);
cudaError_t wf_run_loop(const WfEnqueue& enqueue, const WfCounters* ctr, long long max_iters, cudaStream_t stream,
                        bool use_graph_loop);

// Allocation-free render (see the comment above wf_render_noalloc in
// wavefront.cu): path state in a file-scope device array, direct launches,
// films of at most wf_noalloc_max_slots() pixels.
size_t wf_noalloc_max_slots();
cudaError_t wf_render_noalloc(const WfScene& S, const WfParams& P, double* acc, double* acc_w, cudaStream_t stream,
                              int sm_count, WfCounters* host_counters);

}  // namespace tpt
