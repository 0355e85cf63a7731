// C ABI of the B200 path integrator (include/tinypt_cuda.h).
#include <cuda_runtime.h>

#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tinypt_cuda.h"
#include "adjoint.cuh"
#include "bvh_build.cuh"
#include "checkpoint.hpp"
#include "host_scene.hpp"
#include "image_io.hpp"
#include "plain_f64.cuh"
#include "scene_io.hpp"
#include "wavefront.cuh"

namespace tpt {
namespace {

thread_local std::string g_last_error;

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const char* what)
        : std::runtime_error(std::string(what) + ": " + cudaGetErrorString(c)), code(c) {}
};
struct TptError : std::runtime_error {
    int code;
    TptError(int c, const std::string& w) : std::runtime_error(w), code(c) {}
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(e, what);
}

// Makes a handle's device current for one entry point and gives the
// caller's current device back on the way out, so a caller that drives
// several GPUs from one thread keeps its own selection.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        ck(cudaSetDevice(device), "cudaSetDevice");
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

struct SceneHandle {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
    PlainScene plain{};
    WfScene wf{};
    WfBuffers wfbuf;
    AdjBuffers adjbuf;               // wavefront adjoint state
    double* film = nullptr;          // device film for host-output renders
    size_t film_px = 0;
    unsigned long long* d_counters = nullptr;
    int* d_flags = nullptr;
    int max_stack = 0;
    // Host scene kept for tpt_scene_set_materials (mesh BVHs dropped).
    HostScene hs;
    bool detached = false;           // sampling materials differ from evaluation
    // staging of the host-pointer forward/backward entry points
    float* img = nullptr;
    size_t img_px = 0;
    double* grad = nullptr;
    size_t grad_n = 0;

    // Frees a device array of this handle and uploads v in its place.
    template <class P, class T>
    void reupload(P*& dst, const std::vector<T>& v) {
        if (dst) {
            for (auto& p : allocs)
                if (p == (void*)dst) {
                    cudaFree(p);
                    p = nullptr;
                }
        }
        dst = upload(v);
    }

    template <class T>
    T* upload(const std::vector<T>& v) {
        if (v.empty()) return nullptr;
        void* p = nullptr;
        ck(cudaMalloc(&p, v.size() * sizeof(T)), "cudaMalloc(scene)");
        allocs.push_back(p);
        ck(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream), "upload scene");
        return static_cast<T*>(p);
    }
    ~SceneHandle() {
        if (stream) cudaStreamSynchronize(stream);
        for (void* p : allocs)
            if (p) cudaFree(p);
        if (film) cudaFree(film);
        if (img) cudaFree(img);
        if (grad) cudaFree(grad);
        if (d_counters) cudaFree(d_counters);
        if (d_flags) cudaFree(d_flags);
        wf_release(wfbuf);
        adj_release(adjbuf);
        if (stream) cudaStreamDestroy(stream);
    }
};

template <class F>
int guarded(F&& f) {
    try {
        g_last_error.clear();
        return f();
    } catch (const CudaError& e) {
        g_last_error = e.what();
        cudaGetLastError();
        return e.code == cudaErrorMemoryAllocation ? TPT_ERR_ALLOC : TPT_ERR_CUDA;
    } catch (const TptError& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return TPT_ERR_ALLOC;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return TPT_ERR_INVALID;
    }
}

// Integer tuning knob from the environment: the fallback unless the
// variable holds a whole decimal int (so "16M" or "" cannot turn into a
// 1-slot pool or a 0-sample task).
int env_int(const char* name, int fallback) {
    const char* v = std::getenv(name);
    if (!v || !*v) return fallback;
    char* end = nullptr;
    errno = 0;
    const long x = std::strtol(v, &end, 10);
    if (errno == ERANGE || *end != '\0' || x < INT_MIN || x > INT_MAX) return fallback;
    return (int)x;
}

// The wavefront kernels sweep the whole path pool while more than
// 1/TPT_QUEUE_DIV of it is live and take the compacted extension queue
// below (default 8; 1 = always the queue, a huge value = always sweep).
int queue_div_setting() {
    const int d = env_int("TPT_QUEUE_DIV", 8);
    return d < 1 ? 1 : d;
}

// Leaf visits between lane refills in the trace kernels (TPT_TRACE_CHUNK
// overrides the default of 4; the autotuner sweeps it).
int trace_chunk_setting() {
    const int c = env_int("TPT_TRACE_CHUNK", 4);
    return c < 1 ? 1 : (c > 64 ? 64 : c);
}

// Mesh BVHs of a scene being created: large meshes are built on the device
// (same tree as the host builder), small ones on the host, where the launch
// and copy overheads of the device build are larger than the build itself.
// TPT_BVH_BUILD=host or =device forces one builder for every mesh.  A
// device build that finds no room for its arrays falls back to the host.
HostBvh scene_mesh_bvh(const tpt_mesh_desc& m) {
    const char* v = std::getenv("TPT_BVH_BUILD");
    const bool force_host = v && std::strcmp(v, "host") == 0;
    const bool force_device = v && std::strcmp(v, "device") == 0;
    if (!force_host && (force_device || m.n_tris >= kGpuBvhMinTris)) {
        HostBvh b;
        std::string err;
        const int rc = build_mesh_bvh_gpu(m.positions, m.n_vertices, m.indices, m.n_tris, b, &err);
        if (rc == kGpuBvhOk) return b;
        if (rc == kGpuBvhCudaError) throw TptError(TPT_ERR_CUDA, "device BVH build: " + err);
        // kGpuBvhNoMemory, kGpuBvhUseHost: the host builder makes the same tree
    }
    return build_mesh_bvh(m.positions, m.n_vertices, m.indices, m.n_tris);
}

// Rows of the output film: all rows, or the shard row_begin, row_begin +
// row_step, ... (tpt_render_config).
int film_rows(const tpt_render_config& c) {
    if (c.row_step <= 0) return c.height;
    return (c.height - c.row_begin + c.row_step - 1) / c.row_step;
}
int row_step_of(const tpt_render_config& c) { return c.row_step <= 0 ? 1 : c.row_step; }
int row_begin_of(const tpt_render_config& c) { return c.row_step <= 0 ? 0 : c.row_begin; }

// Samples per pool task unless TPT_TASK_SPP or a batch tuning says
// otherwise.  Short tasks keep the end of a frame short (slots run out of
// work at about the same time) and still leave most camera-ray misses to
// the closest-hit kernel's fast path: 1080p mesh+env frame, one B200, G
// paths/s at task length 16 / 12 / 8 / 4 / 2: 1.58 / 1.70 / 1.72 / 1.71 /
// 1.76 (2-sample tasks need 8.5 GB of per-task sums at 256 spp, 8-sample
// ones 2.1 GB).  A render with fewer tasks than pool slots at that length
// takes shorter ones, down to one sample, until it fills the pool: the
// 512x512 64-spp frame runs at 0.59 / 0.84 / 1.08 G paths/s at task length
// 8 / 4 / 2, and the inverse-rendering step takes 49 / 43 / 38 / 36 ms at
// 8 / 4 / 2 / 1.  The forward and adjoint renders take the same value.
constexpr int kDefaultTaskSpp = 8;

// Path slots in flight unless TPT_POOL or a batch tuning says otherwise: 64
// Mi, ~26 GB of path state (a render halves it while the device has no room;
// a pool larger than the render's task count is clamped to it).  With the
// ordered extension queue every kernel visits only live slots, so a larger
// pool spreads each launch's fixed costs and end-of-launch drain over more
// paths: 1080p mesh+env frame, one B200, G paths/s at 8 / 16 / 32 / 48 / 64
// Mi slots: 1.80 / 2.07 / 2.27 / 2.33 / 2.36.
constexpr int kDefaultPool = 64 << 20;

// Wavefront schedule.  Each pixel's samples are split into tasks of
// task_spp samples (TPT_TASK_SPP, else the longest of 8, 4, 2, 1 that
// gives at least as many tasks as pool slots), each seeded like a reference
// Task with that sample_start; a pool of paths (TPT_POOL slots, default 64
// Mi, about 26 GB of path state) pulls tasks until all are done.
// Adaptive renders use the same tasks and run in rounds (wf_render_adaptive):
// the stopping rule sees every sample of a pixel in sample order, as in the
// reference.  TPT_ADAPTIVE_ROUNDS=0 keeps one task per pixel instead (the
// reference's own per-pixel stream, one path per pixel in flight); so does
// the allocation-free entry point.
// Samples per task of a wavefront render (forward and adjoint alike): as
// above or TPT_TASK_SPP, at most spp, and long enough that the film's task
// ids fit the path state's 32-bit field.
int task_spp_for(const tpt_render_config& c, long long n_pixels) {
    int task_spp = env_int("TPT_TASK_SPP", 0);
    if (task_spp <= 0) {  // the longest of 8, 4, 2, 1 samples that still fills the pool
        const long long pool = std::max(1, env_int("TPT_POOL", kDefaultPool));
        task_spp = kDefaultTaskSpp;
        while (task_spp > 1 && n_pixels * (long long)((c.spp + task_spp - 1) / task_spp) < pool) task_spp /= 2;
    }
    if (task_spp < 1 || task_spp > c.spp) task_spp = c.spp;
    while (task_spp < c.spp && n_pixels * (long long)((c.spp + task_spp - 1) / task_spp) > 0x7fffffffLL)
        task_spp = std::min(c.spp, 2 * task_spp);
    return task_spp;
}

// The FP32 forms keep a path's bounce count and its task's samples done in
// the packed path record (8 and 19 bits): configs beyond them are refused
// (the plain f64 form has neither limit).
void check_wavefront_limits(int max_bounces, int task_spp) {
    if (max_bounces > kMaxWavefrontBounces)
        throw TptError(TPT_ERR_UNSUPPORTED, "the FP32 wavefront form traces at most 255 bounces (max_bounces)");
    if (task_spp > kMaxTaskSamples)
        throw TptError(TPT_ERR_UNSUPPORTED,
                       "a wavefront task holds at most 524,287 samples (spp of a one-task-per-pixel render)");
}

// Adaptive wavefront renders in rounds of tasks (default) or one task per
// pixel (TPT_ADAPTIVE_ROUNDS=0).
bool adaptive_rounds_setting() { return env_int("TPT_ADAPTIVE_ROUNDS", 1) != 0; }

void fill_wf_params(const tpt_render_config& c, WfParams& p, bool noalloc) {
    p.width = c.width; p.height = c.height; p.spp = c.spp;
    p.max_bounces = c.max_bounces; p.rr_start = c.rr_start;
    p.adaptive = c.adaptive_enabled != 0; p.adaptive_min_spp = c.adaptive_min_spp;
    p.adaptive_threshold = c.adaptive_threshold;
    p.seed = c.seed;
    p.n_pixels = c.width * film_rows(c);
    p.row_begin = row_begin_of(c);
    p.row_step = row_step_of(c);
    wf_set_divisors(p);
    const bool one_task = noalloc || (p.adaptive && !adaptive_rounds_setting());
    const int task_spp = one_task ? c.spp : task_spp_for(c, p.n_pixels);
    check_wavefront_limits(c.max_bounces, task_spp);
    p.task_spp = task_spp;
    p.n_chunks = (c.spp + task_spp - 1) / task_spp;
    p.n_tasks = (long long)p.n_pixels * p.n_chunks;
    long long pool = noalloc ? (long long)p.n_pixels : (long long)env_int("TPT_POOL", kDefaultPool);
    if (pool < 1) pool = 1;
    p.n_slots = (int)(p.n_tasks < pool ? p.n_tasks : pool);
    const long long rounds = (p.n_tasks + p.n_slots - 1) / p.n_slots + 1;
    p.max_iters = (long long)task_spp * (long long)(c.max_bounces + 1) * rounds + 16;
    p.trace_chunk = trace_chunk_setting();
    p.shade_sort = env_int("TPT_SHADE_SORT", 0) != 0;
    p.ext_queue = 1;
    p.queue_div = queue_div_setting();
    p.ordered_queue = env_int("TPT_QUEUE_ORDER", 1) != 0;
    // the drain's last live slots run to the end in k_tail; unset: -1, the
    // default (262,144, at most a sixteenth of the pool)
    p.tail_live = noalloc ? 0 : std::max(-1, env_int("TPT_TAIL_SLOTS", -1));
    // one-task adaptive renders run the stopping rule after every sample in
    // finish_sample, so their camera misses go through the shading kernel.
    // Unset: 2 = on unless camera culling takes the open pixels (wf_render).
    {
        const int fast = env_int("TPT_CAMERA_FAST", 2);
        p.camera_fast = (p.adaptive && one_task) || fast == 0 ? 0 : (fast == 1 ? 1 : 2);
    }
    // camera culling (wf_render applies it to pinhole cameras only)
    p.sky_cull = !noalloc && !p.adaptive && env_int("TPT_SKY_CULL", 1) != 0;
    // Adaptive renders spend their samples on the noisy pixels' long paths,
    // where 6 blocks per SM (80 registers, fewer spills) beat 8 (1080p
    // adaptive Cornell frame: 6.72 s at 6, 6.86 s at 8, 7.11 s at 4);
    // TPT_SHADE_CTAS=4|6|8 overrides.
    {
        const int ctas = env_int("TPT_SHADE_CTAS", p.adaptive ? 6 : 8);
        p.shade_ctas = (ctas == 4 || ctas == 6) ? ctas : 8;
    }
    // Per-task f64 sums (32 B, 64 with second moments) held at once: more
    // tasks than this (4.3 GB of sums) and the render runs in chunk batches,
    // each of which drains the pool (the 1080p 256-spp frame, 133 M 4-sample
    // tasks, stays one batch).
    p.max_part_tasks = std::max(1, env_int("TPT_MAX_PART_TASKS", 1 << 27));
}

void check_config(const tpt_render_config& c) {
    if (c.width <= 0 || c.height <= 0) throw TptError(TPT_ERR_INVALID, "width and height must be positive");
    if (c.row_step > 0 && (c.row_begin < 0 || c.row_begin >= c.height))
        throw TptError(TPT_ERR_INVALID, "row_begin outside the film");
    if ((long long)c.width * c.height > (1ll << 30)) throw TptError(TPT_ERR_INVALID, "film too large");
    if (c.spp <= 0) throw TptError(TPT_ERR_INVALID, "spp must be positive");
    if (c.max_bounces < 0 || c.rr_start < 0) throw TptError(TPT_ERR_INVALID, "negative path limits");
    if (c.mode != TPT_MODE_PLAIN_F64 && c.mode != TPT_MODE_WAVEFRONT_FP32)
        throw TptError(TPT_ERR_INVALID, "unknown render mode");
}

void render_device(SceneHandle& h, const tpt_render_config& c, double* acc, double* acc_w, double* acc_sq,
                   tpt_stats* stats) {
    check_config(c);
    DeviceGuard device_guard(h.device);
    tpt_stats s{};
    if (c.mode == TPT_MODE_PLAIN_F64) {
        if (h.detached)
            throw TptError(TPT_ERR_UNSUPPORTED, "the plain f64 form samples with the evaluation materials only");
        PlainParams p{c.width, c.height, c.spp, c.max_bounces, c.rr_start, c.adaptive_enabled != 0,
                      c.adaptive_min_spp, c.adaptive_threshold, c.seed, row_begin_of(c), row_step_of(c), film_rows(c)};
        ck(cudaMemsetAsync(h.d_counters, 0, 4 * sizeof(unsigned long long), h.stream), "memset counters");
        ck(cudaMemsetAsync(h.d_flags, 0, sizeof(int), h.stream), "memset flags");
        struct EventPair {
            cudaEvent_t e[2] = {nullptr, nullptr};
            ~EventPair() {
                for (cudaEvent_t x : e)
                    if (x) cudaEventDestroy(x);
            }
        } ev;
        ck(cudaEventCreate(&ev.e[0]), "event");
        ck(cudaEventCreate(&ev.e[1]), "event");
        cudaEventRecord(ev.e[0], h.stream);
        cudaError_t e = launch_plain(h.plain, p, acc, acc_w, acc_sq, h.d_counters, h.d_flags, h.stream);
        cudaEventRecord(ev.e[1], h.stream);
        unsigned long long cnt[4] = {0, 0, 0, 0};
        int flags = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, h.d_counters, sizeof(cnt), cudaMemcpyDeviceToHost, h.stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&flags, h.d_flags, sizeof(int), cudaMemcpyDeviceToHost, h.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h.stream);
        float ms = 0.0f;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, ev.e[0], ev.e[1]);
        ck(e, "plain f64 render");
        s.render_ms = ms;
        s.paths = cnt[0];
        s.rays_closest = cnt[1];
        s.rays_shadow = cnt[2];
        s.device_flags = flags;
    } else {
        WfParams p{};
        fill_wf_params(c, p, false);
        const char* loop = std::getenv("TPT_WAVEFRONT_HOST_LOOP");
        const bool graph_loop = !(loop && loop[0] == '1');
        WfCounters hc{};
        float ms = 0.0f;
        const bool profile = stats && stats->profile == 1;
        unsigned long long launches[4] = {0, 0, 0, 0};
        const bool rounds_path = p.adaptive && adaptive_rounds_setting();
        if (rounds_path) {
            // rounds of tasks with the stopping rule replayed per pixel in sample order
            // (no instrumented form: profile requests are ignored)
            // sample buffer: TPT_ADAPTIVE_ROUND_MB, else 16 GB but at most half the free device memory
            // (each round ends in a drain of the path pool, so fewer, larger rounds run faster)
            size_t round_bytes = (size_t)std::max(64, env_int("TPT_ADAPTIVE_ROUND_MB", 16384)) << 20;
            if (!std::getenv("TPT_ADAPTIVE_ROUND_MB")) {
                size_t free_b = 0, total_b = 0;
                if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
                    round_bytes = std::max<size_t>(size_t(64) << 20, std::min(round_bytes, free_b / 2));
            }
            int rounds = 0;
            ck(wf_render_adaptive(h.wf, p, h.wfbuf, acc, acc_w, acc_sq, h.stream, h.sm_count, graph_loop, &hc, &ms,
                                  round_bytes, &rounds),
               "adaptive wavefront render");
        } else {
            ck(wf_render(h.wf, p, h.wfbuf, acc, acc_w, acc_sq, h.stream, h.sm_count, graph_loop, &hc, &ms, profile,
                         s.stage_ms, launches),
               "wavefront render");
        }
        s.profile = (profile && !rounds_path) ? 1 : 0;
        for (int k = 0; k < 4; ++k) s.stage_launches[k] = launches[k];
        for (int k = 0; k < 2; ++k) {
            s.nodes_visited[k] = hc.cnt_nodes[k];
            s.tris_tested[k] = hc.cnt_tris[k];
            s.spheres_tested[k] = hc.cnt_spheres[k];
            s.instances_tested[k] = hc.cnt_inst[k];
            s.node_steps[k] = hc.cnt_node_steps[k];
            s.leaf_visits[k] = hc.cnt_leaves[k];
            s.leaf_steps[k] = hc.cnt_leaf_steps[k];
        }
        s.camera_fast = hc.cnt_fast;
        s.fast_steps = hc.cnt_fast_steps;
        s.render_ms = ms;
        s.rays_closest = hc.rays_closest;
        s.rays_shadow = hc.rays_shadow;
        s.iterations = (uint64_t)hc.iters;
        s.device_flags = hc.flags;
        s.paths = hc.samples;
        s.task_spp = p.task_spp;
        s.pool_slots = hc.pool_slots;
        s.sky_samples = hc.sky_samples;
        s.kernel_launches = (uint64_t)hc.launches;
    }
    if (stats) *stats = s;
    if (s.device_flags != 0) {
        char buf[128];
        std::snprintf(buf, sizeof buf, "kernel raised device flags 0x%x", s.device_flags);
        throw TptError(TPT_ERR_DEVICE, buf);
    }
}

// ---- batch handle ----------------------------------------------------------
struct BatchHandle {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
    WfScene wf{};                 // merged arrays; per-job fields come from the job table
    std::vector<BatchScene> scenes;
    WfBuffers wfbuf;
    WfJob* d_jobs = nullptr;
    size_t d_jobs_n = 0;

    template <class T>
    T* upload(const std::vector<T>& v) {
        if (v.empty()) return nullptr;
        void* p = nullptr;
        ck(cudaMalloc(&p, v.size() * sizeof(T)), "cudaMalloc(batch)");
        allocs.push_back(p);
        ck(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream), "upload batch");
        return static_cast<T*>(p);
    }
    ~BatchHandle() {
        if (stream) cudaStreamSynchronize(stream);
        for (void* p : allocs) cudaFree(p);
        if (d_jobs) cudaFree(d_jobs);
        wf_release(wfbuf);
        if (stream) cudaStreamDestroy(stream);
    }
};

// Schedule of a render: tuning fields, else TPT_* environment overrides,
// else the defaults.
struct Schedule {
    long long pool;
    int task_spp;
    int trace_chunk;
    int shade_ctas;  // 4 or 8
};
Schedule schedule_of(const tpt_tuning* t) {
    Schedule sc;
    sc.pool = (t && t->pool_slots > 0) ? t->pool_slots : env_int("TPT_POOL", kDefaultPool);
    sc.task_spp = (t && t->task_spp > 0) ? t->task_spp : env_int("TPT_TASK_SPP", kDefaultTaskSpp);
    sc.trace_chunk = (t && t->trace_chunk > 0) ? std::min(std::max(t->trace_chunk, 1), 64) : trace_chunk_setting();
    const int ctas = (t && t->shade_ctas > 0) ? t->shade_ctas : env_int("TPT_SHADE_CTAS", 4);
    sc.shade_ctas = ctas == 8 ? 8 : 4;
    if (sc.pool < 1) sc.pool = 1;
    if (sc.task_spp < 1) sc.task_spp = 1;
    return sc;
}

// Sums a render's counters into a batch's.
void add_stats(tpt_stats& s, const WfCounters& hc, float ms) {
    s.render_ms += ms;
    s.rays_closest += hc.rays_closest;
    s.rays_shadow += hc.rays_shadow;
    s.iterations += (uint64_t)hc.iters;
    s.device_flags |= hc.flags;
    s.paths += hc.samples;
    s.pool_slots = std::max(s.pool_slots, (int32_t)hc.pool_slots);
    s.sky_samples += hc.sky_samples;
    s.kernel_launches += (uint64_t)hc.launches;
}

// A batch job of at least this many paths (film pixels x spp) keeps the GPU
// busy on its own.  It renders alone, before the shared loop, with the single
// render's schedule (task length, pool, shading variant) on the batch's merged
// arrays, its scene fields set on the host as apply_job sets them per slot on
// the device; its film is that of tpt_render_device on its scene, bit for bit.
// The shared loop reads every job field per slot from the job table, which
// costs such a job about 7%, and mixing several large scenes in flight shares
// the L2 between them.  TPT_BATCH_ALONE_PATHS overrides (0: every job in the
// shared loop).
constexpr long long kBatchAlonePaths = 16ll << 20;

void batch_render(BatchHandle& B, const tpt_batch_job* jobs, int64_t n_jobs, const Schedule& sc, int spp_div,
                  tpt_stats* stats) {
    if (n_jobs <= 0) throw TptError(TPT_ERR_INVALID, "no jobs");
    DeviceGuard device_guard(B.device);
    long long alone_paths = kBatchAlonePaths;
    if (const char* v = std::getenv("TPT_BATCH_ALONE_PATHS")) alone_paths = std::atoll(v);
    std::vector<WfJob> hj;
    hj.reserve((size_t)n_jobs);
    std::vector<int64_t> alone;
    long long tasks = 0, pixels = 0;
    int max_chunks = 1, max_task = 1, max_bounces = 0;
    for (int64_t k = 0; k < n_jobs; ++k) {
        const tpt_batch_job& j = jobs[k];
        tpt_render_config c = j.config;
        check_config(c);
        if (c.mode != TPT_MODE_WAVEFRONT_FP32)
            throw TptError(TPT_ERR_UNSUPPORTED, "batch jobs render in the FP32 wavefront form");
        if (c.adaptive_enabled) throw TptError(TPT_ERR_UNSUPPORTED, "batch jobs cannot use adaptive sampling");
        if (j.scene < 0 || (size_t)j.scene >= B.scenes.size()) throw TptError(TPT_ERR_INVALID, "job scene out of range");
        if (!j.d_acc || !j.d_acc_w) throw TptError(TPT_ERR_INVALID, "null job film");
        // (decided at the job's own spp, so that the autotuner's shorter
        // trials split the jobs as the render will)
        if (alone_paths > 0 && (long long)c.width * film_rows(c) * c.spp >= alone_paths) {
            alone.push_back(k);
            continue;
        }
        if (spp_div > 1) c.spp = std::max(1, c.spp / spp_div);
        const BatchScene& bs = B.scenes[(size_t)j.scene];
        hj.emplace_back();
        WfJob& J = hj.back();
        J.cam = bs.cam;
        J.top_root = bs.top_root;
        J.env_kind = bs.env_kind; J.env_w = bs.env_w; J.env_h = bs.env_h; J.env_has_cdf = bs.env_has_cdf;
        J.env_tex = B.wf.env_tex ? B.wf.env_tex + bs.env_tex_off : nullptr;
        J.env_row = B.wf.env_row ? B.wf.env_row + bs.env_row_off : nullptr;
        J.env_col = B.wf.env_col ? B.wf.env_col + bs.env_col_off : nullptr;
        J.lights = B.wf.lights ? B.wf.lights + bs.light_begin : nullptr;
        J.light_cdf = B.wf.light_cdf ? B.wf.light_cdf + bs.light_begin : nullptr;
        J.lights64 = B.wf.lights64 ? B.wf.lights64 + bs.light_begin : nullptr;
        J.n_lights = bs.n_lights;
        J.width = c.width; J.height = c.height; J.spp = c.spp; J.max_bounces = c.max_bounces; J.rr_start = c.rr_start;
        J.seed = c.seed;
        J.row_begin = row_begin_of(c);
        J.row_step = row_step_of(c);
        J.n_pixels = c.width * film_rows(c);
        J.task_spp = std::min(sc.task_spp, c.spp);
        check_wavefront_limits(c.max_bounces, J.task_spp);
        J.n_chunks = (c.spp + J.task_spp - 1) / J.task_spp;
        J.task_begin = tasks;
        J.n_tasks = (long long)J.n_pixels * J.n_chunks;
        J.pixel_begin = pixels;
        J.acc = j.d_acc;
        J.acc_w = j.d_acc_w;
        J.px_div = make_fastdiv((uint32_t)J.n_pixels);
        J.w_div = make_fastdiv((uint32_t)J.width);
        tasks += J.n_tasks;
        pixels += J.n_pixels;
        max_chunks = std::max(max_chunks, J.n_chunks);
        max_task = std::max(max_task, J.task_spp);
        max_bounces = std::max(max_bounces, c.max_bounces);
    }
    tpt_stats s{};
    for (int64_t k : alone) {
        const tpt_batch_job& j = jobs[k];
        tpt_render_config c = j.config;
        if (spp_div > 1) c.spp = std::max(1, c.spp / spp_div);
        const BatchScene& bs = B.scenes[(size_t)j.scene];
        WfScene S = B.wf;
        S.cam = bs.cam;
        S.top_root = bs.top_root;
        S.env_kind = bs.env_kind; S.env_w = bs.env_w; S.env_h = bs.env_h; S.env_has_cdf = bs.env_has_cdf;
        S.env_tex = B.wf.env_tex ? B.wf.env_tex + bs.env_tex_off : nullptr;
        S.env_row = B.wf.env_row ? B.wf.env_row + bs.env_row_off : nullptr;
        S.env_col = B.wf.env_col ? B.wf.env_col + bs.env_col_off : nullptr;
        S.lights = B.wf.lights ? B.wf.lights + bs.light_begin : nullptr;
        S.light_cdf = B.wf.light_cdf ? B.wf.light_cdf + bs.light_begin : nullptr;
        S.lights64 = B.wf.lights64 ? B.wf.lights64 + bs.light_begin : nullptr;
        S.n_lights = bs.n_lights;
        WfParams p{};
        fill_wf_params(c, p, false);
        WfCounters hc{};
        float ms = 0.0f;
        ck(wf_render(S, p, B.wfbuf, j.d_acc, j.d_acc_w, nullptr, B.stream, B.sm_count, true, &hc, &ms),
           "batch render (job alone)");
        add_stats(s, hc, ms);
        if (hc.flags != 0) break;
    }
    if (hj.empty() || s.device_flags != 0) {
        s.task_spp = sc.task_spp;
        if (stats) *stats = s;
        if (s.device_flags != 0) {
            char buf[128];
            std::snprintf(buf, sizeof buf, "kernel raised device flags 0x%x", s.device_flags);
            throw TptError(TPT_ERR_DEVICE, buf);
        }
        return;
    }
    if (tasks >= (1ll << 31)) throw TptError(TPT_ERR_UNSUPPORTED, "batch has more than 2^31 tasks");
    if (B.d_jobs_n < hj.size()) {
        if (B.d_jobs) cudaFree(B.d_jobs);
        B.d_jobs = nullptr;
        B.d_jobs_n = 0;
        ck(cudaMalloc(&B.d_jobs, hj.size() * sizeof(WfJob)), "cudaMalloc(jobs)");
        B.d_jobs_n = hj.size();
    }
    ck(cudaMemcpyAsync(B.d_jobs, hj.data(), hj.size() * sizeof(WfJob), cudaMemcpyHostToDevice, B.stream),
       "upload jobs");
    WfParams p{};
    p.n_tasks = tasks;
    p.n_slots = (int)std::min(tasks, sc.pool);
    p.n_chunks = max_chunks;
    p.task_spp = max_task;
    p.max_bounces = max_bounces;
    const long long rounds = (tasks + p.n_slots - 1) / p.n_slots + 1;
    p.max_iters = (long long)max_task * (long long)(max_bounces + 1) * rounds + 16;
    p.trace_chunk = sc.trace_chunk;
    {
        const int fast = env_int("TPT_CAMERA_FAST", 2);  // 2: on unless camera culling takes the open pixels
        p.camera_fast = fast == 0 ? 0 : (fast == 1 ? 1 : 2);
    }
    p.sky_cull = env_int("TPT_SKY_CULL", 1) != 0;
    p.tail_live = std::max(-1, env_int("TPT_TAIL_SLOTS", -1));
    p.ext_queue = 1;
    p.queue_div = queue_div_setting();
    p.ordered_queue = env_int("TPT_QUEUE_ORDER", 1) != 0;
    p.shade_ctas = sc.shade_ctas;
    p.jobs = B.d_jobs;
    p.n_jobs = (int)hj.size();
    p.total_pixels = pixels;
    p.n_pixels = 0;
    WfCounters hc{};
    float ms = 0.0f;
    ck(wf_render(B.wf, p, B.wfbuf, nullptr, nullptr, nullptr, B.stream, B.sm_count, true, &hc, &ms),
       "batch render");
    add_stats(s, hc, ms);
    s.task_spp = sc.task_spp;
    if (stats) *stats = s;
    if (s.device_flags != 0) {
        char buf[128];
        std::snprintf(buf, sizeof buf, "kernel raised device flags 0x%x", s.device_flags);
        throw TptError(TPT_ERR_DEVICE, buf);
    }
}

}  // namespace
}  // namespace tpt

using namespace tpt;

extern "C" {

const char* tpt_last_error(void) { return g_last_error.c_str(); }
const char* tpt_version(void) { return "tinypt-b200 0.1 (sm_100a)"; }

int64_t tpt_bvh_build_host(const tpt_mesh_desc* mesh, double* bbox, int32_t* lr, uint32_t* sc, int64_t* indices) {
    int64_t result = 0;
    int rc = guarded([&] {
        if (!mesh) throw TptError(TPT_ERR_INVALID, "null mesh");
        if (mesh->n_tris < 0 || (mesh->n_tris > 0 && (!mesh->positions || !mesh->indices)))
            throw TptError(TPT_ERR_INVALID, "bad mesh description");
        HostBvh b = build_mesh_bvh(mesh->positions, mesh->n_vertices, mesh->indices, mesh->n_tris);
        const size_t n = b.left_right.size() / 2;
        if (bbox) std::memcpy(bbox, b.bbox.data(), n * 6 * sizeof(double));
        if (lr) std::memcpy(lr, b.left_right.data(), n * 2 * sizeof(int32_t));
        if (sc) std::memcpy(sc, b.start_count.data(), n * 2 * sizeof(uint32_t));
        if (indices) std::memcpy(indices, b.indices.data(), b.indices.size() * sizeof(int64_t));
        result = (int64_t)n;
        return TPT_OK;
    });
    return rc == TPT_OK ? result : (int64_t)rc;
}

int64_t tpt_bvh_build_fp32(const tpt_mesh_desc* mesh, double* bbox, int32_t* lr, uint32_t* sc, int64_t* indices) {
    int64_t result = 0;
    int rc = guarded([&] {
        if (!mesh) throw TptError(TPT_ERR_INVALID, "null mesh");
        if (mesh->n_tris < 0 || (mesh->n_tris > 0 && (!mesh->positions || !mesh->indices)))
            throw TptError(TPT_ERR_INVALID, "bad mesh description");
        HostBvh b = build_fp32_mesh_bvh(mesh->positions, mesh->n_vertices, mesh->indices, mesh->n_tris);
        const size_t n = b.left_right.size() / 2;
        if (bbox) std::memcpy(bbox, b.bbox.data(), n * 6 * sizeof(double));
        if (lr) std::memcpy(lr, b.left_right.data(), n * 2 * sizeof(int32_t));
        if (sc) std::memcpy(sc, b.start_count.data(), n * 2 * sizeof(uint32_t));
        if (indices) std::memcpy(indices, b.indices.data(), b.indices.size() * sizeof(int64_t));
        result = (int64_t)n;
        return TPT_OK;
    });
    return rc == TPT_OK ? result : (int64_t)rc;
}

int64_t tpt_bvh_build_device(const tpt_mesh_desc* mesh, double* bbox, int32_t* lr, uint32_t* sc, int64_t* indices) {
    int64_t result = 0;
    int rc = guarded([&] {
        if (!mesh) throw TptError(TPT_ERR_INVALID, "null mesh");
        if (mesh->n_tris < 0 || mesh->n_vertices < 0 || (mesh->n_tris > 0 && (!mesh->positions || !mesh->indices)))
            throw TptError(TPT_ERR_INVALID, "bad mesh description");
        std::string err;
        int64_t n = 0;
        const int r = build_mesh_bvh_gpu(
            mesh->positions, mesh->n_vertices, mesh->indices, mesh->n_tris,
            [&](int64_t) { return GpuBvhSink{bbox, lr, sc, indices}; }, nullptr, &n, &err);
        if (r == kGpuBvhCudaError) throw TptError(TPT_ERR_CUDA, "device BVH build: " + err);
        if (r == kGpuBvhNoMemory) throw TptError(TPT_ERR_ALLOC, "device BVH build: " + err);
        if (r == kGpuBvhUseHost) throw TptError(TPT_ERR_UNSUPPORTED, "device BVH build: " + err);
        result = n;
        return TPT_OK;
    });
    return rc == TPT_OK ? result : (int64_t)rc;
}

int tpt_scene_create(const tpt_scene_desc* desc, void** out_scene) {
    return guarded([&] {
        if (!desc || !out_scene) throw TptError(TPT_ERR_INVALID, "null argument");
        *out_scene = nullptr;
        HostScene hs;
        build_host_scene(*desc, hs, scene_mesh_bvh);
        auto h = std::make_unique<SceneHandle>();
        ck(cudaGetDevice(&h->device), "cudaGetDevice");
        ck(cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device), "device attribute");
        ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ck(cudaMalloc(&h->d_counters, 4 * sizeof(unsigned long long)), "cudaMalloc(counters)");
        ck(cudaMalloc(&h->d_flags, sizeof(int)), "cudaMalloc(flags)");

        PlainImage pi;
        flatten_plain(hs, pi);
        PlainScene& P = h->plain;
        P.nodes = h->upload(pi.nodes);
        P.tris = h->upload(pi.tris);
        P.meshes = h->upload(pi.meshes);
        P.instances = h->upload(pi.instances);
        P.n_instances = (int)pi.instances.size();
        P.spheres = h->upload(pi.spheres);
        P.n_spheres = (int)pi.spheres.size();
        P.mats = h->upload(pi.mats);
        P.lights = h->upload(pi.lights);
        P.light_cdf = h->upload(pi.light_cdf);
        P.n_lights = (int)pi.lights.size();
        P.light_total = hs.light_total;
        P.env_kind = hs.env_kind;
        P.env_w = hs.env_w;
        P.env_h = hs.env_h;
        P.env_data = h->upload(pi.env_data);
        P.env_row_cdf = h->upload(pi.env_row_cdf);
        P.env_col_cdf = h->upload(pi.env_col_cdf);
        P.env_total = hs.env_total;
        P.cam = hs.cam;

        Fp32Image fi;
        flatten_fp32(hs, fi);
        if (fi.max_stack > 64) throw TptError(TPT_ERR_UNSUPPORTED, "BVH deeper than the 64-entry traversal stack");
        h->max_stack = fi.max_stack;
        h->wf.max_stack = fi.max_stack;
        WfScene& W = h->wf;
        W.nodes = h->upload(fi.nodes);
        W.tris = h->upload(fi.tris);
        W.meshes = h->upload(fi.meshes);
        W.inst = h->upload(fi.instances);
        W.n_inst = (int)fi.instances.size();
        W.spheres = h->upload(fi.spheres);
        W.n_spheres = (int)fi.spheres.size();
        W.top_root = fi.top_root;
        W.mats = h->upload(fi.mats);
        W.lights = h->upload(fi.lights);
        W.light_cdf = h->upload(fi.light_cdf);
        W.n_lights = (int)fi.lights.size();
        W.env_kind = hs.env_kind;
        W.env_w = hs.env_w;
        W.env_h = hs.env_h;
        W.env_has_cdf = hs.env_total > 0.0;
        W.env_tex = h->upload(fi.env_texels);
        W.env_row = h->upload(fi.env_row_cdf);
        W.env_col = h->upload(fi.env_col_cdf);
        const CameraF64& c = hs.cam;
        W.cam.o = make_float3((float)c.o[0], (float)c.o[1], (float)c.o[2]);
        W.cam.u = make_float3((float)c.u[0], (float)c.u[1], (float)c.u[2]);
        W.cam.v = make_float3((float)c.v[0], (float)c.v[1], (float)c.v[2]);
        W.cam.w = make_float3((float)c.w[0], (float)c.w[1], (float)c.w[2]);
        W.cam.half_h = (float)c.half_h;
        W.cam.half_w = (float)c.half_w;
        W.cam.lens_radius = (float)c.lens_radius;
        W.cam.focus_dist = (float)c.focus_dist;
        W.lights64 = P.lights;
        W.inst64 = P.instances;
        W.spheres64 = P.spheres;
        ck(cudaStreamSynchronize(h->stream), "scene upload");
        for (HostScene::Mesh& m : hs.meshes) m.bvh = HostBvh{};
        h->hs = std::move(hs);
        *out_scene = h.release();
        return TPT_OK;
    });
}

void tpt_scene_destroy(void* scene) {
    auto* h = static_cast<SceneHandle*>(scene);
    if (!h) return;
    // frees on the handle's device; never throws (no guard object here)
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaSetDevice(h->device);
    delete h;
    if (prev >= 0) cudaSetDevice(prev);
}

int tpt_render_device(void* scene, const tpt_render_config* config, double* d_acc, double* d_acc_w,
                      double* d_acc_sq, tpt_stats* stats) {
    return guarded([&] {
        if (!scene || !config || !d_acc || !d_acc_w) throw TptError(TPT_ERR_INVALID, "null argument");
        render_device(*static_cast<SceneHandle*>(scene), *config, d_acc, d_acc_w, d_acc_sq, stats);
        return TPT_OK;
    });
}

int tpt_render_device_noalloc(void* scene, const tpt_render_config* config, double* d_acc, double* d_acc_w,
                              tpt_stats* stats) {
    return guarded([&] {
        if (!scene || !config || !d_acc || !d_acc_w) throw TptError(TPT_ERR_INVALID, "null argument");
        SceneHandle& h = *static_cast<SceneHandle*>(scene);
        tpt_render_config c = *config;
        c.mode = TPT_MODE_WAVEFRONT_FP32;
        check_config(c);
        const long long px = (long long)c.width * film_rows(c);
        if ((size_t)px > wf_noalloc_max_slots()) {
            char buf[160];
            std::snprintf(buf, sizeof buf,
                          "tpt_render_device_noalloc: film of %lld pixels exceeds the allocation-free limit of %zu",
                          px, wf_noalloc_max_slots());
            throw TptError(TPT_ERR_INVALID, buf);
        }
        DeviceGuard device_guard(h.device);
        WfParams p{};
        fill_wf_params(c, p, true);
        WfCounters hc{};
        ck(wf_render_noalloc(h.wf, p, d_acc, d_acc_w, h.stream, h.sm_count, &hc), "allocation-free render");
        tpt_stats s{};
        s.rays_closest = hc.rays_closest;
        s.rays_shadow = hc.rays_shadow;
        s.iterations = (uint64_t)hc.iters;
        s.device_flags = hc.flags;
        s.paths = hc.samples;
        if (stats) *stats = s;
        if (s.device_flags != 0) {
            char buf[128];
            std::snprintf(buf, sizeof buf, "kernel raised device flags 0x%x", s.device_flags);
            throw TptError(TPT_ERR_DEVICE, buf);
        }
        return TPT_OK;
    });
}

int tpt_render(void* scene, const tpt_render_config* config, double* acc, double* acc_w, tpt_stats* stats) {
    return guarded([&] {
        if (!scene || !config || !acc || !acc_w) throw TptError(TPT_ERR_INVALID, "null argument");
        SceneHandle& h = *static_cast<SceneHandle*>(scene);
        check_config(*config);
        const size_t px = (size_t)config->width * (size_t)film_rows(*config);
        DeviceGuard device_guard(h.device);
        if (h.film_px < px) {
            if (h.film) cudaFree(h.film);
            h.film = nullptr;
            h.film_px = 0;
            ck(cudaMalloc(&h.film, px * 4 * sizeof(double)), "cudaMalloc(film)");
            h.film_px = px;
        }
        double* d_acc = h.film;
        double* d_w = h.film + 3 * px;
        tpt_stats s{};
        s.profile = stats ? stats->profile : 0;
        render_device(h, *config, d_acc, d_w, nullptr, &s);
        ck(cudaMemcpyAsync(acc, d_acc, 3 * px * sizeof(double), cudaMemcpyDeviceToHost, h.stream), "copy acc");
        ck(cudaMemcpyAsync(acc_w, d_w, px * sizeof(double), cudaMemcpyDeviceToHost, h.stream), "copy acc_w");
        ck(cudaStreamSynchronize(h.stream), "render sync");
        if (s.paths == 0)
            for (size_t i = 0; i < px; ++i) s.paths += (uint64_t)acc_w[i];
        if (stats) *stats = s;
        return TPT_OK;
    });
}

int64_t tpt_scene_material_count(void* scene) {
    if (!scene) return -1;
    return (int64_t)static_cast<SceneHandle*>(scene)->hs.mats.size();
}

int tpt_scene_set_materials(void* scene, const tpt_material* materials, const tpt_material* sampling_materials,
                            int64_t n_materials) {
    return guarded([&] {
        if (!scene || !materials || n_materials < 0) throw TptError(TPT_ERR_INVALID, "null argument");
        SceneHandle& h = *static_cast<SceneHandle*>(scene);
        DeviceGuard device_guard(h.device);
        ck(cudaStreamSynchronize(h.stream), "sync before material update");
        set_materials(h.hs, materials, sampling_materials, (size_t)n_materials);
        h.detached = sampling_materials &&
                     std::memcmp(materials, sampling_materials, (size_t)n_materials * sizeof(tpt_material)) != 0;
        std::vector<MaterialF32> fm;
        std::vector<LightF32> fl;
        std::vector<float> fcdf;
        flatten_fp32_materials(h.hs, fm, fl, fcdf);
        std::vector<MaterialF64> pm;
        std::vector<LightF64> pl;
        flatten_plain_materials(h.hs, pm, pl);
        if (!fm.empty())
            ck(cudaMemcpyAsync((void*)h.wf.mats, fm.data(), fm.size() * sizeof(MaterialF32), cudaMemcpyHostToDevice,
                               h.stream), "upload materials");
        if (!pm.empty())
            ck(cudaMemcpyAsync((void*)h.plain.mats, pm.data(), pm.size() * sizeof(MaterialF64),
                               cudaMemcpyHostToDevice, h.stream), "upload materials");
        h.reupload(h.wf.lights, fl);
        h.reupload(h.wf.light_cdf, fcdf);
        h.wf.n_lights = (int)fl.size();
        h.reupload(h.plain.lights, pl);
        h.reupload(h.plain.light_cdf, h.hs.light_cdf);
        h.plain.n_lights = (int)pl.size();
        h.plain.light_total = h.hs.light_total;
        h.wf.lights64 = h.plain.lights;
        ck(cudaStreamSynchronize(h.stream), "material upload");
        return TPT_OK;
    });
}

int tpt_render_forward_device(void* scene, const tpt_render_config* config, float* d_image, tpt_stats* stats) {
    return guarded([&] {
        if (!scene || !config || !d_image) throw TptError(TPT_ERR_INVALID, "null argument");
        SceneHandle& h = *static_cast<SceneHandle*>(scene);
        check_config(*config);
        const size_t px = (size_t)config->width * (size_t)film_rows(*config);
        DeviceGuard device_guard(h.device);
        if (h.film_px < px) {
            if (h.film) cudaFree(h.film);
            h.film = nullptr;
            h.film_px = 0;
            ck(cudaMalloc(&h.film, px * 4 * sizeof(double)), "cudaMalloc(film)");
            h.film_px = px;
        }
        tpt_stats s{};
        s.profile = stats ? stats->profile : 0;
        render_device(h, *config, h.film, h.film + 3 * px, nullptr, &s);
        ck(resolve_film(h.film, h.film + 3 * px, d_image, (int)px, h.stream), "resolve");
        ck(cudaStreamSynchronize(h.stream), "forward sync");
        if (stats) *stats = s;
        return TPT_OK;
    });
}

int tpt_render_forward(void* scene, const tpt_render_config* config, float* image, tpt_stats* stats) {
    return guarded([&] {
        if (!scene || !config || !image) throw TptError(TPT_ERR_INVALID, "null argument");
        SceneHandle& h = *static_cast<SceneHandle*>(scene);
        check_config(*config);
        const size_t px = (size_t)config->width * (size_t)film_rows(*config);
        DeviceGuard device_guard(h.device);
        if (h.img_px < px) {
            if (h.img) cudaFree(h.img);
            h.img = nullptr;
            h.img_px = 0;
            ck(cudaMalloc(&h.img, px * 3 * sizeof(float)), "cudaMalloc(image)");
            h.img_px = px;
        }
        const int rc = tpt_render_forward_device(scene, config, h.img, stats);
        if (rc != TPT_OK) throw TptError(rc, g_last_error);
        ck(cudaMemcpy(image, h.img, px * 3 * sizeof(float), cudaMemcpyDeviceToHost), "copy image");
        return TPT_OK;
    });
}

int tpt_render_backward_device(void* scene, const tpt_render_config* config, const float* d_dL_dimage,
                               double* d_grad, tpt_stats* stats) {
    return guarded([&] {
        if (!scene || !config || !d_dL_dimage || !d_grad) throw TptError(TPT_ERR_INVALID, "null argument");
        SceneHandle& h = *static_cast<SceneHandle*>(scene);
        const tpt_render_config& c = *config;
        check_config(c);
        if (c.mode != TPT_MODE_WAVEFRONT_FP32)
            throw TptError(TPT_ERR_UNSUPPORTED, "the adjoint differentiates the FP32 form (mode WAVEFRONT_FP32)");
        if (c.adaptive_enabled) throw TptError(TPT_ERR_UNSUPPORTED, "the adjoint needs a fixed spp (adaptive off)");
        DeviceGuard device_guard(h.device);
        AdjParams p{};
        p.width = c.width; p.height = c.height; p.spp = c.spp;
        p.max_bounces = c.max_bounces; p.rr_start = c.rr_start;
        p.seed = c.seed;
        p.n_pixels = c.width * film_rows(c);
        p.row_begin = row_begin_of(c);
        p.row_step = row_step_of(c);
        // the forward form's task split, so that sample s of a pixel draws
        // the same PCG32 stream in both renders
        p.task_spp = task_spp_for(c, p.n_pixels);
        check_wavefront_limits(c.max_bounces, p.task_spp);
        p.n_chunks = (c.spp + p.task_spp - 1) / p.task_spp;
        p.n_tasks = (long long)p.n_pixels * p.n_chunks;
        p.px_div = make_fastdiv((uint32_t)p.n_pixels);
        p.w_div = make_fastdiv((uint32_t)p.width);
        p.queue_div = queue_div_setting();
        p.ordered_queue = env_int("TPT_QUEUE_ORDER", 1) != 0;
        p.sky_cull = env_int("TPT_SKY_CULL", 1) != 0;
        p.n_mats = (int)h.hs.mats.size();
        if (p.n_mats == 0) return TPT_OK;
        p.trace_chunk = trace_chunk_setting();
        float ms = 0.0f;
        unsigned long long culled = 0;
        // TPT_ADJOINT=megakernel: the one-kernel two-pass replay (a cross-check)
        const char* form = std::getenv("TPT_ADJOINT");
        if (form && std::strcmp(form, "megakernel") == 0) {
            ck(adj_render_backward(h.wf, p, d_dL_dimage, d_grad, h.d_flags, h.d_counters, h.stream, h.sm_count, &ms),
               "adjoint render");
        } else {
            const long long pool = env_int("TPT_POOL", kDefaultPool);
            const char* loop = std::getenv("TPT_WAVEFRONT_HOST_LOOP");
            const bool graph = !(loop && loop[0] == '1');
            ck(adj_render_backward_wf(h.wf, p, h.wfbuf, h.adjbuf, pool < 1 ? 1 : pool, d_dL_dimage, d_grad, h.d_flags,
                                      h.d_counters, h.stream, h.sm_count, graph, &ms, &culled),
               "adjoint render");
        }
        unsigned long long cnt[2] = {0, 0};
        int flags = 0;
        ck(cudaMemcpyAsync(cnt, h.d_counters, sizeof(cnt), cudaMemcpyDeviceToHost, h.stream), "copy counters");
        ck(cudaMemcpyAsync(&flags, h.d_flags, sizeof(int), cudaMemcpyDeviceToHost, h.stream), "copy flags");
        ck(cudaStreamSynchronize(h.stream), "adjoint sync");
        tpt_stats s{};
        s.render_ms = ms;
        s.paths = cnt[0];
        std::memcpy(&s.adjoint_linear, &cnt[1], sizeof(double));
        s.device_flags = flags;
        s.task_spp = p.task_spp;
        s.sky_samples = culled;
        if (stats) *stats = s;
        if (flags != 0) {
            char buf[128];
            std::snprintf(buf, sizeof buf, "kernel raised device flags 0x%x", flags);
            throw TptError(TPT_ERR_DEVICE, buf);
        }
        return TPT_OK;
    });
}

int tpt_render_backward(void* scene, const tpt_render_config* config, const float* dL_dimage, double* grad,
                        tpt_stats* stats) {
    return guarded([&] {
        if (!scene || !config || !dL_dimage || !grad) throw TptError(TPT_ERR_INVALID, "null argument");
        SceneHandle& h = *static_cast<SceneHandle*>(scene);
        check_config(*config);
        const size_t px = (size_t)config->width * (size_t)film_rows(*config);
        const size_t n_par = 4 * h.hs.mats.size();
        DeviceGuard device_guard(h.device);
        if (h.img_px < px) {
            if (h.img) cudaFree(h.img);
            h.img = nullptr;
            h.img_px = 0;
            ck(cudaMalloc(&h.img, px * 3 * sizeof(float)), "cudaMalloc(image)");
            h.img_px = px;
        }
        if (h.grad_n < n_par) {
            if (h.grad) cudaFree(h.grad);
            h.grad = nullptr;
            h.grad_n = 0;
            ck(cudaMalloc(&h.grad, (n_par ? n_par : 1) * sizeof(double)), "cudaMalloc(grad)");
            h.grad_n = n_par;
        }
        ck(cudaMemcpy(h.img, dL_dimage, px * 3 * sizeof(float), cudaMemcpyHostToDevice), "copy dL/dimage");
        const int rc = tpt_render_backward_device(scene, config, h.img, h.grad, stats);
        if (rc != TPT_OK) throw TptError(rc, g_last_error);
        if (n_par) ck(cudaMemcpy(grad, h.grad, n_par * sizeof(double), cudaMemcpyDeviceToHost), "copy gradient");
        return TPT_OK;
    });
}

int tpt_batch_create(const tpt_scene_desc* scenes, int64_t n_scenes, void** out_batch) {
    return guarded([&] {
        if (!scenes || !out_batch || n_scenes <= 0) throw TptError(TPT_ERR_INVALID, "null argument or no scenes");
        *out_batch = nullptr;
        std::vector<HostScene> hs((size_t)n_scenes);
        std::vector<const HostScene*> ptrs;
        for (int64_t i = 0; i < n_scenes; ++i) {
            build_host_scene(scenes[i], hs[(size_t)i], scene_mesh_bvh);
            ptrs.push_back(&hs[(size_t)i]);
        }
        BatchImage bi;
        merge_scenes(ptrs, bi);
        if (bi.fp.max_stack > 64) throw TptError(TPT_ERR_UNSUPPORTED, "BVH deeper than the 64-entry traversal stack");
        auto b = std::make_unique<BatchHandle>();
        ck(cudaGetDevice(&b->device), "cudaGetDevice");
        ck(cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, b->device), "device attribute");
        ck(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        WfScene& W = b->wf;
        const Fp32Image& F = bi.fp;
        W.nodes = b->upload(F.nodes);
        W.tris = b->upload(F.tris);
        W.meshes = b->upload(F.meshes);
        W.inst = b->upload(F.instances);
        W.n_inst = (int)F.instances.size();
        W.spheres = b->upload(F.spheres);
        W.n_spheres = (int)F.spheres.size();
        W.top_root = TPT_REF_NONE;
        W.mats = b->upload(F.mats);
        W.lights = b->upload(F.lights);
        W.light_cdf = b->upload(F.light_cdf);
        W.n_lights = 0;
        W.env_tex = b->upload(F.env_texels);
        W.env_row = b->upload(F.env_row_cdf);
        W.env_col = b->upload(F.env_col_cdf);
        W.lights64 = b->upload(bi.lights64);
        W.inst64 = b->upload(bi.inst64);
        W.spheres64 = b->upload(bi.spheres64);
        W.max_stack = F.max_stack;
        b->scenes = bi.scenes;
        ck(cudaStreamSynchronize(b->stream), "batch upload");
        *out_batch = b.release();
        return TPT_OK;
    });
}

void tpt_batch_destroy(void* batch) {
    auto* b = static_cast<BatchHandle*>(batch);
    if (!b) return;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaSetDevice(b->device);
    delete b;
    if (prev >= 0) cudaSetDevice(prev);
}

int tpt_batch_render_device(void* batch, const tpt_batch_job* jobs, int64_t n_jobs, const tpt_tuning* tuning,
                            tpt_stats* stats) {
    return guarded([&] {
        if (!batch || !jobs) throw TptError(TPT_ERR_INVALID, "null argument");
        batch_render(*static_cast<BatchHandle*>(batch), jobs, n_jobs, schedule_of(tuning), 1, stats);
        return TPT_OK;
    });
}

int tpt_batch_autotune(void* batch, const tpt_batch_job* jobs, int64_t n_jobs, tpt_tuning* best, double* trial_ms,
                       int32_t n_trials) {
    return guarded([&] {
        if (!batch || !jobs || !best) throw TptError(TPT_ERR_INVALID, "null argument");
        BatchHandle& B = *static_cast<BatchHandle*>(batch);
        long long total_tasks = 0;
        for (int64_t k = 0; k < n_jobs; ++k)
            total_tasks += (long long)jobs[k].config.width * jobs[k].config.height;
        // Trials at half of each job's spp (a quarter picked schedules that
        // were slower at the full spp); coordinate descent over the pool size,
        // the task length, the refill chunk, then the shading kernel's blocks
        // per SM.  Each coordinate skips the value it starts from: that
        // schedule is the one best_ms was measured on.
        const int div = 2;
        Schedule cur = schedule_of(nullptr);
        int trials = 0;
        auto trial = [&](const Schedule& sc) {
            tpt_stats st{};
            batch_render(B, jobs, n_jobs, sc, div, &st);
            if (trial_ms && trials < n_trials) trial_ms[trials] = st.render_ms;
            ++trials;
            return (double)st.render_ms;
        };
        trial(cur);  // warm-up (allocations, graph build)
        double best_ms = trial(cur);
        const long long pools[] = {1 << 20, 4 << 20, 16 << 20, 32 << 20, 64 << 20};
        const long long pool0 = cur.pool;
        for (long long pool : pools) {
            if (pool == pool0 || pool > 2 * total_tasks) continue;
            Schedule sc = cur;
            sc.pool = pool;
            const double ms = trial(sc);
            if (ms < best_ms) { best_ms = ms; cur = sc; }
        }
        const int tasks_spp[] = {4, 8, 16, 32};
        const int task0 = cur.task_spp;
        for (int ts : tasks_spp) {
            if (ts == task0) continue;
            Schedule sc = cur;
            sc.task_spp = ts;
            const double ms = trial(sc);
            if (ms < best_ms) { best_ms = ms; cur = sc; }
        }
        const int chunks[] = {2, 4, 8, 16};
        const int chunk0 = cur.trace_chunk;
        for (int ch : chunks) {
            if (ch == chunk0) continue;
            Schedule sc = cur;
            sc.trace_chunk = ch;
            const double ms = trial(sc);
            if (ms < best_ms) { best_ms = ms; cur = sc; }
        }
        {
            Schedule sc = cur;
            sc.shade_ctas = cur.shade_ctas == 8 ? 4 : 8;
            const double ms = trial(sc);
            if (ms < best_ms) { best_ms = ms; cur = sc; }
        }
        best->pool_slots = (int32_t)cur.pool;
        best->task_spp = cur.task_spp;
        best->trace_chunk = cur.trace_chunk;
        best->shade_ctas = cur.shade_ctas;
        return trials;
    });
}

// ---- scene ingestion and image files (host only) ----------------------------------
int tpt_scene_load_xml(const char* path, tpt_render_config* config, void** out_loaded) {
    return guarded([&] {
        if (!path || !config || !out_loaded) throw TptError(TPT_ERR_INVALID, "null argument");
        *out_loaded = nullptr;
        tpt_render_config c = *config;
        auto sc = load_mitsuba(path, c);
        *config = c;
        *out_loaded = sc.release();
        return TPT_OK;
    });
}

int tpt_scene_default(const tpt_render_config* config, const char* env_path, void** out_loaded) {
    return guarded([&] {
        if (!config || !out_loaded) throw TptError(TPT_ERR_INVALID, "null argument");
        if (config->width <= 0 || config->height <= 0) throw TptError(TPT_ERR_INVALID, "bad film size");
        *out_loaded = default_scene(*config, env_path ? std::string(env_path) : std::string()).release();
        return TPT_OK;
    });
}

const tpt_scene_desc* tpt_loaded_desc(void* loaded) {
    return loaded ? &static_cast<LoadedScene*>(loaded)->desc : nullptr;
}

int64_t tpt_loaded_warning_count(void* loaded) {
    return loaded ? (int64_t)static_cast<LoadedScene*>(loaded)->warnings.size() : 0;
}

const char* tpt_loaded_warning(void* loaded, int64_t i) {
    if (!loaded) return "";
    const auto& w = static_cast<LoadedScene*>(loaded)->warnings;
    return (i >= 0 && (size_t)i < w.size()) ? w[(size_t)i].c_str() : "";
}

void tpt_loaded_destroy(void* loaded) { delete static_cast<LoadedScene*>(loaded); }

int tpt_write_image(const char* path, int32_t width, int32_t height, const double* rgb, double exposure,
                    int32_t tonemap) {
    return guarded([&] {
        if (!path || !rgb) throw TptError(TPT_ERR_INVALID, "null argument");
        if (tonemap != 0 && tonemap != 1) throw TptError(TPT_ERR_INVALID, "tonemap must be 0 (none) or 1 (aces)");
        write_image(path, width, height, rgb, exposure, tonemap);
        return TPT_OK;
    });
}

int tpt_read_hdr(const char* path, int32_t* width, int32_t* height, double* rgb) {
    return guarded([&] {
        if (!path || !width || !height) throw TptError(TPT_ERR_INVALID, "null argument");
        int w = 0, h = 0;
        std::vector<double> px;
        read_hdr(path, w, h, px);
        if (rgb) {
            if (*width != w || *height != h) throw TptError(TPT_ERR_INVALID, "buffer size differs from the image");
            std::memcpy(rgb, px.data(), px.size() * sizeof(double));
        }
        *width = w;
        *height = h;
        return TPT_OK;
    });
}

// ---- checkpoints (src/checkpoint.rs) ------------------------------------------------
int tpt_checkpoint_save(const char* path, uint64_t scene_hash, int32_t width, int32_t height, uint64_t next_id,
                        const double* acc, const double* acc_w) {
    return guarded([&] {
        if (!path || !acc || !acc_w || width <= 0 || height <= 0) throw TptError(TPT_ERR_INVALID, "bad argument");
        save_checkpoint(path, scene_hash, width, height, next_id, acc, acc_w);
        return TPT_OK;
    });
}

int tpt_checkpoint_load(const char* path, uint64_t scene_hash, int32_t width, int32_t height, uint64_t* next_id,
                        double* acc, double* acc_w) {
    int found = 0;
    const int rc = guarded([&] {
        if (!path || !acc || !acc_w || !next_id || width <= 0 || height <= 0)
            throw TptError(TPT_ERR_INVALID, "bad argument");
        uint64_t nid = 0;
        found = load_checkpoint(path, scene_hash, width, height, nid, acc, acc_w) ? 1 : 0;
        if (found) *next_id = nid;
        return TPT_OK;
    });
    return rc == TPT_OK ? found : rc;
}

int64_t tpt_film_tiles(int32_t width, int32_t height, int32_t tile, int32_t morton, int32_t* x0y0x1y1) {
    int64_t n = -1;
    const int rc = guarded([&] {
        const auto t = film_tiles(width, height, tile, morton != 0);
        if (x0y0x1y1)
            for (size_t k = 0; k < t.size(); ++k) {
                x0y0x1y1[4 * k] = t[k].x0; x0y0x1y1[4 * k + 1] = t[k].y0;
                x0y0x1y1[4 * k + 2] = t[k].x1; x0y0x1y1[4 * k + 3] = t[k].y1;
            }
        n = (int64_t)t.size();
        return TPT_OK;
    });
    return rc == TPT_OK ? n : rc;
}

int tpt_render_resume(void* scene, const tpt_render_config* config, const char* ckpt_path, uint64_t scene_hash,
                      double* acc, double* acc_w, tpt_stats* stats) {
    return guarded([&] {
        if (!scene || !config || !ckpt_path || !acc || !acc_w) throw TptError(TPT_ERR_INVALID, "null argument");
        const tpt_render_config& c = *config;
        check_config(c);
        if (c.row_step > 0) throw TptError(TPT_ERR_UNSUPPORTED, "resume renders whole films");
        const size_t n = (size_t)c.width * (size_t)c.height;
        std::vector<double> a(3 * n, 0.0), aw(n, 0.0);
        // src/render.rs:56-68: only Ok(Some(..)) resumes; a file that is
        // absent, does not match or cannot be read starts a fresh film.
        uint64_t next_id = 0;
        bool resumed = false;
        try {
            resumed = load_checkpoint(ckpt_path, scene_hash, c.width, c.height, next_id, a.data(), aw.data());
        } catch (const std::exception&) {
            resumed = false;
        }
        if (!resumed) {
            std::fill(a.begin(), a.end(), 0.0);
            std::fill(aw.begin(), aw.end(), 0.0);
            next_id = 0;
        }
        const auto tiles = film_tiles(c.width, c.height, c.tile > 0 ? c.tile : 16, c.morton_enabled != 0);
        std::vector<double> na(3 * n), nw(n);
        tpt_stats s{};
        s.profile = 0;
        if (next_id < tiles.size()) {
            // every pixel's RNG stream is independent of the tile schedule, so
            // the tiles still to merge are those of a whole-film render
            const int rc = tpt_render(scene, config, na.data(), nw.data(), &s);
            if (rc != TPT_OK) throw TptError(rc, g_last_error);
            merge_tiles(tiles, (size_t)next_id, c.width, na.data(), nw.data(), a.data(), aw.data());
        }
        std::memcpy(acc, a.data(), a.size() * sizeof(double));
        std::memcpy(acc_w, aw.data(), aw.size() * sizeof(double));
        // src/render.rs:268-272: a failed final save is reported on stderr
        // and the film is still returned.
        try {
            save_checkpoint(ckpt_path, scene_hash, c.width, c.height, (uint64_t)tiles.size(), a.data(), aw.data());
        } catch (const std::exception& e) {
            std::fprintf(stderr, "Final checkpoint save failed: %s\n", e.what());
        }
        if (stats) *stats = s;
        return TPT_OK;
    });
}

}  // extern "C"
