// FP32 wavefront path integrator for sm_100a.
//
// The reference runs radiance() (src/integrator.rs:53-135) once per sample on
// CPU threads over Morton-ordered tiles (src/render.rs:116-206).  Here a
// pixel's samples are cut into tasks (the reference's Task with its
// sample_start seeding); a pool of path slots pulls tasks and runs each
// task's samples one after another, so a slot's u64 PCG32 state continues
// the task's reference stream draw for draw.  One bounce of all live paths
// is one iteration of:
//
//   trace<closest> : closest hit of every active slot (BVH2 traversal, FP32)
//   shade          : miss/env, Russian roulette, emitter, NEE sample
//                    generation (env + area light, power-heuristic MIS),
//                    BSDF sample; samples with nothing pending complete here
//   trace<any>     : occlusion of the NEE shadow rays
//   regen          : samples whose shadow rays were pending complete: the
//                    f64 sums (+ Welford for adaptive sampling), then the
//                    next camera ray or the next task
//
// Slots are visited in slot order (an active byte per slot); shadow records
// and pending completions go through queues filled with warp-aggregated
// atomics.  The iterations run inside one CUDA graph whose WHILE
// conditional node is re-armed on the device until no slot is active.
#include "fp32_device.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <type_traits>
#include <vector>

namespace tpt {
namespace wf {

// ---- kernels ------------------------------------------------------------------
// A task is the reference's Task restricted to one pixel (src/task.rs:11-27):
// samples [sample_start, sample_end) of that pixel, with the RNG seeded from
// seed_for(x, y, sample_start) ^ seed (src/render.rs:142).  Task t covers
// pixel t % n_pixels and sample chunk t / n_pixels; chunk 0 starts each
// pixel's reference stream.  With one chunk per pixel the schedule is the
// reference's own.
// Batch renders: a slot's task belongs to one job, whose scene view (root,
// camera, env map, lights), parameters and film overlay the batch-wide ones.
struct Film {
    double* acc;
    double* acc_w;
    double* acc_sq;
};
__device__ __forceinline__ void apply_job(const WfJob& J, WfScene& S, WfParams& P, Film& F, long long& base) {
    S.cam = J.cam;
    S.top_root = J.top_root;
    S.env_kind = J.env_kind; S.env_w = J.env_w; S.env_h = J.env_h; S.env_has_cdf = J.env_has_cdf;
    S.env_tex = J.env_tex; S.env_row = J.env_row; S.env_col = J.env_col;
    S.lights = J.lights; S.light_cdf = J.light_cdf; S.lights64 = J.lights64; S.n_lights = J.n_lights;
    P.width = J.width; P.height = J.height; P.spp = J.spp; P.max_bounces = J.max_bounces; P.rr_start = J.rr_start;
    P.seed = J.seed; P.n_pixels = J.n_pixels; P.task_spp = J.task_spp; P.n_chunks = J.n_chunks;
    P.row_begin = J.row_begin; P.row_step = J.row_step;
    P.px_map = nullptr; P.sample_base = 0; P.sample_end = J.spp;
    P.px_div = J.px_div; P.w_div = J.w_div;
    F.acc = J.acc; F.acc_w = J.acc_w; F.acc_sq = nullptr;
    base = J.task_begin;
}
// Job holding a batch-wide task id (tasks are numbered job after job).
__device__ __forceinline__ int find_job(const WfParams& P, long long task) {
    int lo = 0, hi = P.n_jobs;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (P.jobs[mid].task_begin <= task) lo = mid; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ Film film_of(const WfState& st) { return Film{st.acc, st.acc_w, st.acc_sq}; }

// Where task lt (its index within its job) sits: task-space pixel j = lt %
// n_pixels, sample chunk lt / n_pixels; the film pixel (through px_map in an
// adaptive round), its first sample and its length.
// Task ids are below 2^31 (the host lengthens tasks until they are).
struct TaskPos { int j, pixel, sample_start, len; };
__device__ __forceinline__ TaskPos task_pos(const WfParams& P, long long lt) {
    TaskPos t;
    const uint32_t u = (uint32_t)lt;
    const int chunk = (int)fdiv(P.px_div, u);
    t.j = (int)(u - (uint32_t)chunk * (uint32_t)P.n_pixels);
    t.pixel = P.px_map ? __ldg(P.px_map + t.j) : t.j;
    t.sample_start = P.sample_base + chunk * P.task_spp;
    const int end = P.sample_end > 0 ? P.sample_end : P.spp;
    t.len = min(P.task_spp, end - t.sample_start);
    return t;
}

// The pool's task cursor counts fetch ids from task_first.  Without camera
// culling a fetch id is the task itself.  With it (P.geo_map), the ids of
// the current chunk batch enumerate, chunk by chunk, the tasks of the n_geo
// pixels in geo_map, in film order: the task order of the batch with the
// culled pixels' tasks left out (k_sky_tasks renders those).  A multi-job
// render does the same per job, jobs one after another (WfJob::fetch_begin;
// geo_map then holds batch-wide pixel ids).
__device__ __forceinline__ long long fetch_end(const WfParams& P) {
    if (!P.geo_map) return P.n_tasks;
    if (P.jobs) return P.n_fetch;
    return P.task_first + (P.n_tasks - P.task_first) / P.n_pixels * P.n_geo;
}
// The last job whose begin (a job-ordered id space: fetch ids, sky tasks)
// is at most f; jobs with an empty stretch share the next job's begin.
template <class Begin>
__device__ __forceinline__ int job_at(const WfParams& P, long long f, Begin begin) {
    int lo = 0, hi = P.n_jobs;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (begin(P.jobs[mid]) <= f) lo = mid; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ long long task_of_fetch(const WfParams& P, long long f) {
    if (!P.geo_map) return f;
    if (P.jobs) {
        const WfJob& J = P.jobs[job_at(P, f, [](const WfJob& x) { return x.fetch_begin; })];
        const uint32_t v = (uint32_t)(f - J.fetch_begin);
        const uint32_t c = fdiv(J.geo_div, v);
        const int gp = __ldg(P.geo_map + J.geo_begin + (v - c * (uint32_t)J.n_geo));
        return J.task_begin + (long long)c * J.n_pixels + (gp - J.pixel_begin);
    }
    const uint32_t v = (uint32_t)(f - P.task_first);
    const uint32_t c = fdiv(P.geo_div, v);
    return P.task_first + (long long)c * P.n_pixels + __ldg(P.geo_map + (v - c * (uint32_t)P.n_geo));
}

template <bool BATCH>
__device__ __forceinline__ void start_task(const WfScene& S0, const WfParams& P0, const WfState& st, int slot,
                                           long long task) {
    WfScene S = S0;
    WfParams P = P0;
    Film F = film_of(st);
    long long base = 0;
    if constexpr (BATCH) {
        const int j = find_job(P0, task);
        st.job[slot] = j;
        apply_job(P0.jobs[j], S, P, F, base);
    }
    const TaskPos tp = task_pos(P, task - base);  // task within its job
    const int row = (int)fdiv(P.w_div, (uint32_t)tp.pixel);
    const int x = tp.pixel - row * P.width, y = P.row_begin + row * P.row_step;
    uint64_t rng = task_seed((uint32_t)x, (uint32_t)y, (uint32_t)tp.sample_start, P.seed);
    float3 o, d;
    float time;
    camera_ray(S.cam, x, y, 1.0f / (float)P.width, 1.0f / (float)P.height, rng, o, d, time);
    store_path(st, slot, make_int4(0, 0, 0, (int)task), rng);
    sts(&st.ray_o[slot], make_float4(o.x, o.y, o.z, ifloat(-1)));
    sts(&st.ray_d[slot], make_float4(d.x, d.y, d.z, ifloat(-1)));
    sts(&st.beta[slot], make_float4(1.0f, 1.0f, 1.0f, 0.0f));
    sts(&st.rad[slot], make_float4(0.0f, 0.0f, 0.0f, time));
    sts(&st.sacc[slot], make_double4(0.0, 0.0, 0.0, 0.0));
    if (st.ssq) st.ssq[slot] = make_double4(0.0, 0.0, 0.0, 0.0);
    if (st.welford) st.welford[slot] = make_double2(0.0, 0.0);
}

template <bool BATCH>
__global__ void k_init(WfScene S, WfParams P, WfState st) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const long long avail = fetch_end(P) - P.task_first;  // tasks of this chunk batch
    const int first = (int)(avail < (long long)P.n_slots ? avail : P.n_slots);
    if (i == 0) {
        st.ctr->n_ext[0] = first;
        st.ctr->next_task = P.task_first + first;
    }
    if (i >= P.n_slots) return;
    st.act[i] = i < first ? 1 : 0;
    if (i < first) {
        st.q_ext[0][i] = i;
        start_task<BATCH>(S, P, st, i, task_of_fetch(P, P.task_first + i));
    }
}

// Adds a thread's trace counters to the render totals (one atomic per warp).
template <bool COUNT>
__device__ __forceinline__ void flush_counts(WfCounters* c, int stage, const TraceCount& t) {
    if (!COUNT) return;
    unsigned long long v[8] = {t.nodes, t.tris, t.spheres, t.inst, t.node_steps, t.leaves, t.leaf_steps, t.fast_steps};
    for (int k = 0; k < 8; ++k)
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
    if (lane_id() == 0) {
        atomicAdd(&c->cnt_nodes[stage], v[0]);
        atomicAdd(&c->cnt_tris[stage], v[1]);
        atomicAdd(&c->cnt_spheres[stage], v[2]);
        atomicAdd(&c->cnt_inst[stage], v[3]);
        atomicAdd(&c->cnt_node_steps[stage], v[4]);
        atomicAdd(&c->cnt_leaves[stage], v[5]);
        atomicAdd(&c->cnt_leaf_steps[stage], v[6]);
        atomicAdd(&c->cnt_fast_steps, v[7]);
    }
}

// Persistent trace kernel over the extension queue (ANY = false: closest
// hit) or the shadow records (ANY = true: occlusion).  Each lane traces its
// own ray; every `chunk` leaf visits the warp reconverges and lanes whose
// ray has finished take new rays from the queue (one atomic per warp), so
// short rays (most camera rays miss every box) do not idle their warp
// while long ones traverse.
// Camera-ray misses (src/integrator.rs:71-83 at bounce 0) are the most
// common samples of an open scene: a camera ray that leaves the scene adds
// the env (or sky) radiance and the sample is done.  When such a sample is
// not the last of its task, the closest-hit kernel finishes it in place --
// the f64 task sums, the next camera ray from the pixel's stream
// (src/render.rs:151-158) -- and traces that ray at once, instead of a
// round trip through the shading kernel.  Same arithmetic and draws as
// k_shade + finish_sample; off for adaptive renders (their stopping rule
// runs in finish_sample) and for the adjoint.  Returns false when the slot
// is not such a sample.
template <bool BATCH>
__device__ __forceinline__ bool camera_miss_next(const WfScene& S0, const WfParams& P, const WfState& st, int slot,
                                                 Tracer& T) {
    int4 m;
    uint64_t rng;
    load_path(st, slot, m, rng);
    if (m.y != 0) return false;
    // the render's (or the slot's batch job's) camera, env map and film
    const WfJob* J = BATCH ? P.jobs + st.job[slot] : nullptr;
    const int max_bounces = BATCH ? J->max_bounces : P.max_bounces;
    if (max_bounces <= 0) return false;
    TaskPos tp;
    if constexpr (BATCH) {
        const long long lt = (long long)m.w - J->task_begin;
        const uint32_t chunk = fdiv(J->px_div, (uint32_t)lt);
        tp.j = tp.pixel = (int)((uint32_t)lt - chunk * (uint32_t)J->n_pixels);
        tp.sample_start = (int)chunk * J->task_spp;
        tp.len = min(J->task_spp, J->spp - tp.sample_start);
    } else {
        tp = task_pos(P, (long long)m.w);
    }
    if (m.x + 1 >= tp.len) return false;  // the task's last sample ends in the shading kernel
    WfScene S = S0;
    if constexpr (BATCH) {
        S.env_kind = J->env_kind; S.env_w = J->env_w; S.env_h = J->env_h; S.env_tex = J->env_tex;
    }
    const float3 L = clamp_lum(f3(1.0f, 1.0f, 1.0f) * background(S, T.wd), 50.0f);  // beta = 1 at bounce 0
    if (!BATCH && st.rsamp) {  // adaptive round: the sample itself, for the in-order stopping rule
        sts(&st.rsamp[(size_t)tp.j * P.round_len + (tp.sample_start - P.sample_base) + m.x],
            make_float4(L.x, L.y, L.z, 0.0f));
    } else {
        double4 a = lds(&st.sacc[slot]);
        a.x += (double)L.x; a.y += (double)L.y; a.z += (double)L.z; a.w += 1.0;
        sts(&st.sacc[slot], a);
        if (st.ssq) {
            double4 q = lds(&st.ssq[slot]);
            q.x += (double)L.x * (double)L.x; q.y += (double)L.y * (double)L.y; q.z += (double)L.z * (double)L.z;
            sts(&st.ssq[slot], q);
        }
    }
    m.x += 1;
    const int pixel = tp.pixel;
    const int width = BATCH ? J->width : P.width, height = BATCH ? J->height : P.height;
    const int row_begin = BATCH ? J->row_begin : P.row_begin, row_step = BATCH ? J->row_step : P.row_step;
    float3 o, d;
    float ptime;
    const int row = (int)fdiv(BATCH ? J->w_div : P.w_div, (uint32_t)pixel);
    camera_ray(BATCH ? J->cam : S0.cam, pixel - row * width, row_begin + row * row_step, 1.0f / (float)width,
               1.0f / (float)height, rng, o, d, ptime);
    store_path(st, slot, m, rng);
    sts(&st.ray_o[slot], make_float4(o.x, o.y, o.z, ifloat(-1)));
    sts(&st.ray_d[slot], make_float4(d.x, d.y, d.z, ifloat(-1)));
    sts(&st.rad[slot], make_float4(0.0f, 0.0f, 0.0f, ptime));
    tracer_start_at(BATCH ? J->top_root : S0.top_root, T, o, d, kTMax, -1, -1);
    return true;
}

template <bool ANY, bool COUNT, bool SHARED_STACK, bool BATCH>
__global__ void __launch_bounds__(kTraceBlock) k_trace(WfScene S, WfParams P, WfState st, int n_slots, int chunk,
                                                       const WfJob* __restrict__ jobs, int cur) {
    // Extension rays come from a sweep of every slot's act byte in slot
    // order, or, once few paths are live (forward renders, use_ext_queue),
    // from the compacted queue the shading and completion kernels push;
    // shadow rays from the shadow-record queue.
    const bool queue = ANY || (P.ext_queue && (P.ordered_queue || use_ext_queue(st.ctr->n_ext[cur], n_slots, P.queue_div)));
    const int n = ANY ? st.ctr->n_sh : (queue ? st.ctr->n_ext[cur] : n_slots);
    int* fetch = ANY ? &st.ctr->fetch_sh : &st.ctr->fetch_ext;
    const int* __restrict__ q = ANY ? st.q_sh : st.q_ext[cur];
    int* flags = &st.ctr->flags;
    __shared__ int sstack[SHARED_STACK ? kSharedStack * kTraceBlock : 1];
    int lstack[SHARED_STACK ? 1 : kStack];
    using Stack = typename std::conditional<SHARED_STACK, TStack<kTraceBlock, kSharedStack>, TStack<1, kStack>>::type;
    const Stack stack{SHARED_STACK ? sstack + threadIdx.x : lstack};
    Tracer T;
    TraceCount cnt;
    int item = -1;
    bool exhausted = false;
    const unsigned lt_mask = (1u << lane_id()) - 1u;
    unsigned long long fast_done = 0;  // samples finished by camera_miss_next
    for (;;) {
        const bool want = item < 0 && !exhausted;
        const unsigned m = __ballot_sync(0xffffffffu, want);
        if (m) {
            const int leader = __ffs(m) - 1;
            int base = 0;
            if ((int)lane_id() == leader) base = atomicAdd(fetch, __popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (want) {
                const int k = base + __popc(m & lt_mask);
                if (k < n) {
                    item = queue ? q[k] : (st.act[k] ? k : -1);
                    if (item < 0) {
                        // inactive slot: nothing to trace; refill next round
                    } else if (ANY) {
                        const float4 o4 = lds(&st.sh_o[item]), d4 = lds(&st.sh_d[item]);
                        const int self_inst = fbits(reinterpret_cast<const float*>(st.sh_c + item)[3]);
                        const int root = BATCH ? __ldg(&jobs[st.job[item >> 1]].top_root) : S.top_root;
                        tracer_start_at(root, T, f3(o4), f3(d4), o4.w, fbits(d4.w), self_inst);
                    } else {
                        const float4 o4 = lds(&st.ray_o[item]), d4 = lds(&st.ray_d[item]);
                        const int root = BATCH ? __ldg(&jobs[st.job[item]].top_root) : S.top_root;
                        tracer_start_at(root, T, f3(o4), f3(d4), kTMax, fbits(o4.w), fbits(d4.w));
                    }
                } else {
                    exhausted = true;
                }
            }
        }
        // A window of inactive slots leaves every lane empty but the cursor
        // short of n: the warp keeps fetching until all lanes are exhausted.
        if (!__any_sync(0xffffffffu, item >= 0 || !exhausted)) break;
        if (item >= 0 && tracer_run<ANY, COUNT>(S, T, stack, kEps, chunk, flags, cnt)) {
            if (ANY) {
                reinterpret_cast<float*>(st.sh_c + item)[3] = T.hit_prim >= 0 ? 0.0f : 1.0f;
            } else {
                if (P.camera_fast && T.hit_prim < 0 && camera_miss_next<BATCH>(S, P, st, item, T)) {
                    if (COUNT) count_step(cnt.fast_steps);
                    ++fast_done;
                    continue;  // this lane traces the task's next camera ray
                }
                sts(&st.hit[item], make_float4(T.hit_prim >= 0 ? T.tmax : kTMax, ifloat(T.hit_prim), ifloat(T.hit_inst), 0.0f));
            }
            item = -1;
        }
    }
    flush_counts<COUNT>(st.ctr, ANY ? 1 : 0, cnt);
    if (!ANY) {
        for (int off = 16; off > 0; off >>= 1) fast_done += __shfl_down_sync(0xffffffffu, fast_done, off);
        if (lane_id() == 0 && fast_done) {
            atomicAdd(&st.ctr->samples, fast_done);
            atomicAdd(&st.ctr->rays_closest, fast_done);
            if (COUNT) atomicAdd(&st.ctr->cnt_fast, fast_done);
        }
    }
}


__device__ __forceinline__ float3 take_pending(const WfState& st, int slot, int& fl, float3 L) {
    if (fl & F_PEND_ENV) {
        const float4 c = lds(&st.sh_c[2 * slot]);
        if (c.w > 0.5f) L = L + f3(c);
    }
    if (fl & F_PEND_AREA) {
        const float4 c = lds(&st.sh_c[2 * slot + 1]);
        if (c.w > 0.5f) L = L + f3(c);
    }
    fl &= ~(F_PEND_ENV | F_PEND_AREA);
    return L;
}

// End of one sample of a slot (src/render.rs:143-191): the sample's radiance
// joins the task's f64 sums (and the Welford statistics of adaptive
// sampling).  If the task has samples left, the pixel's next camera ray is
// written and the path state reset (returns true); otherwise the task's sums
// go to the film (one task per pixel) or to the task's partial sums, and
// need_task is set so the slot takes a new task.
__device__ __forceinline__ bool finish_sample(const WfScene& S, const WfParams& P, const WfState& st, int slot,
                                              int4& m, int& fl, float3& L, float3& beta, float& last_pdf,
                                              float& ptime, uint64_t& rng, bool& need_task, const Film& F,
                                              long long base) {
    const long long task = (long long)m.w;       // batch-wide task id
    const long long lt = task - base;            // within its job
    const TaskPos tp = task_pos(P, lt);
    double4 a = make_double4(0.0, 0.0, 0.0, 0.0);
    if (st.rsamp) {  // adaptive round: the sample itself, for the in-order stopping rule
        sts(&st.rsamp[(size_t)tp.j * P.round_len + (tp.sample_start - P.sample_base) + m.x],
            make_float4(L.x, L.y, L.z, 0.0f));
    } else {
        a = lds(&st.sacc[slot]);
        a.x += (double)L.x; a.y += (double)L.y; a.z += (double)L.z; a.w += 1.0;
        sts(&st.sacc[slot], a);
        if (st.ssq) {
            double4 q = st.ssq[slot];
            q.x += (double)L.x * (double)L.x; q.y += (double)L.y * (double)L.y; q.z += (double)L.z * (double)L.z;
            st.ssq[slot] = q;
        }
    }
    m.x += 1;
    const int task_len = tp.len;
    bool stop = m.x >= task_len;
    if (P.adaptive) {  // Welford on luminance (render.rs:160-176)
        double2 wv = st.welford[slot];
        const double l = 0.2126 * (double)L.x + 0.7152 * (double)L.y + 0.0722 * (double)L.z;
        const double delta = l - wv.x;
        wv.x += delta / (double)m.x;
        wv.y += delta * (l - wv.x);
        st.welford[slot] = wv;
        const int min_spp = min(max(P.adaptive_min_spp, 1), max(task_len, 1));
        if (m.x >= min_spp && m.x > 1) {
            const double var = wv.y / (double)(m.x - 1);
            if (sqrt(var) / fmax(fabs(wv.x), 1e-4) < P.adaptive_threshold) stop = true;
        }
    }
    const int pixel = tp.pixel;
    if (stop && st.rsamp) {  // adaptive round: k_round_merge adds the samples
        need_task = true;
        return false;
    }
    if (stop) {
        if (P.n_chunks == 1) {  // one task per pixel: straight into the film
            const size_t px = (size_t)pixel;
            F.acc[3 * px] = a.x; F.acc[3 * px + 1] = a.y; F.acc[3 * px + 2] = a.z;
            F.acc_w[px] = a.w;
            if (F.acc_sq) {
                const double4 q = st.ssq[slot];
                F.acc_sq[3 * px] = q.x; F.acc_sq[3 * px + 1] = q.y; F.acc_sq[3 * px + 2] = q.z;
            }
        } else {  // per-task sums, merged in task order by k_merge
            st.part[task - P.task_first] = a;
            if (st.part_sq) st.part_sq[task - P.task_first] = st.ssq[slot];
        }
        need_task = true;
        return false;
    }
    float3 o, d;
    const int row = (int)fdiv(P.w_div, (uint32_t)pixel);
    camera_ray(S.cam, pixel - row * P.width, P.row_begin + row * P.row_step, 1.0f / (float)P.width,
               1.0f / (float)P.height, rng, o, d,
               ptime);
    sts(&st.ray_o[slot], make_float4(o.x, o.y, o.z, ifloat(-1)));
    sts(&st.ray_d[slot], make_float4(d.x, d.y, d.z, ifloat(-1)));
    beta = f3(1.0f, 1.0f, 1.0f);
    last_pdf = 0.0f;
    L = f3(0, 0, 0);
    m.y = 0;
    fl = 0;
    return true;
}

// Slots whose task finished take the next tasks from the pool (one atomic
// per warp).  Must be called by all lanes of a converged warp.
template <bool BATCH>
__device__ __forceinline__ bool take_next_task(const WfScene& S, const WfParams& P, const WfState& st, int slot,
                                               bool need_task) {
    const unsigned want = __ballot_sync(0xffffffffu, need_task);
    if (!want) return false;
    const int leader = __ffs(want) - 1;
    long long t0 = 0;
    if ((int)lane_id() == leader)
        t0 = (long long)atomicAdd((unsigned long long*)&st.ctr->next_task, (unsigned long long)__popc(want));
    t0 = __shfl_sync(0xffffffffu, t0, leader);
    if (!need_task) return false;
    const long long t = t0 + __popc(want & ((1u << lane_id()) - 1u));
    if (t >= fetch_end(P)) return false;
    start_task<BATCH>(S, P, st, slot, task_of_fetch(P, t));
    return true;
}

// ---- shading -------------------------------------------------------------------
// Material-sorted shading (TPT_SHADE_SORT=1): one bounce of radiance()
// (src/integrator.rs:67-132), split by what the ray found.  k_shade_pre takes every queued path: misses (env + MIS), Russian
// roulette and emitter hits end the sample in place; surface hits are sorted
// into one queue per material kind with warp-ballot compaction.
// k_shade_surface<KIND> then runs NEE and BSDF sampling for one material
// kind, so each kernel carries only its own BSDF and no warp diverges on the
// material.
constexpr int kKinds = 5;  // TPT_MAT_LAMBERT .. TPT_MAT_SUBSURFACE

// Warp-aggregated count of `pred` lanes added to *counter.
__device__ __forceinline__ void warp_count(int* counter, bool pred) {
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (mask && (int)lane_id() == __ffs(mask) - 1) atomicAdd(counter, __popc(mask));
}

__global__ void __launch_bounds__(128) k_shade_pre(WfScene S, WfParams P, WfState st, int cur) {
    const int live = st.ctr->n_ext[cur];  // the slots the closest-hit kernel traced
    const bool use_q = P.ordered_queue || use_ext_queue(live, P.n_slots, P.queue_div);
    const int n = use_q ? live : P.n_slots;
    const int* __restrict__ qe = st.q_ext[cur];
    const int nxt = cur ^ 1;
    const bool has_env = S.env_kind == TPT_ENV_MAP;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const int i = base + (int)lane_id();
        bool again = false, need_task = false, finished = false, surface = false;
        int kind = 0, slot = 0;
        const bool active = i < n && (use_q || st.act[i]);
        if (active) {
            slot = use_q ? qe[i] : i;
            const float4 o4 = lds(&st.ray_o[slot]), d4 = lds(&st.ray_d[slot]);
            const float3 ro = f3(o4), rd = f3(d4);
            const float4 h4 = lds(&st.hit[slot]);
            const int prim = fbits(h4.y), inst = fbits(h4.z);
            const float4 b4 = lds(&st.beta[slot]);
            float3 beta = f3(b4);
            float last_pdf = b4.w;
            const float4 r4 = lds(&st.rad[slot]);
            float3 L = f3(r4);
            float ptime = r4.w;
            int4 m;
            uint64_t rng;
            load_path(st, slot, m, rng);
            int fl = m.z;
            L = take_pending(st, slot, fl, L);
            bool done = m.y >= P.max_bounces;  // max_bounces = 0: radiance() returns 0
            if (!done && prim < 0) {  // miss (:71-83)
                float3 contrib = beta * background(S, rd);
                if (has_env && (fl & F_LAST_ND)) contrib = contrib * mis(last_pdf, env_pdf(S, rd));
                L = L + clamp_lum(contrib, 50.0f);
                done = true;
            }
            if (!done && m.y >= P.rr_start) {  // Russian roulette (:89-95)
                const float p = fmaxf(fminf(max3(beta), 0.95f), 0.05f);
                if (pcg_f32(rng) > p) done = true;
                else beta = beta / p;
            }
            if (!done) {
                const float3 hp = ro + rd * h4.x;
                float3 ng;
                int mid;
                if (inst < 0) {
                    const float4 cr = __ldg(&S.spheres[prim].cr);
                    ng = (hp - f3(cr)) / cr.w;
                    mid = __ldg(&S.spheres[prim].mat);
                } else {
                    const TriF32* tp = S.tris + (prim - S.n_spheres);
                    const float4 v0 = __ldg(&tp->v0), e1 = __ldg(&tp->e1), e2 = __ldg(&tp->e2);
                    const float3 no = cross(f3(e1), f3(e2));
                    const InstanceF32* I = S.inst + inst;
                    const float4 n0 = __ldg(&I->nrm[0]), n1 = __ldg(&I->nrm[1]), n2 = __ldg(&I->nrm[2]);
                    ng = normalize(f3(n0.x * no.x + n0.y * no.y + n0.z * no.z, n1.x * no.x + n1.y * no.y + n1.z * no.z,
                                      n2.x * no.x + n2.y * no.y + n2.z * no.z));
                    const int ov = fbits(__ldg(&I->wbox_max.w));
                    mid = ov >= 0 ? ov : fbits(v0.w);
                }
                kind = __ldg(&S.mats[mid].kind);
                if (kind == TPT_MAT_DIFFUSE_LIGHT) {  // emitter (:100-104)
                    L = L + clamp_lum(beta * f3(__ldg(&S.mats[mid].c)), 50.0f);
                    done = true;
                } else {
                    st.surf_p[slot] = make_float4(hp.x, hp.y, hp.z, h4.x);
                    st.surf_n[slot] = make_float4(ng.x, ng.y, ng.z, ifloat(mid));
                    surface = true;
                }
            }
            if (done) {  // nothing is pending: the sample ends here
                again = finish_sample(S, P, st, slot, m, fl, L, beta, last_pdf, ptime, rng, need_task, film_of(st), 0);
                finished = true;
            }
            sts(&st.beta[slot], make_float4(beta.x, beta.y, beta.z, last_pdf));
            sts(&st.rad[slot], make_float4(L.x, L.y, L.z, ptime));
            m.z = fl;
            store_path(st, slot, m, rng);
        }
        if (take_next_task<false>(S, P, st, slot, need_task)) again = true;
        if (active) st.act[slot] = (again || surface) ? 1 : 0;
        if (!P.ordered_queue) warp_push(st.q_ext[nxt], &st.ctr->n_ext[nxt], again, slot);
        for (int k = 0; k < kKinds; ++k)
            warp_push(st.q_mat + (size_t)k * P.n_slots, &st.ctr->n_mat[k], surface && kind == k, slot);
        warp_count(&st.ctr->n_done_in_shade, finished);
    }
}

// One bounce of radiance() (src/integrator.rs:67-132) per queued path, all
// material kinds in one kernel (the default; it keeps each path's state in
// registers through the whole bounce).
// CTAS: resident blocks per SM the kernel is compiled for (its register
// budget).  More warps hide the latency of the path-state loads; fewer
// registers spill the heavier BSDF paths.  Measured on one B200 (4 vs 8):
// the 1080p mesh+env frame runs 9% faster at 8, the adaptive Cornell frame
// (long GGX/dielectric paths in the noisy pixels) 6% faster at 4, the batch
// workload 8% faster at 4.
// One visit of the shading kernel to a live slot (the per-slot body of
// k_shade, shared with k_tail): the bounce of radiance() (src/integrator.rs:
// 67-132) for the slot's closest hit, its NEE shadow records, the sample's
// completion when nothing is pending.  Returns what the caller's queues and
// task fetch need.
struct ShadeOut {
    bool cont, term, need_task, finished_here;
    int sh_env, sh_area;
};
template <bool BATCH>
__device__ __forceinline__ ShadeOut shade_slot(const WfScene& S0, const WfParams& P0, const WfState& st, int slot) {
    bool cont = false, term = false, need_task = false, finished_here = false;
    int sh_env = 0, sh_area = 0;
    WfScene S = S0;
    WfParams P = P0;
    Film F = film_of(st);
    long long tbase = 0;
    if constexpr (BATCH) apply_job(P0.jobs[st.job[slot]], S, P, F, tbase);
    const bool has_env = S.env_kind == TPT_ENV_MAP;
    const float4 o4 = lds(&st.ray_o[slot]), d4 = lds(&st.ray_d[slot]);
    const float3 ro = f3(o4), rd = f3(d4);
    const float4 h4 = lds(&st.hit[slot]);
    const int prim = fbits(h4.y), inst = fbits(h4.z);
    const float4 b4 = lds(&st.beta[slot]);
    float3 beta = f3(b4);
    float last_pdf = b4.w;
    const float4 r4 = lds(&st.rad[slot]);
    float3 L = f3(r4);
    float ptime = r4.w;
    int4 m;
    uint64_t rng;
    load_path(st, slot, m, rng);
    int fl = m.z;
    L = take_pending(st, slot, fl, L);
    bool done = m.y >= P.max_bounces;  // max_bounces = 0: radiance() returns 0
    if (!done && prim < 0) {  // miss (:71-83)
        float3 contrib = beta * background(S, rd);
        if (has_env && (fl & F_LAST_ND)) contrib = contrib * mis(last_pdf, env_pdf(S, rd));
        L = L + clamp_lum(contrib, 50.0f);
        done = true;
    }
    if (!done && m.y >= P.rr_start) {  // Russian roulette (:89-95)
        const float p = fmaxf(fminf(max3(beta), 0.95f), 0.05f);
        if (pcg_f32(rng) > p) done = true;
        else beta = beta / p;
    }
    if (!done) {
        const float3 hp = ro + rd * h4.x;
        float3 ng;
        int mid;
        if (inst < 0) {
            const SphereF32 sp = S.spheres[prim];
            ng = (hp - f3(sp.cr)) / sp.cr.w;
            mid = sp.mat;
        } else {
            const TriF32* tp = S.tris + (prim - S.n_spheres);
            const float4 v0 = __ldg(&tp->v0), e1 = __ldg(&tp->e1), e2 = __ldg(&tp->e2);
            const float3 no = cross(f3(e1), f3(e2));
            const InstanceF32* I = S.inst + inst;
            const float4 n0 = __ldg(&I->nrm[0]), n1 = __ldg(&I->nrm[1]), n2 = __ldg(&I->nrm[2]);
            ng = normalize(f3(n0.x * no.x + n0.y * no.y + n0.z * no.z, n1.x * no.x + n1.y * no.y + n1.z * no.z,
                              n2.x * no.x + n2.y * no.y + n2.z * no.z));
            const int ov = fbits(__ldg(&I->wbox_max.w));
            mid = ov >= 0 ? ov : fbits(v0.w);
        }
        const MaterialF32 mt = S.mats[mid];
        const float3 mc = f3(mt.c);
        if (mt.kind == TPT_MAT_DIFFUSE_LIGHT) {  // emitter (:100-104)
            L = L + clamp_lum(beta * mc, 50.0f);
            done = true;
        } else {
            const bool entering = dot(ng, rd) < 0.0f;
            const float3 n = entering ? ng : -ng;
            const float3 wo = -rd;
            if (mt.kind != TPT_MAT_METAL && mt.kind != TPT_MAT_DIELECTRIC) {
                if (has_env) {  // nee_environment (:148-172)
                    float3 wi, li;
                    float pe;
                    env_sample_dir(S, rng, wi, li, pe);
                    const float c = fmaxf(dot(n, wi), 0.0f);
                    if (c > 0.0f && pe > 0.0f) {
                        float3 f;
                        float pb;
                        mat_eval(mt, wo, wi, n, f, pb);
                        const float3 contrib = beta * f * li * (c * mis(pe, pb) / pe);
                        if (contrib.x > 0.0f || contrib.y > 0.0f || contrib.z > 0.0f) {
                            const float3 so = hp + wi * kEps;
                            sts(&st.sh_o[2 * slot], make_float4(so.x, so.y, so.z, kTMax));
                            sts(&st.sh_d[2 * slot], make_float4(wi.x, wi.y, wi.z, ifloat(prim)));
                            sts(&st.sh_c[2 * slot], make_float4(contrib.x, contrib.y, contrib.z, ifloat(inst)));
                            sh_env = 1;
                            fl |= F_PEND_ENV;
                        }
                    }
                }
                float3 lp, le;
                float lpdf;
                int lidx;
                double lud, lvd;
                if (sample_light(S, rng, hp, lp, le, lpdf, lidx, lud, lvd)) {  // nee_area_light (:178-213)
                    const float3 tl = lp - hp;
                    const float dist = length(tl);
                    if (dist > 1e-6f) {
                        const float3 wi = tl / dist;
                        const float c = fmaxf(dot(n, wi), 0.0f);
                        if (c > 0.0f && !ref_light_self_occluded(S.lights64, S.spheres64, S.inst64, lidx, ro, rd, h4.x, lud, lvd, (double)ptime)) {
                            float3 f;
                            float pb;
                            mat_eval(mt, wo, wi, n, f, pb);
                            const float3 contrib = beta * f * le * (c * mis(lpdf, pb) / lpdf);
                            if (contrib.x > 0.0f || contrib.y > 0.0f || contrib.z > 0.0f) {
                                const float3 so = hp + wi * kEps;
                                // stops 1e-4 short of the light: the light itself is
                                // handled by ref_light_self_occluded
                                sts(&st.sh_o[2 * slot + 1], make_float4(so.x, so.y, so.z, fmaxf(dist - 2.0f * kEps, kEps)));
                                sts(&st.sh_d[2 * slot + 1], make_float4(wi.x, wi.y, wi.z, ifloat(prim)));
                                sts(&st.sh_c[2 * slot + 1], make_float4(contrib.x, contrib.y, contrib.z, ifloat(inst)));
                                sh_area = 1;
                                fl |= F_PEND_AREA;
                            }
                        }
                    }
                }
            }
            // Material::sample (src/material.rs:76-201)
            float3 nd = f3(0, 0, 0), w = f3(0, 0, 0), no = hp;
            float pdf = 0.0f;
            bool delta = false, ok = true, self_ok = true;
            switch (mt.kind) {
                case TPT_MAT_LAMBERT:
                    nd = cos_hemi(n, rng);
                    w = mc;
                    pdf = fmaxf(dot(n, nd), 0.0f) / kPi;
                    break;
                case TPT_MAT_METAL:
                    nd = rd - n * (2.0f * dot(rd, n));
                    w = mc;
                    delta = true;
                    break;
                case TPT_MAT_DIELECTRIC: {
                    const float ior = mt.c.w;
                    const float eta = entering ? 1.0f / ior : ior;
                    const float ci = fmaxf(dot(wo, n), 0.0f);
                    const float fq = (ior - 1.0f) / (ior + 1.0f);
                    const float f0 = fq * fq;
                    const float fr = f0 + (1.0f - f0) * pow5(1.0f - ci);
                    float3 bt = f3(1, 1, 1);
                    if (!entering) {
                        const float dist = fmaxf(h4.x, 0.0f);
                        bt = f3(__expf(-mc.x * dist), __expf(-mc.y * dist), __expf(-mc.z * dist));
                    }
                    const float cosi = fminf(fmaxf(dot(wo, n), -1.0f), 1.0f);
                    const float sin2t = eta * eta * (1.0f - cosi * cosi);
                    const bool has_refr = !(sin2t >= 1.0f);
                    const bool refl = !has_refr || pcg_f32(rng) < fr;
                    if (refl) {
                        nd = rd - n * (2.0f * dot(rd, n));
                        bt = bt * (fr / fmaxf(fr, 1e-6f));
                    } else {
                        nd = rd * eta + n * (eta * cosi - sqrtf(1.0f - sin2t));
                        bt = bt * ((1.0f - fr) / fmaxf(1.0f - fr, 1e-6f)) * (eta * eta);
                    }
                    w = bt;
                    delta = true;
                    break;
                }
                case TPT_MAT_GGX: {
                    GgxSample gs;
                    if (!ggx_sample(rd, n, mt, rng, gs)) { ok = false; break; }
                    nd = gs.nd;
                    w = gs.w;
                    pdf = gs.pdf;
                    break;
                }
                case TPT_MAT_SUBSURFACE: {
                    const float sc = fmaxf(mt.c.w, 1e-4f);
                    const float u = fmaxf(pcg_f32(rng), 1e-12f);
                    const float dist = -__logf(u) * sc;
                    nd = cos_hemi(ng, rng);  // unoriented normal (material.rs:187-188)
                    w = mc * __expf(-dist / sc);
                    no = hp - ng * dist;
                    pdf = fmaxf(dot(n, nd), 0.0f) / kPi;
                    self_ok = false;     // origin moved off the surface
                    break;
                }
                default:
                    ok = false;
            }
            if (!ok) {
                done = true;
            } else {
                beta = beta * w;
                last_pdf = pdf;
                fl = delta ? (fl & ~F_LAST_ND) : (fl | F_LAST_ND);
                const float3 o2 = no + nd * kEps;
                sts(&st.ray_o[slot], make_float4(o2.x, o2.y, o2.z, ifloat(self_ok ? prim : -1)));
                sts(&st.ray_d[slot], make_float4(nd.x, nd.y, nd.z, ifloat(self_ok ? inst : -1)));
                m.y += 1;
                if (m.y >= P.max_bounces) done = true;  // bounce loop bound (:67)
            }
        }
    }
    if (done && !sh_env && !sh_area) {
        // Nothing pending: finish the sample here instead of in k_regen.
        cont = finish_sample(S, P, st, slot, m, fl, L, beta, last_pdf, ptime, rng, need_task, F, tbase);
        finished_here = true;
    } else {
        cont = !done;
        term = done;
    }
    sts(&st.beta[slot], make_float4(beta.x, beta.y, beta.z, last_pdf));
    sts(&st.rad[slot], make_float4(L.x, L.y, L.z, ptime));
    m.z = fl;
    store_path(st, slot, m, rng);
    return ShadeOut{cont, term, need_task, finished_here, sh_env, sh_area};
}

template <bool BATCH, int CTAS>
__global__ void __launch_bounds__(128, CTAS) k_shade(WfScene S0, WfParams P0, WfState st, int cur) {
    // At 6+ blocks per SM the kernel spills: ptxas may put the spills in
    // shared memory (13 KB per block) instead of local memory, which at
    // 1024 threads per SM does not fit in L1 (1080p frame: +1.0% paths/s).
    if constexpr (CTAS >= 6) asm volatile(".pragma \"enable_smem_spilling\";");
    const int live = st.ctr->n_ext[cur];  // the slots the closest-hit kernel traced
    const bool use_q = P0.ordered_queue || use_ext_queue(live, P0.n_slots, P0.queue_div);
    const int n = use_q ? live : P0.n_slots;
    const int* __restrict__ qe = st.q_ext[cur];
    const int nxt = cur ^ 1;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const int i = base + (int)lane_id();
        const bool active = i < n && (use_q || st.act[i]);
        bool cont = false, term = false, need_task = false, finished_here = false;
        int slot = 0;
        int sh_env = 0, sh_area = 0;
        if (active) {
            slot = use_q ? qe[i] : i;
            const ShadeOut r = shade_slot<BATCH>(S0, P0, st, slot);
            cont = r.cont; term = r.term; need_task = r.need_task; finished_here = r.finished_here;
            sh_env = r.sh_env; sh_area = r.sh_area;
        }
        if (take_next_task<BATCH>(S0, P0, st, slot, need_task)) cont = true;
        if (active) st.act[slot] = cont ? 1 : 0;
        if (!P0.ordered_queue) warp_push(st.q_ext[nxt], &st.ctr->n_ext[nxt], cont, slot);
        warp_push(st.q_term, &st.ctr->n_term, term, slot);
        warp_count(&st.ctr->n_done_in_shade, finished_here);
        warp_push(st.q_sh, &st.ctr->n_sh, sh_env != 0, 2 * slot);
        warp_push(st.q_sh, &st.ctr->n_sh, sh_area != 0, 2 * slot + 1);
    }
}

template <int KIND>
__global__ void __launch_bounds__(128) k_shade_surface(WfScene S, WfParams P, WfState st, int cur) {
    const int n = st.ctr->n_mat[KIND];
    const int* __restrict__ q = st.q_mat + (size_t)KIND * P.n_slots;
    const int nxt = cur ^ 1;
    const bool has_env = S.env_kind == TPT_ENV_MAP;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const int i = base + (int)lane_id();
        bool cont = false, term = false, need_task = false, finished = false;
        int slot = 0;
        int sh_env = 0, sh_area = 0;
        if (i < n) {
            slot = q[i];
            const float3 ro = f3(lds(&st.ray_o[slot])), rd = f3(lds(&st.ray_d[slot]));
            const float4 sp4 = st.surf_p[slot], sn4 = st.surf_n[slot];
            const float3 hp = f3(sp4), ng = f3(sn4);
            const float4 h4 = lds(&st.hit[slot]);
            const int prim = fbits(h4.y), inst = fbits(h4.z);
            const int mid = fbits(sn4.w);
            const float4 b4 = lds(&st.beta[slot]);
            float3 beta = f3(b4);
            float last_pdf = b4.w;
            const float4 r4 = lds(&st.rad[slot]);
            float3 L = f3(r4);
            float ptime = r4.w;
            int4 m;
            uint64_t rng;
            load_path(st, slot, m, rng);
            int fl = m.z;
            const MaterialF32 mt = S.mats[mid];
            const float3 mc = f3(mt.c);
            bool done = false;
            {
                {
                    const bool entering = dot(ng, rd) < 0.0f;
                    const float3 n = entering ? ng : -ng;
                    const float3 wo = -rd;
                    if (KIND != TPT_MAT_METAL && KIND != TPT_MAT_DIELECTRIC) {
                        if (has_env) {  // nee_environment (:148-172)
                            float3 wi, li;
                            float pe;
                            env_sample_dir(S, rng, wi, li, pe);
                            const float c = fmaxf(dot(n, wi), 0.0f);
                            if (c > 0.0f && pe > 0.0f) {
                                float3 f;
                                float pb;
                                mat_eval(mt, wo, wi, n, f, pb);
                                const float3 contrib = beta * f * li * (c * mis(pe, pb) / pe);
                                if (contrib.x > 0.0f || contrib.y > 0.0f || contrib.z > 0.0f) {
                                    const float3 so = hp + wi * kEps;
                                    sts(&st.sh_o[2 * slot], make_float4(so.x, so.y, so.z, kTMax));
                                    sts(&st.sh_d[2 * slot], make_float4(wi.x, wi.y, wi.z, ifloat(prim)));
                                    sts(&st.sh_c[2 * slot], make_float4(contrib.x, contrib.y, contrib.z, ifloat(inst)));
                                    sh_env = 1;
                                    fl |= F_PEND_ENV;
                                }
                            }
                        }
                        float3 lp, le;
                        float lpdf;
                        int lidx;
                        double lud, lvd;
                        if (sample_light(S, rng, hp, lp, le, lpdf, lidx, lud, lvd)) {  // nee_area_light (:178-213)
                            const float3 tl = lp - hp;
                            const float dist = length(tl);
                            if (dist > 1e-6f) {
                                const float3 wi = tl / dist;
                                const float c = fmaxf(dot(n, wi), 0.0f);
                                if (c > 0.0f && !ref_light_self_occluded(S.lights64, S.spheres64, S.inst64, lidx, ro, rd, h4.x, lud, lvd, (double)ptime)) {
                                    float3 f;
                                    float pb;
                                    mat_eval(mt, wo, wi, n, f, pb);
                                    const float3 contrib = beta * f * le * (c * mis(lpdf, pb) / lpdf);
                                    if (contrib.x > 0.0f || contrib.y > 0.0f || contrib.z > 0.0f) {
                                        const float3 so = hp + wi * kEps;
                                        // stops 1e-4 short of the light: the light itself is
                                        // handled by ref_light_self_occluded
                                        sts(&st.sh_o[2 * slot + 1], make_float4(so.x, so.y, so.z, fmaxf(dist - 2.0f * kEps, kEps)));
                                        sts(&st.sh_d[2 * slot + 1], make_float4(wi.x, wi.y, wi.z, ifloat(prim)));
                                        sts(&st.sh_c[2 * slot + 1], make_float4(contrib.x, contrib.y, contrib.z, ifloat(inst)));
                                        sh_area = 1;
                                        fl |= F_PEND_AREA;
                                    }
                                }
                            }
                        }
                    }
                    // Material::sample (src/material.rs:76-201)
                    float3 nd = f3(0, 0, 0), w = f3(0, 0, 0), no = hp;
                    float pdf = 0.0f;
                    bool delta = false, ok = true, self_ok = true;
                    switch (KIND) {
                        case TPT_MAT_LAMBERT:
                            nd = cos_hemi(n, rng);
                            w = mc;
                            pdf = fmaxf(dot(n, nd), 0.0f) / kPi;
                            break;
                        case TPT_MAT_METAL:
                            nd = rd - n * (2.0f * dot(rd, n));
                            w = mc;
                            delta = true;
                            break;
                        case TPT_MAT_DIELECTRIC: {
                            const float ior = mt.c.w;
                            const float eta = entering ? 1.0f / ior : ior;
                            const float ci = fmaxf(dot(wo, n), 0.0f);
                            const float fq = (ior - 1.0f) / (ior + 1.0f);
                            const float f0 = fq * fq;
                            const float fr = f0 + (1.0f - f0) * pow5(1.0f - ci);
                            float3 bt = f3(1, 1, 1);
                            if (!entering) {
                                const float dist = fmaxf(h4.x, 0.0f);
                                bt = f3(__expf(-mc.x * dist), __expf(-mc.y * dist), __expf(-mc.z * dist));
                            }
                            const float cosi = fminf(fmaxf(dot(wo, n), -1.0f), 1.0f);
                            const float sin2t = eta * eta * (1.0f - cosi * cosi);
                            const bool has_refr = !(sin2t >= 1.0f);
                            const bool refl = !has_refr || pcg_f32(rng) < fr;
                            if (refl) {
                                nd = rd - n * (2.0f * dot(rd, n));
                                bt = bt * (fr / fmaxf(fr, 1e-6f));
                            } else {
                                nd = rd * eta + n * (eta * cosi - sqrtf(1.0f - sin2t));
                                bt = bt * ((1.0f - fr) / fmaxf(1.0f - fr, 1e-6f)) * (eta * eta);
                            }
                            w = bt;
                            delta = true;
                            break;
                        }
                        case TPT_MAT_GGX: {
                            GgxSample gs;
                            if (!ggx_sample(rd, n, mt, rng, gs)) { ok = false; break; }
                            nd = gs.nd;
                            w = gs.w;
                            pdf = gs.pdf;
                            break;
                        }
                        case TPT_MAT_SUBSURFACE: {
                            const float sc = fmaxf(mt.c.w, 1e-4f);
                            const float u = fmaxf(pcg_f32(rng), 1e-12f);
                            const float dist = -__logf(u) * sc;
                            nd = cos_hemi(ng, rng);  // unoriented normal (material.rs:187-188)
                            w = mc * __expf(-dist / sc);
                            no = hp - ng * dist;
                            pdf = fmaxf(dot(n, nd), 0.0f) / kPi;
                            self_ok = false;     // origin moved off the surface
                            break;
                        }
                        default:
                            ok = false;
                    }
                    if (!ok) {
                        done = true;
                    } else {
                        beta = beta * w;
                        last_pdf = pdf;
                        fl = delta ? (fl & ~F_LAST_ND) : (fl | F_LAST_ND);
                        const float3 o2 = no + nd * kEps;
                        sts(&st.ray_o[slot], make_float4(o2.x, o2.y, o2.z, ifloat(self_ok ? prim : -1)));
                        sts(&st.ray_d[slot], make_float4(nd.x, nd.y, nd.z, ifloat(self_ok ? inst : -1)));
                        m.y += 1;
                        if (m.y >= P.max_bounces) done = true;  // bounce loop bound (:67)
                    }
                }
            }
            if (done && !sh_env && !sh_area) {
                cont = finish_sample(S, P, st, slot, m, fl, L, beta, last_pdf, ptime, rng, need_task, film_of(st), 0);
                finished = true;
            } else {
                cont = !done;
                term = done;
            }
            sts(&st.beta[slot], make_float4(beta.x, beta.y, beta.z, last_pdf));
            sts(&st.rad[slot], make_float4(L.x, L.y, L.z, ptime));
            m.z = fl;
            store_path(st, slot, m, rng);
        }
        if (take_next_task<false>(S, P, st, slot, need_task)) cont = true;
        if (i < n) st.act[slot] = cont ? 1 : 0;
        if (!P.ordered_queue) warp_push(st.q_ext[nxt], &st.ctr->n_ext[nxt], cont, slot);
        warp_push(st.q_term, &st.ctr->n_term, term, slot);
        warp_push(st.q_sh, &st.ctr->n_sh, sh_env != 0, 2 * slot);
        warp_push(st.q_sh, &st.ctr->n_sh, sh_area != 0, 2 * slot + 1);
        warp_count(&st.ctr->n_done_in_shade, finished);
    }
}

// Samples that ended with shadow rays pending finish here, after k_shadow
// has resolved their visibility.
// The completion kernel's per-slot body (k_regen, shared with k_tail): a
// path that ended with shadow rays pending takes their results, then
// finish_sample.  Returns whether the slot traces on (the task's next
// camera ray); need_task when its task is done.
template <bool BATCH>
__device__ __forceinline__ bool regen_slot(const WfScene& S0, const WfParams& P0, const WfState& st, int slot,
                                           bool& need_task) {
    bool again = false;
    WfScene S = S0;
    WfParams P = P0;
    Film F = film_of(st);
    long long tbase = 0;
    if constexpr (BATCH) apply_job(P0.jobs[st.job[slot]], S, P, F, tbase);
    int4 m;
    uint64_t rng;
    load_path(st, slot, m, rng);
    int fl = m.z;
    const float4 r4 = lds(&st.rad[slot]);
    float ptime = r4.w;
    float3 L = take_pending(st, slot, fl, f3(r4));
    float3 beta = f3(1.0f, 1.0f, 1.0f);
    float last_pdf = 0.0f;
    again = finish_sample(S, P, st, slot, m, fl, L, beta, last_pdf, ptime, rng, need_task, F, tbase);
    if (again) sts(&st.beta[slot], make_float4(1.0f, 1.0f, 1.0f, 0.0f));
    sts(&st.rad[slot], make_float4(L.x, L.y, L.z, ptime));
    m.z = fl;
    store_path(st, slot, m, rng);
    return again;
}

template <bool BATCH>
__global__ void __launch_bounds__(128) k_regen(WfScene S0, WfParams P0, WfState st, int cur) {
    const int n = st.ctr->n_term;
    const int nxt = cur ^ 1;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const int i = base + (int)lane_id();
        bool again = false, need_task = false;
        int slot = 0;
        if (i < n) {
            slot = st.q_term[i];
            again = regen_slot<BATCH>(S0, P0, st, slot, need_task);
        }
        if (take_next_task<BATCH>(S0, P0, st, slot, need_task)) again = true;
        if (i < n) st.act[slot] = again ? 1 : 0;
        if (!P0.ordered_queue) warp_push(st.q_ext[nxt], &st.ctr->n_ext[nxt], again, slot);
    }
}

// Film of a multi-chunk render: each pixel's task sums added in task order
// (the reference merges task results in task-id order, src/render.rs:226-241).
// A render in chunk batches merges each batch onto the film the previous
// ones left: the same additions in the same order.
// ---- camera culling -------------------------------------------------------------
// A film pixel is "open" when no camera ray through it can reach a leaf of
// the top-level tree (a sphere group or an instance): then each of its
// samples is a camera ray that leaves the scene (src/integrator.rs:71-83 at
// bounce 0), and k_sky_tasks computes it without a trace.  The test is
// conservative: the pixel's footprint, widened by 1% of a pixel on every
// side, spans a pyramid from the pinhole; each side plane is turned outward
// by a bound on the FP32 error of camera_ray's direction (cull_may_hit)
// and every box is padded by 1e-5 of the coordinates' magnitude
// (far above the FP32 error of the trace kernels' slab tests), and a box is
// passed over only when one side plane has it wholly outside.  All in f64.
struct CullFrustum {
    double3 o;
    double3 n[4];  // unit inward side normals
    double sin_m;
    double o_mag;  // largest |o| component
};
__device__ __forceinline__ double3 dd3(float3 a) { return make_double3(a.x, a.y, a.z); }
__device__ __forceinline__ double3 dsub(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double ddot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double3 dcross(double3 a, double3 b) {
    return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// Unnormalised camera direction at screen position (sx, sy), as camera_ray
// forms it before normalising.
__device__ __forceinline__ double3 cull_dir(const CameraF32& c, double sx, double sy) {
    const double hw = c.half_w, hh = c.half_h;
    return make_double3(-(double)c.w.x + c.u.x * (sx * hw) + c.v.x * (sy * hh),
                        -(double)c.w.y + c.u.y * (sx * hw) + c.v.y * (sy * hh),
                        -(double)c.w.z + c.u.z * (sx * hw) + c.v.z * (sy * hh));
}
// true when the box [lo, hi] lies wholly outside the frustum (padded).
__device__ __forceinline__ bool cull_outside(const CullFrustum& F, double3 lo, double3 hi) {
    const double mag = fmax(fmax(fmax(fabs(lo.x), fabs(hi.x)), fmax(fabs(lo.y), fabs(hi.y))), fmax(fabs(lo.z), fabs(hi.z)));
    const double pad = 1e-5 * (mag + F.o_mag) + 1e-30;
    const double3 c = make_double3(0.5 * (lo.x + hi.x), 0.5 * (lo.y + hi.y), 0.5 * (lo.z + hi.z));
    const double3 h = make_double3(0.5 * (hi.x - lo.x) + pad, 0.5 * (hi.y - lo.y) + pad, 0.5 * (hi.z - lo.z) + pad);
    const double3 co = dsub(c, F.o);
    const double3 far = make_double3(fabs(co.x) + h.x, fabs(co.y) + h.y, fabs(co.z) + h.z);
    const double reach = F.sin_m * sqrt(ddot(far, far));  // the outward turn at the box's farthest point
    for (int k = 0; k < 4; ++k) {
        const double3 n = F.n[k];
        const double s = ddot(n, co) + fabs(n.x) * h.x + fabs(n.y) * h.y + fabs(n.z) * h.z + reach;
        if (s < 0.0) return true;
    }
    return false;
}

// True when a camera ray through pixel (x, y) of a width x height film may
// reach a leaf of the top-level tree rooted at `root` (see above).  Lens
// cameras, and renders whose paths end before their first bounce, are
// never culled.
// What the primitives of a leaf code (not TPT_REF_NONE) leave to the walk
// of cull_may_hit: keep = true when they may be hit (spheres, triangles, a
// transformed instance), else the node to walk on (the mesh tree of an
// identity instance, which the traversal tests with the world ray, so its
// boxes are world boxes under the same slab test) or TPT_REF_NONE (an
// empty leaf or mesh: nothing to hit).
__device__ __forceinline__ int cull_leaf(const WfScene& S, int ref, bool& keep) {
    const uint32_t code = (uint32_t)(~ref), first = code >> 3, count = code & 7u;
    keep = false;
    if (count == 0u) return TPT_REF_NONE;  // an empty leaf (exit markers never sit in nodes)
    keep = true;
    if (count != 7u) return TPT_REF_NONE;  // spheres or triangles
    const int mw = __float_as_int(S.inst[first].wbox_min.w);
    if (!(mw & kInstIdentity)) return TPT_REF_NONE;
    const int mroot = S.meshes[mw & kInstMeshMask].root_ref;
    if (mroot < 0) {  // an empty mesh, or one leaf whose box the instance box was
        keep = mroot != TPT_REF_NONE;
        return TPT_REF_NONE;
    }
    keep = false;
    return mroot;
}

// Most nodes one pixel's walk visits; past them the pixel stays in the path pool.
constexpr int kCullMaxVisits = 1024;

__device__ bool cull_may_hit(const WfScene& S, const CameraF32& c, int root, int x, int y, int width, int height,
                             int max_bounces) {
    if (!(c.lens_radius == 0.0f && c.focus_dist > 0.0f && max_bounces > 0)) return true;
    // camera_ray: sx = (x + jx) * inv_w * 2 - 1, sy = 1 - (y + jy) * inv_h * 2, jx, jy in [0, 1)
    const double iw = (double)(1.0f / (float)width), ih = (double)(1.0f / (float)height);
    const double sx0 = ((double)x - 0.01) * iw * 2.0 - 1.0, sx1 = ((double)x + 1.01) * iw * 2.0 - 1.0;
    const double sy0 = 1.0 - ((double)y + 1.01) * ih * 2.0, sy1 = 1.0 - ((double)y - 0.01) * ih * 2.0;
    const double3 d[4] = {cull_dir(c, sx0, sy0), cull_dir(c, sx1, sy0), cull_dir(c, sx1, sy1), cull_dir(c, sx0, sy1)};
    const double3 mid = cull_dir(c, 0.5 * (sx0 + sx1), 0.5 * (sy0 + sy1));
    CullFrustum F;
    F.o = dd3(c.o);
    F.o_mag = fmax(fmax(fabs(F.o.x), fabs(F.o.y)), fabs(F.o.z));
    // FP32 error bound of camera_ray's direction: a few ulps of the screen
    // basis, and of (o + base * focus_dist) - o relative to focus_dist
    F.sin_m = sin(1e-5 + 4e-6 * (1.0 + F.o_mag / (double)c.focus_dist));
    for (int k = 0; k < 4; ++k) {
        double3 n = dcross(d[k], d[(k + 1) & 3]);
        const double len = sqrt(ddot(n, n));
        if (!(len > 0.0)) return true;  // degenerate footprint: keep the pixel
        n = make_double3(n.x / len, n.y / len, n.z / len);
        if (ddot(n, mid) < 0.0) n = make_double3(-n.x, -n.y, -n.z);
        F.n[k] = n;
    }
    if (root == TPT_REF_NONE) return false;
    int ref = root;
    if (root < 0) {  // a single leaf at the root: the bounds of its instance or spheres
        const uint32_t code = (uint32_t)(~root), first = code >> 3, count = code & 7u;
        double3 lo, hi;
        if (count == 7u) {
            const InstanceF32& I = S.inst[first];
            lo = make_double3(I.wbox_min.x, I.wbox_min.y, I.wbox_min.z);
            hi = make_double3(I.wbox_max.x, I.wbox_max.y, I.wbox_max.z);
            if (!(lo.x <= hi.x)) return false;  // an empty mesh
            if (cull_outside(F, lo, hi)) return false;
            bool keep;
            ref = cull_leaf(S, root, keep);
            if (keep) return true;
            if (ref == TPT_REF_NONE) return false;
        } else {
            lo = make_double3(INFINITY, INFINITY, INFINITY);
            hi = make_double3(-INFINITY, -INFINITY, -INFINITY);
            for (uint32_t k = first; k < first + count; ++k) {
                const float4 cr = S.spheres[k].cr;
                const double r = fabs((double)cr.w);
                lo = make_double3(fmin(lo.x, cr.x - r), fmin(lo.y, cr.y - r), fmin(lo.z, cr.z - r));
                hi = make_double3(fmax(hi.x, cr.x + r), fmax(hi.y, cr.y + r), fmax(hi.z, cr.z + r));
            }
            return !cull_outside(F, lo, hi);
        }
    }
    int stack[64];
    int sp = 0;
    for (int visits = 1;; ++visits) {
        if (visits > kCullMaxVisits) return true;
        const BvhNode2 nd = S.nodes[ref];
        const double3 lo0 = make_double3(fmin(nd.lx.x, nd.lx.y), fmin(nd.lx.z, nd.lx.w), fmin(nd.zz.x, nd.zz.y));
        const double3 hi0 = make_double3(fmax(nd.lx.x, nd.lx.y), fmax(nd.lx.z, nd.lx.w), fmax(nd.zz.x, nd.zz.y));
        const double3 lo1 = make_double3(fmin(nd.rx.x, nd.rx.y), fmin(nd.rx.z, nd.rx.w), fmin(nd.zz.z, nd.zz.w));
        const double3 hi1 = make_double3(fmax(nd.rx.x, nd.rx.y), fmax(nd.rx.z, nd.rx.w), fmax(nd.zz.z, nd.zz.w));
        const int r[2] = {nd.refs.x, nd.refs.y};
        const bool in[2] = {r[0] != TPT_REF_NONE && !cull_outside(F, lo0, hi0),
                            r[1] != TPT_REF_NONE && !cull_outside(F, lo1, hi1)};
        for (int k = 0; k < 2; ++k) {
            if (!in[k]) continue;
            int next = r[k];
            if (next < 0) {  // a leaf's box
                bool keep;
                next = cull_leaf(S, next, keep);
                if (keep) return true;
                if (next == TPT_REF_NONE) continue;
            }
            if (sp == 64) return true;  // deeper than the walk keeps: keep the pixel
            stack[sp++] = next;
        }
        if (sp == 0) return false;
        ref = stack[--sp];
    }
}

// One thread per film pixel (a multi-job render: per pixel of all jobs,
// numbered job after job): may[j] = 1 when a camera ray through pixel j
// may reach a top-level leaf, open[j] = 1 otherwise.
template <bool BATCH>
__global__ void k_cull_classify(WfScene S, WfParams P, uint8_t* __restrict__ may, uint8_t* __restrict__ open) {
    const long long gp = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool hit;
    if constexpr (BATCH) {
        if (gp >= P.total_pixels) return;
        const WfJob& J = P.jobs[job_at(P, gp, [](const WfJob& x) { return x.pixel_begin; })];
        const int j = (int)(gp - J.pixel_begin);
        const int row = (int)fdiv(J.w_div, (uint32_t)j);
        hit = cull_may_hit(S, J.cam, J.top_root, j - row * J.width, J.row_begin + row * J.row_step, J.width, J.height,
                           J.max_bounces);
    } else {
        if (gp >= P.n_pixels) return;
        const int j = (int)gp;
        const int row = (int)fdiv(P.w_div, (uint32_t)j);
        hit = cull_may_hit(S, S.cam, S.top_root, j - row * P.width, P.row_begin + row * P.row_step, P.width, P.height,
                           P.max_bounces);
    }
    may[gp] = hit ? 1 : 0;
    open[gp] = hit ? 0 : 1;
}

// Multi-job renders, one block: each job's stretch of the two compacted
// pixel lists (batch-wide pixel ids, ascending), then, job after job, the
// first pool fetch id and the first sky task of each job.  out[0] / out[1]
// = the fetch ids / sky tasks of the whole batch.
__device__ __forceinline__ int lower_bound_int(const int* __restrict__ a, int n, long long key) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((long long)a[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}
__global__ void __launch_bounds__(1024) k_cull_jobs(WfJob* jobs, int n_jobs, const int* __restrict__ may_list,
                                                    const int* __restrict__ open_list, const int* __restrict__ counts,
                                                    long long* out) {
    const int n_may = counts[0], n_open = counts[1];
    for (int k = threadIdx.x; k < n_jobs; k += blockDim.x) {
        WfJob& J = jobs[k];
        J.geo_begin = lower_bound_int(may_list, n_may, J.pixel_begin);
        J.n_geo = lower_bound_int(may_list, n_may, J.pixel_begin + J.n_pixels) - J.geo_begin;
        J.sky_begin = lower_bound_int(open_list, n_open, J.pixel_begin);
        J.n_sky = lower_bound_int(open_list, n_open, J.pixel_begin + J.n_pixels) - J.sky_begin;
        J.geo_div = make_fastdiv((uint32_t)(J.n_geo > 0 ? J.n_geo : 1));
        J.sky_div = make_fastdiv((uint32_t)(J.n_sky > 0 ? J.n_sky : 1));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        long long f = 0, u = 0;
        for (int k = 0; k < n_jobs; ++k) {
            WfJob& J = jobs[k];
            J.fetch_begin = f;
            J.sky_task_begin = u;
            f += (long long)J.n_chunks * J.n_geo;
            u += (long long)J.n_chunks * J.n_sky;
        }
        out[0] = f;
        out[1] = u;
    }
}

// One thread per task of an open pixel (single renders: in the current
// chunk batch, chunk by chunk, the open pixels in film order; multi-job
// renders: job after job): the task's samples exactly as the pool would
// run them -- the stream from seed_for(x, y, sample_start) ^ seed, per
// sample camera_ray, the background at bounce 0 (beta = 1, no MIS),
// clamp_lum, the f64 sums in sample order -- then the film (one task per
// pixel) or the task's partial sums, like finish_sample.
template <bool BATCH>
__global__ void k_sky_tasks(WfScene S0, WfParams P0, WfState st, const int* __restrict__ open_map, int n_open,
                            FastDiv open_div, long long count) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long done = 0;
    if (v < count) {
        WfScene S = S0;
        WfParams P = P0;
        Film F = film_of(st);
        long long task, base = 0;
        int pixel;
        if constexpr (BATCH) {
            const WfJob& J = P0.jobs[job_at(P0, v, [](const WfJob& x) { return x.sky_task_begin; })];
            apply_job(J, S, P, F, base);
            const uint32_t w = (uint32_t)(v - J.sky_task_begin);
            const uint32_t c = fdiv(J.sky_div, w);
            pixel = (int)(__ldg(open_map + J.sky_begin + (w - c * (uint32_t)J.n_sky)) - J.pixel_begin);
            task = J.task_begin + (long long)c * J.n_pixels + pixel;
        } else {
            const uint32_t c = fdiv(open_div, (uint32_t)v);
            pixel = __ldg(open_map + ((uint32_t)v - c * (uint32_t)n_open));
            task = P.task_first + (long long)c * P.n_pixels + pixel;
        }
        const TaskPos tp = task_pos(P, task - base);
        const int row = (int)fdiv(P.w_div, (uint32_t)pixel);
        const int x = pixel - row * P.width, y = P.row_begin + row * P.row_step;
        uint64_t rng = task_seed((uint32_t)x, (uint32_t)y, (uint32_t)tp.sample_start, P.seed);
        double4 a = make_double4(0.0, 0.0, 0.0, 0.0);
        double4 q = make_double4(0.0, 0.0, 0.0, 0.0);
        for (int k = 0; k < tp.len; ++k) {
            float3 o, d;
            float time;
            camera_ray(S.cam, x, y, 1.0f / (float)P.width, 1.0f / (float)P.height, rng, o, d, time);
            const float3 L = clamp_lum(f3(1.0f, 1.0f, 1.0f) * background(S, d), 50.0f);
            a.x += (double)L.x; a.y += (double)L.y; a.z += (double)L.z; a.w += 1.0;
            q.x += (double)L.x * (double)L.x; q.y += (double)L.y * (double)L.y; q.z += (double)L.z * (double)L.z;
        }
        if (P.n_chunks == 1) {
            const size_t px = (size_t)pixel;
            F.acc[3 * px] = a.x; F.acc[3 * px + 1] = a.y; F.acc[3 * px + 2] = a.z;
            F.acc_w[px] = a.w;
            if (F.acc_sq) { F.acc_sq[3 * px] = q.x; F.acc_sq[3 * px + 1] = q.y; F.acc_sq[3 * px + 2] = q.z; }
        } else {
            st.part[task - P0.task_first] = a;
            if (st.part_sq) st.part_sq[task - P0.task_first] = q;
        }
        done = (unsigned long long)tp.len;
    }
    for (int off = 16; off > 0; off >>= 1) done += __shfl_down_sync(0xffffffffu, done, off);
    if (lane_id() == 0 && done) atomicAdd(&st.ctr->sky_samples, done);  // beside k_step: its own counter
}

// The end of a render's bounce loop: when every task has been taken and at
// most P.tail_live slots are still live, the loop stops and this kernel
// runs each live slot (the queue the last iteration left, q_ext[0]) to the
// end of its task, one thread per slot: closest hit, shade_slot, the shadow
// rays at once, regen_slot when the path ended with shadow rays pending,
// and on to the task's next sample.  These are the wavefront kernels'
// per-slot steps in their order, so the film is that of the loop run to
// the end; the drain's per-iteration launches and compactions go away.
// Each slot is bounded by P.max_iters visits (TPT_FLAG_ITER_LIMIT).
template <bool BATCH>
__global__ void __launch_bounds__(128) k_tail(WfScene S, WfParams P, WfState st) {
    const int n = st.ctr->n_ext[0];
    const int* __restrict__ q = st.q_ext[0];
    int* flags = &st.ctr->flags;
    int lstack[kStack];
    const TStack<1, kStack> stack{lstack};
    unsigned long long samples = 0, rays_c = 0, rays_s = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int slot = q[i];
        const int root = BATCH ? P.jobs[st.job[slot]].top_root : S.top_root;
        for (long long visit = 0;; ++visit) {
            if (visit >= P.max_iters) {
                raise_flag(flags, TPT_FLAG_ITER_LIMIT);
                break;
            }
            Tracer T;
            TraceCount cnt;
            const float4 o4 = lds(&st.ray_o[slot]), d4 = lds(&st.ray_d[slot]);
            tracer_start_at(root, T, f3(o4), f3(d4), kTMax, fbits(o4.w), fbits(d4.w));
            while (!tracer_run<false, false>(S, T, stack, kEps, 1 << 30, flags, cnt)) {
            }
            sts(&st.hit[slot], make_float4(T.hit_prim >= 0 ? T.tmax : kTMax, ifloat(T.hit_prim), ifloat(T.hit_inst),
                                           0.0f));
            ++rays_c;
            const ShadeOut r = shade_slot<BATCH>(S, P, st, slot);
            if (r.finished_here) ++samples;
            for (int k = 0; k < 2; ++k) {
                if (!(k == 0 ? r.sh_env : r.sh_area)) continue;
                const int rec = 2 * slot + k;
                const float4 so = lds(&st.sh_o[rec]), sd = lds(&st.sh_d[rec]);
                float* vis = reinterpret_cast<float*>(st.sh_c + rec) + 3;
                tracer_start_at(root, T, f3(so), f3(sd), so.w, fbits(sd.w), fbits(*vis));
                while (!tracer_run<true, false>(S, T, stack, kEps, 1 << 30, flags, cnt)) {
                }
                *vis = T.hit_prim >= 0 ? 0.0f : 1.0f;
                ++rays_s;
            }
            bool cont = r.cont;
            if (r.term) {
                bool need_task = false;
                cont = regen_slot<BATCH>(S, P, st, slot, need_task);
                ++samples;
            }
            if (!cont) break;  // its task is done, and no task is left to take
        }
        st.act[slot] = 0;
    }
    for (int off = 16; off > 0; off >>= 1) {
        samples += __shfl_down_sync(0xffffffffu, samples, off);
        rays_c += __shfl_down_sync(0xffffffffu, rays_c, off);
        rays_s += __shfl_down_sync(0xffffffffu, rays_s, off);
    }
    if (lane_id() == 0) {
        if (samples) atomicAdd(&st.ctr->samples, samples);
        if (rays_c) atomicAdd(&st.ctr->rays_closest, rays_c);
        if (rays_s) atomicAdd(&st.ctr->rays_shadow, rays_s);
    }
}

__global__ void k_merge(WfParams P, WfState st) {
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    if (px >= P.n_pixels) return;
    const int c0 = (int)(P.task_first / P.n_pixels), c1 = (int)(P.n_tasks / P.n_pixels);
    double ax = 0.0, ay = 0.0, az = 0.0, aw = 0.0, qx = 0.0, qy = 0.0, qz = 0.0;
    if (c0 > 0) {
        ax = st.acc[3 * (size_t)px]; ay = st.acc[3 * (size_t)px + 1]; az = st.acc[3 * (size_t)px + 2];
        aw = st.acc_w[px];
        if (st.acc_sq) { qx = st.acc_sq[3 * (size_t)px]; qy = st.acc_sq[3 * (size_t)px + 1]; qz = st.acc_sq[3 * (size_t)px + 2]; }
    }
    for (int k = c0; k < c1; ++k) {
        const long long t = (long long)(k - c0) * P.n_pixels + px;
        const double4 a = st.part[t];
        ax += a.x; ay += a.y; az += a.z; aw += a.w;
        if (st.acc_sq) {
            const double4 q = st.part_sq[t];
            qx += q.x; qy += q.y; qz += q.z;
        }
    }
    st.acc[3 * (size_t)px] = ax; st.acc[3 * (size_t)px + 1] = ay; st.acc[3 * (size_t)px + 2] = az;
    st.acc_w[px] = aw;
    if (st.acc_sq) { st.acc_sq[3 * (size_t)px] = qx; st.acc_sq[3 * (size_t)px + 1] = qy; st.acc_sq[3 * (size_t)px + 2] = qz; }
}

// End of an iteration: statistics, queue reset, loop condition.
// Batch films: one thread per pixel of all jobs (pixels numbered job after job).
__global__ void k_merge_batch(WfParams P, WfState st) {
    const long long gp = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gp >= P.total_pixels) return;
    int lo = 0, hi = P.n_jobs;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (P.jobs[mid].pixel_begin <= gp) lo = mid; else hi = mid;
    }
    const WfJob& J = P.jobs[lo];
    const long long px = gp - J.pixel_begin;
    if (J.n_chunks == 1) return;  // one task per pixel: finish_sample wrote the film
    double ax = 0.0, ay = 0.0, az = 0.0, aw = 0.0;
    for (int k = 0; k < J.n_chunks; ++k) {
        const double4 a = st.part[J.task_begin + (long long)k * J.n_pixels + px];
        ax += a.x; ay += a.y; az += a.z; aw += a.w;
    }
    J.acc[3 * px] = ax; J.acc[3 * px + 1] = ay; J.acc[3 * px + 2] = az;
    J.acc_w[px] = aw;
}

// ---- adaptive renders in rounds -------------------------------------------------
// Round r renders samples [sample_base, sample_end) of every film pixel still
// sampling (active list, n of them) as ordinary tasks and stores each
// sample's radiance.  This kernel then runs the reference's per-pixel loop
// (src/render.rs:143-180) over those samples in sample order: each joins the
// f64 film sums, the Welford statistics of its luminance are updated, and
// after min_spp samples the pixel stops once the sample relative standard
// deviation sqrt(m2 / (n - 1)) / max(|mean|, 1e-4) is below the threshold.
// A pixel that has not stopped goes to the next round's active list.  The
// sums, counts and the stopping decision are those of one loop over the
// pixel's samples; only the streams differ from the reference's (each task
// of task_spp samples starts at seed_for(x, y, sample_start) ^ seed).
__global__ void k_round_merge(WfParams P, WfState st, const int* __restrict__ active, int n, double4* wstate,
                              int* next_active, int* n_next, unsigned long long* taken) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    bool keep = false;
    int px = 0;
    unsigned long long used = 0;
    if (j < n) {
        px = active[j];
        double4 w = wstate[px];  // n, mean, m2, (unused)
        double ax = st.acc[3 * (size_t)px], ay = st.acc[3 * (size_t)px + 1], az = st.acc[3 * (size_t)px + 2];
        double aw = st.acc_w[px];
        double qx = 0.0, qy = 0.0, qz = 0.0;
        if (st.acc_sq) { qx = st.acc_sq[3 * (size_t)px]; qy = st.acc_sq[3 * (size_t)px + 1]; qz = st.acc_sq[3 * (size_t)px + 2]; }
        const int min_spp = min(max(P.adaptive_min_spp, 1), max(P.spp, 1));
        const float4* smp = st.rsamp + (size_t)j * P.round_len;
        const int len = P.sample_end - P.sample_base;
        bool stop = false;
        for (int k = 0; k < len && !stop; ++k, ++used) {
            const float4 L = smp[k];
            ax += (double)L.x; ay += (double)L.y; az += (double)L.z; aw += 1.0;
            if (st.acc_sq) {
                qx += (double)L.x * (double)L.x; qy += (double)L.y * (double)L.y; qz += (double)L.z * (double)L.z;
            }
            w.x += 1.0;
            const double l = 0.2126 * (double)L.x + 0.7152 * (double)L.y + 0.0722 * (double)L.z;
            const double delta = l - w.y;
            w.y += delta / w.x;
            w.z += delta * (l - w.y);
            if (w.x >= (double)min_spp && w.x > 1.0) {
                const double var = w.z / (w.x - 1.0);
                if (sqrt(var) / fmax(fabs(w.y), 1e-4) < P.adaptive_threshold) stop = true;
            }
        }
        wstate[px] = w;
        st.acc[3 * (size_t)px] = ax; st.acc[3 * (size_t)px + 1] = ay; st.acc[3 * (size_t)px + 2] = az;
        st.acc_w[px] = aw;
        if (st.acc_sq) { st.acc_sq[3 * (size_t)px] = qx; st.acc_sq[3 * (size_t)px + 1] = qy; st.acc_sq[3 * (size_t)px + 2] = qz; }
        keep = !stop && P.sample_end < P.spp;
    }
    warp_push(next_active, n_next, keep, px);
    for (int off = 16; off > 0; off >>= 1) used += __shfl_down_sync(0xffffffffu, used, off);
    if (lane_id() == 0 && used) atomicAdd(taken, used);
}

// Round 0: every film pixel active, film and statistics zero.
__global__ void k_round_init(int n_pixels, int* active, double4* wstate, double* acc, double* acc_w, double* acc_sq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pixels) return;
    active[i] = i;
    wstate[i] = make_double4(0.0, 0.0, 0.0, 0.0);
    acc[3 * (size_t)i] = 0.0; acc[3 * (size_t)i + 1] = 0.0; acc[3 * (size_t)i + 2] = 0.0;
    acc_w[i] = 0.0;
    if (acc_sq) { acc_sq[3 * (size_t)i] = 0.0; acc_sq[3 * (size_t)i + 1] = 0.0; acc_sq[3 * (size_t)i + 2] = 0.0; }
}

// ---- ordered extension queue ----------------------------------------------------
// After an iteration the live slots (act byte 1) are compacted, in slot
// order, into the next iteration's extension queue: per 16384-slot span a
// count, one block's exclusive scan of the counts, and a scatter.  The
// kernels then visit only live slots, consecutive lanes on ascending slots.
// A thread covers 64 consecutive act bytes (four 16-byte loads in flight).
constexpr int kCmpBlock = 256, kCmpPerThread = 64, kCmpSpan = kCmpBlock * kCmpPerThread;
constexpr int kCmpScanTiles = 16;  // the scan prefetches up to 16 x 1024 counts (2^28 slots)

// Live-slot bits of slots [t0, t0 + 64) (bit k = slot t0 + k).
__device__ __forceinline__ unsigned long long live_bits(const uint8_t* __restrict__ act, int n, int t0) {
    unsigned long long bits = 0;
    if (t0 + kCmpPerThread <= n) {
        const uint4* a = reinterpret_cast<const uint4*>(act + t0);  // t0 is a multiple of 64
        uint4 v[4];
        for (int k = 0; k < 4; ++k) v[k] = a[k];
        for (int k = 0; k < 4; ++k) {
            const unsigned w[4] = {v[k].x, v[k].y, v[k].z, v[k].w};
            for (int q = 0; q < 4; ++q)
                for (int b = 0; b < 4; ++b)
                    if ((w[q] >> (8 * b)) & 0xffu) bits |= 1ull << (16 * k + 4 * q + b);
        }
    } else {
        for (int k = 0; k < kCmpPerThread; ++k)
            if (t0 + k < n && act[t0 + k]) bits |= 1ull << k;
    }
    return bits;
}

// Exclusive prefix of v over the block's threads; *total gets the sum.
__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_sums, int* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        int ws = lane < nw ? warp_sums[lane] : 0;
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, ws, off);
            if (lane >= off) ws += y;
        }
        if (lane < nw) warp_sums[lane] = ws;  // inclusive per warp
    }
    __syncthreads();
    const int before = w > 0 ? warp_sums[w - 1] : 0;
    if (total) *total = warp_sums[(blockDim.x >> 5) - 1];
    const int excl = before + x - v;
    __syncthreads();  // warp_sums may be reused by the caller
    return excl;
}

__global__ void __launch_bounds__(kCmpBlock) k_cmp_count(const uint8_t* __restrict__ act, int n, int* counts) {
    __shared__ int ws[kCmpBlock / 32];
    const int t0 = blockIdx.x * kCmpSpan + threadIdx.x * kCmpPerThread;
    const int c = __popcll(live_bits(act, n, t0));
    int total = 0;
    block_exclusive_scan(c, ws, &total);
    if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

// One block of 1024: counts[0..nb) -> exclusive offsets in place; *n_out =
// the total.  The first 16 x 1024 counts are loaded at once (coalesced),
// then scanned tile by tile; any further tiles load one after another.
__global__ void __launch_bounds__(1024) k_cmp_scan(int* counts, int nb, int* n_out) {
    __shared__ int ws[32];
    int v[kCmpScanTiles];
#pragma unroll
    for (int k = 0; k < kCmpScanTiles; ++k) {
        const int i = k * 1024 + (int)threadIdx.x;
        v[k] = i < nb ? counts[i] : 0;
    }
    int run = 0;
#pragma unroll
    for (int k = 0; k < kCmpScanTiles; ++k) {
        if (k * 1024 >= nb) break;  // uniform over the block
        int total = 0;
        const int ex = block_exclusive_scan(v[k], ws, &total);
        const int i = k * 1024 + (int)threadIdx.x;
        if (i < nb) counts[i] = run + ex;
        run += total;
    }
    for (int b0 = kCmpScanTiles * 1024; b0 < nb; b0 += 1024) {
        const int i = b0 + (int)threadIdx.x;
        int total = 0;
        const int ex = block_exclusive_scan(i < nb ? counts[i] : 0, ws, &total);
        if (i < nb) counts[i] = run + ex;
        run += total;
    }
    if (threadIdx.x == 0) *n_out = run;
}

// The scatter takes its span in four rounds of 4096 slots (16 per thread,
// one 16-byte load): each round's live slot ids are ranked into shared
// memory, then written out by the whole block in consecutive addresses.
__global__ void __launch_bounds__(kCmpBlock) k_cmp_scatter(const uint8_t* __restrict__ act, int n,
                                                          const int* __restrict__ offsets, int* __restrict__ q) {
    constexpr int kRound = kCmpBlock * 16;
    __shared__ int ws[kCmpBlock / 32];
    __shared__ int stage[kRound];
    int out = offsets[blockIdx.x];
    for (int r = 0; r < kCmpSpan / kRound; ++r) {
        const int t0 = blockIdx.x * kCmpSpan + r * kRound + threadIdx.x * 16;
        unsigned bits = 0;
        if (t0 + 16 <= n) {
            const uint4 v = *reinterpret_cast<const uint4*>(act + t0);  // t0 is a multiple of 16
            const unsigned w[4] = {v.x, v.y, v.z, v.w};
            for (int q4 = 0; q4 < 4; ++q4)
                for (int b = 0; b < 4; ++b)
                    if ((w[q4] >> (8 * b)) & 0xffu) bits |= 1u << (4 * q4 + b);
        } else {
            for (int k = 0; k < 16; ++k)
                if (t0 + k < n && act[t0 + k]) bits |= 1u << k;
        }
        int total = 0;
        int pos = block_exclusive_scan(__popc(bits), ws, &total);  // ends with a barrier
        while (bits) {
            const int k = __ffs(bits) - 1;
            bits &= bits - 1;
            stage[pos++] = t0 + k;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < total; i += kCmpBlock) q[out + i] = stage[i];
        out += total;
        __syncthreads();  // stage is refilled next round
    }
}

__global__ void k_step(WfState st, int cur, long long max_iters, cudaGraphConditionalHandle handle, int use_cond,
                       long long fetch_end = 0, int tail_live = 0) {
    WfCounters* c = st.ctr;
    c->rays_closest += (unsigned long long)c->n_ext[cur];
    c->rays_shadow += (unsigned long long)c->n_sh;
    c->samples += (unsigned long long)c->n_term + (unsigned long long)c->n_done_in_shade;
    c->n_done_in_shade = 0;
    for (int k = 0; k < 5; ++k) c->n_mat[k] = 0;
    c->n_ext[cur] = 0;
    c->n_sh = 0;
    c->n_term = 0;
    c->fetch_ext = 0;
    c->fetch_sh = 0;
    c->iters += 1;
    bool more = c->n_ext[cur ^ 1] > 0;
    if (more && tail_live > 0 && c->n_ext[cur ^ 1] <= tail_live && c->next_task >= fetch_end) {
        c->tail = 1;  // the pool's tasks are all taken: k_tail finishes the few live slots
        more = false;
    }
    if (more && c->iters >= max_iters) {
        c->flags |= TPT_FLAG_ITER_LIMIT;
        more = false;
        c->n_ext[cur ^ 1] = 0;  // iterations a host loop has already enqueued find nothing to do
    }
    if (use_cond) cudaGraphSetConditional(handle, more ? 1u : 0u);
}

}  // namespace wf

// ---- buffers ---------------------------------------------------------------
namespace {
size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }
}

namespace {
// Frees the path-state block only (the adaptive-round arrays stay).
void release_state(WfBuffers& b) {
    if (b.block) cudaFree(b.block);
    b.block = nullptr;
    b.slots = 0;
    b.part_tasks = 0;
}
}  // namespace

cudaError_t wf_reserve(WfBuffers& b, size_t slots, size_t part_tasks) {
    if (b.block && b.slots >= slots && b.part_tasks >= part_tasks) return cudaSuccess;
    release_state(b);
    const size_t S = slots, T = part_tasks;
    // (entry 5 holds the two extension queues)
    size_t sz[] = {S * 16, S * 16, S * 16, S * 16, S * 16, 2 * S * 4, S * 16, 2 * S * 16, 2 * S * 16, 2 * S * 16,
                   S * 16, S * 1, 2 * S * 4, S * 4, sizeof(WfCounters), S * 32, S * 32, T * 32, T * 32,
                   S * 16, S * 16, 5 * S * 4, S * 4, wf_compact_spans(S) * 4};
    size_t total = 0;
    for (size_t s : sz) total += align_up(s);
    char* p = nullptr;
    cudaError_t e = cudaMalloc(&p, total);
    if (e != cudaSuccess) return e;
    b.block = p;
    b.slots = slots;
    b.part_tasks = part_tasks;
    size_t off = 0;
    auto take = [&](size_t bytes) { char* r = p + off; off += align_up(bytes); return (void*)r; };
    WfState& st = b.st;
    st.path = (int4*)take(sz[0]);
    st.ray_o = (float4*)take(sz[1]);
    st.ray_d = (float4*)take(sz[2]);
    st.beta = (float4*)take(sz[3]);
    st.rad = (float4*)take(sz[4]);
    st.q_ext[0] = (int*)take(sz[5]);
    st.q_ext[1] = st.q_ext[0] + S;
    st.hit = (float4*)take(sz[6]);
    st.sh_o = (float4*)take(sz[7]);
    st.sh_d = (float4*)take(sz[8]);
    st.sh_c = (float4*)take(sz[9]);
    st.welford = (double2*)take(sz[10]);
    st.act = (uint8_t*)take(sz[11]);
    st.q_sh = (int*)take(sz[12]);
    st.q_term = (int*)take(sz[13]);
    st.ctr = (WfCounters*)take(sz[14]);
    st.sacc = (double4*)take(sz[15]);
    st.ssq = (double4*)take(sz[16]);
    st.part = T ? (double4*)take(sz[17]) : nullptr;
    st.part_sq = T ? (double4*)take(sz[18]) : nullptr;
    st.surf_p = (float4*)take(sz[19]);
    st.surf_n = (float4*)take(sz[20]);
    st.q_mat = (int*)take(sz[21]);
    st.job = (int*)take(sz[22]);
    st.cmp_counts = (int*)take(sz[23]);
    return cudaSuccess;
}

void wf_release(WfBuffers& b) {
    release_state(b);
    if (b.round_block) cudaFree(b.round_block);
    b.round_block = nullptr;
    b.round_pixels = b.round_samples = 0;
    if (b.cull_block) cudaFree(b.cull_block);
    b.cull_block = nullptr;
    b.cull_pixels = 0;
    if (b.ev_fork) cudaEventDestroy(b.ev_fork);
    if (b.ev_join) cudaEventDestroy(b.ev_join);
    if (b.side) cudaStreamDestroy(b.side);
    b.ev_fork = b.ev_join = nullptr;
    b.side = nullptr;
}

namespace {
// Camera-culling arrays for a film of `pixels`: two flag bytes and two
// compacted lists per pixel, the compaction's span counts, two lengths.
cudaError_t cull_reserve(WfBuffers& b, size_t pixels) {
    if (b.cull_block && b.cull_pixels >= pixels) return cudaSuccess;
    if (b.cull_block) cudaFree(b.cull_block);
    b.cull_block = nullptr;
    b.cull_pixels = 0;
    const size_t spans = wf_compact_spans(pixels);
    const size_t sz[] = {pixels, pixels, pixels * 4, pixels * 4, spans * 4, spans * 4, 256};
    size_t total = 0;
    for (size_t x : sz) total += align_up(x);
    char* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, total);
    if (e != cudaSuccess) return e;
    size_t off = 0;
    auto take = [&](size_t bytes) { char* r = p + off; off += align_up(bytes); return (void*)r; };
    b.cull_block = p;
    b.cull_flag[0] = (uint8_t*)take(sz[0]);
    b.cull_flag[1] = (uint8_t*)take(sz[1]);
    b.cull_map[0] = (int*)take(sz[2]);
    b.cull_map[1] = (int*)take(sz[3]);
    b.cull_counts[0] = (int*)take(sz[4]);
    b.cull_counts[1] = (int*)take(sz[5]);
    b.cull_n = (int*)take(sz[6]);
    b.cull_pixels = pixels;
    return cudaSuccess;
}

// Classifies the film's pixels (a multi-job render: every job's) for
// camera culling and compacts both kinds in pixel order: B.cull_map[0] =
// the n_may pixels a camera ray may reach geometry from, B.cull_map[1] =
// the n_open others.  A multi-job render then also gets each job's
// stretches and first ids in the device job table, and n_fetch / n_sky_tasks
// for the whole batch.  7 launches (8 for multi-job renders), one read-back.
cudaError_t cull_classify(const WfScene& S, const WfParams& P, WfBuffers& B, cudaStream_t s, int& n_may, int& n_open,
                          long long& n_fetch, long long& n_sky_tasks) {
    const long long n_ll = P.jobs ? P.total_pixels : (long long)P.n_pixels;
    cudaError_t e = cull_reserve(B, (size_t)n_ll);
    if (e != cudaSuccess) return e;
    const int n = (int)n_ll;
    if (P.jobs) wf::k_cull_classify<true><<<(n + 255) / 256, 256, 0, s>>>(S, P, B.cull_flag[0], B.cull_flag[1]);
    else wf::k_cull_classify<false><<<(n + 255) / 256, 256, 0, s>>>(S, P, B.cull_flag[0], B.cull_flag[1]);
    const int nb = (int)((n + wf::kCmpSpan - 1) / wf::kCmpSpan);
    for (int k = 0; k < 2; ++k) {
        wf::k_cmp_count<<<nb, wf::kCmpBlock, 0, s>>>(B.cull_flag[k], n, B.cull_counts[k]);
        wf::k_cmp_scan<<<1, 1024, 0, s>>>(B.cull_counts[k], nb, B.cull_n + k);
        wf::k_cmp_scatter<<<nb, wf::kCmpBlock, 0, s>>>(B.cull_flag[k], n, B.cull_counts[k], B.cull_map[k]);
    }
    long long* totals = reinterpret_cast<long long*>(B.cull_n + 2);  // 8-byte aligned: cull_n is 256-byte aligned
    if (P.jobs)
        wf::k_cull_jobs<<<1, 1024, 0, s>>>(const_cast<WfJob*>(P.jobs), P.n_jobs, B.cull_map[0], B.cull_map[1],
                                           B.cull_n, totals);
    struct { int n[2]; long long t[2]; } h{{n, 0}, {0, 0}};
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, B.cull_n, sizeof h, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    n_may = h.n[0];
    n_open = h.n[1];
    n_fetch = P.jobs ? h.t[0] : 0;
    n_sky_tasks = P.jobs ? h.t[1] : 0;
    return e;
}
}  // namespace

cudaError_t wf_cull_pixels(const WfScene& S, const WfParams& P, WfBuffers& B, cudaStream_t s, int* n_may,
                           int* n_open) {
    long long f = 0, u = 0;
    return cull_classify(S, P, B, s, *n_may, *n_open, f, u);
}

namespace {
// Adaptive-round arrays: Welford state (32 B) and two active lists (4 B
// each) per film pixel, a counter, and `samples` float4 sample records.
cudaError_t round_reserve(WfBuffers& b, size_t pixels, size_t samples) {
    if (b.round_block && b.round_pixels >= pixels && b.round_samples >= samples) return cudaSuccess;
    if (b.round_block) cudaFree(b.round_block);
    b.round_block = nullptr;
    b.round_pixels = b.round_samples = 0;
    const size_t sz[] = {pixels * 32, pixels * 4, pixels * 4, 256, samples * 16};
    size_t total = 0;
    for (size_t x : sz) total += align_up(x);
    char* p = nullptr;
    cudaError_t e = cudaMalloc(&p, total);
    if (e != cudaSuccess) return e;
    size_t off = 0;
    auto take = [&](size_t bytes) { char* r = p + off; off += align_up(bytes); return (void*)r; };
    b.round_block = p;
    b.wstate = (double4*)take(sz[0]);
    b.active[0] = (int*)take(sz[1]);
    b.active[1] = (int*)take(sz[2]);
    b.n_active = (int*)take(sz[3]);
    b.rsamp = (float4*)take(sz[4]);
    b.round_pixels = pixels;
    b.round_samples = samples;
    return cudaSuccess;
}
}  // namespace

// ---- host driver -------------------------------------------------------------
namespace {

struct Grids { int extend, shade, shadow, regen, surface[5], shade_all, shade_all4, shade_all6, shade_batch, shade_batch8; };

// Shading: the classify kernel, then one surface kernel per material kind
// (each returns at once when its queue is empty).
void launch_shade(const Grids& g, cudaStream_t s, const WfScene& S, const WfParams& P, const WfState& st, int cur) {
    if (P.jobs) {  // batch renders: fused shading only
        if (P.shade_ctas == 8) wf::k_shade<true, 8><<<g.shade_batch8, 128, 0, s>>>(S, P, st, cur);
        else wf::k_shade<true, 4><<<g.shade_batch, 128, 0, s>>>(S, P, st, cur);
        return;
    }
    if (!P.shade_sort) {
        if (P.shade_ctas == 4) wf::k_shade<false, 4><<<g.shade_all4, 128, 0, s>>>(S, P, st, cur);
        else if (P.shade_ctas == 6) wf::k_shade<false, 6><<<g.shade_all6, 128, 0, s>>>(S, P, st, cur);
        else wf::k_shade<false, 8><<<g.shade_all, 128, 0, s>>>(S, P, st, cur);
        return;
    }
    wf::k_shade_pre<<<g.shade, 128, 0, s>>>(S, P, st, cur);
    wf::k_shade_surface<TPT_MAT_LAMBERT><<<g.surface[0], 128, 0, s>>>(S, P, st, cur);
    wf::k_shade_surface<TPT_MAT_METAL><<<g.surface[1], 128, 0, s>>>(S, P, st, cur);
    wf::k_shade_surface<TPT_MAT_DIELECTRIC><<<g.surface[2], 128, 0, s>>>(S, P, st, cur);
    wf::k_shade_surface<TPT_MAT_GGX><<<g.surface[3], 128, 0, s>>>(S, P, st, cur);
    wf::k_shade_surface<TPT_MAT_SUBSURFACE><<<g.surface[4], 128, 0, s>>>(S, P, st, cur);
}

// Trace kernels keep their stack in shared memory when the scene's deepest
// path (top level + exit marker + mesh tree) fits kSharedStack entries.
template <bool ANY, bool COUNT>
void launch_trace(int grid, cudaStream_t s, const WfScene& S, const WfParams& P, const WfState& st, int n_slots,
                  int chunk, int cur) {
    const bool shared = S.max_stack <= wf::kSharedStack;
    if (P.jobs) {
        if (shared)
            wf::k_trace<ANY, COUNT, true, true><<<grid, wf::kTraceBlock, 0, s>>>(S, P, st, n_slots, chunk, P.jobs, cur);
        else
            wf::k_trace<ANY, COUNT, false, true><<<grid, wf::kTraceBlock, 0, s>>>(S, P, st, n_slots, chunk, P.jobs, cur);
    } else if (shared) {
        wf::k_trace<ANY, COUNT, true, false><<<grid, wf::kTraceBlock, 0, s>>>(S, P, st, n_slots, chunk, nullptr, cur);
    } else {
        wf::k_trace<ANY, COUNT, false, false><<<grid, wf::kTraceBlock, 0, s>>>(S, P, st, n_slots, chunk, nullptr, cur);
    }
}
void launch_regen(int grid, cudaStream_t s, const WfScene& S, const WfParams& P, const WfState& st, int cur) {
    if (P.jobs) wf::k_regen<true><<<grid, 128, 0, s>>>(S, P, st, cur);
    else wf::k_regen<false><<<grid, 128, 0, s>>>(S, P, st, cur);
}

template <class K>
int grid_for(K kernel, int sm_count) {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, 128, 0);
    return sm_count * (occ > 0 ? occ : 1);
}

Grids pick_grids(int sm_count) {
    Grids g{};
    g.extend = grid_for(wf::k_trace<false, false, true, false>, sm_count);
    g.shadow = grid_for(wf::k_trace<true, false, true, false>, sm_count);
    g.shade = grid_for(wf::k_shade_pre, sm_count);
    g.shade_all = grid_for(wf::k_shade<false, 8>, sm_count);
    g.shade_all4 = grid_for(wf::k_shade<false, 4>, sm_count);
    g.shade_all6 = grid_for(wf::k_shade<false, 6>, sm_count);
    g.shade_batch = grid_for(wf::k_shade<true, 4>, sm_count);
    g.shade_batch8 = grid_for(wf::k_shade<true, 8>, sm_count);
    g.surface[0] = grid_for(wf::k_shade_surface<TPT_MAT_LAMBERT>, sm_count);
    g.surface[1] = grid_for(wf::k_shade_surface<TPT_MAT_METAL>, sm_count);
    g.surface[2] = grid_for(wf::k_shade_surface<TPT_MAT_DIELECTRIC>, sm_count);
    g.surface[3] = grid_for(wf::k_shade_surface<TPT_MAT_GGX>, sm_count);
    g.surface[4] = grid_for(wf::k_shade_surface<TPT_MAT_SUBSURFACE>, sm_count);
    g.regen = grid_for(wf::k_regen<false>, sm_count);
    return g;
}

// The pool's end of fetch ids (fetch_end on the device).
long long host_fetch_end(const WfParams& P) {
    if (!P.geo_map) return P.n_tasks;
    if (P.jobs) return P.n_fetch;
    return P.task_first + (P.n_tasks - P.task_first) / P.n_pixels * P.n_geo;
}

void enqueue_iteration(const WfScene& S, const WfParams& P, const WfState& st, const Grids& g, cudaStream_t s,
                       cudaGraphConditionalHandle h, int use_cond) {
    for (int cur = 0; cur < 2; ++cur) {
        launch_trace<false, false>(g.extend, s, S, P, st, P.n_slots, P.trace_chunk, cur);
        launch_shade(g, s, S, P, st, cur);
        launch_trace<true, false>(g.shadow, s, S, P, st, P.n_slots, P.trace_chunk, cur);
        launch_regen(g.regen, s, S, P, st, cur);
        if (P.ordered_queue) wf_launch_compact(s, st, cur, P.n_slots);
        wf::k_step<<<1, 1, 0, s>>>(st, cur, P.max_iters, h, use_cond, P.tail_live > 0 ? host_fetch_end(P) : 0,
                                   P.tail_live);
    }
}

struct Events {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    Events() { cudaEventCreate(&e0); cudaEventCreate(&e1); }
    ~Events() { cudaEventDestroy(e0); cudaEventDestroy(e1); }
};

struct GraphGuard {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~GraphGuard() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

// Device-driven loop: one WHILE conditional node whose body is two
// iterations; the last kernel of each iteration re-arms the condition on the
// device.
cudaError_t run_graph_loop(const WfEnqueue& enqueue, cudaStream_t stream, bool* built) {
    GraphGuard gg;
    cudaError_t e = cudaGraphCreate(&gg.graph, 0);
    cudaGraphConditionalHandle handle{};
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&handle, gg.graph, 1, cudaGraphCondAssignDefault);
    cudaGraphNode_t node{};
    cudaGraphNodeParams np{};
    if (e == cudaSuccess) {
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = handle;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        e = cudaGraphAddNode(&node, gg.graph, nullptr, 0, &np);
    }
    cudaStream_t cap = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        cudaGraph_t body = np.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            enqueue(cap, handle, 1);
            e = cudaStreamEndCapture(cap, &body);
        }
    }
    if (cap) cudaStreamDestroy(cap);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&gg.exec, gg.graph, 0);
    if (e != cudaSuccess) {
        // Nothing ran yet: report "not supported" so the caller can use the
        // host-driven loop instead.
        cudaGetLastError();
        *built = false;
        return e;
    }
    *built = true;
    e = cudaGraphLaunch(gg.exec, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    return e;
}

// Host-driven loop: the two-iteration body launched directly on the stream
// (no graph, so every kernel launch is visible to a profiler's launch list),
// 8 bodies between checks of the extension queue.
cudaError_t run_host_loop(const WfEnqueue& enqueue, const WfCounters* ctr, long long max_iters,
                          cudaStream_t stream) {
    WfCounters probe{};
    long long launched = 0;
    cudaError_t e = cudaSuccess;
    // one graph body (two iterations) between probes, so the loop ends where
    // the device-side loop would
    while (e == cudaSuccess) {
        enqueue(stream, cudaGraphConditionalHandle{}, 0);
        launched += 2;
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&probe, ctr, sizeof(WfCounters), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) break;
        if (probe.n_ext[0] == 0 && probe.n_ext[1] == 0) break;
        if (probe.tail) break;  // k_tail finishes the live slots
        if ((probe.flags & TPT_FLAG_ITER_LIMIT) || launched > max_iters + 16) break;
    }
    return e;
}

// Profiling loop: plain launches with events around every stage and the
// counting variants of the trace kernels.
cudaError_t run_profile_loop(const WfScene& S, const WfParams& P, const WfState& st, const Grids& g,
                             cudaStream_t s, double* stage_ms, unsigned long long* stage_launches) {
    Events ev[4];
    cudaError_t e = cudaSuccess;
    WfCounters probe{};
    for (long long it = 0; it <= P.max_iters + 1 && e == cudaSuccess; it += 2) {
        for (int cur = 0; cur < 2 && e == cudaSuccess; ++cur) {
            cudaEventRecord(ev[0].e0, s);
            launch_trace<false, true>(g.extend, s, S, P, st, P.n_slots, P.trace_chunk, cur);
            cudaEventRecord(ev[0].e1, s);
            cudaEventRecord(ev[1].e0, s);
            launch_shade(g, s, S, P, st, cur);
            cudaEventRecord(ev[1].e1, s);
            cudaEventRecord(ev[2].e0, s);
            launch_trace<true, true>(g.shadow, s, S, P, st, P.n_slots, P.trace_chunk, cur);
            cudaEventRecord(ev[2].e1, s);
            cudaEventRecord(ev[3].e0, s);
            launch_regen(g.regen, s, S, P, st, cur);
            if (P.ordered_queue) wf_launch_compact(s, st, cur, P.n_slots);
            cudaEventRecord(ev[3].e1, s);
            wf::k_step<<<1, 1, 0, s>>>(st, cur, P.max_iters, cudaGraphConditionalHandle{}, 0);
            e = cudaMemcpyAsync(&probe, st.ctr, sizeof(WfCounters), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) break;
            for (int k = 0; k < 4; ++k) {
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, ev[k].e0, ev[k].e1);
                stage_ms[k] += ms;
                stage_launches[k] += 1;
            }
            if (probe.n_ext[0] == 0 && probe.n_ext[1] == 0) return cudaSuccess;
        }
    }
    return e;
}

}  // namespace

cudaError_t wf_run_loop(const WfEnqueue& enqueue, const WfCounters* ctr, long long max_iters, cudaStream_t stream,
                        bool use_graph_loop) {
    if (use_graph_loop) {
        bool built = false;
        const cudaError_t e = run_graph_loop(enqueue, stream, &built);
        if (e == cudaSuccess || built) return e;
    }
    return run_host_loop(enqueue, ctr, max_iters, stream);
}

void wf_trace_grids(int sm_count, int* extend, int* shadow) {
    *extend = grid_for(wf::k_trace<false, false, true, false>, sm_count);
    *shadow = grid_for(wf::k_trace<true, false, true, false>, sm_count);
}

void wf_launch_trace(bool any, int grid, cudaStream_t s, const WfScene& S, const WfParams& P, const WfState& st,
                     int cur) {
    if (any) launch_trace<true, false>(grid, s, S, P, st, P.n_slots, P.trace_chunk, cur);
    else launch_trace<false, false>(grid, s, S, P, st, P.n_slots, P.trace_chunk, cur);
}

void wf_launch_step(cudaStream_t s, const WfState& st, int cur, long long max_iters, cudaGraphConditionalHandle h,
                    int use_cond) {
    wf::k_step<<<1, 1, 0, s>>>(st, cur, max_iters, h, use_cond);
}

size_t wf_compact_spans(size_t n_slots) { return (n_slots + wf::kCmpSpan - 1) / wf::kCmpSpan + 1; }

void wf_launch_compact(cudaStream_t s, const WfState& st, int cur, int n_slots) {
    const int nb = (int)((n_slots + wf::kCmpSpan - 1) / wf::kCmpSpan);
    const int nxt = cur ^ 1;
    wf::k_cmp_count<<<nb, wf::kCmpBlock, 0, s>>>(st.act, n_slots, st.cmp_counts);
    wf::k_cmp_scan<<<1, 1024, 0, s>>>(st.cmp_counts, nb, &st.ctr->n_ext[nxt]);
    wf::k_cmp_scatter<<<nb, wf::kCmpBlock, 0, s>>>(st.act, n_slots, st.cmp_counts, st.q_ext[nxt]);
}

namespace {
void add_counters(WfCounters& a, const WfCounters& b) {
    a.iters += b.iters;
    a.flags |= b.flags;
    a.rays_closest += b.rays_closest;
    a.rays_shadow += b.rays_shadow;
    a.samples += b.samples;
    for (int k = 0; k < 2; ++k) {
        a.cnt_nodes[k] += b.cnt_nodes[k];
        a.cnt_tris[k] += b.cnt_tris[k];
        a.cnt_spheres[k] += b.cnt_spheres[k];
        a.cnt_inst[k] += b.cnt_inst[k];
        a.cnt_node_steps[k] += b.cnt_node_steps[k];
        a.cnt_leaves[k] += b.cnt_leaves[k];
        a.cnt_leaf_steps[k] += b.cnt_leaf_steps[k];
    }
    a.cnt_fast += b.cnt_fast;
    a.cnt_fast_steps += b.cnt_fast_steps;
    a.sky_samples += b.sky_samples;
}

// Kernels one iteration of the bounce loop launches (enqueue_iteration).
long long launches_per_iteration(const WfParams& P) {
    return 3 + (P.shade_sort && !P.jobs ? 6 : 1) + (P.ordered_queue ? 3 : 0) + 1;
}
}  // namespace

namespace {
// Reserves the path state of P.n_slots slots, halving the pool (down to 2^20
// slots) while the device has no room for it; the iteration bound grows to
// match.  A render does not depend on the pool size: each task's samples run
// in one slot and task sums merge in task order.
cudaError_t reserve_pool(WfBuffers& B, WfParams& P, size_t part_tasks) {
    for (;;) {
        const cudaError_t e = wf_reserve(B, (size_t)P.n_slots, part_tasks);
        if (e != cudaErrorMemoryAllocation || P.n_slots <= (1 << 20)) return e;
        cudaGetLastError();
        P.n_slots /= 2;
        P.max_iters *= 2;
    }
}
}  // namespace

// A single render whose per-task sums would exceed P.max_part_tasks runs its
// sample chunks in batches (chunks [c0, c1) of every pixel, then the next
// batch), merging each onto the film in task order: device memory for the
// sums stays bounded however many samples a pixel takes.
cudaError_t wf_render(const WfScene& S, const WfParams& P_in, WfBuffers& B, double* acc, double* acc_w, double* acc_sq,
                      cudaStream_t stream, int sm_count, bool use_graph_loop, WfCounters* hc, float* ms, bool profile,
                      double* stage_ms, unsigned long long* stage_launches) {
    WfParams P = P_in;
    long long batch_chunks = P.n_chunks;
    if (!P.jobs && P.n_chunks > 1 && P.max_part_tasks > 0 && P.n_tasks > P.max_part_tasks)
        batch_chunks = std::max<long long>(1, P.max_part_tasks / P.n_pixels);
    // per-task sums of one chunk batch (single renders) or of all tasks (a
    // multi-job render, whose P.n_pixels is 0: every job has its own)
    size_t part_tasks = 0;
    if (P.n_chunks > 1)
        part_tasks = P.jobs ? (size_t)P.n_tasks : (size_t)std::min<long long>(P.n_tasks, batch_chunks * P.n_pixels);
    cudaError_t e = reserve_pool(B, P, part_tasks);
    if (e != cudaSuccess) return e;
    WfState st = B.st;
    st.acc = acc;
    st.acc_w = acc_w;
    st.acc_sq = acc_sq;
    if (!P.adaptive) st.welford = nullptr;
    if (!acc_sq) { st.ssq = nullptr; st.part_sq = nullptr; }
    const Grids g = pick_grids(sm_count);

    Events total;
    cudaEventRecord(total.e0, stream);
    if (profile)
        for (int k = 0; k < 4; ++k) { stage_ms[k] = 0.0; stage_launches[k] = 0; }
    // Camera culling: forward renders (single or multi-job) through pinhole
    // cameras (cull_may_hit keeps every pixel of a lens camera).
    long long launches = 0;
    int n_may = P.n_pixels, n_open = 0;
    long long n_fetch = 0, n_sky_tasks = 0;
    const bool cull_single = !P.jobs && P.max_bounces > 0 && P.n_pixels > 0 && S.cam.lens_radius == 0.0f &&
                             S.cam.focus_dist > 0.0f;
    const bool cull_batch = P.jobs && P.total_pixels > 0 && P.total_pixels < (1ll << 31);
    if (P.sky_cull && !P.adaptive && (cull_single || cull_batch)) {
        e = cull_classify(S, P, B, stream, n_may, n_open, n_fetch, n_sky_tasks);
        launches += P.jobs ? 8 : 7;
        if (e != cudaSuccess) {
            cudaGetLastError();
            return e;
        }
    }
    // With the open pixels culled, the camera rays left that miss are few:
    // the fast path then costs the closest-hit kernel more than it saves
    // (1080p frame: 2.76 -> 2.80 G paths/s without it).
    if (P.camera_fast == 2) P.camera_fast = n_open > 0 ? 0 : 1;
    WfCounters sum{};
    for (long long c0 = 0; c0 < P.n_chunks && e == cudaSuccess; c0 += batch_chunks) {
        WfParams Pb = P;
        if (!P.jobs) {
            Pb.task_first = c0 * P.n_pixels;
            Pb.n_tasks = std::min<long long>(c0 + batch_chunks, P.n_chunks) * P.n_pixels;
        }
        const long long batch_chunk_count = P.jobs ? 0 : (Pb.n_tasks - Pb.task_first) / P.n_pixels;
        if (n_open > 0) {
            // the pool takes the other pixels' tasks; no more slots than those
            Pb.geo_map = B.cull_map[0];
            Pb.n_geo = n_may;
            Pb.geo_div = make_fastdiv((uint32_t)std::max(n_may, 1));
            Pb.n_fetch = n_fetch;
            const long long pooled = P.jobs ? n_fetch : batch_chunk_count * n_may;
            if (pooled > 0 && pooled < Pb.n_slots) Pb.n_slots = (int)pooled;
        }
        // the drain's handover to k_tail (1080p frame, 64 Mi slots: 2.838 -> 2.931 G paths/s at
        // 262,144; 2.921 at 65,536, 2.930 at 1 Mi, 2.781 at 4 Mi)
        if (Pb.tail_live < 0) Pb.tail_live = std::min(262144, Pb.n_slots / 16);
        cudaMemsetAsync(st.ctr, 0, sizeof(WfCounters), stream);
        // The culled tasks run on a side stream beside the bounce loop: they
        // write other tasks' sums, read only the classification, and count
        // into sky_samples alone; the merge waits for them.
        bool sky_side = false;
        if (n_open > 0) {
            const long long count = P.jobs ? n_sky_tasks : batch_chunk_count * n_open;
            const unsigned grid = (unsigned)((count + 255) / 256);
            const FastDiv od = make_fastdiv((uint32_t)n_open);
            if (!B.side) {
                if (cudaStreamCreateWithFlags(&B.side, cudaStreamNonBlocking) != cudaSuccess ||
                    cudaEventCreateWithFlags(&B.ev_fork, cudaEventDisableTiming) != cudaSuccess ||
                    cudaEventCreateWithFlags(&B.ev_join, cudaEventDisableTiming) != cudaSuccess) {
                    cudaGetLastError();
                    if (B.side) cudaStreamDestroy(B.side);
                    B.side = nullptr;
                }
            }
            cudaStream_t ss = stream;
            if (B.side && B.ev_fork && B.ev_join) {
                cudaEventRecord(B.ev_fork, stream);
                cudaStreamWaitEvent(B.side, B.ev_fork, 0);
                ss = B.side;
                sky_side = true;
            }
            if (P.jobs) wf::k_sky_tasks<true><<<grid, 256, 0, ss>>>(S, Pb, st, B.cull_map[1], n_open, od, count);
            else wf::k_sky_tasks<false><<<grid, 256, 0, ss>>>(S, Pb, st, B.cull_map[1], n_open, od, count);
            if (sky_side) cudaEventRecord(B.ev_join, B.side);
            ++launches;
        }
        if (P.jobs) wf::k_init<true><<<(Pb.n_slots + 255) / 256, 256, 0, stream>>>(S, Pb, st);
        else wf::k_init<false><<<(Pb.n_slots + 255) / 256, 256, 0, stream>>>(S, Pb, st);
        ++launches;
        e = cudaGetLastError();
        if (e == cudaSuccess) {
            if (profile) {
                e = run_profile_loop(S, Pb, st, g, stream, stage_ms, stage_launches);
            } else {
                e = wf_run_loop([&](cudaStream_t s, cudaGraphConditionalHandle h, int use_cond) {
                    enqueue_iteration(S, Pb, st, g, s, h, use_cond);
                }, st.ctr, P.max_iters, stream, use_graph_loop);
                if (e == cudaSuccess && Pb.tail_live > 0) {
                    // the slots the loop left (none when it drained the pool)
                    const unsigned grid = (unsigned)((Pb.tail_live + 127) / 128);
                    if (P.jobs) wf::k_tail<true><<<grid, 128, 0, stream>>>(S, Pb, st);
                    else wf::k_tail<false><<<grid, 128, 0, stream>>>(S, Pb, st);
                    ++launches;
                    e = cudaGetLastError();
                }
            }
        }
        if (sky_side) cudaStreamWaitEvent(stream, B.ev_join, 0);
        if (e == cudaSuccess && P.n_chunks > 1) {
            if (P.jobs)
                wf::k_merge_batch<<<(unsigned)((P.total_pixels + 255) / 256), 256, 0, stream>>>(Pb, st);
            else
                wf::k_merge<<<(P.n_pixels + 255) / 256, 256, 0, stream>>>(Pb, st);
            ++launches;
            e = cudaGetLastError();
        }
        WfCounters part{};
        if (e == cudaSuccess) e = cudaMemcpyAsync(&part, st.ctr, sizeof(WfCounters), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e == cudaSuccess) {
            part.samples += part.sky_samples;  // counted apart by k_sky_tasks
            part.rays_closest += part.sky_samples;
            add_counters(sum, part);
            launches += part.iters * launches_per_iteration(Pb);
        }
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return e;
    }
    cudaEventRecord(total.e1, stream);
    e = cudaEventSynchronize(total.e1);
    sum.pool_slots = P.n_slots;
    sum.launches = launches;
    *hc = sum;
    if (e == cudaSuccess && ms) cudaEventElapsedTime(ms, total.e0, total.e1);
    return e;
}

cudaError_t wf_render_adaptive(const WfScene& S, const WfParams& P_in, WfBuffers& B, double* acc, double* acc_w,
                               double* acc_sq, cudaStream_t stream, int sm_count, bool use_graph_loop, WfCounters* hc,
                               float* ms, size_t round_bytes, int* rounds_out) {
    WfParams P0 = P_in;
    const int n_film = P0.n_pixels, tspp = P0.task_spp;
    // round 0 takes the first min_spp samples (whole tasks): no pixel can stop before them
    const int min_spp = std::min(std::max(P0.adaptive_min_spp, 1), std::max(P0.spp, 1));
    const int first_len = std::min(P0.spp, (min_spp + tspp - 1) / tspp * tspp);
    const size_t cap = std::max(round_bytes / 16, (size_t)n_film * (size_t)first_len);
    cudaError_t e = round_reserve(B, (size_t)n_film, cap);
    if (e == cudaSuccess) e = reserve_pool(B, P0, 0);
    if (e != cudaSuccess) return e;
    WfState st = B.st;
    st.acc = acc;
    st.acc_w = acc_w;
    st.acc_sq = acc_sq;
    st.welford = nullptr;
    st.ssq = nullptr;
    st.part = nullptr;
    st.part_sq = nullptr;
    st.rsamp = B.rsamp;
    unsigned long long* taken = reinterpret_cast<unsigned long long*>(B.n_active + 2);
    const Grids g = pick_grids(sm_count);
    Events total;
    cudaEventRecord(total.e0, stream);
    wf::k_round_init<<<(n_film + 255) / 256, 256, 0, stream>>>(n_film, B.active[0], B.wstate, acc, acc_w, acc_sq);
    e = cudaMemsetAsync(B.n_active, 0, 256, stream);
    WfCounters sum{};
    int n_active = n_film, cur = 0, base = 0, rounds = 0;
    while (e == cudaSuccess && n_active > 0 && base < P0.spp) {
        int len = first_len;
        if (rounds > 0) {
            // as many samples as the buffer holds for every active pixel, whole tasks, and a task count that
            // fits the path state's 32-bit task ids
            long long fit = (long long)(cap / (size_t)n_active) / tspp * tspp;
            const long long id_fit = (0x7fffffffLL / n_active) * tspp;
            fit = std::min(fit, id_fit);
            len = (int)std::min<long long>(P0.spp - base, std::max<long long>(fit, tspp));
        }
        WfParams Pb = P0;
        Pb.adaptive = 0;  // the stopping rule runs in k_round_merge
        Pb.n_pixels = n_active;
        wf_set_divisors(Pb);
        Pb.px_map = B.active[cur];
        Pb.sample_base = base;
        Pb.sample_end = base + len;
        Pb.round_len = len;
        Pb.n_chunks = (len + tspp - 1) / tspp;
        Pb.n_tasks = (long long)n_active * Pb.n_chunks;
        Pb.task_first = 0;
        Pb.n_slots = (int)std::min<long long>(P0.n_slots, Pb.n_tasks);
        Pb.max_iters = (long long)tspp * (long long)(P0.max_bounces + 1) * ((Pb.n_tasks + Pb.n_slots - 1) / Pb.n_slots + 1) + 16;
        if (Pb.tail_live < 0) Pb.tail_live = std::min(262144, Pb.n_slots / 16);  // each round's drain
        cudaMemsetAsync(st.ctr, 0, sizeof(WfCounters), stream);
        wf::k_init<false><<<(Pb.n_slots + 255) / 256, 256, 0, stream>>>(S, Pb, st);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = wf_run_loop([&](cudaStream_t s, cudaGraphConditionalHandle h, int use_cond) {
                enqueue_iteration(S, Pb, st, g, s, h, use_cond);
            }, st.ctr, Pb.max_iters, stream, use_graph_loop);
        if (e == cudaSuccess && Pb.tail_live > 0) {
            wf::k_tail<false><<<(unsigned)((Pb.tail_live + 127) / 128), 128, 0, stream>>>(S, Pb, st);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemsetAsync(B.n_active, 0, sizeof(int), stream);
        if (e == cudaSuccess) {
            wf::k_round_merge<<<(n_active + 255) / 256, 256, 0, stream>>>(Pb, st, B.active[cur], n_active, B.wstate,
                                                                         B.active[cur ^ 1], B.n_active, taken);
            e = cudaGetLastError();
        }
        WfCounters part{};
        int next = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&part, st.ctr, sizeof(WfCounters), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&next, B.n_active, sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) break;
        add_counters(sum, part);
        n_active = next;
        cur ^= 1;
        base += len;
        ++rounds;
    }
    unsigned long long used = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&used, taken, sizeof(used), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return e;
    }
    cudaEventRecord(total.e1, stream);
    e = cudaEventSynchronize(total.e1);
    sum.samples = used;  // samples that joined the film; later samples of a round that stopped are dropped
    sum.pool_slots = P0.n_slots;
    *hc = sum;
    if (rounds_out) *rounds_out = rounds;
    if (e == cudaSuccess && ms) cudaEventElapsedTime(ms, total.e0, total.e1);
    return e;
}

}  // namespace tpt

// ---- allocation-free variant ---------------------------------------------------
// Some callers cannot allocate device memory while they render: a process
// that reserves the whole GPU for its own allocator at start-up, or one that
// cannot afford the device-wide synchronisation cudaMalloc/cudaFree imply in
// the middle of a frame loop.  wf_render_noalloc runs the same wavefront
// kernels with their path state and queues carved out of one file-scope
// device array instead of a cudaMalloc'd block, launches them directly (no
// graph or event objects are created) and allocates nothing.
//
// Limits: films of at most kNoAllocMaxSlots pixels.  Every call shares the
// array: calls that overlap on the GPU (other streams or host threads) race
// on it, and each call re-initialises the counters and path state it uses.
namespace tpt {
namespace {

constexpr size_t kNoAllocMaxSlots = 16384;  // e.g. 128 x 128

constexpr size_t na_align(size_t x) { return (x + 255) & ~(size_t)255; }
// Same arrays as wf_reserve, for kNoAllocMaxSlots slots.
constexpr size_t kNoAllocBytes =
    na_align(2 * kNoAllocMaxSlots * 4) + 6 * na_align(kNoAllocMaxSlots * 16) + 3 * na_align(2 * kNoAllocMaxSlots * 16) +
    na_align(kNoAllocMaxSlots * 16) + na_align(kNoAllocMaxSlots) + na_align(2 * kNoAllocMaxSlots * 4) +
    na_align(kNoAllocMaxSlots * 4) + na_align(sizeof(WfCounters)) + na_align(kNoAllocMaxSlots * 32) +
    2 * na_align(kNoAllocMaxSlots * 16) + na_align(5 * kNoAllocMaxSlots * 4) + na_align(64);

}  // namespace
}  // namespace tpt

// 5,128,704 bytes (about 5.1 MB), held by every GPU that loads the library
// until the process exits.
static_assert(tpt::kNoAllocBytes == 5128704, "the documented size of the allocation-free scratch array");
static __device__ __align__(256) unsigned char g_noalloc_scratch[tpt::kNoAllocBytes];

namespace tpt {
namespace {

std::mutex g_noalloc_mu;
void* g_noalloc_addr[256] = {};

// Device address of g_noalloc_scratch on the current device, looked up once
// per device (the host-side name of the array is not a device address).
cudaError_t noalloc_scratch(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return cudaSuccess;
}

}  // namespace

size_t wf_noalloc_max_slots() { return kNoAllocMaxSlots; }

cudaError_t wf_render_noalloc(const WfScene& S, const WfParams& P, double* acc, double* acc_w, cudaStream_t stream,
                              int sm_count, WfCounters* hc) {
    if (P.n_slots <= 0 || (size_t)P.n_slots > kNoAllocMaxSlots || P.n_chunks != 1 || P.n_tasks != P.n_slots)
        return cudaErrorInvalidValue;
    void* base = nullptr;
    cudaError_t e = noalloc_scratch(&base);
    if (e != cudaSuccess) return e;
    const size_t n = kNoAllocMaxSlots;
    char* p = static_cast<char*>(base);
    size_t off = 0;
    auto take = [&](size_t bytes) { char* r = p + off; off += na_align(bytes); return (void*)r; };
    WfState st{};
    st.q_ext[0] = (int*)take(2 * n * 4);
    st.q_ext[1] = st.q_ext[0] + n;
    st.path = (int4*)take(n * 16);
    st.ray_o = (float4*)take(n * 16);
    st.ray_d = (float4*)take(n * 16);
    st.beta = (float4*)take(n * 16);
    st.rad = (float4*)take(n * 16);
    st.hit = (float4*)take(n * 16);
    st.sh_o = (float4*)take(2 * n * 16);
    st.sh_d = (float4*)take(2 * n * 16);
    st.sh_c = (float4*)take(2 * n * 16);
    st.welford = P.adaptive ? (double2*)take(n * 16) : (take(n * 16), nullptr);
    st.act = (uint8_t*)take(n);
    st.q_sh = (int*)take(2 * n * 4);
    st.q_term = (int*)take(n * 4);
    st.ctr = (WfCounters*)take(sizeof(WfCounters));
    st.sacc = (double4*)take(n * 32);
    st.surf_p = (float4*)take(n * 16);
    st.surf_n = (float4*)take(n * 16);
    st.q_mat = (int*)take(5 * n * 4);
    st.cmp_counts = (int*)take(64);  // wf_compact_spans(16384) = 2 ints
    st.job = nullptr;  // single-scene renders only
    st.ssq = nullptr;
    st.part = nullptr;
    st.part_sq = nullptr;
    st.acc = acc;
    st.acc_w = acc_w;
    st.acc_sq = nullptr;
    const Grids g = pick_grids(sm_count);
    // The counters must start at zero; k_init initialises every slot it uses.
    e = cudaMemsetAsync(st.ctr, 0, sizeof(WfCounters), stream);
    if (e != cudaSuccess) return e;
    wf::k_init<false><<<(P.n_slots + 255) / 256, 256, 0, stream>>>(S, P, st);
    e = cudaGetLastError();
    long long iters = 0;
    while (e == cudaSuccess) {
        for (int k = 0; k < 8; ++k) {  // 8 x two iterations between host checks
            for (int cur = 0; cur < 2; ++cur) {
                launch_trace<false, false>(g.extend, stream, S, P, st, P.n_slots, P.trace_chunk, cur);
                launch_shade(g, stream, S, P, st, cur);
                launch_trace<true, false>(g.shadow, stream, S, P, st, P.n_slots, P.trace_chunk, cur);
                launch_regen(g.regen, stream, S, P, st, cur);
                if (P.ordered_queue) wf_launch_compact(stream, st, cur, P.n_slots);
                wf::k_step<<<1, 1, 0, stream>>>(st, cur, P.max_iters, cudaGraphConditionalHandle{}, 0);
            }
        }
        iters += 16;
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(hc, st.ctr, sizeof(WfCounters), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) break;
        if (hc->n_ext[0] == 0 && hc->n_ext[1] == 0) break;
        if ((hc->flags & TPT_FLAG_ITER_LIMIT) || iters > P.max_iters + 16) break;
    }
    return e;
}

}  // namespace tpt
