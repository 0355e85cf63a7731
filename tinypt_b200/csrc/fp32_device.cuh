// FP32 device routines shared by the wavefront kernels and the adjoint
// kernel: BVH2 traversal, ray-primitive tests, BSDFs, env-map and area-light
// sampling, the reference's f64 self-occlusion replay, and the camera ray.
// Each routine cites the reference function it restates.
#pragma once

#include "wavefront.cuh"

namespace tpt {
namespace wf {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTau = 6.28318530717958647692f;
constexpr float kEps = 1e-4f;          // RAY_EPSILON (src/constants.rs:4)
constexpr float kTMax = 1e30f;         // RAY_T_MAX (src/constants.rs:7)
constexpr int kStack = 64;        // local-memory traversal stack (deep trees)
constexpr int kSharedStack = 40;  // shared-memory traversal stack (default)
constexpr int kTraceBlock = 128;

// Traversal stack: element k at p[k * STRIDE] (STRIDE = block size for the
// shared-memory stack, so a warp's accesses fall in distinct banks).
template <int STRIDE, int CAP>
struct TStack {
    int* p;
    __device__ __forceinline__ int& operator[](int k) const { return p[k * STRIDE]; }
    static constexpr int capacity = CAP;
};

// meta.z flags
constexpr int F_LAST_ND = 1;           // last BSDF sample was non-delta
constexpr int F_PEND_ENV = 2;          // shadow record 0 pending
constexpr int F_PEND_AREA = 4;         // shadow record 1 pending
constexpr int F_DONE = 8;              // pixel finished all samples

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// Path-state records are read and written once per iteration: streaming
// (evict-first) accesses keep them from pushing the BVH nodes and triangles
// out of L2.  (lds returns a const value, so a misplaced assignment to it
// does not compile.)
template <class T>
__device__ __forceinline__ const T lds(const T* p) { return __ldcs(p); }
// (an overload, not a specialisation: a const scalar return means nothing)
__device__ __forceinline__ uint64_t lds(const uint64_t* p) {
    return (uint64_t)__ldcs(reinterpret_cast<const unsigned long long*>(p));
}
template <>
__device__ __forceinline__ const double4 lds(const double4* p) {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p)), b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
template <class T>
__device__ __forceinline__ void sts(T* p, const T& v) { __stcs(p, v); }
template <>
__device__ __forceinline__ void sts(uint64_t* p, const uint64_t& v) {
    __stcs(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}
template <>
__device__ __forceinline__ void sts(double4* p, const double4& v) {
    __stcs(reinterpret_cast<double2*>(p), make_double2(v.x, v.y));
    __stcs(reinterpret_cast<double2*>(p) + 1, make_double2(v.z, v.w));
}

// The path record in registers: m = {samples done, bounce, flags, task}
// and the PCG32 state; in memory one 16-byte record (WfState::path).
__device__ __forceinline__ void load_path(const WfState& st, int slot, int4& m, uint64_t& rng) {
    const int4 v = lds(&st.path[slot]);
    rng = ((uint64_t)(uint32_t)v.y << 32) | (uint64_t)(uint32_t)v.x;
    const uint32_t w = (uint32_t)v.w;
    m = make_int4((int)(w & ((1u << kPathDoneBits) - 1u)),
                  (int)((w >> kPathDoneBits) & ((1u << kPathBounceBits) - 1u)),
                  (int)(w >> (kPathDoneBits + kPathBounceBits)), v.z);
}
__device__ __forceinline__ void store_path(const WfState& st, int slot, const int4& m, uint64_t rng) {
    const uint32_t w = (uint32_t)m.x | ((uint32_t)m.y << kPathDoneBits) |
                       ((uint32_t)m.z << (kPathDoneBits + kPathBounceBits));
    sts(&st.path[slot], make_int4((int)(uint32_t)rng, (int)(uint32_t)(rng >> 32), m.w, (int)w));
}

// Which slots an iteration's kernels visit.  While more than 1/div of the
// pool is live (div = WfParams::queue_div, default 8) they sweep every slot
// in slot order and skip dead ones by their act byte: consecutive lanes read
// consecutive slots' records.  Below that they take the compacted extension
// queue, so the long tail of a frame -- dozens of iterations with few live
// paths -- does not pay for sweeping (and fetching, one atomic per 32 slots)
// the whole pool each time.  (The queue alone is slower while the pool is
// full: its order scrambles over the iterations and the record accesses
// stop coalescing.)
__device__ __forceinline__ bool use_ext_queue(int live, int n_slots, int div) {
    return (long long)live * div <= n_slots;
}

// Appends `pred` lanes to a queue with one atomic per warp.  Must be called
// by every lane of a converged warp.
__device__ __forceinline__ void warp_push(int* __restrict__ q, int* counter, bool pred, int value) {
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (mask == 0) return;
    const int leader = __ffs(mask) - 1;
    int base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) q[base + __popc(mask & ((1u << lane_id()) - 1u))] = value;
}

// Three-input minimum / maximum (one instruction on sm_100a).  Exact, like
// fminf/fmaxf, so a slab test written with them takes the same decisions.
__device__ __forceinline__ float fmin3f(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float fmax3f(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

__device__ __forceinline__ float3 safe_inv(float3 d) {
    const float e = 1e-20f;
    return f3(1.0f / (fabsf(d.x) > e ? d.x : copysignf(e, d.x)), 1.0f / (fabsf(d.y) > e ? d.y : copysignf(e, d.y)),
              1.0f / (fabsf(d.z) > e ? d.z : copysignf(e, d.z)));
}

// ---- traversal ------------------------------------------------------------
struct TraceHit { float t; int prim; int inst; };
// Work counters of the profiling variant of the trace kernels.
struct TraceCount {
    uint32_t nodes = 0, tris = 0, spheres = 0, inst = 0, node_steps = 0;
    uint32_t leaves = 0, leaf_steps = 0;  // leaf / instance / exit visits, and the warp-wide steps they took
    uint32_t fast_steps = 0;              // warp-wide steps of the camera-miss fast path
};

// Counts one warp-wide step of the code this is placed in: the lowest lane
// that takes it adds one.
__device__ __forceinline__ void count_step(uint32_t& steps) {
    const unsigned am = __activemask();
    if ((int)(threadIdx.x & 31u) == __ffs(am) - 1) steps++;
}

__device__ __forceinline__ bool tri_test(const TriF32* __restrict__ tris, uint32_t k, float3 o, float3 d, float tmin,
                                         float tmax, float& t_out) {
    const float4* tp = reinterpret_cast<const float4*>(tris + k);
    const float4 v0 = __ldg(tp), e1 = __ldg(tp + 1), e2 = __ldg(tp + 2);
    const float3 E1 = f3(e1), E2 = f3(e2);
    const float3 pvec = cross(d, E2);
    const float det = dot(E1, pvec);
    if (fabsf(det) < 1e-10f) return false;
    const float inv = 1.0f / det;
    const float3 tvec = o - f3(v0);
    const float u = dot(tvec, pvec) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    const float3 qvec = cross(tvec, E1);
    const float v = dot(d, qvec) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    const float t = dot(E2, qvec) * inv;
    if (t < tmin || t > tmax) return false;
    t_out = t;
    return true;
}

// Ray-sphere (src/geometry.rs:174-195) in the numerically robust form:
// the discriminant is r^2 - |f - (f.d)d|^2 and the near root is c/q.  A ray
// that starts on this sphere (self) cannot hit it again going outward and
// only hits the far side going inward; the reference gets the same outcome
// from its f64 epsilon offsets.
__device__ __forceinline__ bool sphere_test(float4 cr, float3 o, float3 d, float tmin, float tmax, bool self,
                                            float& t_out) {
    const float3 f = o - f3(cr);
    const float a = dot(d, d);
    const float b = dot(f, d);
    const float3 l = f - d * (b / a);
    const float r2 = cr.w * cr.w;
    const float disc = a * (r2 - dot(l, l));
    if (disc <= 0.0f) return false;
    const float sq = sqrtf(disc);
    if (self) {
        if (b >= 0.0f) return false;
        const float t = (-b + sq) / a;
        if (t < tmin || t > tmax) return false;
        t_out = t;
        return true;
    }
    const float c = dot(f, f) - r2;
    const float q = -(b + copysignf(sq, b));
    float t0 = c / q, t1 = q / a;
    if (t0 > t1) { float tmp = t0; t0 = t1; t1 = tmp; }
    float t = t0;
    if (t < tmin || t > tmax) {
        t = t1;
        if (t < tmin || t > tmax) return false;
    }
    t_out = t;
    return true;
}

// Top-level walk (src/world.rs:81-121 World::hit, src/bvh.rs:248-351
// Bvh::hit).  One child-pair BVH2 walk covers the world: the top-level
// tree over spheres and instances, and below each instance leaf that
// instance's mesh tree, entered by taking the ray to object space (the
// direction is not renormalised, so t stays the world t) and pushing an
// exit marker that restores the world ray when popped.  Near child first,
// like src/bvh.rs:321-346.
constexpr int32_t kRefExit = ~0;          // leaf code 0/0: leave the current instance
constexpr int32_t kRefExitIdentity = ~8;  // leaf code 1/0: leave an identity instance (the ray is the world ray)

struct Tracer {
    float3 wo, wd;       // world-space ray
    float3 o, d, idir;   // ray in the current space
    float tmax;
    int ref, sp, inst;   // next node, stack size, entered instance (-1 = world)
    int self_prim, self_inst;
    int hit_prim, hit_inst;
};

// root = the top-level tree to walk (S.top_root, or a batch job's root).
__device__ __forceinline__ void tracer_start_at(int root, Tracer& T, float3 o, float3 d, float tmax, int self_prim,
                                                int self_inst) {
    T.wo = o; T.wd = d;
    T.o = o; T.d = d; T.idir = safe_inv(d);
    T.tmax = tmax;
    T.ref = root; T.sp = 0; T.inst = -1;
    T.self_prim = self_prim; T.self_inst = self_inst;
    T.hit_prim = -1; T.hit_inst = -1;
}
__device__ __forceinline__ void tracer_start(const WfScene& S, Tracer& T, float3 o, float3 d, float tmax, int self_prim,
                                             int self_inst) {
    T.wo = o; T.wd = d;
    T.o = o; T.d = d; T.idir = safe_inv(d);
    T.tmax = tmax;
    T.ref = S.top_root; T.sp = 0; T.inst = -1;
    T.self_prim = self_prim; T.self_inst = self_inst;
    T.hit_prim = -1; T.hit_inst = -1;
}

template <class Stack>
__device__ __forceinline__ void tracer_pop(Tracer& T, const Stack& stack) {
    T.ref = T.sp > 0 ? stack[--T.sp] : TPT_REF_NONE;
}

// Runs up to `chunk` leaf visits of one ray.  Returns true when the ray is
// finished: stack exhausted, or (ANY) an occluder found.
template <bool ANY, bool COUNT, class Stack>
__device__ __forceinline__ bool tracer_run(const WfScene& S, Tracer& T, const Stack& stack, float tmin, int chunk, int* flags,
                                           TraceCount& cnt) {
    for (int it = 0; it < chunk; ++it) {
        const float3 ood = f3(T.o.x * T.idir.x, T.o.y * T.idir.y, T.o.z * T.idir.z);
        while (T.ref >= 0) {
            if (COUNT) {
                cnt.nodes++;
                count_step(cnt.node_steps);
            }
            const float4* np = reinterpret_cast<const float4*>(S.nodes + T.ref);
            const float4 lx = __ldg(np), rx = __ldg(np + 1), zz = __ldg(np + 2);
            const int4 rf = __ldg(reinterpret_cast<const int4*>(np + 3));
            const float3 idir = T.idir;
            // slab distances (box - o) * idir as one explicit FMA each: the
            // unit is compiled without automatic contraction, so results
            // do not depend on how a kernel instantiation is scheduled
            const float a0 = __fmaf_rn(lx.x, idir.x, -ood.x), a1 = __fmaf_rn(lx.y, idir.x, -ood.x);
            const float a2 = __fmaf_rn(lx.z, idir.y, -ood.y), a3 = __fmaf_rn(lx.w, idir.y, -ood.y);
            const float a4 = __fmaf_rn(zz.x, idir.z, -ood.z), a5 = __fmaf_rn(zz.y, idir.z, -ood.z);
            const float b0 = __fmaf_rn(rx.x, idir.x, -ood.x), b1 = __fmaf_rn(rx.y, idir.x, -ood.x);
            const float b2 = __fmaf_rn(rx.z, idir.y, -ood.y), b3 = __fmaf_rn(rx.w, idir.y, -ood.y);
            const float b4 = __fmaf_rn(zz.z, idir.z, -ood.z), b5 = __fmaf_rn(zz.w, idir.z, -ood.z);
            const float ln = fmax3f(fminf(a0, a1), fminf(a2, a3), fmaxf(fminf(a4, a5), tmin));
            const float lf = fmin3f(fmaxf(a0, a1), fmaxf(a2, a3), fminf(fmaxf(a4, a5), T.tmax));
            const float rn = fmax3f(fminf(b0, b1), fminf(b2, b3), fmaxf(fminf(b4, b5), tmin));
            const float rfar = fmin3f(fmaxf(b0, b1), fmaxf(b2, b3), fminf(fmaxf(b4, b5), T.tmax));
            // every child of an interior node is a node or a leaf (emit_bvh2)
            const bool hl = ln <= lf;
            const bool hr = rn <= rfar;
            if (hl && hr) {
                int near = rf.x, far = rf.y;
                if (rn < ln) { near = rf.y; far = rf.x; }
                if (T.sp < Stack::capacity) stack[T.sp++] = far;
                else raise_flag(flags, TPT_FLAG_STACK_OVERFLOW);
                T.ref = near;
            } else if (hl) {
                T.ref = rf.x;
            } else if (hr) {
                T.ref = rf.y;
            } else {
                tracer_pop(T, stack);
            }
        }
        if (T.ref == TPT_REF_NONE) return true;
        if (COUNT) {
            cnt.leaves++;
            count_step(cnt.leaf_steps);
        }
        if (T.ref == kRefExit || T.ref == kRefExitIdentity) {  // back to world space
            if (T.ref == kRefExit) { T.o = T.wo; T.d = T.wd; T.idir = safe_inv(T.wd); }
            T.inst = -1;
            tracer_pop(T, stack);
            continue;
        }
        const uint32_t code = (uint32_t)(~T.ref);
        const uint32_t first = code >> 3, count = code & 7u;
        if (count == 7u) {  // instance leaf: enter its mesh tree
            if (COUNT) cnt.inst++;
            const InstanceF32* I = S.inst + first;
            const int mw = fbits(__ldg(&I->wbox_min.w));
            const int root = __ldg(&S.meshes[mw & kInstMeshMask].root_ref);
            if (root != TPT_REF_NONE && T.sp < Stack::capacity && (mw & kInstIdentity)) {
                // identity transform: the object-space ray is the world ray (up to the sign of zeros)
                T.inst = (int)first;
                stack[T.sp++] = kRefExitIdentity;
                T.ref = root;
            } else if (root != TPT_REF_NONE && T.sp < Stack::capacity) {
                const float4 r0 = __ldg(&I->w2o[0]), r1 = __ldg(&I->w2o[1]), r2 = __ldg(&I->w2o[2]);
                const float3 wo = T.wo, wd = T.wd;
                T.o = f3(r0.x * wo.x + r0.y * wo.y + r0.z * wo.z + r0.w, r1.x * wo.x + r1.y * wo.y + r1.z * wo.z + r1.w,
                         r2.x * wo.x + r2.y * wo.y + r2.z * wo.z + r2.w);
                T.d = f3(r0.x * wd.x + r0.y * wd.y + r0.z * wd.z, r1.x * wd.x + r1.y * wd.y + r1.z * wd.z,
                         r2.x * wd.x + r2.y * wd.y + r2.z * wd.z);
                T.idir = safe_inv(T.d);
                T.inst = (int)first;
                stack[T.sp++] = kRefExit;
                T.ref = root;
            } else {
                if (root != TPT_REF_NONE) raise_flag(flags, TPT_FLAG_STACK_OVERFLOW);
                tracer_pop(T, stack);
            }
            continue;
        }
        bool stop = false;
        if (T.inst >= 0) {  // triangles of the entered mesh
            const uint32_t self_tri = (T.self_inst == T.inst && T.self_prim >= S.n_spheres)
                                          ? (uint32_t)(T.self_prim - S.n_spheres) : 0xffffffffu;
            for (uint32_t k = first; k < first + count; ++k) {
                if (k == self_tri) continue;
                if (COUNT) cnt.tris++;
                float t;
                if (tri_test(S.tris, k, T.o, T.d, tmin, T.tmax, t)) {
                    T.tmax = t;
                    T.hit_prim = S.n_spheres + (int)k;
                    T.hit_inst = T.inst;
                    if (ANY) { stop = true; break; }
                }
            }
        } else {  // spheres (world space)
            const int self_sphere = T.self_inst < 0 ? T.self_prim : -1;
            for (uint32_t k = first; k < first + count; ++k) {
                if (COUNT) cnt.spheres++;
                const float4 cr = __ldg(&S.spheres[k].cr);
                float t;
                if (sphere_test(cr, T.o, T.d, tmin, T.tmax, (int)k == self_sphere, t)) {
                    T.tmax = t;
                    T.hit_prim = (int)k;
                    T.hit_inst = -1;
                    if (ANY) { stop = true; break; }
                }
            }
        }
        if (stop) return true;
        tracer_pop(T, stack);
    }
    return false;
}

// ---- shading helpers (src/material.rs, src/env.rs, src/world.rs) ------------
__device__ __forceinline__ float mis(float a, float b) {  // integrator.rs:221-225
    const float a2 = a * a, b2 = b * b;
    return (a2 + b2 > 0.0f) ? a2 / (a2 + b2) : 0.0f;
}
__device__ __forceinline__ float3 clamp_lum(float3 c, float m) {  // math.rs:42-49
    const float l = luminance(c);
    return (l > m && l > 0.0f) ? c * (m / l) : c;
}
__device__ __forceinline__ float pow5(float x) { const float x2 = x * x; return x2 * x2 * x; }
__device__ __forceinline__ float3 fresnel_schlick(float c, float3 f0) {
    const float x = 1.0f - fmaxf(c, 0.0f);
    return f0 + (f3(1.0f, 1.0f, 1.0f) - f0) * pow5(x);
}
__device__ __forceinline__ float ggx_d(float alpha, float ch) {
    if (ch <= 0.0f) return 0.0f;
    const float a2 = alpha * alpha;
    const float den = ch * ch * (a2 - 1.0f) + 1.0f;
    return a2 / (kPi * den * den);
}
__device__ __forceinline__ float ggx_g1(float alpha, float c) {
    if (c <= 0.0f) return 0.0f;
    const float a = alpha * sqrtf(fmaxf(1.0f - c * c, 0.0f)) / fmaxf(c, 1e-6f);
    return 2.0f / (1.0f + sqrtf(1.0f + a * a));
}
static __device__ float3 ggx_eval(float3 albedo, float alpha, float3 n, float3 wo, float3 wi) {
    const float ci = dot(n, wo), co = dot(n, wi);
    if (ci <= 0.0f || co <= 0.0f) return f3(0, 0, 0);
    const float3 m = normalize(wo + wi);
    const float ch = fmaxf(dot(n, m), 0.0f);
    const float g = ggx_g1(alpha, ci) * ggx_g1(alpha, co);
    const float3 f = fresnel_schlick(fabsf(dot(wi, m)), albedo);
    return f * (ggx_d(alpha, ch) * g / (4.0f * ci * co + 1e-6f));
}
static __device__ float ggx_pdf(float alpha, float3 n, float3 wo, float3 wi) {
    const float ci = dot(n, wo), co = dot(n, wi);
    if (ci <= 0.0f || co <= 0.0f) return 0.0f;
    const float3 m = normalize(wo + wi);
    const float ch = fmaxf(dot(n, m), 0.0f);
    const float pdf_m = ggx_d(alpha, ch) * ggx_g1(alpha, ci) * ch / fmaxf(ci, 1e-6f);
    return fmaxf(pdf_m / (4.0f * fmaxf(fabsf(dot(wi, m)), 1e-6f)), 0.0f);
}
__device__ __forceinline__ void tangent_frame(float3 n, float3& t, float3& b) {
    const float3 a = fabsf(n.x) > 0.9f ? f3(0, 1, 0) : f3(1, 0, 0);
    t = normalize(cross(n, a));
    b = cross(t, n);
}
__device__ __forceinline__ float3 cos_hemi(float3 n, uint64_t& rng) {
    const float u = pcg_f32(rng), v = pcg_f32(rng);
    const float r = sqrtf(u);
    float s, c;
    __sincosf(kTau * v, &s, &c);
    float3 t, b;
    tangent_frame(n, t, b);
    return t * (r * c) + b * (r * s) + n * sqrtf(1.0f - u);
}
static __device__ float3 vndf(float3 wo, float alpha, float u1, float u2) {
    const float3 v = normalize(f3(alpha * wo.x, alpha * wo.y, wo.z));
    float3 t1, t2;
    if (v.z < 0.9999f) { t1 = normalize(f3(-v.y, v.x, 0.0f)); t2 = cross(v, t1); }
    else { t1 = f3(1, 0, 0); t2 = f3(0, 1, 0); }
    const float r = sqrtf(u1);
    float sp, cp;
    __sincosf(kTau * u2, &sp, &cp);
    const float t1p = r * cp;
    const float s = 0.5f * (1.0f + v.z);
    const float t2p = sqrtf(1.0f - s) * (r * sp) + s * sqrtf(fmaxf(1.0f - t1p * t1p, 0.0f));
    const float3 nh = normalize(t1 * t1p + t2 * t2p + v * sqrtf(fmaxf(1.0f - t1p * t1p - t2p * t2p, 0.0f)));
    return normalize(f3(alpha * nh.x, alpha * nh.y, nh.z));
}

// Material::eval (src/material.rs:207-223).  The BSDF value takes the
// material's own parameters; the pdf (used only in MIS weights) takes the
// sampler's GGX alpha, which differs only when sampling is detached.
__device__ __forceinline__ void mat_eval(const MaterialF32& mt, float3 wo, float3 wi, float3 n, float3& f, float& pdf) {
    if (mt.kind == TPT_MAT_LAMBERT || mt.kind == TPT_MAT_SUBSURFACE) {
        const float c = fmaxf(dot(n, wi), 0.0f);
        if (c <= 0.0f) { f = f3(0, 0, 0); pdf = 0.0f; return; }
        f = f3(mt.c) * (1.0f / kPi);
        pdf = c / kPi;
    } else if (mt.kind == TPT_MAT_GGX) {
        f = ggx_eval(f3(mt.c), fmaxf(mt.c.w, 1e-3f), n, wo, wi);
        pdf = ggx_pdf(fmaxf(mt.s_param, 1e-3f), n, wo, wi);
    } else {
        f = f3(0, 0, 0);
        pdf = 0.0f;
    }
}

// The Ggx arm of Material::sample (src/material.rs:140-173): VNDF sample of
// the microfacet normal with the sampler's alpha, weight f*cos/pdf with the
// BSDF at the material's alpha and the pdf at the sampler's.
struct GgxSample {
    float3 nd, mh;       // scattered direction, microfacet normal
    float ci, co, ch;    // n.wo, n.nd, n.mh
    float3 w;            // throughput weight
    float pdf;
};
__device__ __forceinline__ bool ggx_sample(float3 rd, float3 n, const MaterialF32& mt, uint64_t& rng, GgxSample& g) {
    const float av = fmaxf(mt.c.w, 1e-3f), as = fmaxf(mt.s_param, 1e-3f);
    const float3 wo = -rd;
    float3 t, b;
    tangent_frame(n, t, b);
    const float3 wl = f3(dot(wo, t), dot(wo, b), dot(wo, n));
    if (wl.z <= 0.0f) return false;
    const float u1 = pcg_f32(rng), u2 = pcg_f32(rng);
    const float3 ml = vndf(wl, as, u1, u2);
    g.mh = t * ml.x + b * ml.y + n * ml.z;
    g.nd = rd - g.mh * (2.0f * dot(rd, g.mh));
    g.co = dot(g.nd, n);
    g.ci = dot(wo, n);
    if (g.co <= 1e-6f || g.ci <= 1e-6f) return false;
    g.ch = fmaxf(dot(n, g.mh), 0.0f);
    const float gg = ggx_g1(av, g.ci) * ggx_g1(av, g.co);
    const float3 fr = fresnel_schlick(fabsf(dot(g.nd, g.mh)), f3(mt.c));
    const float3 spec = fr * (ggx_d(av, g.ch) * gg / (4.0f * g.ci * g.co + 1e-6f));
    g.pdf = ggx_pdf(as, n, wo, g.nd);
    g.w = spec * (g.co / fmaxf(g.pdf, 1e-6f));
    return true;
}

// Env map (src/env.rs:92-210); texel .w holds the nearest-texel pdf_uv.
__device__ __forceinline__ void dir_uv(float3 d, float& u, float& v, float& theta) {
    const float3 n = normalize(d);
    theta = acosf(fminf(fmaxf(n.y, -1.0f), 1.0f));
    float phi = atan2f(n.z, n.x);
    if (phi < 0.0f) phi += kTau;
    u = phi / kTau;
    v = theta / kPi;
}
static __device__ float3 env_lookup(const WfScene& S, float3 d) {
    float u, v, theta;
    dir_uv(d, u, v, theta);
    const int W = S.env_w, H = S.env_h;
    const float x = u * (float)W, y = v * ((float)H - 1.0f);
    const float fxf = floorf(x);
    int x0 = (int)fxf % W;
    if (x0 < 0) x0 = 0;
    const int x1 = (x0 + 1) % W;
    int y0 = (int)floorf(fminf(fmaxf(y, 0.0f), (float)(H - 1)));
    const int y1 = min(y0 + 1, H - 1);
    const float fx = x - fxf, fy = y - floorf(y);
    const float3 c00 = f3(__ldg(S.env_tex + y0 * W + x0)), c10 = f3(__ldg(S.env_tex + y0 * W + x1));
    const float3 c01 = f3(__ldg(S.env_tex + y1 * W + x0)), c11 = f3(__ldg(S.env_tex + y1 * W + x1));
    const float3 c0 = c00 * (1.0f - fx) + c10 * fx;
    const float3 c1 = c01 * (1.0f - fx) + c11 * fx;
    return c0 * (1.0f - fy) + c1 * fy;
}
// What a ray that leaves the scene sees (src/integrator.rs:71-83): the env
// map, or without one the sky gradient (:25-28).
__device__ __forceinline__ float3 background(const WfScene& S, float3 rd) {
    if (S.env_kind == TPT_ENV_MAP) return env_lookup(S, rd);
    const float t = 0.5f * (rd.y + 1.0f);
    return f3(0.9f, 0.95f, 1.0f) * (1.0f - t) + f3(0.6f, 0.75f, 1.0f) * t;
}
static __device__ float env_pdf(const WfScene& S, float3 d) {
    if (!S.env_has_cdf) return 1.0f / (4.0f * kPi);
    float u, v, theta;
    dir_uv(d, u, v, theta);
    const int W = S.env_w, H = S.env_h;
    const int x = (int)fminf(fmaxf(floorf(u * (float)W), 0.0f), (float)(W - 1));
    const int y = (int)fminf(fmaxf(floorf(v * (float)H), 0.0f), (float)(H - 1));
    const float pdf_uv = __ldg(&S.env_tex[y * W + x].w);
    if (pdf_uv <= 0.0f) return 0.0f;
    return pdf_uv / (2.0f * kPi * kPi * fmaxf(sinf(theta), 1e-6f));
}
// Largest index lo in [0, n-2] with cdf[lo] <= x (src/env.rs:185-197).
__device__ __forceinline__ int cdf_search(const float* __restrict__ cdf, int n, float x) {
    int lo = 0, hi = n > 0 ? n - 1 : 0;
    while (lo + 1 < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) <= x) lo = mid; else hi = mid;
    }
    return lo;
}
static __device__ void env_uniform(const WfScene& S, uint64_t& rng, float3& dir, float3& rad, float& pdf) {
    const float u = pcg_f32(rng), v = pcg_f32(rng);
    const float z = 1.0f - 2.0f * u;
    const float r = sqrtf(fmaxf(1.0f - z * z, 0.0f));
    float s, c;
    __sincosf(kTau * v, &s, &c);
    dir = f3(r * c, z, r * s);
    rad = env_lookup(S, dir);
    pdf = 1.0f / (4.0f * kPi);
}
static __device__ void env_sample_dir(const WfScene& S, uint64_t& rng, float3& dir, float3& rad, float& pdf) {
    if (!S.env_has_cdf) { env_uniform(S, rng, dir, rad, pdf); return; }
    const int W = S.env_w, H = S.env_h;
    const float r0 = pcg_f32(rng);
    const int y = min(cdf_search(S.env_row, H + 1, r0), H - 1);
    if (__ldg(S.env_row + y + 1) - __ldg(S.env_row + y) <= 0.0f) { env_uniform(S, rng, dir, rad, pdf); return; }
    const float r1 = pcg_f32(rng);
    const int x = min(cdf_search(S.env_col + (size_t)y * (W + 1), W + 1, r1), W - 1);
    const float u = ((float)x + pcg_f32(rng)) / (float)W;
    const float v = ((float)y + pcg_f32(rng)) / (float)H;
    float st, ct, sp, cp;
    sincosf(kPi * v, &st, &ct);
    sincosf(kTau * u, &sp, &cp);
    dir = f3(cp * st, ct, sp * st);
    rad = env_lookup(S, dir);
    pdf = env_pdf(S, dir);
}

// World::sample_light (src/world.rs:171-209) with the reference's CDF quirk:
// the CDF has no leading zero, so the search never returns the last light.
// The surface variates u, v are also returned at full 53-bit precision
// (ud, vd) for the f64 self-occlusion test below.
static __device__ bool sample_light(const WfScene& S, uint64_t& rng, float3 p, float3& pos, float3& emit, float& pdf,
                             int& idx, double& ud, double& vd) {
    if (S.n_lights == 0) return false;
    const float r = pcg_f32(rng);
    idx = min(cdf_search(S.light_cdf, S.n_lights, r), S.n_lights - 1);
    const LightF32* L = S.lights + idx;
    const float4 e = __ldg(&L->emit);
    const float4 p0 = __ldg(&L->p0);
    float3 nrm;
    float area;
    ud = pcg_f64(rng);
    vd = pcg_f64(rng);
    const float u = (float)ud, v = (float)vd;
    if (__ldg(&L->is_sphere)) {
        const float z = 1.0f - 2.0f * u;
        const float rr = sqrtf(fmaxf(1.0f - z * z, 0.0f));
        float s, c;
        __sincosf(kTau * v, &s, &c);
        const float3 dir = f3(rr * c, z, rr * s);
        pos = f3(p0) + dir * p0.w;
        nrm = dir;
        area = 4.0f * kPi * p0.w * p0.w;
    } else {
        const float3 w0 = f3(p0), w1 = f3(__ldg(&L->p1)), w2 = f3(__ldg(&L->p2));
        const float su = sqrtf(u);
        const float b0 = 1.0f - su, b1 = v * su;
        pos = w0 * b0 + w1 * b1 + w2 * (1.0f - b0 - b1);
        const float3 nn = cross(w1 - w0, w2 - w0);
        area = 0.5f * length(nn);
        nrm = area > 0.0f ? nn / (2.0f * area) : f3(0, 1, 0);
    }
    if (area <= 0.0f) return false;
    const float3 tl = pos - p;
    const float d2 = dot(tl, tl);
    if (d2 <= 1e-12f) return false;
    const float dist = sqrtf(d2);
    const float cl = fmaxf(-dot(nrm, tl) / dist, 0.0f);
    if (cl <= 0.0f) return false;
    pdf = e.w * (d2 / (area * cl));
    if (!(pdf > 0.0f)) return false;
    emit = f3(e);
    return true;
}

// ---- the reference's self-occlusion of area-light shadow rays -------------------
// nee_area_light (src/integrator.rs:178-213) traces the shadow ray from
// hit_p + 1e-4 wi with tmax = dist - 1e-4, which is also the distance from
// that origin to the sampled light point.  Whether World::hit reports the
// light's own primitive (instances: t_world < tmax, src/world.rs:104; spheres:
// t <= tmax, src/geometry.rs:183-189) is therefore decided by f64 rounding;
// in the reference about a quarter of otherwise unobstructed samples are
// lost this way.  The FP32 shadow ray excludes the sampled light, and this
// function replays the reference's f64 test on that one primitive, with
// explicitly rounded operations (no FMA contraction), to reproduce the loss.
namespace ref64 {
struct D3 { double x, y, z; };
__device__ __forceinline__ D3 add(D3 a, D3 b) { return {__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y), __dadd_rn(a.z, b.z)}; }
__device__ __forceinline__ D3 sub(D3 a, D3 b) { return {__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z)}; }
__device__ __forceinline__ D3 mul(D3 a, double s) { return {__dmul_rn(a.x, s), __dmul_rn(a.y, s), __dmul_rn(a.z, s)}; }
__device__ __forceinline__ D3 dv(D3 a, double s) { return {__ddiv_rn(a.x, s), __ddiv_rn(a.y, s), __ddiv_rn(a.z, s)}; }
__device__ __forceinline__ double dot(D3 a, D3 b) {
    return __dadd_rn(__dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dmul_rn(a.z, b.z));
}
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
    return {__dsub_rn(__dmul_rn(a.y, b.z), __dmul_rn(a.z, b.y)), __dsub_rn(__dmul_rn(a.z, b.x), __dmul_rn(a.x, b.z)),
            __dsub_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x))};
}
__device__ __forceinline__ D3 norm(D3 a) { return dv(a, fmax(__dsqrt_rn(dot(a, a)), 1e-30)); }
__device__ __forceinline__ D3 mv(const double* m, D3 v) {
    return {__dadd_rn(__dadd_rn(__dmul_rn(m[0], v.x), __dmul_rn(m[1], v.y)), __dmul_rn(m[2], v.z)),
            __dadd_rn(__dadd_rn(__dmul_rn(m[3], v.x), __dmul_rn(m[4], v.y)), __dmul_rn(m[5], v.z)),
            __dadd_rn(__dadd_rn(__dmul_rn(m[6], v.x), __dmul_rn(m[7], v.y)), __dmul_rn(m[8], v.z))};
}
__device__ __forceinline__ D3 ld(const double* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ D3 lerp_static(D3 v, double t) {  // Triangle::vertices_at (geometry.rs:212-218)
    return add(mul(v, __dsub_rn(1.0, t)), mul(v, t));
}
}  // namespace ref64

// The hit point is taken as the reference forms it, o + t * d rounded in
// f64 (src/ray.rs `Ray::at`), from the FP32 ray and distance: a point whose
// low-order bits carry that rounding, like the reference's f64 hit points.
// Rounding the FP32 hit point instead (its low 29 bits zero) made the coin
// below land on the "occluded" side less often than in the reference:
// +2.5% direct light on the sphere scene.
// The scene's f64 arrays come by value: a reference to the whole WfScene
// would make every caller keep its scene view in addressable local memory.
static __device__ __noinline__ bool ref_light_self_occluded(const LightF64* __restrict__ lights64,
                                                            const SphereF64* __restrict__ spheres64,
                                                            const InstanceF64* __restrict__ inst64, int idx, float3 ro,
                                                            float3 rd, float t_hit, double ud, double vd, double time) {
    using namespace ref64;
    const LightF64& L = lights64[idx];
    const double t = (double)t_hit;
    const D3 hp{__dadd_rn((double)ro.x, __dmul_rn(t, (double)rd.x)), __dadd_rn((double)ro.y, __dmul_rn(t, (double)rd.y)),
                __dadd_rn((double)ro.z, __dmul_rn(t, (double)rd.z))};
    D3 pos;
    D3 w0, w1, w2;
    const InstanceF64* inst = nullptr;
    if (L.is_sphere) {  // Light::sample_surface, sphere (world.rs:244-254)
        const SphereF64& s = spheres64[L.sphere];
        const double z = __dsub_rn(1.0, __dmul_rn(2.0, ud));
        const double rr = __dsqrt_rn(fmax(__dsub_rn(1.0, __dmul_rn(z, z)), 0.0));
        const double phi = __dmul_rn(6.28318530717958647692528676655900577, vd);
        const D3 dir{__dmul_rn(rr, cos(phi)), z, __dmul_rn(rr, sin(phi))};
        pos = add(ld(s.c), mul(dir, s.r));
    } else {  // tri_world_verts + Light::sample_surface, triangle (world.rs:256-270)
        inst = inst64 + L.inst;
        w0 = add(mv(inst->a, lerp_static(ld(L.v), time)), ld(inst->t));
        w1 = add(mv(inst->a, lerp_static(ld(L.v + 3), time)), ld(inst->t));
        w2 = add(mv(inst->a, lerp_static(ld(L.v + 6), time)), ld(inst->t));
        const double su = __dsqrt_rn(ud);
        const double b0 = __dsub_rn(1.0, su), b1 = __dmul_rn(vd, su);
        const double b2 = __dsub_rn(__dsub_rn(1.0, b0), b1);
        pos = add(add(mul(w0, b0), mul(w1, b1)), mul(w2, b2));
    }
    const D3 tl = sub(pos, hp);
    const double dist = __dsqrt_rn(dot(tl, tl));
    const D3 wi = dv(tl, dist);
    const D3 o = add(hp, mul(wi, 1e-4));
    const double tmin = 1e-4, tmax = fmax(__dsub_rn(dist, 1e-4), 1e-4);
    if (L.is_sphere) {  // Sphere::hit (geometry.rs:174-195)
        const SphereF64& s = spheres64[L.sphere];
        const D3 oc = sub(o, ld(s.c));
        const double a = dot(wi, wi), b = dot(oc, wi);
        const double c = __dsub_rn(dot(oc, oc), __dmul_rn(s.r, s.r));
        const double d = __dsub_rn(__dmul_rn(b, b), __dmul_rn(a, c));
        if (d <= 0.0) return false;
        const double sd = __dsqrt_rn(d);
        double t = __ddiv_rn(__dsub_rn(-b, sd), a);
        if (t < tmin || t > tmax) {
            t = __ddiv_rn(__dadd_rn(-b, sd), a);
            if (t < tmin || t > tmax) return false;
        }
        return true;
    }
    // World::hit, instance branch (world.rs:92-108), against the sampled triangle.
    const D3 o_obj = mv(inst->a_inv, sub(o, ld(inst->t)));
    const D3 d_obj = norm(mv(inst->a_inv, wi));
    const D3 v0 = lerp_static(ld(L.v), time), v1 = lerp_static(ld(L.v + 3), time), v2 = lerp_static(ld(L.v + 6), time);
    const D3 e1 = sub(v1, v0), e2 = sub(v2, v0);
    const D3 pvec = cross(d_obj, e2);
    const double det = dot(e1, pvec);
    if (fabs(det) < 1e-10) return false;
    const double inv_det = __ddiv_rn(1.0, det);
    const D3 tvec = sub(o_obj, v0);
    const double u = __dmul_rn(dot(tvec, pvec), inv_det);
    if (u < 0.0 || u > 1.0) return false;
    const D3 qvec = cross(tvec, e1);
    const double v = __dmul_rn(dot(d_obj, qvec), inv_det);
    if (v < 0.0 || __dadd_rn(u, v) > 1.0) return false;
    const double th = __dmul_rn(dot(e2, qvec), inv_det);
    if (th < tmin) return false;
    const D3 p_obj = add(o_obj, mul(d_obj, th));
    const D3 p_world = add(mv(inst->a, p_obj), ld(inst->t));
    const double t_world = dot(sub(p_world, o), wi);
    return t_world > tmin && t_world < tmax;
}

// Camera::ray (src/ray.rs:91-108) after the pixel jitter (src/render.rs:153-158).
static __device__ void camera_ray(const CameraF32& c, int x, int y, float inv_w, float inv_h, uint64_t& rng, float3& o,
                           float3& d, float& time) {
    const float jx = pcg_f32(rng), jy = pcg_f32(rng);
    const float sx = ((float)x + jx) * inv_w * 2.0f - 1.0f;
    const float sy = 1.0f - ((float)y + jy) * inv_h * 2.0f;
    const float3 base = normalize((-c.w) + c.u * (sx * c.half_w) + c.v * (sy * c.half_h));
    float3 lens = f3(0, 0, 0);
    if (c.lens_radius > 0.0f) {
        float dx = 0.0f, dy = 0.0f;
        for (int k = 0; k < 256; ++k) {  // rejection sampling of the unit disk (:112-120)
            dx = 2.0f * pcg_f32(rng) - 1.0f;
            dy = 2.0f * pcg_f32(rng) - 1.0f;
            if (dx * dx + dy * dy < 1.0f) break;
        }
        lens = c.u * (dx * c.lens_radius) + c.v * (dy * c.lens_radius);
    }
    o = c.o + lens;
    d = normalize((c.o + base * c.focus_dist) - o);
    time = pcg_f32(rng);  // shutter time; only the self-occlusion replay reads it
}

}  // namespace wf
}  // namespace tpt
