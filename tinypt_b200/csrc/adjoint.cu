// Path-replay backpropagation (PRB) of an image loss through the FP32 path
// integrator.
//
// The reference renders only; it has no derivative.  This kernel
// differentiates the estimator the FP32 forward form evaluates: radiance()
// (src/integrator.rs:53-135) with its BSDFs (src/material.rs:76-223), NEE
// with power-heuristic MIS (:148-225) and the luminance clamp of emitter and
// environment hits (src/math.rs:42-49).
//
// Sampling is detached: directions, light choices, pdfs, MIS weights and
// Russian-roulette probabilities are held fixed, and only the BSDF values,
// emission and absorption vary with the parameters.  A sample's radiance is
//     L = sum_k clamp_k(c_k),  c_k = beta_k * E_k,  beta_k = prod_{j<k} w_j,
// so its derivative along a parameter t is
//     dL = sum_k J_k (beta_k dE_k + c_k * sum_{j<k} dlog w_j)
// with J_k the Jacobian of the clamp.  With the pixel's adjoint delta (dLoss
// / dI_p divided by spp) each term is projected to a_k = (delta^T J_k) * c_k
// (per channel), and
//     dLoss/dt = sum_k a_k . dlog E_k/dt + sum_j dlog w_j/dt . (sum_{k>j} a_k).
// A first pass over the sample computes A = sum_k a_k; a second pass replays
// the same path from the same PCG32 state (nothing is stored per vertex),
// subtracting each a_k as it is met, so that after vertex j's own NEE terms
// the remainder is the suffix sum_{k>j} a_k that multiplies dlog w_j.
// Both passes run the same machine code (one non-inlined function with a
// runtime flag), so every branch is taken identically.
//
// Parameters per material m: 4m+0..2 = rgb (Lambert/Metal/Ggx/Subsurface
// albedo, Dielectric absorption, DiffuseLight emission), 4m+3 = Ggx alpha.
// Not differentiated (gradient 0): Dielectric ior and Subsurface
// scatter_dist, whose effect is through ray directions and origins; albedo
// channels that are exactly 0 (the path's suffix carries the factor 0).
#include "adjoint.cuh"

#include "fp32_device.cuh"

#include <algorithm>
#include <type_traits>

namespace tpt {
namespace wf {

constexpr float kClamp = 50.0f;  // FIREFLY_CLAMP (src/constants.rs)

// Gradient accumulation: per-thread f32 partials in local memory when the
// parameter vector is small (summed over the warp in f64 and added to the
// f64 result once per thread), else f64 atomics into a per-block shared copy
// (or straight into global memory for very large material counts).
constexpr int kPrivateParams = 64;
struct GradSink {
    float* pv;   // private partials, or nullptr
    double* sh;  // per-block shared copy, or nullptr
    double* gl;
    __device__ __forceinline__ void add(int k, float v) const {
        if (v == 0.0f) return;
        if (pv) pv[k] += v;
        else atomicAdd((sh ? sh : gl) + k, (double)v);
    }
    __device__ __forceinline__ void add_rgb(int m, float3 v) const {
        add(4 * m, v.x);
        add(4 * m + 1, v.y);
        add(4 * m + 2, v.z);
    }
};

// a = (delta^T J) * c for the luminance clamp of src/math.rs:42-49 (clamp =
// true) or a = delta * c (no clamp).
__device__ __forceinline__ float3 adj_weight(float3 c, float3 delta, bool clamp) {
    if (clamp) {
        const float l = luminance(c);
        if (l > kClamp && l > 0.0f) {
            const float s = kClamp / l;
            const float dc = dot(delta, c) / l;
            return f3(s * c.x * (delta.x - dc * 0.2126f), s * c.y * (delta.y - dc * 0.7152f),
                      s * c.z * (delta.z - dc * 0.0722f));
        }
    }
    return delta * c;
}

__device__ __forceinline__ float inv_or_zero(float x) { return x > 0.0f ? 1.0f / x : 0.0f; }

// d log D / d alpha of the GGX NDF (src/material.rs:273-281).
__device__ __forceinline__ float dlog_ggx_d(float alpha, float ch) {
    if (ch <= 0.0f) return 0.0f;
    const float den = ch * ch * (alpha * alpha - 1.0f) + 1.0f;
    return 2.0f / alpha - 4.0f * alpha * ch * ch / den;
}
// d log G1 / d alpha of Smith's G1 (src/material.rs:284-290).
__device__ __forceinline__ float dlog_ggx_g1(float alpha, float c) {
    if (c <= 0.0f) return 0.0f;
    const float a = alpha * sqrtf(fmaxf(1.0f - c * c, 0.0f)) / fmaxf(c, 1e-6f);
    const float s = sqrtf(1.0f + a * a);
    return -(a * a) / (alpha * s * (1.0f + s));
}
// Scatters a . dlog f/dtheta for a GGX value f = F(c_dm) D(ch) G1(ci) G1(co) / (...)
// (src/material.rs:227-239) to material m.
__device__ __forceinline__ void ggx_grad(const GradSink& g, int m, const MaterialF32& mt, float ci, float co, float ch,
                                         float c_dm, float3 a) {
    const float x5 = pow5(1.0f - fmaxf(c_dm, 0.0f));
    const float3 al = f3(mt.c);
    const float3 F = al + (f3(1.0f, 1.0f, 1.0f) - al) * x5;
    const float dF = 1.0f - x5;
    g.add_rgb(m, f3(a.x * dF * inv_or_zero(F.x), a.y * dF * inv_or_zero(F.y), a.z * dF * inv_or_zero(F.z)));
    if (mt.c.w >= 1e-3f) {  // alpha.max(1e-3) (:150) has no derivative below the clamp
        const float al_ = mt.c.w;
        g.add(4 * m + 3, (a.x + a.y + a.z) * (dlog_ggx_d(al_, ch) + dlog_ggx_g1(al_, ci) + dlog_ggx_g1(al_, co)));
    }
}
// a . dlog f/dtheta for the value Material::eval returns at (wo, wi).
__device__ __forceinline__ void eval_grad(const GradSink& g, int m, const MaterialF32& mt, float3 wo, float3 wi, float3 n,
                                          float3 a) {
    if (mt.kind == TPT_MAT_LAMBERT || mt.kind == TPT_MAT_SUBSURFACE) {
        const float3 al = f3(mt.c);
        g.add_rgb(m, f3(a.x * inv_or_zero(al.x), a.y * inv_or_zero(al.y), a.z * inv_or_zero(al.z)));
    } else if (mt.kind == TPT_MAT_GGX) {
        const float3 mh = normalize(wo + wi);
        ggx_grad(g, m, mt, dot(n, wo), dot(n, wi), fmaxf(dot(n, mh), 0.0f), fabsf(dot(wi, mh)), a);
    }
}

// Path state of one sample pass.  acc holds sum_k a_k during the first pass
// and the remaining suffix during the replay.
struct AdjPath {
    float3 o, d, beta, acc;
    uint64_t rng;
    float last_pdf, ptime, lin;
    int bounce, self_prim, self_inst;
    bool last_nd, grad;
};

// Starts a pass of one sample at the given PCG32 state: the camera ray of
// src/render.rs:151-158 and the initial state of radiance() (:61-65).
__device__ __noinline__ void adj_begin(const WfScene& S, const AdjParams& P, int x, int y, uint64_t rng, bool grad,
                                       float3 acc, AdjPath& p) {
    p.rng = rng;
    camera_ray(S.cam, x, y, 1.0f / (float)P.width, 1.0f / (float)P.height, p.rng, p.o, p.d, p.ptime);
    p.beta = f3(1.0f, 1.0f, 1.0f);
    p.acc = acc;
    p.last_pdf = 0.0f;
    p.lin = 0.0f;
    p.bounce = 0;
    p.self_prim = -1;
    p.self_inst = -1;
    p.last_nd = false;
    p.grad = grad;
}

// One bounce of radiance() (src/integrator.rs:67-132) for a pass.  First
// pass (grad = false): adds each a_k to acc and the clamped contribution to
// lin.  Replay (grad = true): subtracts each a_k from acc and scatters the
// gradient terms to `sink`.  Returns false when the path has ended.  Both
// passes run this one function, so they take the same branches.
template <class Stack>
__device__ __noinline__ bool adj_step(const WfScene& S, const AdjParams& P, AdjPath& p, float3 delta,
                                      const GradSink& sink, int* flags, const Stack stack) {
    if (p.bounce >= P.max_bounces) return false;
    const bool has_env = S.env_kind == TPT_ENV_MAP;
    Tracer T;
    TraceCount cnt;
    tracer_start(S, T, p.o, p.d, kTMax, p.self_prim, p.self_inst);
    tracer_run<false, false>(S, T, stack, kEps, 1 << 30, flags, cnt);
    const int prim = T.hit_prim, inst = T.hit_inst;
    const float th = T.tmax;
    if (prim < 0) {  // miss (:71-83)
        float3 bg;
        if (has_env) {
            bg = env_lookup(S, p.d);
        } else {
            const float t = 0.5f * (p.d.y + 1.0f);
            bg = f3(0.9f, 0.95f, 1.0f) * (1.0f - t) + f3(0.6f, 0.75f, 1.0f) * t;
        }
        float3 c = p.beta * bg;
        if (has_env && p.last_nd) c = c * mis(p.last_pdf, env_pdf(S, p.d));
        const float3 a = adj_weight(c, delta, true);
        if (p.grad) p.acc = p.acc - a; else { p.acc = p.acc + a; p.lin += dot(delta, clamp_lum(c, kClamp)); }
        return false;
    }
    if (p.bounce >= P.rr_start) {  // Russian roulette (:89-95), probability detached
        const float q = fmaxf(fminf(max3(p.beta), 0.95f), 0.05f);
        if (pcg_f32(p.rng) > q) return false;
        p.beta = p.beta / q;
    }
    const float3 hp = p.o + p.d * th;
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
        const float3 a = adj_weight(p.beta * mc, delta, true);
        if (p.grad) {
            p.acc = p.acc - a;
            sink.add_rgb(mid, f3(a.x * inv_or_zero(mc.x), a.y * inv_or_zero(mc.y), a.z * inv_or_zero(mc.z)));
        } else {
            p.acc = p.acc + a;
            p.lin += dot(delta, clamp_lum(p.beta * mc, kClamp));
        }
        return false;
    }
    const bool entering = dot(ng, p.d) < 0.0f;
    const float3 n = entering ? ng : -ng;
    const float3 wo = -p.d;
    if (mt.kind != TPT_MAT_METAL && mt.kind != TPT_MAT_DIELECTRIC) {
        if (has_env) {  // nee_environment (:148-172)
            float3 wi, li;
            float pe;
            env_sample_dir(S, p.rng, wi, li, pe);
            const float c = fmaxf(dot(n, wi), 0.0f);
            if (c > 0.0f && pe > 0.0f) {
                float3 f;
                float pb;
                mat_eval(mt, wo, wi, n, f, pb);
                const float3 contrib = p.beta * f * li * (c * mis(pe, pb) / pe);
                if (contrib.x > 0.0f || contrib.y > 0.0f || contrib.z > 0.0f) {
                    tracer_start(S, T, hp + wi * kEps, wi, kTMax, prim, inst);
                    tracer_run<true, false>(S, T, stack, kEps, 1 << 30, flags, cnt);
                    if (T.hit_prim < 0) {
                        const float3 a = delta * contrib;
                        if (p.grad) {
                            p.acc = p.acc - a;
                            eval_grad(sink, mid, mt, wo, wi, n, a);
                        } else {
                            p.acc = p.acc + a;
                            p.lin += dot(delta, contrib);
                        }
                    }
                }
            }
        }
        float3 lp, le;
        float lpdf;
        int lidx;
        double lud, lvd;
        if (sample_light(S, p.rng, hp, lp, le, lpdf, lidx, lud, lvd)) {  // nee_area_light (:178-213)
            const float3 tl = lp - hp;
            const float dist = length(tl);
            if (dist > 1e-6f) {
                const float3 wi = tl / dist;
                const float c = fmaxf(dot(n, wi), 0.0f);
                if (c > 0.0f && !ref_light_self_occluded(S.lights64, S.spheres64, S.inst64, lidx, p.o, p.d, th, lud, lvd, (double)p.ptime)) {
                    float3 f;
                    float pb;
                    mat_eval(mt, wo, wi, n, f, pb);
                    const float3 contrib = p.beta * f * le * (c * mis(lpdf, pb) / lpdf);
                    if (contrib.x > 0.0f || contrib.y > 0.0f || contrib.z > 0.0f) {
                        tracer_start(S, T, hp + wi * kEps, wi, fmaxf(dist - 2.0f * kEps, kEps), prim, inst);
                        tracer_run<true, false>(S, T, stack, kEps, 1 << 30, flags, cnt);
                        if (T.hit_prim < 0) {
                            const float3 a = delta * contrib;
                            if (p.grad) {
                                p.acc = p.acc - a;
                                eval_grad(sink, mid, mt, wo, wi, n, a);
                                const int lm = __ldg(&S.lights[lidx].mat);
                                sink.add_rgb(lm, f3(a.x * inv_or_zero(le.x), a.y * inv_or_zero(le.y),
                                                    a.z * inv_or_zero(le.z)));
                            } else {
                                p.acc = p.acc + a;
                                p.lin += dot(delta, contrib);
                            }
                        }
                    }
                }
            }
        }
    }
    // Material::sample (src/material.rs:76-201) and dlog w of the sample
    float3 nd = f3(0, 0, 0), w = f3(0, 0, 0), no = hp;
    float pdf = 0.0f;
    bool delta_s = false, self_ok = true;
    if (mt.kind == TPT_MAT_LAMBERT) {
        nd = cos_hemi(n, p.rng);
        w = mc;
        pdf = fmaxf(dot(n, nd), 0.0f) / kPi;
        if (p.grad) sink.add_rgb(mid, f3(p.acc.x * inv_or_zero(mc.x), p.acc.y * inv_or_zero(mc.y), p.acc.z * inv_or_zero(mc.z)));
    } else if (mt.kind == TPT_MAT_METAL) {
        nd = p.d - n * (2.0f * dot(p.d, n));
        w = mc;
        delta_s = true;
        if (p.grad) sink.add_rgb(mid, f3(p.acc.x * inv_or_zero(mc.x), p.acc.y * inv_or_zero(mc.y), p.acc.z * inv_or_zero(mc.z)));
    } else if (mt.kind == TPT_MAT_DIELECTRIC) {
        const float ior = mt.c.w;
        const float eta = entering ? 1.0f / ior : ior;
        const float ci = fmaxf(dot(wo, n), 0.0f);
        const float fq = (ior - 1.0f) / (ior + 1.0f);
        const float f0 = fq * fq;
        const float fr = f0 + (1.0f - f0) * pow5(1.0f - ci);
        float3 bt = f3(1, 1, 1);
        float dist = 0.0f;
        if (!entering) {
            dist = fmaxf(th, 0.0f);
            bt = f3(__expf(-mc.x * dist), __expf(-mc.y * dist), __expf(-mc.z * dist));
        }
        const float cosi = fminf(fmaxf(dot(wo, n), -1.0f), 1.0f);
        const float sin2t = eta * eta * (1.0f - cosi * cosi);
        const bool has_refr = !(sin2t >= 1.0f);
        const bool refl = !has_refr || pcg_f32(p.rng) < fr;
        if (refl) {
            nd = p.d - n * (2.0f * dot(p.d, n));
            bt = bt * (fr / fmaxf(fr, 1e-6f));
        } else {
            nd = p.d * eta + n * (eta * cosi - sqrtf(1.0f - sin2t));
            bt = bt * ((1.0f - fr) / fmaxf(1.0f - fr, 1e-6f)) * (eta * eta);
        }
        w = bt;
        delta_s = true;
        if (p.grad && !entering) sink.add_rgb(mid, p.acc * (-dist));  // Beer-Lambert: dlog att/dsigma = -dist
    } else if (mt.kind == TPT_MAT_GGX) {
        GgxSample gs;
        if (!ggx_sample(p.d, n, mt, p.rng, gs)) return false;
        nd = gs.nd;
        w = gs.w;
        pdf = gs.pdf;
        if (p.grad) ggx_grad(sink, mid, mt, gs.ci, gs.co, gs.ch, fabsf(dot(gs.nd, gs.mh)), p.acc);
    } else if (mt.kind == TPT_MAT_SUBSURFACE) {
        const float sc = fmaxf(mt.c.w, 1e-4f);
        const float u = fmaxf(pcg_f32(p.rng), 1e-12f);
        const float dist = -__logf(u) * sc;
        nd = cos_hemi(ng, p.rng);  // unoriented normal (material.rs:187-188)
        w = mc * __expf(-dist / sc);
        no = hp - ng * dist;
        pdf = fmaxf(dot(n, nd), 0.0f) / kPi;
        self_ok = false;
        if (p.grad) sink.add_rgb(mid, f3(p.acc.x * inv_or_zero(mc.x), p.acc.y * inv_or_zero(mc.y), p.acc.z * inv_or_zero(mc.z)));
    } else {
        return false;
    }
    p.beta = p.beta * w;
    p.last_pdf = pdf;
    p.last_nd = !delta_s;
    p.o = no + nd * kEps;
    p.d = nd;
    p.self_prim = self_ok ? prim : -1;
    p.self_inst = self_ok ? inst : -1;
    return ++p.bounce < P.max_bounces;  // bounce loop bound (:67)
}

// Each thread runs tasks (a pixel's run of task_spp samples, seeded like the
// forward form's tasks) one bounce at a time: when a lane's pass ends it
// starts the replay of that sample, or the next sample, or the next task, so
// the warp's lanes stay busy until the work runs out.
template <bool SHARED_STACK>
__global__ void __launch_bounds__(128) k_adjoint(WfScene S, AdjParams P, const float* __restrict__ dimg,
                                                 double* __restrict__ grad, int* flags,
                                                 unsigned long long* counters, int mode) {
    extern __shared__ double sgrad[];
    __shared__ int sstack[SHARED_STACK ? kSharedStack * 128 : 1];
    int lstack[SHARED_STACK ? 1 : kStack];
    using Stack = typename std::conditional<SHARED_STACK, TStack<128, kSharedStack>, TStack<1, kStack>>::type;
    const Stack stack{SHARED_STACK ? sstack + threadIdx.x : lstack};
    const int n_params = 4 * P.n_mats;
    float pv[kPrivateParams];
    if (mode == 0) {
        for (int k = 0; k < kPrivateParams; ++k) pv[k] = 0.0f;
    } else if (mode == 1) {
        for (int k = threadIdx.x; k < n_params; k += blockDim.x) sgrad[k] = 0.0;
        __syncthreads();
    }
    const GradSink sink{mode == 0 ? pv : nullptr, mode == 1 ? sgrad : nullptr, grad};
    const long long stride = (long long)gridDim.x * blockDim.x;
    const float inv_spp = 1.0f / (float)P.spp;
    unsigned long long paths = 0;
    double lin = 0.0;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int x = 0, y = 0, s = 0, n = 0;
    float3 delta = f3(0, 0, 0);
    uint64_t rng = 0, sample_rng = 0;
    // next task with a non-zero adjoint (no gradient flows through the others)
    auto take_task = [&]() -> bool {
        for (; t < P.n_tasks; t += stride) {
            const int chunk = (int)fdiv(P.px_div, (uint32_t)t);
            const int pixel = (int)t - chunk * P.n_pixels;
            delta = f3(dimg[3 * (size_t)pixel], dimg[3 * (size_t)pixel + 1], dimg[3 * (size_t)pixel + 2]) * inv_spp;
            if (delta.x == 0.0f && delta.y == 0.0f && delta.z == 0.0f) continue;
            const int row = (int)fdiv(P.w_div, (uint32_t)pixel);
            x = pixel - row * P.width;
            y = P.row_begin + row * P.row_step;
            rng = task_seed((uint32_t)x, (uint32_t)y, (uint32_t)(chunk * P.task_spp), P.seed);
            n = min(P.task_spp, P.spp - chunk * P.task_spp);
            s = 0;
            return true;
        }
        return false;
    };
    AdjPath p;
    bool ok = take_task();
    if (ok) {
        sample_rng = rng;
        adj_begin(S, P, x, y, sample_rng, false, f3(0, 0, 0), p);
    }
    // The loop runs while any lane of the warp has work, and the warp
    // reconverges after every bounce, so lanes that start a new pass rejoin
    // the others instead of running the bounce code as a separate group.
    while (__any_sync(0xffffffffu, ok)) {
        if (ok && !adj_step(S, P, p, delta, sink, flags, stack)) {
            if (!p.grad) {  // first pass done: replay the sample from its start
                lin += (double)p.lin;
                adj_begin(S, P, x, y, sample_rng, true, p.acc, p);
            } else {
                ++paths;  // replay done; the stream continues with the next sample
                rng = p.rng;
                if (++s >= n) {
                    t += stride;
                    ok = take_task();
                }
                if (ok) {
                    sample_rng = rng;
                    adj_begin(S, P, x, y, sample_rng, false, f3(0, 0, 0), p);
                }
            }
        }
        __syncwarp();
    }
    if (paths) atomicAdd(counters, paths);
    if (lin != 0.0) atomicAdd(reinterpret_cast<double*>(counters + 1), lin);
    if (mode == 0) {
        for (int k = 0; k < n_params; ++k) {
            double v = (double)pv[k];
            for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
            if ((threadIdx.x & 31u) == 0 && v != 0.0) atomicAdd(grad + k, v);
        }
    } else if (mode == 1) {
        __syncthreads();
        for (int k = threadIdx.x; k < n_params; k += blockDim.x)
            if (sgrad[k] != 0.0) atomicAdd(grad + k, sgrad[k]);
    }
}

__global__ void k_resolve(const double* __restrict__ acc, const double* __restrict__ acc_w, float* __restrict__ img,
                          int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double w = fmax(acc_w[i], 1.0);
    img[3 * (size_t)i] = (float)(acc[3 * (size_t)i] / w);
    img[3 * (size_t)i + 1] = (float)(acc[3 * (size_t)i + 1] / w);
    img[3 * (size_t)i + 2] = (float)(acc[3 * (size_t)i + 2] / w);
}

// ---- wavefront form ---------------------------------------------------------------
// The same derivative, computed on the forward form's wavefront machinery
// (dense slot order, persistent lane-refilling traversal, queues) in ONE
// pass per sample instead of a first pass and a replay.  The suffix sums are
// regrouped:
//     sum_j dlog w_j . (sum_{k>j} a_k) = sum_j dlog w_j . (A - C_j),
// A = sum_k a_k of the whole sample, C_j = the part of it known once vertex
// j's NEE terms are resolved.  Each BSDF sample stores its dlog w and
// material in a per-slot vertex list; C_j joins the entry when the next
// iteration has resolved vertex j's shadow rays; when the sample ends every
// entry scatters dlog w_j . (A - C_j).  The difference is taken per path, in
// f32 like the replay's running suffix, so no large terms cancel in the
// gradient sums.  The last vertex of a path cut by the bounce limit has
// C_j = A and is skipped (F_ADJ_OPEN marks an entry still without C_j).
//
// Per iteration: closest hit (the forward kernel) -> k_adj_shade (resolves
// pending NEE, miss / emitter terms, NEE records with their gradient
// packets, BSDF sample and its vertex entry) -> occlusion (the forward
// kernel) -> k_adj_regen (samples that ended with shadow rays pending).
constexpr int F_ADJ_OPEN = 16;    // the last vertex entry has no C_j yet
constexpr int kAdjBlock = 128;

// Gradient partials of one block for one launch, flushed to the f64 totals
// at its end: mode 0 per-thread partials in shared memory ([param][thread],
// no bank conflicts), mode 1 shared f32 atomics, mode 2 f64 atomics straight
// into the totals.  Index n_params holds the linearised loss.
struct GradAcc {
    float* sh;
    double* gl;
    int mode;
    __device__ __forceinline__ void add(int k, float v) const {
        if (v == 0.0f) return;
        if (mode == 0) sh[k * kAdjBlock + threadIdx.x] += v;
        else if (mode == 1) atomicAdd(sh + k, v);
        else atomicAdd(gl + k, (double)v);
    }
    __device__ __forceinline__ void add4(int m, float4 v) const {
        add(4 * m, v.x);
        add(4 * m + 1, v.y);
        add(4 * m + 2, v.z);
        add(4 * m + 3, v.w);
    }
};
__device__ __forceinline__ GradAcc grad_begin(float* sh, double* gl, int mode, int n) {
    if (mode == 0)
        for (int k = 0; k < n; ++k) sh[k * kAdjBlock + threadIdx.x] = 0.0f;
    else if (mode == 1)
        for (int k = threadIdx.x; k < n; k += blockDim.x) sh[k] = 0.0f;
    __syncthreads();
    return GradAcc{sh, gl, mode};
}
__device__ __forceinline__ void grad_end(const GradAcc& g, int n) {
    if (g.mode == 2) return;
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double v = 0.0;
        if (g.mode == 0)
            for (int t = 0; t < kAdjBlock; ++t) v += (double)g.sh[k * kAdjBlock + t];
        else
            v = (double)g.sh[k];
        if (v != 0.0) atomicAdd(g.gl + k, v);
    }
}

// Per-channel and alpha factors of dlog f for Material::eval's value at
// (wo, wi) (src/material.rs:204-223): w = (dlog f/drgb_c per channel, dlog
// f/dalpha).  Metal and Dielectric have no eval term (delta lobes).
__device__ __forceinline__ float4 ggx_dlog(const MaterialF32& mt, float ci, float co, float ch, float c_dm) {
    const float x5 = pow5(1.0f - fmaxf(c_dm, 0.0f));
    const float3 al = f3(mt.c);
    const float3 F = al + (f3(1.0f, 1.0f, 1.0f) - al) * x5;
    const float dF = 1.0f - x5;
    float da = 0.0f;
    if (mt.c.w >= 1e-3f) {  // alpha.max(1e-3) (:150) has no derivative below the clamp
        const float al_ = mt.c.w;
        da = dlog_ggx_d(al_, ch) + dlog_ggx_g1(al_, ci) + dlog_ggx_g1(al_, co);
    }
    return make_float4(dF * inv_or_zero(F.x), dF * inv_or_zero(F.y), dF * inv_or_zero(F.z), da);
}
__device__ __forceinline__ float4 albedo_dlog(float3 al) {
    return make_float4(inv_or_zero(al.x), inv_or_zero(al.y), inv_or_zero(al.z), 0.0f);
}
__device__ __forceinline__ float4 eval_dlog(const MaterialF32& mt, float3 wo, float3 wi, float3 n) {
    if (mt.kind == TPT_MAT_LAMBERT || mt.kind == TPT_MAT_SUBSURFACE) return albedo_dlog(f3(mt.c));
    if (mt.kind == TPT_MAT_GGX) {
        const float3 mh = normalize(wo + wi);
        return ggx_dlog(mt, dot(n, wo), dot(n, wi), fmaxf(dot(n, mh), 0.0f), fabsf(dot(wi, mh)));
    }
    return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}
// a . dlog: per channel for rgb, the channel sum for alpha.
__device__ __forceinline__ float4 project(float4 dl, float3 a) {
    return make_float4(a.x * dl.x, a.y * dl.y, a.z * dl.z, (a.x + a.y + a.z) * dl.w);
}

__device__ __forceinline__ void adj_warp_count(int* counter, bool pred) {
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (mask && (int)lane_id() == __ffs(mask) - 1) atomicAdd(counter, __popc(mask));
}

__device__ __forceinline__ float3 pixel_delta(const AdjParams& P, const float* __restrict__ dimg, long long task,
                                              float inv_spp) {
    const size_t px = (size_t)((uint32_t)task - fdiv(P.px_div, (uint32_t)task) * (uint32_t)P.n_pixels);
    return f3(__ldg(dimg + 3 * px), __ldg(dimg + 3 * px + 1), __ldg(dimg + 3 * px + 2)) * inv_spp;
}

// Task t: pixel t % n_pixels, samples from chunk t / n_pixels, seeded like
// the forward form's tasks (src/render.rs:142).
__device__ __forceinline__ void adj_start_task(const WfScene& S, const AdjParams& P, const WfState& st,
                                               const AdjWfState& A, int slot, long long task) {
    const int chunk = (int)fdiv(P.px_div, (uint32_t)task);
    const int pixel = (int)task - chunk * P.n_pixels;
    const int row = (int)fdiv(P.w_div, (uint32_t)pixel);
    const int x = pixel - row * P.width, y = P.row_begin + row * P.row_step;
    uint64_t rng = task_seed((uint32_t)x, (uint32_t)y, (uint32_t)(chunk * P.task_spp), P.seed);
    float3 o, d;
    float time;
    camera_ray(S.cam, x, y, 1.0f / (float)P.width, 1.0f / (float)P.height, rng, o, d, time);
    store_path(st, slot, make_int4(0, 0, 0, (int)task), rng);
    sts(&st.ray_o[slot], make_float4(o.x, o.y, o.z, ifloat(-1)));
    sts(&st.ray_d[slot], make_float4(d.x, d.y, d.z, ifloat(-1)));
    sts(&st.beta[slot], make_float4(1.0f, 1.0f, 1.0f, 0.0f));
    sts(&A.acc[slot], make_float4(0.0f, 0.0f, 0.0f, time));
}

// Fetch ids of the task pool: the tasks themselves, or with camera culling
// the tasks of the pixels in geo_map, chunk by chunk, in film order.
__device__ __forceinline__ long long adj_fetch_end(const AdjParams& P) {
    return P.geo_map ? (long long)P.n_chunks * P.n_geo : P.n_tasks;
}
__device__ __forceinline__ long long adj_task_of(const AdjParams& P, long long f) {
    if (!P.geo_map) return f;
    const uint32_t c = fdiv(P.geo_div, (uint32_t)f);
    return (long long)c * P.n_pixels + __ldg(P.geo_map + ((uint32_t)f - c * (uint32_t)P.n_geo));
}

// Must be called by all lanes of a converged warp.
__device__ __forceinline__ bool adj_take_task(const WfScene& S, const AdjParams& P, const WfState& st,
                                              const AdjWfState& A, int slot, bool need_task) {
    const unsigned want = __ballot_sync(0xffffffffu, need_task);
    if (!want) return false;
    const int leader = __ffs(want) - 1;
    long long t0 = 0;
    if ((int)lane_id() == leader)
        t0 = (long long)atomicAdd((unsigned long long*)&st.ctr->next_task, (unsigned long long)__popc(want));
    t0 = __shfl_sync(0xffffffffu, t0, leader);
    if (!need_task) return false;
    const long long t = t0 + __popc(want & ((1u << lane_id()) - 1u));
    if (t >= adj_fetch_end(P)) return false;
    adj_start_task(S, P, st, A, slot, adj_task_of(P, t));
    return true;
}

__global__ void k_adj_init(WfScene S, AdjParams P, WfState st, AdjWfState A, int n_slots) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const long long avail = adj_fetch_end(P);
    const int first = (int)(avail < (long long)n_slots ? avail : n_slots);
    if (i == 0) {
        st.ctr->n_ext[0] = first;
        st.ctr->next_task = first;
    }
    if (i >= n_slots) return;
    st.act[i] = i < first ? 1 : 0;
    if (i < first) {
        st.q_ext[0][i] = i;
        adj_start_task(S, P, st, A, i, adj_task_of(P, i));
    }
}

// One thread per task of a culled pixel (chunk by chunk, the pixels of
// open_map in film order): every sample is a camera ray that leaves the
// scene, whose only term is the linearised loss dot(dL/dpixel / spp,
// clamp_lum(background)) -- no material gradient.  Same draws as the
// replay (adj_start_task + camera_ray per sample).  Adds the terms (f64,
// one atomic per block) and the samples to the render's counters.
__global__ void __launch_bounds__(256) k_adj_sky(WfScene S, AdjParams P, WfState st, const float* __restrict__ dimg,
                                                 double* gtot, int lin_k, const int* __restrict__ open_map, int n_open,
                                                 FastDiv open_div, long long count) {
    __shared__ double red[256 / 32];
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double lin = 0.0;
    unsigned long long done = 0;
    if (v < count) {
        const uint32_t c = fdiv(open_div, (uint32_t)v);
        const int pixel = __ldg(open_map + ((uint32_t)v - c * (uint32_t)n_open));
        const long long task = (long long)c * P.n_pixels + pixel;
        const int row = (int)fdiv(P.w_div, (uint32_t)pixel);
        const int x = pixel - row * P.width, y = P.row_begin + row * P.row_step;
        const int start = (int)c * P.task_spp;
        const int len = min(P.task_spp, P.spp - start);
        uint64_t rng = task_seed((uint32_t)x, (uint32_t)y, (uint32_t)start, P.seed);
        const float3 delta = pixel_delta(P, dimg, task, 1.0f / (float)P.spp);
        for (int k = 0; k < len; ++k) {
            float3 o, d;
            float time;
            camera_ray(S.cam, x, y, 1.0f / (float)P.width, 1.0f / (float)P.height, rng, o, d, time);
            lin += (double)dot(delta, clamp_lum(background(S, d), kClamp));
        }
        done = (unsigned long long)len;
    }
    for (int off = 16; off > 0; off >>= 1) {
        lin += __shfl_down_sync(0xffffffffu, lin, off);
        done += __shfl_down_sync(0xffffffffu, done, off);
    }
    if (lane_id() == 0) {
        red[threadIdx.x >> 5] = lin;
        if (done) atomicAdd(&st.ctr->samples, done);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        if (t != 0.0) atomicAdd(gtot + lin_k, t);
    }
}

// Shadow records of the previous vertex: visible ones add their a to the
// sample's sum and scatter their gradient packets.
__device__ __forceinline__ float3 adj_take_pending(const WfState& st, const AdjWfState& A, int slot, int& fl,
                                                   float3 acc, const GradAcc& g, int lin_k) {
    for (int r = 0; r < 2; ++r) {
        if (!(fl & (r ? F_PEND_AREA : F_PEND_ENV))) continue;
        const float4 c = lds(&st.sh_c[2 * slot + r]);
        if (c.w > 0.5f) {
            const float3 a = f3(c);
            acc = acc + a;
            g.add(lin_k, a.x + a.y + a.z);
            g.add4(A.sh_mat[2 * slot + r], lds(&A.sh_gm[2 * slot + r]));
            if (r) {
                const float4 gl = lds(&A.sh_gl[2 * slot + 1]);
                g.add4(fbits(gl.w), make_float4(gl.x, gl.y, gl.z, 0.0f));
            }
        }
    }
    fl &= ~(F_PEND_ENV | F_PEND_AREA);
    return acc;
}

// End of a sample: dlog w_j . (A - C_j) for its vertex entries (the last
// one skipped while open: its C_j is A).
__device__ __forceinline__ void adj_final(const AdjWfState& A, const GradAcc& g, int slot, int n_slots, int nb, int fl,
                                          float3 acc) {
    const int last = (fl & F_ADJ_OPEN) ? nb - 1 : nb;
    for (int j = 0; j < last; ++j) {
        const size_t e = (size_t)j * n_slots + slot;
        const float4 c = lds(&A.vc[e]);
        const int vm = fbits(c.w);
        if (vm >= 0) g.add4(vm, project(lds(&A.vg[e]), acc - f3(c)));
    }
}

// The next sample of the task (its camera ray continues the PCG32 stream),
// or need_task when the task is done.
__device__ __forceinline__ bool adj_next_sample(const WfScene& S, const AdjParams& P, const WfState& st, int slot,
                                                int4& m, int& fl, float3& acc, float3& beta, float& last_pdf,
                                                float& ptime, uint64_t& rng, bool& need_task) {
    m.x += 1;
    const int task = m.w;
    const int chunk = (int)fdiv(P.px_div, (uint32_t)task);
    const int task_len = min(P.task_spp, P.spp - chunk * P.task_spp);
    if (m.x >= task_len) {
        need_task = true;
        return false;
    }
    const int pixel = task - chunk * P.n_pixels;
    const int row = (int)fdiv(P.w_div, (uint32_t)pixel);
    float3 o, d;
    camera_ray(S.cam, pixel - row * P.width, P.row_begin + row * P.row_step, 1.0f / (float)P.width,
               1.0f / (float)P.height, rng, o, d, ptime);
    sts(&st.ray_o[slot], make_float4(o.x, o.y, o.z, ifloat(-1)));
    sts(&st.ray_d[slot], make_float4(d.x, d.y, d.z, ifloat(-1)));
    beta = f3(1.0f, 1.0f, 1.0f);
    last_pdf = 0.0f;
    acc = f3(0.0f, 0.0f, 0.0f);
    m.y = 0;
    fl = 0;
    return true;
}

// One bounce of radiance() (src/integrator.rs:67-132) per active slot, with
// the adjoint bookkeeping.  The sampling arithmetic is k_shade's, so every
// slot follows the forward form's path.
__global__ void __launch_bounds__(kAdjBlock, 6) k_adj_shade(WfScene S, AdjParams P, WfState st, AdjWfState A,
                                                            const float* __restrict__ dimg, double* gtot, int gmode,
                                                            int cur, int n_slots) {
    extern __shared__ float gsh[];
    const int lin_k = 4 * P.n_mats;
    const GradAcc g = grad_begin(gsh, gtot, gmode, lin_k + 1);
    const int ns = n_slots;
    const int nxt = cur ^ 1;
    const int stride = gridDim.x * blockDim.x;
    const bool has_env = S.env_kind == TPT_ENV_MAP;
    const float inv_spp = 1.0f / (float)P.spp;
    // slots in slot order while many are live, from the extension queue when few are (use_ext_queue)
    const int live = st.ctr->n_ext[cur];
    const bool use_q = P.ordered_queue || use_ext_queue(live, ns, P.queue_div);
    const int n = use_q ? live : ns;
    const int* __restrict__ qe = st.q_ext[cur];
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const int i = base + (int)lane_id();
        const bool active = i < n && (use_q || st.act[i]);
        bool cont = false, term = false, need_task = false, finished_here = false;
        int slot = 0;
        int sh_env = 0, sh_area = 0;
        if (active) {
            slot = use_q ? qe[i] : i;
            const float4 o4 = lds(&st.ray_o[slot]), d4 = lds(&st.ray_d[slot]);
            const float3 ro = f3(o4), rd = f3(d4);
            const float4 h4 = lds(&st.hit[slot]);
            const int prim = fbits(h4.y), inst = fbits(h4.z);
            const float4 b4 = lds(&st.beta[slot]);
            float3 beta = f3(b4);
            float last_pdf = b4.w;
            const float4 a4 = lds(&A.acc[slot]);
            float3 acc = f3(a4);
            float ptime = a4.w;
            int4 m;
            uint64_t rng;
            load_path(st, slot, m, rng);
            int fl = m.z;
            const float3 delta = pixel_delta(P, dimg, (long long)m.w, inv_spp);
            acc = adj_take_pending(st, A, slot, fl, acc, g, lin_k);
            if (fl & F_ADJ_OPEN) {  // the previous vertex's C_j is known now
                const size_t e = (size_t)(m.y - 1) * ns + slot;
                const float4 c = lds(&A.vc[e]);
                sts(&A.vc[e], make_float4(acc.x, acc.y, acc.z, c.w));
                fl &= ~F_ADJ_OPEN;
            }
            bool done = m.y >= P.max_bounces;  // max_bounces = 0: radiance() returns 0
            if (!done && prim < 0) {  // miss (:71-83)
                float3 bg;
                if (has_env) {
                    bg = env_lookup(S, rd);
                } else {
                    const float t = 0.5f * (rd.y + 1.0f);  // sky (:25-28)
                    bg = f3(0.9f, 0.95f, 1.0f) * (1.0f - t) + f3(0.6f, 0.75f, 1.0f) * t;
                }
                float3 c = beta * bg;
                if (has_env && (fl & F_LAST_ND)) c = c * mis(last_pdf, env_pdf(S, rd));
                acc = acc + adj_weight(c, delta, true);
                g.add(lin_k, dot(delta, clamp_lum(c, kClamp)));
                done = true;
            }
            if (!done && m.y >= P.rr_start) {  // Russian roulette (:89-95), probability detached
                const float q = fmaxf(fminf(max3(beta), 0.95f), 0.05f);
                if (pcg_f32(rng) > q) done = true;
                else beta = beta / q;
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
                    const float3 c = beta * mc;
                    const float3 a = adj_weight(c, delta, true);
                    acc = acc + a;
                    g.add4(mid, make_float4(a.x * inv_or_zero(mc.x), a.y * inv_or_zero(mc.y), a.z * inv_or_zero(mc.z),
                                            0.0f));
                    g.add(lin_k, dot(delta, clamp_lum(c, kClamp)));
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
                                    const float3 a = delta * contrib;
                                    sts(&st.sh_o[2 * slot], make_float4(so.x, so.y, so.z, kTMax));
                                    sts(&st.sh_d[2 * slot], make_float4(wi.x, wi.y, wi.z, ifloat(prim)));
                                    sts(&st.sh_c[2 * slot], make_float4(a.x, a.y, a.z, ifloat(inst)));
                                    sts(&A.sh_gm[2 * slot], project(eval_dlog(mt, wo, wi, n), a));
                                    A.sh_mat[2 * slot] = mid;
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
                                        const float3 a = delta * contrib;
                                        sts(&st.sh_o[2 * slot + 1],
                                            make_float4(so.x, so.y, so.z, fmaxf(dist - 2.0f * kEps, kEps)));
                                        sts(&st.sh_d[2 * slot + 1], make_float4(wi.x, wi.y, wi.z, ifloat(prim)));
                                        sts(&st.sh_c[2 * slot + 1], make_float4(a.x, a.y, a.z, ifloat(inst)));
                                        sts(&A.sh_gm[2 * slot + 1], project(eval_dlog(mt, wo, wi, n), a));
                                        A.sh_mat[2 * slot + 1] = mid;
                                        const int lm = __ldg(&S.lights[lidx].mat);
                                        sts(&A.sh_gl[2 * slot + 1], make_float4(a.x * inv_or_zero(le.x), a.y * inv_or_zero(le.y),
                                                                            a.z * inv_or_zero(le.z), ifloat(lm)));
                                        sh_area = 1;
                                        fl |= F_PEND_AREA;
                                    }
                                }
                            }
                        }
                    }
                    // Material::sample (src/material.rs:76-201) and its dlog w
                    float3 nd = f3(0, 0, 0), w = f3(0, 0, 0), no = hp;
                    float pdf = 0.0f;
                    bool delta_s = false, ok = true, self_ok = true;
                    float4 dlw = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    bool has_dlw = true;
                    switch (mt.kind) {
                        case TPT_MAT_LAMBERT:
                            nd = cos_hemi(n, rng);
                            w = mc;
                            pdf = fmaxf(dot(n, nd), 0.0f) / kPi;
                            dlw = albedo_dlog(mc);
                            break;
                        case TPT_MAT_METAL:
                            nd = rd - n * (2.0f * dot(rd, n));
                            w = mc;
                            delta_s = true;
                            dlw = albedo_dlog(mc);
                            break;
                        case TPT_MAT_DIELECTRIC: {
                            const float ior = mt.c.w;
                            const float eta = entering ? 1.0f / ior : ior;
                            const float ci = fmaxf(dot(wo, n), 0.0f);
                            const float fq = (ior - 1.0f) / (ior + 1.0f);
                            const float f0 = fq * fq;
                            const float fr = f0 + (1.0f - f0) * pow5(1.0f - ci);
                            float3 bt = f3(1, 1, 1);
                            float dist = 0.0f;
                            if (!entering) {
                                dist = fmaxf(h4.x, 0.0f);
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
                            delta_s = true;
                            has_dlw = !entering;  // Beer-Lambert: dlog att/dsigma = -dist
                            dlw = make_float4(-dist, -dist, -dist, 0.0f);
                            break;
                        }
                        case TPT_MAT_GGX: {
                            GgxSample gs;
                            if (!ggx_sample(rd, n, mt, rng, gs)) { ok = false; break; }
                            nd = gs.nd;
                            w = gs.w;
                            pdf = gs.pdf;
                            dlw = ggx_dlog(mt, gs.ci, gs.co, gs.ch, fabsf(dot(gs.nd, gs.mh)));
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
                            dlw = albedo_dlog(mc);
                            break;
                        }
                        default:
                            ok = false;
                    }
                    if (!ok) {
                        done = true;
                    } else {
                        const size_t e = (size_t)m.y * ns + slot;
                        sts(&A.vc[e], make_float4(0.0f, 0.0f, 0.0f, ifloat(has_dlw ? mid : -1)));
                        sts(&A.vg[e], dlw);
                        if (has_dlw) fl |= F_ADJ_OPEN;
                        beta = beta * w;
                        last_pdf = pdf;
                        fl = delta_s ? (fl & ~F_LAST_ND) : (fl | F_LAST_ND);
                        const float3 o2 = no + nd * kEps;
                        sts(&st.ray_o[slot], make_float4(o2.x, o2.y, o2.z, ifloat(self_ok ? prim : -1)));
                        sts(&st.ray_d[slot], make_float4(nd.x, nd.y, nd.z, ifloat(self_ok ? inst : -1)));
                        m.y += 1;
                        if (m.y >= P.max_bounces) done = true;  // bounce loop bound (:67)
                    }
                }
            }
            if (done && !sh_env && !sh_area) {
                // nothing pending: the sample ends here
                adj_final(A, g, slot, ns, m.y, fl, acc);
                cont = adj_next_sample(S, P, st, slot, m, fl, acc, beta, last_pdf, ptime, rng, need_task);
                finished_here = true;
            } else {
                cont = !done;
                term = done;
            }
            sts(&st.beta[slot], make_float4(beta.x, beta.y, beta.z, last_pdf));
            sts(&A.acc[slot], make_float4(acc.x, acc.y, acc.z, ptime));
            m.z = fl;
            store_path(st, slot, m, rng);
        }
        if (adj_take_task(S, P, st, A, slot, need_task)) cont = true;
        if (active) st.act[slot] = cont ? 1 : 0;
        if (!P.ordered_queue) warp_push(st.q_ext[nxt], &st.ctr->n_ext[nxt], cont, slot);
        warp_push(st.q_term, &st.ctr->n_term, term, slot);
        adj_warp_count(&st.ctr->n_done_in_shade, finished_here);
        warp_push(st.q_sh, &st.ctr->n_sh, sh_env != 0, 2 * slot);
        warp_push(st.q_sh, &st.ctr->n_sh, sh_area != 0, 2 * slot + 1);
    }
    grad_end(g, lin_k + 1);
}

// Samples that ended with shadow rays pending finish here, after the
// occlusion kernel has resolved them.
__global__ void __launch_bounds__(kAdjBlock) k_adj_regen(WfScene S, AdjParams P, WfState st, AdjWfState A,
                                                         double* gtot, int gmode, int cur, int n_slots) {
    extern __shared__ float gsh[];
    const int lin_k = 4 * P.n_mats;
    const GradAcc g = grad_begin(gsh, gtot, gmode, lin_k + 1);
    const int n = st.ctr->n_term;
    const int nxt = cur ^ 1;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const int i = base + (int)lane_id();
        bool again = false, need_task = false;
        int slot = 0;
        if (i < n) {
            slot = st.q_term[i];
            int4 m;
            uint64_t rng;
            load_path(st, slot, m, rng);
            int fl = m.z;
            const float4 a4 = lds(&A.acc[slot]);
            float ptime = a4.w;
            float3 acc = adj_take_pending(st, A, slot, fl, f3(a4), g, lin_k);
            adj_final(A, g, slot, n_slots, m.y, fl, acc);
            float3 beta = f3(1.0f, 1.0f, 1.0f);
            float last_pdf = 0.0f;
            again = adj_next_sample(S, P, st, slot, m, fl, acc, beta, last_pdf, ptime, rng, need_task);
            if (again) sts(&st.beta[slot], make_float4(1.0f, 1.0f, 1.0f, 0.0f));
            sts(&A.acc[slot], make_float4(acc.x, acc.y, acc.z, ptime));
            m.z = fl;
            store_path(st, slot, m, rng);
        }
        if (adj_take_task(S, P, st, A, slot, need_task)) again = true;
        if (i < n) st.act[slot] = again ? 1 : 0;
        if (!P.ordered_queue) warp_push(st.q_ext[nxt], &st.ctr->n_ext[nxt], again, slot);
    }
    grad_end(g, lin_k + 1);
}

// Totals out: gradients, paths and the linearised loss, device flags.
__global__ void k_adj_out(const double* __restrict__ gtot, int n_params, const WfCounters* ctr, double* grad,
                          unsigned long long* counters, int* flags) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n_params) grad[k] = gtot[k];
    if (k == 0) {
        counters[0] = ctr->samples;
        counters[1] = __double_as_longlong(gtot[n_params]);
        *flags |= ctr->flags;
    }
}

}  // namespace wf

cudaError_t adj_render_backward(const WfScene& S, const AdjParams& P, const float* d_dimg, double* d_grad, int* d_flags,
                                unsigned long long* d_counters, cudaStream_t s, int sm_count, float* elapsed_ms) {
    const size_t n_params = 4 * (size_t)P.n_mats;
    cudaError_t e = cudaMemsetAsync(d_grad, 0, n_params * sizeof(double), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_flags, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_counters, 0, 2 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    const size_t shared = n_params * sizeof(double);
    // 0: private partials, 1: shared f64 atomics, 2: global f64 atomics
    const int mode = n_params <= (size_t)wf::kPrivateParams ? 0 : (shared <= 32 * 1024 ? 1 : 2);
    const size_t dyn = mode == 1 ? shared : 0;
    // shared-memory traversal stack when the deepest path fits it
    const bool shared_stack = S.max_stack <= wf::kSharedStack;
    auto kern = shared_stack ? wf::k_adjoint<true> : wf::k_adjoint<false>;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, dyn);
    if (e != cudaSuccess) return e;
    long long grid = (long long)sm_count * (per_sm > 0 ? per_sm : 1);
    const long long need = (P.n_tasks + 127) / 128;
    if (grid > need) grid = need > 0 ? need : 1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (elapsed_ms) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, s);
    }
    kern<<<(unsigned)grid, 128, dyn, s>>>(S, P, d_dimg, d_grad, d_flags, d_counters, mode);
    e = cudaGetLastError();
    if (elapsed_ms) {
        cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.0f;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        *elapsed_ms = ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return e;
}

cudaError_t resolve_film(const double* acc, const double* acc_w, float* img, int n_pixels, cudaStream_t s) {
    if (n_pixels <= 0) return cudaSuccess;
    wf::k_resolve<<<(n_pixels + 255) / 256, 256, 0, s>>>(acc, acc_w, img, n_pixels);
    return cudaGetLastError();
}


// ---- wavefront adjoint: buffers and host driver ------------------------------------
cudaError_t adj_reserve(AdjBuffers& b, size_t slots, int max_bounces, int n_params) {
    const size_t nb = (size_t)(max_bounces > 0 ? max_bounces : 1);
    if (b.block && b.slots >= slots && b.bounces >= nb && b.params >= (size_t)n_params + 1) return cudaSuccess;
    adj_release(b);
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t S = slots;
    const size_t sz[] = {S * 16, S * nb * 16, S * nb * 16, 2 * S * 16, 2 * S * 16, 2 * S * 4,
                         ((size_t)n_params + 1) * 8};
    size_t total = 0;
    for (size_t x : sz) total += up(x);
    char* p = nullptr;
    cudaError_t e = cudaMalloc(&p, total);
    if (e != cudaSuccess) return e;
    b.block = p;
    b.slots = slots;
    b.bounces = nb;
    b.params = (size_t)n_params + 1;
    size_t off = 0;
    auto take = [&](size_t bytes) { char* r = p + off; off += up(bytes); return (void*)r; };
    b.st.acc = (float4*)take(sz[0]);
    b.st.vg = (float4*)take(sz[1]);
    b.st.vc = (float4*)take(sz[2]);
    b.st.sh_gm = (float4*)take(sz[3]);
    b.st.sh_gl = (float4*)take(sz[4]);
    b.st.sh_mat = (int*)take(sz[5]);
    b.gtot = (double*)take(sz[6]);
    return cudaSuccess;
}

void adj_release(AdjBuffers& b) {
    if (b.block) cudaFree(b.block);
    b = AdjBuffers{};
}

cudaError_t adj_render_backward_wf(const WfScene& S, const AdjParams& P0, WfBuffers& B, AdjBuffers& AB,
                                   long long pool, const float* d_dimg, double* d_grad, int* d_flags,
                                   unsigned long long* d_counters, cudaStream_t s, int sm_count, bool use_graph_loop,
                                   float* elapsed_ms, unsigned long long* culled_samples) {
    const int n_params = 4 * P0.n_mats;
    // Camera culling (pinhole cameras, as in the forward render): the pool
    // replays only the tasks of pixels a camera ray may reach geometry from.
    AdjParams P = P0;
    int n_may = P.n_pixels, n_open = 0;
    if (P.sky_cull && P.max_bounces > 0 && P.n_pixels > 0 && S.cam.lens_radius == 0.0f && S.cam.focus_dist > 0.0f) {
        WfParams CP{};
        CP.width = P.width; CP.height = P.height; CP.n_pixels = P.n_pixels;
        CP.row_begin = P.row_begin; CP.row_step = P.row_step; CP.w_div = P.w_div;
        CP.max_bounces = P.max_bounces;
        const cudaError_t ce = wf_cull_pixels(S, CP, B, s, &n_may, &n_open);
        if (ce != cudaSuccess) return ce;
    }
    if (n_open > 0) {
        P.geo_map = B.cull_map[0];
        P.n_geo = n_may;
        P.geo_div = make_fastdiv((uint32_t)std::max(n_may, 1));
    }
    if (culled_samples) *culled_samples = (unsigned long long)n_open * (unsigned long long)P.spp;
    const long long pooled = P.geo_map ? (long long)P.n_chunks * n_may : P.n_tasks;
    // the vertex lists bound the pool: at most 2 GB of them
    const long long per_slot = 32LL * (P.max_bounces > 0 ? P.max_bounces : 1);
    long long slots = std::min<long long>(pooled, pool);
    slots = std::min<long long>(slots, std::max<long long>(1, (2LL << 30) / std::max<long long>(per_slot, 1)));
    if (slots < 1) slots = 1;
    cudaError_t e = wf_reserve(B, (size_t)slots, 0);
    if (e == cudaSuccess) e = adj_reserve(AB, (size_t)slots, P.max_bounces, n_params);
    if (e != cudaSuccess) return e;
    WfState st = B.st;
    st.welford = nullptr;
    st.ssq = nullptr;
    st.part = nullptr;
    st.part_sq = nullptr;
    const AdjWfState A = AB.st;
    // trace kernels' view of the loop
    WfParams TP{};
    TP.n_slots = (int)slots;
    TP.trace_chunk = P.trace_chunk;
    TP.jobs = nullptr;
    TP.ext_queue = 1;
    TP.queue_div = P.queue_div;
    TP.ordered_queue = P.ordered_queue;
    const int rounds = (int)((pooled + slots - 1) / slots + 1);
    const long long max_iters = (long long)P.task_spp * (long long)(P.max_bounces + 1) * rounds + 16;
    int g_ext = 0, g_sh = 0;
    wf_trace_grids(sm_count, &g_ext, &g_sh);
    const int n_acc = n_params + 1;
    const int gmode = n_acc <= 65 ? 0 : (n_acc * 4 <= 32 * 1024 ? 1 : 2);
    const size_t dyn = gmode == 0 ? (size_t)n_acc * wf::kAdjBlock * 4 : (gmode == 1 ? (size_t)n_acc * 4 : 0);
    int occ_shade = 0, occ_regen = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_shade, wf::k_adj_shade, wf::kAdjBlock, dyn);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_regen, wf::k_adj_regen, wf::kAdjBlock, dyn);
    const int g_shade = sm_count * std::max(occ_shade, 1), g_regen = sm_count * std::max(occ_regen, 1);

    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (elapsed_ms) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, s);
    }
    e = cudaMemsetAsync(st.ctr, 0, sizeof(WfCounters), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(AB.gtot, 0, (size_t)n_acc * sizeof(double), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_flags, 0, sizeof(int), s);
    if (e == cudaSuccess && n_open > 0) {
        const long long count = (long long)P.n_chunks * n_open;
        wf::k_adj_sky<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(S, P, st, d_dimg, AB.gtot, n_params,
                                                                      B.cull_map[1], n_open,
                                                                      make_fastdiv((uint32_t)n_open), count);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        wf::k_adj_init<<<(unsigned)((slots + 255) / 256), 256, 0, s>>>(S, P, st, A, (int)slots);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        e = wf_run_loop([&](cudaStream_t q, cudaGraphConditionalHandle h, int use_cond) {
            for (int cur = 0; cur < 2; ++cur) {
                wf_launch_trace(false, g_ext, q, S, TP, st, cur);
                wf::k_adj_shade<<<g_shade, wf::kAdjBlock, dyn, q>>>(S, P, st, A, d_dimg, AB.gtot, gmode, cur, (int)slots);
                wf_launch_trace(true, g_sh, q, S, TP, st, cur);
                wf::k_adj_regen<<<g_regen, wf::kAdjBlock, dyn, q>>>(S, P, st, A, AB.gtot, gmode, cur, (int)slots);
                if (P.ordered_queue) wf_launch_compact(q, st, cur, (int)slots);
                wf_launch_step(q, st, cur, max_iters, h, use_cond);
            }
        }, st.ctr, max_iters, s, use_graph_loop);
    }
    if (e == cudaSuccess) {
        wf::k_adj_out<<<(unsigned)((n_params + 255) / 256 + 1), 256, 0, s>>>(AB.gtot, n_params, st.ctr, d_grad,
                                                                             d_counters, d_flags);
        e = cudaGetLastError();
    }
    if (elapsed_ms) {
        cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.0f;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        *elapsed_ms = ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    if (e != cudaSuccess) cudaGetLastError();
    return e;
}

}  // namespace tpt
