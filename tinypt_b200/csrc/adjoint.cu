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

namespace tpt {
namespace wf {

constexpr float kClamp = 50.0f;  // FIREFLY_CLAMP (src/constants.rs)

struct GradSink {
    double* sh;  // per-block shared copy, or nullptr
    double* gl;
    __device__ __forceinline__ void add(int k, float v) const {
        if (v != 0.0f) atomicAdd((sh ? sh : gl) + k, (double)v);
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

// One sample of radiance(), replayed.  grad = false: returns sum_k a_k.
// grad = true: A is that sum; gradients are scattered to `sink`.
__device__ __noinline__ float3 adj_path(const WfScene& S, const AdjParams& P, int x, int y, uint64_t& rng, float3 delta,
                                        float3 A, bool grad, const GradSink& sink, int* flags, float& lin) {
    const bool has_env = S.env_kind == TPT_ENV_MAP;
    int lstack[kStack];
    const TStack<1, kStack> stack{lstack};
    Tracer T;
    TraceCount cnt;
    float3 o, d;
    float ptime;
    camera_ray(S.cam, x, y, 1.0f / (float)P.width, 1.0f / (float)P.height, rng, o, d, ptime);
    int self_prim = -1, self_inst = -1;
    float3 beta = f3(1.0f, 1.0f, 1.0f);
    float last_pdf = 0.0f;
    bool last_nd = false;
    float3 sum = f3(0.0f, 0.0f, 0.0f);
    for (int bounce = 0; bounce < P.max_bounces; ++bounce) {
        tracer_start(S, T, o, d, kTMax, self_prim, self_inst);
        tracer_run<false, false>(S, T, stack, kEps, 1 << 30, flags, cnt);
        const int prim = T.hit_prim, inst = T.hit_inst;
        const float th = T.tmax;
        if (prim < 0) {  // miss (:71-83)
            float3 bg;
            if (has_env) {
                bg = env_lookup(S, d);
            } else {
                const float t = 0.5f * (d.y + 1.0f);
                bg = f3(0.9f, 0.95f, 1.0f) * (1.0f - t) + f3(0.6f, 0.75f, 1.0f) * t;
            }
            float3 c = beta * bg;
            if (has_env && last_nd) c = c * mis(last_pdf, env_pdf(S, d));
            const float3 a = adj_weight(c, delta, true);
            if (grad) A = A - a; else { sum = sum + a; lin += dot(delta, clamp_lum(c, kClamp)); }
            break;
        }
        if (bounce >= P.rr_start) {  // Russian roulette (:89-95), probability detached
            const float p = fmaxf(fminf(max3(beta), 0.95f), 0.05f);
            if (pcg_f32(rng) > p) break;
            beta = beta / p;
        }
        const float3 hp = o + d * th;
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
            const float3 a = adj_weight(beta * mc, delta, true);
            if (grad) {
                A = A - a;
                sink.add_rgb(mid, f3(a.x * inv_or_zero(mc.x), a.y * inv_or_zero(mc.y), a.z * inv_or_zero(mc.z)));
            } else {
                sum = sum + a;
                lin += dot(delta, clamp_lum(beta * mc, kClamp));
            }
            break;
        }
        const bool entering = dot(ng, d) < 0.0f;
        const float3 n = entering ? ng : -ng;
        const float3 wo = -d;
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
                        tracer_start(S, T, hp + wi * kEps, wi, kTMax, prim, inst);
                        tracer_run<true, false>(S, T, stack, kEps, 1 << 30, flags, cnt);
                        if (T.hit_prim < 0) {
                            const float3 a = delta * contrib;
                            if (grad) {
                                A = A - a;
                                eval_grad(sink, mid, mt, wo, wi, n, a);
                            } else {
                                sum = sum + a;
                                lin += dot(delta, contrib);
                            }
                        }
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
                    if (c > 0.0f && !ref_light_self_occluded(S, lidx, hp, lud, lvd, (double)ptime)) {
                        float3 f;
                        float pb;
                        mat_eval(mt, wo, wi, n, f, pb);
                        const float3 contrib = beta * f * le * (c * mis(lpdf, pb) / lpdf);
                        if (contrib.x > 0.0f || contrib.y > 0.0f || contrib.z > 0.0f) {
                            tracer_start(S, T, hp + wi * kEps, wi, fmaxf(dist - 2.0f * kEps, kEps), prim, inst);
                            tracer_run<true, false>(S, T, stack, kEps, 1 << 30, flags, cnt);
                            if (T.hit_prim < 0) {
                                const float3 a = delta * contrib;
                                if (grad) {
                                    A = A - a;
                                    eval_grad(sink, mid, mt, wo, wi, n, a);
                                    const int lm = __ldg(&S.lights[lidx].mat);
                                    sink.add_rgb(lm, f3(a.x * inv_or_zero(le.x), a.y * inv_or_zero(le.y),
                                                        a.z * inv_or_zero(le.z)));
                                } else {
                                    sum = sum + a;
                                    lin += dot(delta, contrib);
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
            nd = cos_hemi(n, rng);
            w = mc;
            pdf = fmaxf(dot(n, nd), 0.0f) / kPi;
            if (grad) sink.add_rgb(mid, f3(A.x * inv_or_zero(mc.x), A.y * inv_or_zero(mc.y), A.z * inv_or_zero(mc.z)));
        } else if (mt.kind == TPT_MAT_METAL) {
            nd = d - n * (2.0f * dot(d, n));
            w = mc;
            delta_s = true;
            if (grad) sink.add_rgb(mid, f3(A.x * inv_or_zero(mc.x), A.y * inv_or_zero(mc.y), A.z * inv_or_zero(mc.z)));
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
            const bool refl = !has_refr || pcg_f32(rng) < fr;
            if (refl) {
                nd = d - n * (2.0f * dot(d, n));
                bt = bt * (fr / fmaxf(fr, 1e-6f));
            } else {
                nd = d * eta + n * (eta * cosi - sqrtf(1.0f - sin2t));
                bt = bt * ((1.0f - fr) / fmaxf(1.0f - fr, 1e-6f)) * (eta * eta);
            }
            w = bt;
            delta_s = true;
            if (grad && !entering) sink.add_rgb(mid, A * (-dist));  // Beer-Lambert: dlog att/dsigma = -dist
        } else if (mt.kind == TPT_MAT_GGX) {
            GgxSample gs;
            if (!ggx_sample(d, n, mt, rng, gs)) break;
            nd = gs.nd;
            w = gs.w;
            pdf = gs.pdf;
            if (grad) ggx_grad(sink, mid, mt, gs.ci, gs.co, gs.ch, fabsf(dot(gs.nd, gs.mh)), A);
        } else if (mt.kind == TPT_MAT_SUBSURFACE) {
            const float sc = fmaxf(mt.c.w, 1e-4f);
            const float u = fmaxf(pcg_f32(rng), 1e-12f);
            const float dist = -__logf(u) * sc;
            nd = cos_hemi(ng, rng);  // unoriented normal (material.rs:187-188)
            w = mc * __expf(-dist / sc);
            no = hp - ng * dist;
            pdf = fmaxf(dot(n, nd), 0.0f) / kPi;
            self_ok = false;
            if (grad) sink.add_rgb(mid, f3(A.x * inv_or_zero(mc.x), A.y * inv_or_zero(mc.y), A.z * inv_or_zero(mc.z)));
        } else {
            break;
        }
        beta = beta * w;
        last_pdf = pdf;
        last_nd = !delta_s;
        o = no + nd * kEps;
        d = nd;
        self_prim = self_ok ? prim : -1;
        self_inst = self_ok ? inst : -1;
    }
    return sum;
}

__global__ void __launch_bounds__(128) k_adjoint(WfScene S, AdjParams P, const float* __restrict__ dimg,
                                                 double* __restrict__ grad, int* flags,
                                                 unsigned long long* counters, int use_shared) {
    extern __shared__ double sgrad[];
    const int n_params = 4 * P.n_mats;
    if (use_shared) {
        for (int k = threadIdx.x; k < n_params; k += blockDim.x) sgrad[k] = 0.0;
        __syncthreads();
    }
    const GradSink sink{use_shared ? sgrad : nullptr, grad};
    const long long stride = (long long)gridDim.x * blockDim.x;
    unsigned long long paths = 0;
    double lin = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < P.n_tasks; t += stride) {
        const int pixel = (int)(t % P.n_pixels);
        const int chunk = (int)(t / P.n_pixels);
        const int x = pixel % P.width, y = pixel / P.width;
        const float inv_spp = 1.0f / (float)P.spp;
        const float3 delta = f3(dimg[3 * (size_t)pixel], dimg[3 * (size_t)pixel + 1], dimg[3 * (size_t)pixel + 2]) * inv_spp;
        if (delta.x == 0.0f && delta.y == 0.0f && delta.z == 0.0f) continue;  // no gradient through this pixel
        uint64_t rng = task_seed((uint32_t)x, (uint32_t)y, (uint32_t)(chunk * P.task_spp), P.seed);
        const int n = min(P.task_spp, P.spp - chunk * P.task_spp);
        for (int s = 0; s < n; ++s) {
            uint64_t replay = rng;
            float lp = 0.0f, unused = 0.0f;
            const float3 A = adj_path(S, P, x, y, rng, delta, f3(0, 0, 0), false, sink, flags, lp);
            adj_path(S, P, x, y, replay, delta, A, true, sink, flags, unused);
            lin += (double)lp;
            ++paths;
        }
    }
    if (paths) atomicAdd(counters, paths);
    if (lin != 0.0) atomicAdd(reinterpret_cast<double*>(counters + 1), lin);
    if (use_shared) {
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

}  // namespace wf

cudaError_t adj_render_backward(const WfScene& S, const AdjParams& P, const float* d_dimg, double* d_grad, int* d_flags,
                                unsigned long long* d_counters, cudaStream_t s, int sm_count, float* elapsed_ms) {
    const size_t n_params = 4 * (size_t)P.n_mats;
    cudaError_t e = cudaMemsetAsync(d_grad, 0, n_params * sizeof(double), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_flags, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_counters, 0, 2 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    const size_t shared = n_params * sizeof(double);
    const int use_shared = shared <= 32 * 1024 ? 1 : 0;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wf::k_adjoint, 128, use_shared ? shared : 0);
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
    wf::k_adjoint<<<(unsigned)grid, 128, use_shared ? shared : 0, s>>>(S, P, d_dimg, d_grad, d_flags, d_counters,
                                                                       use_shared);
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

}  // namespace tpt
