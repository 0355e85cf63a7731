// Plain f64 form of the path integrator: one thread per pixel runs the
// pixel's samples in order, continuing the reference's per-pixel RNG stream
// (src/render.rs:141-158) through radiance() (src/integrator.rs:53-135) with
// the reference's f64 arithmetic.  This translation unit is compiled with
// -fmad=false so a*b+c rounds twice, as in the reference; f64 division and
// sqrt are IEEE-rounded on the GPU.  Transcendentals come from CUDA's libm,
// whose last-bit results can differ from glibc's, so a pixel's stream can
// diverge from the reference's after such a difference flips a branch.
#include "plain_f64.cuh"

namespace tpt {
namespace plain {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kTau = 6.28318530717958647692528676655900577;
constexpr double kEps = 1e-4;     // RAY_EPSILON (src/constants.rs:4)
constexpr double kTMax = 1e30;    // RAY_T_MAX (src/constants.rs:7)
constexpr int kStack = 64;        // bvh.rs:255 fixed stack

struct V { double x, y, z; };
__device__ __forceinline__ V mk(double x, double y, double z) { return V{x, y, z}; }
__device__ __forceinline__ V ld(const double* p) { return V{p[0], p[1], p[2]}; }
__device__ __forceinline__ V operator+(V a, V b) { return V{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V operator-(V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V operator-(V a) { return V{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V operator*(V a, double s) { return V{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V operator*(double s, V a) { return a * s; }
__device__ __forceinline__ V operator/(V a, double s) { return V{a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ V had(V a, V b) { return V{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ double dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V cross(V a, V b) { return V{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ double len(V a) { return sqrt(dot(a, a)); }
__device__ __forceinline__ V norm(V a) { double l = fmax(len(a), 1e-30); return a / l; }
__device__ __forceinline__ double lum(V c) { return 0.2126 * c.x + 0.7152 * c.y + 0.0722 * c.z; }
__device__ __forceinline__ V clamp_lum(V c, double m) {             // math.rs:42-49
    double l = lum(c);
    return (l > m && l > 0.0) ? c * (m / l) : c;
}
__device__ __forceinline__ V reflect(V v, V n) { return v - (2.0 * dot(v, n)) * n; }  // math.rs:193
__device__ __forceinline__ double clampd(double x, double a, double b) { return fmin(fmax(x, a), b); }
// Rust `f as usize` (saturating; NaN -> 0) for the small ranges used here.
__device__ __forceinline__ size_t as_usize(double f) { return f > 0.0 ? (size_t)f : 0; }

struct Ray { V o, d; double time; };
struct Hit { double t; V p, n; int mat; };

struct Ctx {
    const PlainScene* S;
    uint32_t shadow_rays;
    uint32_t closest_rays;
    int* flags;
};

// ---- src/geometry.rs ------------------------------------------------------
__device__ bool box_hit(const double* bmin, const double* bmax, const Ray& r, V inv, double tmin, double tmax,
                        double* t_enter) {  // Aabb::hit_inv / hit_range_inv (:117-165)
    double t0 = (bmin[0] - r.o.x) * inv.x, t1 = (bmax[0] - r.o.x) * inv.x;
    tmin = fmax(tmin, fmin(t0, t1)); tmax = fmin(tmax, fmax(t0, t1));
    if (tmax <= tmin) return false;
    t0 = (bmin[1] - r.o.y) * inv.y; t1 = (bmax[1] - r.o.y) * inv.y;
    tmin = fmax(tmin, fmin(t0, t1)); tmax = fmin(tmax, fmax(t0, t1));
    if (tmax <= tmin) return false;
    t0 = (bmin[2] - r.o.z) * inv.z; t1 = (bmax[2] - r.o.z) * inv.z;
    tmin = fmax(tmin, fmin(t0, t1)); tmax = fmin(tmax, fmax(t0, t1));
    if (tmax <= tmin) return false;
    if (t_enter) *t_enter = tmin;
    return true;
}

__device__ bool tri_hit(const TriF64& tr, const Ray& r, double tmin, double tmax, Hit& h) {  // :236-273
    const double t = r.time;
    V v0 = ld(tr.v0) * (1.0 - t) + ld(tr.v0) * t;  // vertices_at (:212-218), static
    V v1 = ld(tr.v1) * (1.0 - t) + ld(tr.v1) * t;
    V v2 = ld(tr.v2) * (1.0 - t) + ld(tr.v2) * t;
    V e1 = v1 - v0, e2 = v2 - v0;
    V pvec = cross(r.d, e2);
    double det = dot(e1, pvec);
    if (fabs(det) < 1e-10) return false;
    double inv_det = 1.0 / det;
    V tvec = r.o - v0;
    double u = dot(tvec, pvec) * inv_det;
    if (u < 0.0 || u > 1.0) return false;
    V qvec = cross(tvec, e1);
    double v = dot(r.d, qvec) * inv_det;
    if (v < 0.0 || u + v > 1.0) return false;
    double th = dot(e2, qvec) * inv_det;
    if (th < tmin || th > tmax) return false;
    h.t = th;
    h.p = r.o + r.d * th;
    h.n = norm(cross(e1, e2));
    h.mat = tr.mat;
    return true;
}

__device__ bool sphere_hit(const SphereF64& s, const Ray& r, double tmin, double tmax, Hit& h) {  // :174-195
    V c = ld(s.c);
    V oc = r.o - c;
    double a = dot(r.d, r.d);
    double b = dot(oc, r.d);
    double cc = dot(oc, oc) - s.r * s.r;
    double d = b * b - a * cc;
    if (d <= 0.0) return false;
    double sd = sqrt(d);
    double t = (-b - sd) / a;
    if (t < tmin || t > tmax) {
        t = (-b + sd) / a;
        if (t < tmin || t > tmax) return false;
    }
    h.t = t;
    h.p = r.o + r.d * t;
    h.n = (h.p - c) / s.r;
    h.mat = s.mat;
    return true;
}

// ---- src/bvh.rs:248-351 ---------------------------------------------------
__device__ bool bvh_hit(Ctx& cx, const MeshF64& m, const Ray& r, double tmin, double tmax, Hit& best) {
    if (m.n_nodes == 0) return false;
    const NodeF64* nodes = cx.S->nodes + m.node_offset;
    const TriF64* tris = cx.S->tris + m.tri_offset;
    V inv = mk(1.0 / r.d.x, 1.0 / r.d.y, 1.0 / r.d.z);
    int stack[kStack];
    int sp = 0;
    stack[sp++] = 0;
    bool found = false;
    while (sp > 0) {
        const NodeF64& n = nodes[stack[--sp]];
        if (!box_hit(n.bmin, n.bmax, r, inv, tmin, tmax, nullptr)) continue;
        if (n.left == -1 && n.right == -1) {
            for (uint32_t k = n.start; k < n.start + n.count; ++k) {
                Hit h;
                if (tri_hit(tris[k], r, tmin, tmax, h)) { tmax = h.t; best = h; found = true; }
            }
            continue;
        }
        int a_id = n.left, b_id = n.right;
        int push[2];
        int np = 0;
        if (a_id == -1) {
            if (b_id != -1) push[np++] = b_id;
        } else if (b_id == -1) {
            push[np++] = a_id;
        } else {
            double ta, tb;
            bool ha = box_hit(nodes[a_id].bmin, nodes[a_id].bmax, r, inv, tmin, tmax, &ta);
            bool hb = box_hit(nodes[b_id].bmin, nodes[b_id].bmax, r, inv, tmin, tmax, &tb);
            if (ha && hb) {
                if (ta <= tb) { push[np++] = b_id; push[np++] = a_id; }  // far then near
                else { push[np++] = a_id; push[np++] = b_id; }
            } else if (ha) {
                push[np++] = a_id;
            } else if (hb) {
                push[np++] = b_id;
            }
        }
        for (int k = 0; k < np; ++k) {
            if (sp < kStack) stack[sp++] = push[k];
            else raise_flag(cx.flags, TPT_FLAG_STACK_OVERFLOW);
        }
    }
    return found;
}

__device__ V xf_point(const InstanceF64& x, V p) {          // apply_point (transform.rs:75-77)
    const double* a = x.a;
    return mk(a[0] * p.x + a[1] * p.y + a[2] * p.z, a[3] * p.x + a[4] * p.y + a[5] * p.z,
              a[6] * p.x + a[7] * p.y + a[8] * p.z) + ld(x.t);
}
__device__ V mat_vec(const double* a, V p) {
    return mk(a[0] * p.x + a[1] * p.y + a[2] * p.z, a[3] * p.x + a[4] * p.y + a[5] * p.z,
              a[6] * p.x + a[7] * p.y + a[8] * p.z);
}

// World::hit (src/world.rs:81-121)
__device__ bool world_hit(Ctx& cx, const Ray& r, double tmin, double tmax, Hit& best) {
    const PlainScene& S = *cx.S;
    double closest = tmax;
    bool found = false;
    for (int i = 0; i < S.n_instances; ++i) {
        const InstanceF64& inst = S.instances[i];
        const MeshF64& mesh = S.meshes[inst.mesh_id];
        Ray ro{mat_vec(inst.a_inv, r.o - ld(inst.t)), norm(mat_vec(inst.a_inv, r.d)), r.time};
        Hit h;
        if (bvh_hit(cx, mesh, ro, tmin, 1e30, h)) {
            V p_world = xf_point(inst, h.p);
            V n_world = norm(mat_vec(inst.nmat, h.n));
            double t_world = dot(p_world - r.o, r.d);
            if (t_world > tmin && t_world < closest) {
                closest = t_world;
                best = Hit{t_world, p_world, n_world, inst.mat_override >= 0 ? inst.mat_override : h.mat};
                found = true;
            }
        }
    }
    for (int i = 0; i < S.n_spheres; ++i) {
        Hit h;
        if (sphere_hit(S.spheres[i], r, tmin, closest, h)) { closest = h.t; best = h; found = true; }
    }
    return found;
}

// ---- src/material.rs -------------------------------------------------------
__device__ __forceinline__ double pow5(double x) { double x2 = x * x; return x2 * x2 * x; }
__device__ V fresnel_schlick(double c, V f0) {
    double x = 1.0 - fmax(c, 0.0);
    return f0 + (mk(1.0, 1.0, 1.0) - f0) * pow5(x);
}
__device__ double ggx_d(double alpha, double ch) {
    if (ch <= 0.0) return 0.0;
    double a2 = alpha * alpha;
    double den = ch * ch * (a2 - 1.0) + 1.0;
    return a2 / (kPi * den * den);
}
__device__ double ggx_g1(double alpha, double c) {
    if (c <= 0.0) return 0.0;
    double a = alpha * sqrt(fmax(1.0 - c * c, 0.0)) / fmax(c, 1e-6);
    return 2.0 / (1.0 + sqrt(1.0 + a * a));
}
__device__ V ggx_eval(V albedo, double alpha, V n, V wo, V wi) {
    double ci = dot(n, wo), co = dot(n, wi);
    if (ci <= 0.0 || co <= 0.0) return mk(0, 0, 0);
    V m = norm(wo + wi);
    double ch = fmax(dot(n, m), 0.0);
    double d = ggx_d(alpha, ch);
    double g = ggx_g1(alpha, ci) * ggx_g1(alpha, co);
    V f = fresnel_schlick(fabs(dot(wi, m)), albedo);
    double den = 4.0 * ci * co + 1e-6;
    return f * (d * g / den);
}
__device__ double ggx_pdf(double alpha, V n, V wo, V wi) {
    double ci = dot(n, wo), co = dot(n, wi);
    if (ci <= 0.0 || co <= 0.0) return 0.0;
    V m = norm(wo + wi);
    double ch = fmax(dot(n, m), 0.0);
    double d = ggx_d(alpha, ch);
    double g1 = ggx_g1(alpha, ci);
    double pdf_m = d * g1 * ch / fmax(ci, 1e-6);
    double den = 4.0 * fmax(fabs(dot(wi, m)), 1e-6);
    return fmax(pdf_m / den, 0.0);
}
__device__ void tangent_frame(V n, V& t, V& b) {
    V a = fabs(n.x) > 0.9 ? mk(0, 1, 0) : mk(1, 0, 0);
    t = norm(cross(n, a));
    b = cross(t, n);
}
__device__ V cos_hemi(V n, uint64_t& rng) {
    double u = pcg_f64(rng);
    double v = pcg_f64(rng);
    double r = sqrt(u);
    double phi = 2.0 * kPi * v;
    double x = r * cos(phi), y = r * sin(phi), z = sqrt(1.0 - u);
    V t, b;
    tangent_frame(n, t, b);
    return t * x + b * y + n * z;
}
__device__ V vndf(V wo, double alpha, double u1, double u2) {
    V v = norm(mk(alpha * wo.x, alpha * wo.y, wo.z));
    V t1, t2;
    if (v.z < 0.9999) { t1 = norm(mk(-v.y, v.x, 0.0)); t2 = cross(v, t1); }
    else { t1 = mk(1, 0, 0); t2 = mk(0, 1, 0); }
    double r = sqrt(u1);
    double phi = kTau * u2;
    double t1p = r * cos(phi);
    double t2pi = r * sin(phi);
    double s = 0.5 * (1.0 + v.z);
    double t2p = sqrt(1.0 - s) * t2pi + s * sqrt(fmax(1.0 - t1p * t1p, 0.0));
    V nh = norm(t1 * t1p + t2 * t2p + v * sqrt(fmax(1.0 - t1p * t1p - t2p * t2p, 0.0)));
    return norm(mk(alpha * nh.x, alpha * nh.y, nh.z));
}

struct Bsdf { Ray ray; V w; double pdf; bool delta; };

__device__ bool mat_sample(const MaterialF64& m, const Ray& in, const Hit& h, uint64_t& rng, Bsdf& s) {  // :76-201
    bool entering = dot(h.n, in.d) < 0.0;
    V n = entering ? h.n : -h.n;
    V c = ld(m.c);
    switch (m.kind) {
        case TPT_MAT_LAMBERT: {
            V d = cos_hemi(n, rng);
            s = Bsdf{Ray{h.p + kEps * d, d, in.time}, c, fmax(dot(n, d), 0.0) / kPi, false};
            return true;
        }
        case TPT_MAT_METAL: {
            V d = reflect(in.d, n);
            s = Bsdf{Ray{h.p + kEps * d, d, in.time}, c, 0.0, true};
            return true;
        }
        case TPT_MAT_DIELECTRIC: {
            double ior = m.p;
            double eta = entering ? 1.0 / ior : ior;
            double ci = fmax(dot(-in.d, n), 0.0);
            double fq = (ior - 1.0) / (ior + 1.0);
            double f0 = fq * fq;
            double fr = f0 + (1.0 - f0) * pow5(1.0 - ci);
            V beta = mk(1, 1, 1);
            if (!entering) {
                double dist = fmax(h.t, 0.0);
                beta = had(beta, mk(exp(-c.x * dist), exp(-c.y * dist), exp(-c.z * dist)));
            }
            V refl = reflect(in.d, n);
            // refract (math.rs:199-207)
            double cosi = fmin(fmax(dot(-in.d, n), -1.0), 1.0);
            double sin2t = eta * eta * (1.0 - cosi * cosi);
            bool has_refr = !(sin2t >= 1.0);
            V refr = mk(0, 0, 0);
            if (has_refr) {
                double cost = sqrt(1.0 - sin2t);
                refr = eta * in.d + (eta * cosi - cost) * n;
            }
            bool choose_refl = !has_refr || pcg_f64(rng) < fr;
            V d;
            if (choose_refl) {
                beta = beta * (fr / fmax(fr, 1e-6));
                d = refl;
            } else {
                double sc = (1.0 - fr) / fmax(1.0 - fr, 1e-6);
                beta = beta * sc * (eta * eta);
                d = refr;
            }
            s = Bsdf{Ray{h.p + kEps * d, d, in.time}, beta, 0.0, true};
            return true;
        }
        case TPT_MAT_GGX: {
            double av = fmax(m.p, 1e-3);
            V t, b;
            tangent_frame(n, t, b);
            V wo = norm(-in.d);
            V wl = mk(dot(wo, t), dot(wo, b), dot(wo, n));
            if (wl.z <= 0.0) return false;
            double u1 = pcg_f64(rng);
            double u2 = pcg_f64(rng);
            V ml = vndf(wl, av, u1, u2);
            V mh = t * ml.x + b * ml.y + n * ml.z;
            V d = reflect(in.d, mh);
            double co = dot(d, n);
            double ci = dot(-in.d, n);
            if (co <= 1e-6 || ci <= 1e-6) return false;
            double ch = fmax(dot(n, mh), 0.0);
            double dg = ggx_d(av, ch);
            double g = ggx_g1(av, ci) * ggx_g1(av, co);
            V f = fresnel_schlick(fabs(dot(d, mh)), c);
            double den = 4.0 * ci * co + 1e-6;
            V spec = f * (dg * g / den);
            double pdf = ggx_pdf(av, n, wo, d);
            s = Bsdf{Ray{h.p + kEps * d, d, in.time}, spec * (co / fmax(pdf, 1e-6)), pdf, false};
            return true;
        }
        case TPT_MAT_SUBSURFACE: {
            double sc = fmax(m.p, 1e-4);
            double u = fmax(pcg_f64(rng), 1e-12);
            double dist = -log(u) * sc;
            V no = h.n;
            V d = cos_hemi(no, rng);
            V att = c * exp(-dist / sc);
            V o = h.p - no * dist + kEps * d;
            s = Bsdf{Ray{o, d, in.time}, att, fmax(dot(n, d), 0.0) / kPi, false};
            return true;
        }
        default:
            return false;
    }
}

__device__ void mat_eval(const MaterialF64& m, V wo, V wi, V n, V& f, double& pdf) {  // :207-223
    if (m.kind == TPT_MAT_LAMBERT || m.kind == TPT_MAT_SUBSURFACE) {
        double c = fmax(dot(n, wi), 0.0);
        if (c <= 0.0) { f = mk(0, 0, 0); pdf = 0.0; return; }
        f = ld(m.c) * (1.0 / kPi);
        pdf = c / kPi;
        return;
    }
    if (m.kind == TPT_MAT_GGX) {
        double a = fmax(m.p, 1e-3);
        f = ggx_eval(ld(m.c), a, n, wo, wi);
        pdf = ggx_pdf(a, n, wo, wi);
        return;
    }
    f = mk(0, 0, 0);
    pdf = 0.0;
}

// ---- src/env.rs ------------------------------------------------------------
__device__ V env_lookup(const PlainScene& S, V dir) {                        // :92-121
    V d = norm(dir);
    double theta = acos(clampd(d.y, -1.0, 1.0));
    double phi = atan2(d.z, d.x);
    if (phi < 0.0) phi += kTau;
    double u = phi / kTau, v = theta / kPi;
    const size_t W = (size_t)S.env_w, H = (size_t)S.env_h;
    double x = u * (double)W;
    double y = v * ((double)H - 1.0);
    size_t x0 = as_usize(floor(x)) % W;
    size_t x1 = (x0 + 1) % W;
    size_t y0 = as_usize(floor(clampd(y, 0.0, (double)(H - 1))));
    size_t y1 = y0 + 1 < H - 1 ? y0 + 1 : H - 1;
    double fx = x - floor(x), fy = y - floor(y);
    const double* D = S.env_data;
    V c00 = ld(D + 3 * (y0 * W + x0)), c10 = ld(D + 3 * (y0 * W + x1));
    V c01 = ld(D + 3 * (y1 * W + x0)), c11 = ld(D + 3 * (y1 * W + x1));
    V c0 = c00 * (1.0 - fx) + c10 * fx;
    V c1 = c01 * (1.0 - fx) + c11 * fx;
    return c0 * (1.0 - fy) + c1 * fy;
}
__device__ double env_pdf(const PlainScene& S, V dir) {                      // :156-182
    if (S.env_total <= 0.0) return 1.0 / (4.0 * kPi);
    V d = norm(dir);
    double theta = acos(clampd(d.y, -1.0, 1.0));
    double phi = atan2(d.z, d.x);
    if (phi < 0.0) phi += kTau;
    double u = phi / kTau, v = theta / kPi;
    const size_t W = (size_t)S.env_w, H = (size_t)S.env_h;
    double fxw = floor(u * (double)W), fyh = floor(v * (double)H);
    fxw = fxw < 0.0 ? 0.0 : (fxw > (double)(W - 1) ? (double)(W - 1) : fxw);
    fyh = fyh < 0.0 ? 0.0 : (fyh > (double)(H - 1) ? (double)(H - 1) : fyh);
    size_t x = as_usize(fxw), y = as_usize(fyh);
    double th0 = kPi * (double)y / (double)H, th1 = kPi * (double)(y + 1) / (double)H;
    double st = fmax(sin(theta), 1e-6);
    double rw = fmax(cos(th0) - cos(th1), 0.0);
    double l = fmax(lum(ld(S.env_data + 3 * (y * W + x))), 0.0);
    double wgt = l * rw;
    if (wgt <= 0.0) return 0.0;
    double pdf_uv = (wgt / S.env_total) * (double)W * (double)H;
    return pdf_uv / (2.0 * kPi * kPi * st);
}
__device__ size_t cdf_search(const double* cdf, size_t n, double x) {      // env.rs:185-197, world.rs:324-336
    size_t lo = 0, hi = n == 0 ? 0 : n - 1;
    while (lo + 1 < hi) {
        size_t mid = (lo + hi) / 2;
        if (cdf[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}
__device__ void env_uniform(const PlainScene& S, uint64_t& rng, V& dir, V& rad, double& pdf) {  // :200-210
    double u = pcg_f64(rng), v = pcg_f64(rng);
    double z = 1.0 - 2.0 * u;
    double r = sqrt(fmax(1.0 - z * z, 0.0));
    double phi = kTau * v;
    dir = mk(r * cos(phi), z, r * sin(phi));
    rad = env_lookup(S, dir);
    pdf = 1.0 / (4.0 * kPi);
}
__device__ void env_sample_dir(const PlainScene& S, uint64_t& rng, V& dir, V& rad, double& pdf) {  // :124-152
    if (S.env_total <= 0.0) { env_uniform(S, rng, dir, rad, pdf); return; }
    const size_t W = (size_t)S.env_w, H = (size_t)S.env_h;
    double r0 = pcg_f64(rng) * S.env_total;
    size_t y = cdf_search(S.env_row_cdf, H + 1, r0);
    if (y > H - 1) y = H - 1;
    double row_sum = fmax(S.env_row_cdf[y + 1] - S.env_row_cdf[y], 0.0);
    if (row_sum <= 0.0) { env_uniform(S, rng, dir, rad, pdf); return; }
    double r1 = pcg_f64(rng) * row_sum;
    size_t x = cdf_search(S.env_col_cdf + y * (W + 1), W + 1, r1);
    if (x > W - 1) x = W - 1;
    double u = ((double)x + pcg_f64(rng)) / (double)W;
    double v = ((double)y + pcg_f64(rng)) / (double)H;
    double theta = kPi * v, phi = kTau * u;
    double st = sin(theta);
    dir = mk(cos(phi) * st, cos(theta), sin(phi) * st);
    rad = env_lookup(S, dir);
    pdf = env_pdf(S, dir);
}

// ---- src/world.rs:171-272 --------------------------------------------------
__device__ bool sample_light(const PlainScene& S, uint64_t& rng, double time, V p, V& pos, V& nrm, V& emit,
                             double& pdf) {
    if (S.light_total <= 0.0 || S.n_lights == 0) return false;
    double r = pcg_f64(rng) * S.light_total;
    size_t idx = cdf_search(S.light_cdf, (size_t)S.n_lights, r);
    if (idx > (size_t)S.n_lights - 1) idx = (size_t)S.n_lights - 1;
    const LightF64& L = S.lights[idx];
    double pdf_sel = L.weight / S.light_total;
    double area;
    if (L.is_sphere) {
        const SphereF64& s = S.spheres[L.sphere];
        double u = pcg_f64(rng), v = pcg_f64(rng);
        double z = 1.0 - 2.0 * u;
        double rr = sqrt(fmax(1.0 - z * z, 0.0));
        double phi = kTau * v;
        V dir = mk(rr * cos(phi), z, rr * sin(phi));
        pos = ld(s.c) + dir * s.r;
        nrm = dir;
        area = 4.0 * kPi * s.r * s.r;
    } else {
        const InstanceF64& inst = S.instances[L.inst];
        V w0 = xf_point(inst, ld(L.v) * (1.0 - time) + ld(L.v) * time);
        V w1 = xf_point(inst, ld(L.v + 3) * (1.0 - time) + ld(L.v + 3) * time);
        V w2 = xf_point(inst, ld(L.v + 6) * (1.0 - time) + ld(L.v + 6) * time);
        double u = pcg_f64(rng), v = pcg_f64(rng);
        double su = sqrt(u);
        double b0 = 1.0 - su, b1 = v * su, b2 = 1.0 - b0 - b1;
        pos = w0 * b0 + w1 * b1 + w2 * b2;
        V nn = cross(w1 - w0, w2 - w0);
        area = 0.5 * len(nn);
        nrm = area > 0.0 ? nn / (2.0 * area) : mk(0.0, 1.0, 0.0);
    }
    if (area <= 0.0) return false;
    V tl = pos - p;
    double d2 = dot(tl, tl);
    if (d2 <= 1e-12) return false;
    double dist = sqrt(d2);
    V wi = tl / dist;
    double cl = fmax(dot(nrm, -wi), 0.0);
    if (cl <= 0.0) return false;
    double pdf_area = 1.0 / area;
    double pdf_omega = pdf_area * d2 / cl;
    pdf = pdf_sel * pdf_omega;
    if (pdf <= 0.0) return false;
    emit = ld(L.emit);
    return true;
}

// ---- src/integrator.rs -----------------------------------------------------
__device__ __forceinline__ double mis(double a, double b) {
    double a2 = a * a, b2 = b * b;
    return (a2 + b2 > 0.0) ? a2 / (a2 + b2) : 0.0;
}

__device__ V radiance(Ctx& cx, Ray ray, uint64_t& rng, int max_bounces, int rr_start) {  // :53-135
    const PlainScene& S = *cx.S;
    const bool has_env = S.env_kind == TPT_ENV_MAP;
    V acc = mk(0, 0, 0), beta = mk(1, 1, 1);
    double last_pdf = 0.0;
    bool last_nd = false;
    for (int bounce = 0; bounce < max_bounces; ++bounce) {
        Hit hit;
        cx.closest_rays++;
        if (!world_hit(cx, ray, kEps, kTMax, hit)) {
            V bg;
            if (has_env) {
                bg = env_lookup(S, ray.d);
            } else {
                double t = 0.5 * (ray.d.y + 1.0);  // sky (:25-28)
                bg = (1.0 - t) * mk(0.9, 0.95, 1.0) + t * mk(0.6, 0.75, 1.0);
            }
            V contrib = had(beta, bg);
            if (has_env && last_nd) contrib = contrib * mis(last_pdf, env_pdf(S, ray.d));
            acc = acc + clamp_lum(contrib, 50.0);
            break;
        }
        if (bounce >= rr_start) {
            double p = fmax(fmin(fmax(fmax(beta.x, beta.y), beta.z), 0.95), 0.05);
            if (pcg_f64(rng) > p) break;
            beta = beta / p;
        }
        const MaterialF64& mat = S.mats[hit.mat];
        if (mat.kind == TPT_MAT_DIFFUSE_LIGHT) {
            acc = acc + clamp_lum(had(beta, ld(mat.c)), 50.0);
            break;
        }
        V n = dot(hit.n, ray.d) < 0.0 ? hit.n : -hit.n;
        if (mat.kind != TPT_MAT_METAL && mat.kind != TPT_MAT_DIELECTRIC) {
            if (has_env) {  // nee_environment (:148-172)
                V wi, li;
                double pe;
                env_sample_dir(S, rng, wi, li, pe);
                double c = fmax(dot(n, wi), 0.0);
                if (c > 0.0 && pe > 0.0) {
                    Ray sh{hit.p + kEps * wi, wi, ray.time};
                    Hit tmp;
                    cx.shadow_rays++;
                    if (!world_hit(cx, sh, kEps, kTMax, tmp)) {
                        V f;
                        double pb;
                        mat_eval(mat, norm(-ray.d), wi, n, f, pb);
                        acc = acc + had(had(beta, f), li) * (c * mis(pe, pb) / pe);
                    }
                }
            }
            V lp, ln, le;
            double lpdf;
            if (sample_light(S, rng, ray.time, hit.p, lp, ln, le, lpdf)) {  // nee_area_light (:178-213)
                V tl = lp - hit.p;
                double d2 = dot(tl, tl);
                double dist = sqrt(d2);
                if (dist > 1e-6) {
                    V wi = tl / dist;
                    double c = fmax(dot(n, wi), 0.0);
                    if (c > 0.0) {
                        Ray sh{hit.p + kEps * wi, wi, ray.time};
                        double tm = fmax(dist - kEps, kEps);
                        Hit tmp;
                        cx.shadow_rays++;
                        if (!world_hit(cx, sh, kEps, tm, tmp)) {
                            V f;
                            double pb;
                            mat_eval(mat, norm(-ray.d), wi, n, f, pb);
                            if (lpdf > 0.0) acc = acc + had(had(beta, f), le) * (c * mis(lpdf, pb) / lpdf);
                        }
                    }
                }
            }
        }
        Bsdf s;
        if (!mat_sample(mat, ray, hit, rng, s)) break;
        last_pdf = s.pdf;
        last_nd = !s.delta;
        beta = had(beta, s.w);
        ray = s.ray;
    }
    return acc;
}

__device__ Ray camera_ray(const CameraF64& c, double sx, double sy, uint64_t& rng) {  // ray.rs:91-108
    V u = ld(c.u), v = ld(c.v), w = ld(c.w), o = ld(c.o);
    V dir_base = norm(((-w) + (sx * c.half_w) * u) + (sy * c.half_h) * v);
    V lens = mk(0, 0, 0);
    if (c.lens_radius > 0.0) {
        double dx = 0.0, dy = 0.0;
        // sample_unit_disk (:112-120); the acceptance rate is pi/4, so the
        // 256-try bound is never reached in practice ((1-pi/4)^256 ~ 1e-171).
        for (int k = 0; k < 256; ++k) {
            dx = 2.0 * pcg_f64(rng) - 1.0;
            dy = 2.0 * pcg_f64(rng) - 1.0;
            if (dx * dx + dy * dy < 1.0) break;
        }
        lens = u * (dx * c.lens_radius) + v * (dy * c.lens_radius);
    }
    V origin = o + lens;
    V focus = o + dir_base * c.focus_dist;
    V dir = norm(focus - origin);
    double time = c.shutter_open + (c.shutter_close - c.shutter_open) * pcg_f64(rng);
    return Ray{origin, dir, time};
}

// One thread per pixel; blocks tile the image 16x8.
__global__ void __launch_bounds__(128) k_render(PlainScene S, PlainParams P, double* __restrict__ acc,
                                                double* __restrict__ acc_w, double* __restrict__ acc_sq,
                                                unsigned long long* __restrict__ counters, int* flags) {
    const int x = blockIdx.x * 16 + (threadIdx.x & 15);
    const int fy = blockIdx.y * 8 + (threadIdx.x >> 4);  // film row
    const int y = P.row_begin + fy * P.row_step;          // image row
    Ctx cx{&S, 0u, 0u, flags};
    uint32_t nsamp = 0;
    if (x < P.width && fy < P.n_rows) {
        uint64_t rng = pixel_seed((uint32_t)x, (uint32_t)y, P.seed);
        const double inv_w = 1.0 / (double)P.width, inv_h = 1.0 / (double)P.height;
        V c = mk(0, 0, 0), c2 = mk(0, 0, 0);
        int max_spp = P.spp > 1 ? P.spp : 1;
        int min_spp = P.adaptive_min_spp > 1 ? P.adaptive_min_spp : 1;
        if (min_spp > max_spp) min_spp = max_spp;
        double mean = 0.0, m2 = 0.0;
        int n = 0;
        for (int s = 0; s < P.spp; ++s) {
            double jx = pcg_f64(rng);
            double jy = pcg_f64(rng);
            double sx = ((double)x + jx) * inv_w * 2.0 - 1.0;
            double sy = 1.0 - ((double)y + jy) * inv_h * 2.0;
            Ray r = camera_ray(S.cam, sx, sy, rng);
            V smp = radiance(cx, r, rng, P.max_bounces, P.rr_start);
            c = c + smp;
            c2 = c2 + had(smp, smp);
            n += 1;
            if (P.adaptive) {  // render.rs:160-176
                double l = lum(smp);
                double delta = l - mean;
                mean += delta / (double)n;
                double delta2 = l - mean;
                m2 += delta * delta2;
                if (n >= min_spp) {
                    double var = n > 1 ? m2 / (double)(n - 1) : __longlong_as_double(0x7ff0000000000000ll);
                    double den = fmax(fabs(mean), 1e-4);
                    if (sqrt(var) / den < P.adaptive_threshold) break;
                }
            }
        }
        const size_t gi = (size_t)fy * (size_t)P.width + (size_t)x;
        acc[3 * gi] = c.x; acc[3 * gi + 1] = c.y; acc[3 * gi + 2] = c.z;
        acc_w[gi] = (double)n;
        if (acc_sq) { acc_sq[3 * gi] = c2.x; acc_sq[3 * gi + 1] = c2.y; acc_sq[3 * gi + 2] = c2.z; }
        nsamp = (uint32_t)n;
    }
    // Warp-reduce the ray/path counters, one atomic per warp.
    unsigned long long cr = cx.closest_rays, sr = cx.shadow_rays, np = nsamp;
    for (int off = 16; off > 0; off >>= 1) {
        cr += __shfl_down_sync(0xffffffffu, cr, off);
        sr += __shfl_down_sync(0xffffffffu, sr, off);
        np += __shfl_down_sync(0xffffffffu, np, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&counters[0], np);
        atomicAdd(&counters[1], cr);
        atomicAdd(&counters[2], sr);
    }
}

}  // namespace plain

cudaError_t launch_plain(const PlainScene& S, const PlainParams& P, double* acc, double* acc_w, double* acc_sq,
                         unsigned long long* counters, int* flags, cudaStream_t stream) {
    dim3 grid((unsigned)((P.width + 15) / 16), (unsigned)((P.n_rows + 7) / 8));
    plain::k_render<<<grid, 128, 0, stream>>>(S, P, acc, acc_w, acc_sq, counters, flags);
    return cudaGetLastError();
}

}  // namespace tpt
