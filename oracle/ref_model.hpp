// ORACLE -- test infrastructure only.  Nothing in the product (tinypt_b200/)
// links, includes or calls this file; only tests/, the smoke check and the
// CPU-baseline leg of bench.py load the oracle library built from it.
//
// CPU f64 restatement of tinypt's per-sample path integrator (Rust crate
// toshinoritakata/tinypt).  Every function follows the reference function
// cited beside it, with the same operation order, so that with
// -ffp-contract=off and glibc's libm the f64 results equal the Rust ones
// (Rust std calls the platform libm on Linux; powi(2) is a plain multiply).
//
// Parity status: the reference cannot be compiled or run in this
// environment (no Rust toolchain, crates not vendored), so this restatement
// is pinned only by the reference's own unit-test assertions (restated in
// tests/test_oracle_kats.py) and by an independent pure-Python restatement
// of the integer paths (tests/golden/make_golden.py).  Image-level parity
// against the Rust binary itself is unpinned.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <optional>
#include <utility>
#include <vector>
#include <algorithm>

namespace ref {

constexpr double PI = 3.14159265358979323846264338327950288;
constexpr double TAU = 6.28318530717958647692528676655900577;

// src/constants.rs:4-24
constexpr double RAY_EPSILON = 1e-4;
constexpr double RAY_T_MAX = 1e30;
constexpr double FIREFLY_CLAMP = 50.0;
constexpr size_t SAH_BINS = 8;
constexpr size_t LEAF_SIZE = 4;

// Rust f64::max / f64::min return the non-NaN operand (IEEE maxNum), as fmax.
inline double rmax(double a, double b) { return std::fmax(a, b); }
inline double rmin(double a, double b) { return std::fmin(a, b); }
// src/math.rs:173  clamp(x, a, b) = x.max(a).min(b)
inline double clamp(double x, double a, double b) { return rmin(rmax(x, a), b); }
// Rust `f as usize`: saturating, NaN -> 0.
inline size_t as_usize(double f) {
    if (!(f > 0.0)) return 0;
    if (f >= 18446744073709551616.0) return SIZE_MAX;
    return (size_t)f;
}
// Rust f64::to_radians = self * (PI / 180)
inline double to_radians(double d) { return d * (PI / 180.0); }

// ---- src/math.rs:9-96 ----------------------------------------------------
struct Vec3 {
    double x = 0, y = 0, z = 0;
    Vec3() = default;
    Vec3(double x_, double y_, double z_) : x(x_), y(y_), z(z_) {}
};
inline Vec3 operator+(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 operator-(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 operator*(Vec3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline Vec3 operator*(double s, Vec3 a) { return a * s; }
inline Vec3 operator/(Vec3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline Vec3 operator-(Vec3 a) { return {-a.x, -a.y, -a.z}; }
inline double dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }       // :57
inline Vec3 cross(Vec3 a, Vec3 b) {                                                   // :59-65
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double len(Vec3 a) { return std::sqrt(dot(a, a)); }                           // :67
inline Vec3 norm(Vec3 a) { double l = rmax(len(a), 1e-30); return a / l; }           // :69-72
inline Vec3 hadamard(Vec3 a, Vec3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }    // :80

// Color is Vec3 with colour helpers (src/math.rs:20-52).
using Color = Vec3;
inline double luminance(Color c) { return 0.2126 * c.x + 0.7152 * c.y + 0.0722 * c.z; }  // :40
inline Color clamp_luminance(Color c, double max_luma) {                               // :42-49
    double l = luminance(c);
    if (l > max_luma && l > 0.0) return c * (max_luma / l);
    return c;
}
// src/math.rs:176-182
inline double srgb_to_linear(double c) {
    if (c <= 0.04045) return c / 12.92;
    return std::pow((c + 0.055) / 1.055, 2.4);
}
// src/math.rs:185-191
inline double linear_to_srgb(double c) {
    if (c <= 0.0031308) return 12.92 * c;
    return 1.055 * std::pow(c, 1.0 / 2.4) - 0.055;
}
// Color::from_srgb (src/math.rs:26-28)
inline Color color_from_srgb(double r, double g, double b) {
    return {srgb_to_linear(r), srgb_to_linear(g), srgb_to_linear(b)};
}
// :193  R = v - 2(v.n)n
inline Vec3 reflect(Vec3 v, Vec3 n) { return v - (2.0 * dot(v, n)) * n; }
// :199-207
inline std::optional<Vec3> refract(Vec3 v, Vec3 n, double eta) {
    double cosi = rmin(rmax(dot(-v, n), -1.0), 1.0);
    double sin2t = eta * eta * (1.0 - cosi * cosi);
    if (sin2t >= 1.0) return std::nullopt;
    double cost = std::sqrt(1.0 - sin2t);
    return (eta * v) + ((eta * cosi - cost) * n);
}

// ---- src/math.rs:100-170 Mat3 -------------------------------------------
struct Mat3 {
    double m[3][3];
    static Mat3 identity() { return Mat3{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}}; }
    Mat3 mul(const Mat3& b) const {                                                   // :117-127
        Mat3 r{};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                r.m[i][j] = m[i][0] * b.m[0][j] + m[i][1] * b.m[1][j] + m[i][2] * b.m[2][j];
        return r;
    }
    Vec3 mul_vec(Vec3 v) const {                                                      // :130-136
        return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z,
                m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
                m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
    }
    Mat3 transpose() const {                                                          // :139-148
        return Mat3{{{m[0][0], m[1][0], m[2][0]}, {m[0][1], m[1][1], m[2][1]}, {m[0][2], m[1][2], m[2][2]}}};
    }
    Mat3 invert() const {                                                             // :151-169
        double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1])
                   - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0])
                   + m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
        double inv_det = 1.0 / det;
        Mat3 r{};
        r.m[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) * inv_det;
        r.m[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * inv_det;
        r.m[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * inv_det;
        r.m[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * inv_det;
        r.m[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * inv_det;
        r.m[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * inv_det;
        r.m[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * inv_det;
        r.m[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * inv_det;
        r.m[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * inv_det;
        return r;
    }
};

// ---- src/rng.rs:9-47 -----------------------------------------------------
struct Rng {
    uint64_t state;
    explicit Rng(uint64_t seed) : state(seed == 0 ? 0x9E3779B97F4A7C15ull : seed) {}  // :12-15
    uint32_t next_u32() {                                                             // :18-27
        uint64_t old = state;
        state = old * 6364136223846793005ull + 1442695040888963407ull;
        uint32_t xorshifted = (uint32_t)(((old >> 18) ^ old) >> 27);
        uint32_t rot = (uint32_t)(old >> 59);
        return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
    }
    double next_f64() {                                                               // :30-36
        uint64_t hi = (uint64_t)next_u32() << 21;
        uint64_t lo = (uint64_t)next_u32() & ((1ull << 21) - 1);
        uint64_t u = hi | lo;
        return (double)u * (1.0 / (double)(1ull << 53));
    }
};
// :41-47
inline uint64_t seed_for(uint32_t px, uint32_t py, uint32_t s) {
    uint64_t h = 0xD1B54A32D192ED03ull;
    h ^= (uint64_t)px * 0x9E3779B185EBCA87ull;
    h ^= (uint64_t)py * 0xC2B2AE3D27D4EB4Full;
    h ^= (uint64_t)s * 0x165667B19E3779F9ull;
    return h ^ (h >> 32);
}

// ---- src/ray.rs ----------------------------------------------------------
struct Ray { Vec3 o, d; double time = 0; };
inline Vec3 ray_at(const Ray& r, double t) { return r.o + r.d * t; }                  // :15

// :112-120 rejection sampling of the unit disk
inline std::pair<double, double> sample_unit_disk(Rng& rng) {
    for (;;) {
        double x = 2.0 * rng.next_f64() - 1.0;
        double y = 2.0 * rng.next_f64() - 1.0;
        if (x * x + y * y < 1.0) return {x, y};
    }
}

struct Camera {                                                                       // :22-33
    Vec3 o, u, v, w;
    double half_h = 0, half_w = 0, lens_radius = 0, focus_dist = 0;
    double shutter_open = 0, shutter_close = 1;

    static Camera look_at(Vec3 eye, Vec3 target, Vec3 up, double fov_deg, double aspect) {  // :36-56
        Camera c;
        double theta = to_radians(fov_deg);
        c.half_h = std::tan(theta * 0.5);
        c.half_w = aspect * c.half_h;
        c.w = norm(eye - target);
        c.u = norm(cross(up, c.w));
        c.v = cross(c.w, c.u);
        c.focus_dist = len(eye - target);
        c.o = eye;
        c.lens_radius = 0.0;
        return c;
    }
    static Camera look_at_dof(Vec3 eye, Vec3 target, Vec3 up, double fov_deg, double aspect,
                              double focus_dist, double aperture) {                   // :59-86
        Camera c;
        double theta = to_radians(fov_deg);
        c.half_h = std::tan(theta * 0.5);
        c.half_w = aspect * c.half_h;
        c.w = norm(eye - target);
        c.u = norm(cross(up, c.w));
        c.v = cross(c.w, c.u);
        c.o = eye;
        c.lens_radius = 0.5 * rmax(aperture, 0.0);
        c.focus_dist = rmax(focus_dist, 1e-6);
        return c;
    }
    Ray ray(double sx, double sy, Rng& rng) const {                                   // :91-108
        Vec3 dir_base = norm(((-w) + (sx * half_w) * u) + (sy * half_h) * v);
        Vec3 lens_offset(0.0, 0.0, 0.0);
        if (lens_radius > 0.0) {
            auto [dx, dy] = sample_unit_disk(rng);
            lens_offset = u * (dx * lens_radius) + v * (dy * lens_radius);
        }
        Vec3 origin = o + lens_offset;
        Vec3 focus_point = o + dir_base * focus_dist;
        Vec3 dir = norm(focus_point - origin);
        double time = shutter_open + (shutter_close - shutter_open) * rng.next_f64();
        return Ray{origin, dir, time};
    }
};

// ---- src/geometry.rs -----------------------------------------------------
struct Hit { double t; Vec3 p, n; size_t mat_id; };                                    // :14-23
struct Sphere { Vec3 c; double r; size_t mat_id; };                                    // :26-34

struct Aabb {                                                                         // :54-57
    Vec3 min, max;
    static Aabb empty() {                                                             // :62-67
        const double inf = std::numeric_limits<double>::infinity();
        return Aabb{{inf, inf, inf}, {-inf, -inf, -inf}};
    }
    Aabb grow(Vec3 p) const {                                                         // :83-87
        return Aabb{{rmin(min.x, p.x), rmin(min.y, p.y), rmin(min.z, p.z)},
                    {rmax(max.x, p.x), rmax(max.y, p.y), rmax(max.z, p.z)}};
    }
    static Aabb from_points(Vec3 a, Vec3 b, Vec3 c) {                                 // :70-80
        Aabb bb = empty().grow(a).grow(b).grow(c);
        const double eps = 1e-9;
        bb.min = Vec3(bb.min.x - eps, bb.min.y - eps, bb.min.z - eps);
        bb.max = Vec3(bb.max.x + eps, bb.max.y + eps, bb.max.z + eps);
        return bb;
    }
    Aabb unite(const Aabb& b) const {                                                 // :90-95
        return Aabb{{rmin(min.x, b.min.x), rmin(min.y, b.min.y), rmin(min.z, b.min.z)},
                    {rmax(max.x, b.max.x), rmax(max.y, b.max.y), rmax(max.z, b.max.z)}};
    }
    Vec3 centroid() const { return (min + max) * 0.5; }                               // :98-100
    Vec3 extent() const { return max - min; }                                         // :103-105
    bool hit_inv(const Ray& r, Vec3 inv, double tmin, double tmax) const {            // :117-136
        double t0x = (min.x - r.o.x) * inv.x, t1x = (max.x - r.o.x) * inv.x;
        tmin = rmax(tmin, rmin(t0x, t1x)); tmax = rmin(tmax, rmax(t0x, t1x));
        if (tmax <= tmin) return false;
        double t0y = (min.y - r.o.y) * inv.y, t1y = (max.y - r.o.y) * inv.y;
        tmin = rmax(tmin, rmin(t0y, t1y)); tmax = rmin(tmax, rmax(t0y, t1y));
        if (tmax <= tmin) return false;
        double t0z = (min.z - r.o.z) * inv.z, t1z = (max.z - r.o.z) * inv.z;
        tmin = rmax(tmin, rmin(t0z, t1z)); tmax = rmin(tmax, rmax(t0z, t1z));
        if (tmax <= tmin) return false;
        return true;
    }
    std::optional<std::pair<double, double>> hit_range_inv(const Ray& r, Vec3 inv, double tmin,
                                                           double tmax) const {       // :146-165
        double t0x = (min.x - r.o.x) * inv.x, t1x = (max.x - r.o.x) * inv.x;
        tmin = rmax(tmin, rmin(t0x, t1x)); tmax = rmin(tmax, rmax(t0x, t1x));
        if (tmax <= tmin) return std::nullopt;
        double t0y = (min.y - r.o.y) * inv.y, t1y = (max.y - r.o.y) * inv.y;
        tmin = rmax(tmin, rmin(t0y, t1y)); tmax = rmin(tmax, rmax(t0y, t1y));
        if (tmax <= tmin) return std::nullopt;
        double t0z = (min.z - r.o.z) * inv.z, t1z = (max.z - r.o.z) * inv.z;
        tmin = rmax(tmin, rmin(t0z, t1z)); tmax = rmin(tmax, rmax(t0z, t1z));
        if (tmax <= tmin) return std::nullopt;
        return std::make_pair(tmin, tmax);
    }
};

// :174-195
inline std::optional<Hit> sphere_hit(const Sphere& s, const Ray& r, double tmin, double tmax) {
    Vec3 oc = r.o - s.c;
    double a = dot(r.d, r.d);
    double b = dot(oc, r.d);
    double c = dot(oc, oc) - s.r * s.r;
    double d = b * b - a * c;
    if (d <= 0.0) return std::nullopt;
    double sd = std::sqrt(d);
    double t = (-b - sd) / a;
    if (t < tmin || t > tmax) {
        t = (-b + sd) / a;
        if (t < tmin || t > tmax) return std::nullopt;
    }
    Vec3 p = ray_at(r, t);
    Vec3 n = (p - s.c) / s.r;
    return Hit{t, p, n, s.mat_id};
}

struct Triangle {                                                                     // :41-47
    Vec3 v0_0, v1_0, v2_0, v0_1, v1_1, v2_1;
    size_t mat_id;
    static Triangle new_static(Vec3 v0, Vec3 v1, Vec3 v2, size_t mat) {               // :199-210
        return Triangle{v0, v1, v2, v0, v1, v2, mat};
    }
    void vertices_at(double t, Vec3& v0, Vec3& v1, Vec3& v2) const {                  // :212-218
        v0 = v0_0 * (1.0 - t) + v0_1 * t;
        v1 = v1_0 * (1.0 - t) + v1_1 * t;
        v2 = v2_0 * (1.0 - t) + v2_1 * t;
    }
    Aabb bounds() const {                                                             // :221-225
        return Aabb::from_points(v0_0, v1_0, v2_0).unite(Aabb::from_points(v0_1, v1_1, v2_1));
    }
    std::optional<Hit> hit(const Ray& r, double tmin, double tmax) const {            // :236-273
        Vec3 v0, v1, v2;
        vertices_at(r.time, v0, v1, v2);
        Vec3 e1 = v1 - v0, e2 = v2 - v0;
        Vec3 pvec = cross(r.d, e2);
        double det = dot(e1, pvec);
        if (std::fabs(det) < 1e-10) return std::nullopt;
        double inv_det = 1.0 / det;
        Vec3 tvec = r.o - v0;
        double u = dot(tvec, pvec) * inv_det;
        if (u < 0.0 || u > 1.0) return std::nullopt;
        Vec3 qvec = cross(tvec, e1);
        double v = dot(r.d, qvec) * inv_det;
        if (v < 0.0 || u + v > 1.0) return std::nullopt;
        double thit = dot(e2, qvec) * inv_det;
        if (thit < tmin || thit > tmax) return std::nullopt;
        Vec3 p = ray_at(r, thit);
        Vec3 n = norm(cross(e1, e2));
        return Hit{thit, p, n, mat_id};
    }
};

// ---- src/transform.rs ----------------------------------------------------
struct Transform {                                                                    // :11-21
    Mat3 a, a_inv, normal_mat;
    Vec3 t;
    static Transform from_affine(const Mat3& a, Vec3 t) {                             // :24-27
        Transform x;
        x.a = a; x.t = t; x.a_inv = a.invert(); x.normal_mat = x.a_inv.transpose();
        return x;
    }
    static Transform identity() { return from_affine(Mat3::identity(), Vec3(0, 0, 0)); }
    static Transform translate(Vec3 t) { return from_affine(Mat3::identity(), t); }  // :43-45
    static Transform scale(Vec3 s) {                                                  // :53-58
        return from_affine(Mat3{{{s.x, 0, 0}, {0, s.y, 0}, {0, 0, s.z}}}, Vec3(0, 0, 0));
    }
    static Mat3 rotation(Vec3 axis, double deg) {                                     // :101-111
        Vec3 k = norm(axis);
        double rad = to_radians(deg);
        double s = std::sin(rad), c = std::cos(rad);
        double one_c = 1.0 - c;
        double x = k.x, y = k.y, z = k.z;
        return Mat3{{{c + x * x * one_c, x * y * one_c - z * s, x * z * one_c + y * s},
                     {y * x * one_c + z * s, c + y * y * one_c, y * z * one_c - x * s},
                     {z * x * one_c - y * s, z * y * one_c + x * s, c + z * z * one_c}}};
    }
    static Transform rotate(Vec3 axis, double deg) { return from_affine(rotation(axis, deg), Vec3(0, 0, 0)); }
    static Transform legacy(Vec3 t, double rot_y_deg, double s) {                    // :38-40
        return from_affine(rotation(Vec3(0, 1, 0), rot_y_deg).mul(Mat3{{{s, 0, 0}, {0, s, 0}, {0, 0, s}}}), t);
    }
    Transform compose(const Transform& inner) const {                                 // :70-72
        return from_affine(a.mul(inner.a), a.mul_vec(inner.t) + t);
    }
    Vec3 apply_point(Vec3 p) const { return a.mul_vec(p) + t; }                      // :75-77
    Vec3 apply_point_inv(Vec3 p) const { return a_inv.mul_vec(p - t); }              // :80-82
    Vec3 apply_vec_inv(Vec3 v) const { return a_inv.mul_vec(v); }                    // :85-87
    Vec3 apply_normal(Vec3 n) const { return norm(normal_mat.mul_vec(n)); }          // :90-92
};

// ---- src/bvh.rs ----------------------------------------------------------
struct BvhNode { Aabb bbox; int32_t left, right; uint32_t start, count; };            // :24-35

struct TraversalCounts {
    uint64_t world_hits = 0, node_pops = 0, node_box_tests = 0, tri_tests = 0, sphere_tests = 0;
};

struct Bvh {                                                                          // :38-43
    std::vector<BvhNode> nodes;
    std::vector<size_t> indices;

    static Bvh build(const std::vector<Triangle>& tris);
    std::optional<Hit> hit(const std::vector<Triangle>& tris, const Ray& r, double tmin, double tmax,
                           TraversalCounts* cnt) const;
};

// ---- src/material.rs -----------------------------------------------------
enum class MatKind { Lambert, Metal, Dielectric, Ggx, Subsurface, DiffuseLight };
struct Material {                                                                     // :30-43
    MatKind kind;
    Color c;       // albedo | absorption | emit
    double p = 0;  // ior | alpha | scatter_dist
    // Test extension (no counterpart in the reference): the GGX alpha of the
    // VNDF sampler and of the pdfs, when sampling is detached from
    // evaluation for finite-difference checks of derivatives; < 0 = p.
    double sp = -1;
};
inline double sampling_alpha(const Material& m) { return m.sp >= 0 ? m.sp : m.p; }
struct BsdfSample { Ray scattered; Color weight; double pdf; bool is_delta; };       // :49-58

std::optional<BsdfSample> material_sample(const Material& m, const Ray& ray_in, const Hit& hit, Rng& rng);
std::pair<Color, double> material_eval(const Material& m, Vec3 wo, Vec3 wi, Vec3 n);
inline bool material_is_delta(const Material& m) {                                    // :70-72
    return m.kind == MatKind::Metal || m.kind == MatKind::Dielectric;
}
inline std::optional<Color> material_emitted(const Material& m) {                     // :62-67
    if (m.kind == MatKind::DiffuseLight) return m.c;
    return std::nullopt;
}
Vec3 sample_cosine_hemisphere(Vec3 n, Rng& rng);
void tangent_frame(Vec3 n, Vec3& t, Vec3& b);

// ---- src/env.rs ----------------------------------------------------------
struct EnvMap {                                                                       // :20-33
    size_t width = 0, height = 0;
    std::vector<Color> data;
    std::vector<double> row_cdf, col_cdf;
    double total_weight = 0;

    static EnvMap from_pixels(size_t w, size_t h, std::vector<Color> data);
    static EnvMap constant(Color c) { return from_pixels(1, 1, {c}); }
    Color sample(Vec3 dir) const;
    void sample_dir(Rng& rng, Vec3& dir, Color& radiance, double& pdf) const;
    double pdf(Vec3 dir) const;
};

// ---- src/world.rs --------------------------------------------------------
struct Mesh { std::vector<Triangle> tris; Bvh bvh; };                                // :20-33
struct Instance { size_t mesh_id; Transform xform; std::optional<size_t> mat_override; };  // :39-46
struct Light {                                                                        // :218-221
    bool is_sphere;
    size_t idx;                                  // sphere index
    size_t mesh_id, tri_id, inst_id;             // triangle light
};
struct LightInfo { Light light; Color emit; double weight; };                         // :296-300
struct LightSample { Vec3 position, normal; Color emit; double pdf; };              // :304-313

struct World {                                                                        // :49-62
    std::vector<Sphere> spheres;
    std::vector<Mesh> meshes;
    std::vector<Instance> instances;
    std::vector<LightInfo> lights;
    std::vector<double> light_cdf;
    double light_total = 0;

    std::optional<Hit> hit(const Ray& r, double tmin, double tmax, TraversalCounts* cnt) const;
    void build_lights(const std::vector<Material>& mats, const std::vector<Material>* sampling = nullptr);
    std::optional<LightSample> sample_light(Rng& rng, double time, Vec3 p) const;
    double light_area(const Light& l, double time) const;
    bool light_sample_surface(const Light& l, double time, Rng& rng, Vec3& pos, Vec3& n, double& area) const;
    bool tri_world_verts(size_t mesh_id, size_t tri_id, size_t inst_id, double time, Vec3& v0, Vec3& v1,
                         Vec3& v2) const;
};

// ---- src/scene.rs, src/integrator.rs -------------------------------------
struct Scene {                                                                        // scene.rs:14-23
    Camera cam;
    World world;
    std::vector<Material> mats;
    std::optional<EnvMap> env;
};
struct PathLimits { size_t max_bounces, rr_start; };                                 // integrator.rs:41-46

Color radiance(const World& world, const std::vector<Material>& mats, const EnvMap* env, Ray ray,
               Rng& rng, PathLimits limits, TraversalCounts* cnt);

// ---- src/render.rs, src/config.rs ----------------------------------------
struct RenderConfig {                                                                 // config.rs:5-46 (hot-path fields)
    size_t width = 1920, height = 1080, spp = 512, max_bounces = 8, rr_start = 3, tile = 16;
    bool adaptive_enabled = false;
    size_t adaptive_min_spp = 8;
    double adaptive_threshold = 0.02;
    bool morton_enabled = true;
    uint64_t seed = 0;
};
uint64_t interleave_bits(uint64_t v);                                                // render.rs:291-299
uint64_t morton2(size_t tx, size_t ty, size_t tiles_x, size_t tiles_y);              // render.rs:284-288
struct Task { size_t id, x0, y0, x1, y1, sample_start, sample_end; };                 // task.rs:11-27
std::vector<Task> make_tasks(const RenderConfig& cfg);                                // render.rs:75-100

// Renders into acc (w*h*3) / acc_w (w*h); acc_sq (optional) receives the sum
// of squared per-sample radiance per channel (not part of the reference
// output; used for per-pixel variance in parity tests).
// rect (x0, y0, x1, y1) restricts the render to a sub-rectangle of the film
// (pixels keep their full-film RNG streams); outputs are then rect-sized.
struct Rect { size_t x0, y0, x1, y1; };
// sample_chunk > 0 cuts every tile task's sample range [0, spp) into tasks of
// sample_chunk samples, [k*sample_chunk, min((k+1)*sample_chunk, spp)), the
// reference worker's Task { sample_start, sample_end } (task.rs:11-27), each
// seeded from seed_for(x, y, sample_start) (render.rs:142).  Task ids run
// chunk by chunk (all tiles of chunk 0 in tile order, then chunk 1, ...) and
// results merge in task-id order (render.rs:226-241), so a pixel's film value
// is ((0 + chunk 0) + chunk 1) + ...  sample_chunk = 0 (or >= spp) is the
// reference's own task list (sample_start 0 for every tile, render.rs:75-100).
// reseed > 0 (with sample_chunk 0) keeps the reference's task list and loop
// but restarts each pixel's RNG from seed_for(x, y, s) ^ seed at every sample
// s that is a multiple of reseed: the streams of tasks of `reseed` samples
// under one per-pixel loop (sums in sample order, one Welford statistic).
void render(const Scene& scene, const RenderConfig& cfg, double* acc, double* acc_w, double* acc_sq,
            int threads, TraversalCounts* cnt, const Rect* rect = nullptr, size_t sample_chunk = 0,
            size_t reseed = 0);

}  // namespace ref
