// ORACLE -- test infrastructure only (see ref_model.hpp).
// f64 restatement of tinypt's bvh.rs, material.rs, env.rs, world.rs,
// integrator.rs and render.rs.  Comments cite the reference lines followed.
#include "ref_model.hpp"

#include <atomic>
#include <thread>

namespace ref {

// ======================= src/bvh.rs:51-242 ===============================
namespace {

void bounds_for_range(const std::vector<Aabb>& bounds, const std::vector<Vec3>& centroids,
                      const size_t* idx, size_t n, Aabb& bbox, Aabb& cbox) {  // :58-67
    bbox = Aabb::empty();
    cbox = Aabb::empty();
    for (size_t k = 0; k < n; ++k) {
        size_t i = idx[k];
        bbox = bbox.unite(bounds[i]);
        cbox = cbox.grow(centroids[i]);
    }
}

double axis_of(Vec3 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

size_t bin_of(double cv, double minc, double inv_extent) {  // :126-127, :180-181
    size_t bi = as_usize((cv - minc) * inv_extent * (double)SAH_BINS);
    if (bi >= SAH_BINS) bi = SAH_BINS - 1;
    return bi;
}

int32_t build_node(std::vector<BvhNode>& nodes, std::vector<size_t>& indices,
                   const std::vector<Aabb>& bounds, const std::vector<Vec3>& centroids, size_t start,
                   size_t end) {  // :69-233
    size_t n = end - start;
    Aabb bbox, cbox;
    bounds_for_range(bounds, centroids, indices.data() + start, n, bbox, cbox);
    int32_t node_index = (int32_t)nodes.size();
    nodes.push_back(BvhNode{bbox, -1, -1, 0, 0});
    if (n <= LEAF_SIZE) {  // :93-98
        nodes[node_index].start = (uint32_t)start;
        nodes[node_index].count = (uint32_t)n;
        return node_index;
    }
    Vec3 ext = cbox.extent();  // :101-108
    int axis = (ext.x >= ext.y && ext.x >= ext.z) ? 0 : (ext.y >= ext.z ? 1 : 2);

    size_t mid;
    if (n >= SAH_BINS * 2) {  // :110
        double minc = axis_of(cbox.min, axis), maxc = axis_of(cbox.max, axis);
        double extent = maxc - minc;
        if (extent > 1e-12) {
            double inv_extent = 1.0 / extent;
            Aabb bin_box[SAH_BINS];
            size_t bin_cnt[SAH_BINS];
            for (size_t b = 0; b < SAH_BINS; ++b) { bin_box[b] = Aabb::empty(); bin_cnt[b] = 0; }
            for (size_t k = start; k < end; ++k) {  // :123-130
                size_t idx = indices[k];
                size_t bi = bin_of(axis_of(centroids[idx], axis), minc, inv_extent);
                bin_box[bi] = bin_box[bi].unite(bounds[idx]);
                bin_cnt[bi] += 1;
            }
            Aabb left_bbox[SAH_BINS], right_bbox[SAH_BINS];
            size_t left_count[SAH_BINS], right_count[SAH_BINS];
            Aabb acc_bbox = Aabb::empty();
            size_t acc_count = 0;
            for (size_t i = 0; i < SAH_BINS; ++i) {  // :139-146
                if (bin_cnt[i] > 0) { acc_bbox = acc_bbox.unite(bin_box[i]); acc_count += bin_cnt[i]; }
                left_bbox[i] = acc_bbox; left_count[i] = acc_count;
            }
            acc_bbox = Aabb::empty(); acc_count = 0;
            for (size_t i = SAH_BINS; i-- > 0;) {  // :150-157
                if (bin_cnt[i] > 0) { acc_bbox = acc_bbox.unite(bin_box[i]); acc_count += bin_cnt[i]; }
                right_bbox[i] = acc_bbox; right_count[i] = acc_count;
            }
            double best_cost = std::numeric_limits<double>::infinity();
            size_t best_split = 0;
            for (size_t i = 0; i < SAH_BINS - 1; ++i) {  // :161-174
                size_t lc = left_count[i], rc = right_count[i + 1];
                if (lc == 0 || rc == 0) continue;
                Vec3 la = left_bbox[i].extent(), ra = right_bbox[i + 1].extent();
                double left_area = 2.0 * (la.x * la.y + la.y * la.z + la.z * la.x);
                double right_area = 2.0 * (ra.x * ra.y + ra.y * ra.z + ra.z * ra.x);
                double cost = left_area * (double)lc + right_area * (double)rc;
                if (cost < best_cost) { best_cost = cost; best_split = i + 1; }
            }
            if (std::isfinite(best_cost)) {  // :176-192
                // slice::sort_by_key is a stable sort.
                std::stable_sort(indices.begin() + start, indices.begin() + end, [&](size_t a, size_t b) {
                    return bin_of(axis_of(centroids[a], axis), minc, inv_extent) <
                           bin_of(axis_of(centroids[b], axis), minc, inv_extent);
                });
                size_t left_total = 0;
                for (size_t i = 0; i < best_split; ++i) left_total += bin_cnt[i];
                mid = (left_total > 0 && left_total < n) ? start + left_total : start + n / 2;
            } else {
                mid = start + n / 2;
            }
        } else {
            mid = start + n / 2;
        }
    } else {
        mid = start + n / 2;
    }
    // :203-222 (mid == start || mid == end) cannot occur: n > LEAF_SIZE gives
    // 0 < n/2 < n and the SAH branch requires 0 < left_total < n.
    int32_t left = build_node(nodes, indices, bounds, centroids, start, mid);
    int32_t right = build_node(nodes, indices, bounds, centroids, mid, end);
    nodes[node_index].left = left;
    nodes[node_index].right = right;
    nodes[node_index].start = 0;
    nodes[node_index].count = 0;
    return node_index;
}

}  // namespace

Bvh Bvh::build(const std::vector<Triangle>& tris) {
    Bvh b;
    b.indices.resize(tris.size());
    for (size_t i = 0; i < tris.size(); ++i) b.indices[i] = i;
    std::vector<Aabb> tri_bounds(tris.size());
    std::vector<Vec3> tri_centroids(tris.size());
    for (size_t i = 0; i < tris.size(); ++i) {
        tri_bounds[i] = tris[i].bounds();
        tri_centroids[i] = tri_bounds[i].centroid();
    }
    if (!b.indices.empty()) build_node(b.nodes, b.indices, tri_bounds, tri_centroids, 0, b.indices.size());
    return b;
}

// src/bvh.rs:248-351.  The 64-entry stack with heap fallback is a growable
// vector here; the visiting order is the same.
std::optional<Hit> Bvh::hit(const std::vector<Triangle>& tris, const Ray& r, double tmin, double tmax,
                            TraversalCounts* cnt) const {
    if (nodes.empty()) return std::nullopt;
    Vec3 inv(1.0 / r.d.x, 1.0 / r.d.y, 1.0 / r.d.z);
    std::vector<int32_t> stack;
    stack.reserve(64);
    stack.push_back(0);
    std::optional<Hit> best;
    while (!stack.empty()) {
        int32_t nid = stack.back();
        stack.pop_back();
        const BvhNode& n = nodes[(size_t)nid];
        if (cnt) { cnt->node_pops++; cnt->node_box_tests++; }
        if (!n.bbox.hit_inv(r, inv, tmin, tmax)) continue;
        if (n.left == -1 && n.right == -1) {
            size_t s = n.start, e = s + n.count;
            for (size_t k = s; k < e; ++k) {
                if (cnt) cnt->tri_tests++;
                if (auto h = tris[indices[k]].hit(r, tmin, tmax)) { tmax = h->t; best = h; }
            }
        } else {
            int32_t a_id = n.left, b_id = n.right;
            if (a_id == -1) { if (b_id != -1) stack.push_back(b_id); continue; }
            if (b_id == -1) { stack.push_back(a_id); continue; }
            const BvhNode& a = nodes[(size_t)a_id];
            const BvhNode& b = nodes[(size_t)b_id];
            if (cnt) cnt->node_box_tests += 2;
            auto a_hit = a.bbox.hit_range_inv(r, inv, tmin, tmax);
            auto b_hit = b.bbox.hit_range_inv(r, inv, tmin, tmax);
            if (a_hit && b_hit) {
                if (a_hit->first <= b_hit->first) { stack.push_back(b_id); stack.push_back(a_id); }
                else { stack.push_back(a_id); stack.push_back(b_id); }
            } else if (a_hit) {
                stack.push_back(a_id);
            } else if (b_hit) {
                stack.push_back(b_id);
            }
        }
    }
    return best;
}

// ======================= src/material.rs ==================================
namespace {
double pow5(double x) { double x2 = x * x; return x2 * x2 * x; }                     // :259-262
Color fresnel_schlick(double cos_theta, Color f0) {                                   // :265-269
    Color one(1.0, 1.0, 1.0);
    double x = 1.0 - rmax(cos_theta, 0.0);
    return f0 + (one - f0) * pow5(x);
}
double ggx_distribution(double alpha, double cos_h) {                                 // :272-279
    if (cos_h <= 0.0) return 0.0;
    double a2 = alpha * alpha;
    double denom = cos_h * cos_h * (a2 - 1.0) + 1.0;
    return a2 / (PI * denom * denom);
}
double ggx_smith_g1(double alpha, double cos_theta) {                                 // :282-288
    if (cos_theta <= 0.0) return 0.0;
    double a = alpha * std::sqrt(rmax(1.0 - cos_theta * cos_theta, 0.0)) / rmax(cos_theta, 1e-6);
    return 2.0 / (1.0 + std::sqrt(1.0 + a * a));
}
double ggx_smith(double alpha, double ci, double co) { return ggx_smith_g1(alpha, ci) * ggx_smith_g1(alpha, co); }
Color ggx_eval(Color albedo, double alpha, Vec3 n, Vec3 wo, Vec3 wi) {                // :227-240
    double cos_i = dot(n, wo), cos_o = dot(n, wi);
    if (cos_i <= 0.0 || cos_o <= 0.0) return Color(0, 0, 0);
    Vec3 m = norm(wo + wi);
    double cos_h = rmax(dot(n, m), 0.0);
    double d = ggx_distribution(alpha, cos_h);
    double g = ggx_smith(alpha, cos_i, cos_o);
    Color f = fresnel_schlick(std::fabs(dot(wi, m)), albedo);
    double denom = 4.0 * cos_i * cos_o + 1e-6;
    return f * (d * g / denom);
}
double ggx_pdf(double alpha, Vec3 n, Vec3 wo, Vec3 wi) {                              // :243-256
    double cos_i = dot(n, wo), cos_o = dot(n, wi);
    if (cos_i <= 0.0 || cos_o <= 0.0) return 0.0;
    Vec3 m = norm(wo + wi);
    double cos_h = rmax(dot(n, m), 0.0);
    double d = ggx_distribution(alpha, cos_h);
    double g1 = ggx_smith_g1(alpha, cos_i);
    double pdf_m = d * g1 * cos_h / rmax(cos_i, 1e-6);
    double denom = 4.0 * rmax(std::fabs(dot(wi, m)), 1e-6);
    return rmax(pdf_m / denom, 0.0);
}
Vec3 sample_ggx_vndf(Vec3 wo, double alpha, double u1, double u2) {                   // :327-347
    Vec3 v = norm(Vec3(alpha * wo.x, alpha * wo.y, wo.z));
    Vec3 t1, t2;
    if (v.z < 0.9999) { t1 = norm(Vec3(-v.y, v.x, 0.0)); t2 = cross(v, t1); }
    else { t1 = Vec3(1, 0, 0); t2 = Vec3(0, 1, 0); }
    double r = std::sqrt(u1);
    double phi = TAU * u2;
    double t1p = r * std::cos(phi);
    double t2p_init = r * std::sin(phi);
    double s = 0.5 * (1.0 + v.z);
    double t2p = std::sqrt(1.0 - s) * t2p_init + s * std::sqrt(rmax(1.0 - t1p * t1p, 0.0));
    Vec3 nh = norm(t1 * t1p + t2 * t2p + v * std::sqrt(rmax(1.0 - t1p * t1p - t2p * t2p, 0.0)));
    return norm(Vec3(alpha * nh.x, alpha * nh.y, nh.z));
}
}  // namespace

void tangent_frame(Vec3 n, Vec3& t, Vec3& b) {                                        // :313-318
    Vec3 a = std::fabs(n.x) > 0.9 ? Vec3(0, 1, 0) : Vec3(1, 0, 0);
    t = norm(cross(n, a));
    b = cross(t, n);
}

Vec3 sample_cosine_hemisphere(Vec3 n, Rng& rng) {                                     // :299-310
    double u = rng.next_f64();
    double v = rng.next_f64();
    double r = std::sqrt(u);
    double phi = 2.0 * PI * v;
    double x = r * std::cos(phi);
    double y = r * std::sin(phi);
    double z = std::sqrt(1.0 - u);
    Vec3 t, b;
    tangent_frame(n, t, b);
    return t * x + b * y + n * z;
}

std::optional<BsdfSample> material_sample(const Material& m, const Ray& ray_in, const Hit& hit,
                                          Rng& rng) {  // :76-201
    bool entering = dot(hit.n, ray_in.d) < 0.0;
    Vec3 n = entering ? hit.n : -hit.n;
    switch (m.kind) {
        case MatKind::Lambert: {
            Vec3 d = sample_cosine_hemisphere(n, rng);
            return BsdfSample{Ray{hit.p + RAY_EPSILON * d, d, ray_in.time}, m.c, rmax(dot(n, d), 0.0) / PI, false};
        }
        case MatKind::Metal: {
            Vec3 d = reflect(ray_in.d, n);
            return BsdfSample{Ray{hit.p + RAY_EPSILON * d, d, ray_in.time}, m.c, 0.0, true};
        }
        case MatKind::Dielectric: {
            double ior = m.p;
            Color absorption = m.c;
            double eta = entering ? 1.0 / ior : ior;
            double cos_i = rmax(dot(-ray_in.d, n), 0.0);
            double f0q = (ior - 1.0) / (ior + 1.0);
            double f0 = f0q * f0q;  // powi(2)
            double fresnel = f0 + (1.0 - f0) * pow5(1.0 - cos_i);
            Color current_beta(1.0, 1.0, 1.0);
            if (!entering) {
                double dist = rmax(hit.t, 0.0);
                Color att(std::exp(-absorption.x * dist), std::exp(-absorption.y * dist),
                          std::exp(-absorption.z * dist));
                current_beta = hadamard(current_beta, att);
            }
            Vec3 refl_dir = reflect(ray_in.d, n);
            auto refr_dir = refract(ray_in.d, n, eta);
            bool choose_refl = !refr_dir.has_value() || rng.next_f64() < fresnel;
            Vec3 d;
            if (choose_refl) {
                current_beta = current_beta * (fresnel / rmax(fresnel, 1e-6));
                d = refl_dir;
            } else {
                double scale = (1.0 - fresnel) / rmax(1.0 - fresnel, 1e-6);
                current_beta = current_beta * scale * (eta * eta);
                d = *refr_dir;
            }
            return BsdfSample{Ray{hit.p + RAY_EPSILON * d, d, ray_in.time}, current_beta, 0.0, true};
        }
        case MatKind::Ggx: {
            double alpha_val = rmax(m.p, 1e-3);
            double alpha_s = rmax(sampling_alpha(m), 1e-3);  // = alpha_val unless detached
            Vec3 t, b;
            tangent_frame(n, t, b);
            Vec3 wo = norm(-ray_in.d);
            Vec3 wo_local(dot(wo, t), dot(wo, b), dot(wo, n));
            if (wo_local.z <= 0.0) return std::nullopt;
            double u1 = rng.next_f64();
            double u2 = rng.next_f64();
            Vec3 m_local = sample_ggx_vndf(wo_local, alpha_s, u1, u2);
            Vec3 mh = t * m_local.x + b * m_local.y + n * m_local.z;
            Vec3 d = reflect(ray_in.d, mh);
            double cos_o = dot(d, n);
            double cos_i = dot(-ray_in.d, n);
            if (cos_o <= 1e-6 || cos_i <= 1e-6) return std::nullopt;
            double cos_h = rmax(dot(n, mh), 0.0);
            double d_ggx = ggx_distribution(alpha_val, cos_h);
            double g = ggx_smith(alpha_val, cos_i, cos_o);
            Color f = fresnel_schlick(std::fabs(dot(d, mh)), m.c);
            double denom = 4.0 * cos_i * cos_o + 1e-6;
            Color spec = f * (d_ggx * g / denom);
            double pdf = ggx_pdf(alpha_s, n, wo, d);
            return BsdfSample{Ray{hit.p + RAY_EPSILON * d, d, ray_in.time}, spec * (cos_o / rmax(pdf, 1e-6)), pdf,
                              false};
        }
        case MatKind::Subsurface: {
            double scale = rmax(m.p, 1e-4);
            double u = rmax(rng.next_f64(), 1e-12);
            double dist = -std::log(u) * scale;
            Vec3 normal_out = hit.n;  // unoriented normal (material.rs:187)
            Vec3 d = sample_cosine_hemisphere(normal_out, rng);
            Color att = m.c * std::exp(-dist / scale);
            Vec3 origin = hit.p - normal_out * dist + RAY_EPSILON * d;
            return BsdfSample{Ray{origin, d, ray_in.time}, att, rmax(dot(n, d), 0.0) / PI, false};
        }
        case MatKind::DiffuseLight:
            return std::nullopt;
    }
    return std::nullopt;
}

std::pair<Color, double> material_eval(const Material& m, Vec3 wo, Vec3 wi, Vec3 n) {  // :207-223
    switch (m.kind) {
        case MatKind::Lambert:
        case MatKind::Subsurface: {
            double c = rmax(dot(n, wi), 0.0);
            if (c <= 0.0) return {Color(0, 0, 0), 0.0};
            return {m.c * (1.0 / PI), c / PI};
        }
        case MatKind::Ggx: {
            double a = rmax(m.p, 1e-3);
            return {ggx_eval(m.c, a, n, wo, wi), ggx_pdf(rmax(sampling_alpha(m), 1e-3), n, wo, wi)};
        }
        default:
            return {Color(0, 0, 0), 0.0};
    }
}

// ======================= src/env.rs =======================================
EnvMap EnvMap::from_pixels(size_t w, size_t h, std::vector<Color> data) {            // :61-89
    EnvMap e;
    e.width = w; e.height = h;
    e.row_cdf.assign(h + 1, 0.0);
    e.col_cdf.assign(h * (w + 1), 0.0);
    double total = 0.0;
    for (size_t y = 0; y < h; ++y) {
        double theta0 = PI * (double)y / (double)h;
        double theta1 = PI * (double)(y + 1) / (double)h;
        double row_weight = rmax(std::cos(theta0) - std::cos(theta1), 0.0);
        size_t row_offset = y * (w + 1);
        double row_sum = 0.0;
        e.col_cdf[row_offset] = 0.0;
        for (size_t x = 0; x < w; ++x) {
            double lum = rmax(luminance(data[y * w + x]), 0.0);
            row_sum += lum * row_weight;
            e.col_cdf[row_offset + x + 1] = row_sum;
        }
        total += row_sum;
        e.row_cdf[y + 1] = total;
    }
    e.data = std::move(data);
    e.total_weight = total;
    return e;
}

Color EnvMap::sample(Vec3 dir) const {                                                // :92-121
    Vec3 d = norm(dir);
    double theta = std::acos(clamp(d.y, -1.0, 1.0));
    double phi = std::atan2(d.z, d.x);
    if (phi < 0.0) phi += TAU;
    double u = phi / TAU;
    double v = theta / PI;
    double x = u * (double)width;
    double y = v * ((double)height - 1.0);
    size_t x0 = as_usize(std::floor(x)) % width;
    size_t x1 = (x0 + 1) % width;
    size_t y0 = as_usize(std::floor(clamp(y, 0.0, (double)(height - 1))));
    size_t y1 = std::min(y0 + 1, height - 1);
    double fx = x - std::floor(x);
    double fy = y - std::floor(y);
    Color c00 = data[y0 * width + x0], c10 = data[y0 * width + x1];
    Color c01 = data[y1 * width + x0], c11 = data[y1 * width + x1];
    Color c0 = c00 * (1.0 - fx) + c10 * fx;
    Color c1 = c01 * (1.0 - fx) + c11 * fx;
    return c0 * (1.0 - fy) + c1 * fy;
}

namespace {
size_t env_cdf_search(const double* cdf, size_t len, double x) {                      // env.rs:185-197
    size_t lo = 0, hi = len == 0 ? 0 : len - 1;
    while (lo + 1 < hi) {
        size_t mid = (lo + hi) / 2;
        if (cdf[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}
void sample_uniform_env(const EnvMap& env, Rng& rng, Vec3& dir, Color& rad, double& pdf) {  // :200-210
    double u = rng.next_f64();
    double v = rng.next_f64();
    double z = 1.0 - 2.0 * u;
    double r = std::sqrt(rmax(1.0 - z * z, 0.0));
    double phi = TAU * v;
    dir = Vec3(r * std::cos(phi), z, r * std::sin(phi));
    rad = env.sample(dir);
    pdf = 1.0 / (4.0 * PI);
}
}  // namespace

void EnvMap::sample_dir(Rng& rng, Vec3& dir, Color& rad, double& pdf_out) const {   // :124-152
    if (total_weight <= 0.0) { sample_uniform_env(*this, rng, dir, rad, pdf_out); return; }
    double r0 = rng.next_f64() * total_weight;
    size_t y = std::min(env_cdf_search(row_cdf.data(), row_cdf.size(), r0), height - 1);
    double row_start = row_cdf[y], row_end = row_cdf[y + 1];
    double row_sum = rmax(row_end - row_start, 0.0);
    if (row_sum <= 0.0) { sample_uniform_env(*this, rng, dir, rad, pdf_out); return; }
    double r1 = rng.next_f64() * row_sum;
    size_t row_offset = y * (width + 1);
    size_t x = std::min(env_cdf_search(col_cdf.data() + row_offset, width + 1, r1), width - 1);
    double u = ((double)x + rng.next_f64()) / (double)width;
    double v = ((double)y + rng.next_f64()) / (double)height;
    double theta = PI * v;
    double phi = TAU * u;
    double sin_theta = std::sin(theta);
    dir = Vec3(std::cos(phi) * sin_theta, std::cos(theta), std::sin(phi) * sin_theta);
    rad = sample(dir);
    pdf_out = pdf(dir);
}

double EnvMap::pdf(Vec3 dir) const {                                                  // :156-182
    if (total_weight <= 0.0) return 1.0 / (4.0 * PI);
    Vec3 d = norm(dir);
    double theta = std::acos(clamp(d.y, -1.0, 1.0));
    double phi = std::atan2(d.z, d.x);
    if (phi < 0.0) phi += TAU;
    double u = phi / TAU;
    double v = theta / PI;
    auto fclamp = [](double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); };
    size_t x = as_usize(fclamp(std::floor(u * (double)width), 0.0, (double)(width - 1)));
    size_t y = as_usize(fclamp(std::floor(v * (double)height), 0.0, (double)(height - 1)));
    double theta0 = PI * (double)y / (double)height;
    double theta1 = PI * (double)(y + 1) / (double)height;
    double sin_theta = rmax(std::sin(theta), 1e-6);
    double row_weight = rmax(std::cos(theta0) - std::cos(theta1), 0.0);
    double lum = rmax(luminance(data[y * width + x]), 0.0);
    double weight = lum * row_weight;
    if (weight <= 0.0) return 0.0;
    double pdf_uv = (weight / total_weight) * (double)width * (double)height;
    return pdf_uv / (2.0 * PI * PI * sin_theta);
}

// ======================= src/world.rs =====================================
std::optional<Hit> World::hit(const Ray& r, double tmin, double tmax, TraversalCounts* cnt) const {  // :81-121
    if (cnt) cnt->world_hits++;
    double closest = tmax;
    std::optional<Hit> best;
    for (const Instance& inst : instances) {
        if (inst.mesh_id >= meshes.size()) continue;
        const Mesh& mesh = meshes[inst.mesh_id];
        Vec3 o_obj = inst.xform.apply_point_inv(r.o);
        Vec3 d_obj = norm(inst.xform.apply_vec_inv(r.d));
        Ray r_obj{o_obj, d_obj, r.time};
        if (auto h_obj = mesh.bvh.hit(mesh.tris, r_obj, tmin, 1e30, cnt)) {
            Vec3 p_world = inst.xform.apply_point(h_obj->p);
            Vec3 n_world = inst.xform.apply_normal(h_obj->n);
            double t_world = dot(p_world - r.o, r.d);
            if (t_world > tmin && t_world < closest) {
                closest = t_world;
                size_t mat_id = inst.mat_override ? *inst.mat_override : h_obj->mat_id;
                best = Hit{t_world, p_world, n_world, mat_id};
            }
        }
    }
    for (const Sphere& s : spheres) {
        if (cnt) cnt->sphere_tests++;
        if (auto h = sphere_hit(s, r, tmin, closest)) { closest = h->t; best = h; }
    }
    return best;
}

bool World::tri_world_verts(size_t mesh_id, size_t tri_id, size_t inst_id, double time, Vec3& v0, Vec3& v1,
                            Vec3& v2) const {  // :276-292
    if (mesh_id >= meshes.size() || tri_id >= meshes[mesh_id].tris.size() || inst_id >= instances.size())
        return false;
    const Instance& inst = instances[inst_id];
    Vec3 a, b, c;
    meshes[mesh_id].tris[tri_id].vertices_at(time, a, b, c);
    v0 = inst.xform.apply_point(a);
    v1 = inst.xform.apply_point(b);
    v2 = inst.xform.apply_point(c);
    return true;
}

double World::light_area(const Light& l, double time) const {                         // :226-238
    if (l.is_sphere) {
        if (l.idx >= spheres.size()) return 0.0;
        const Sphere& s = spheres[l.idx];
        return 4.0 * PI * s.r * s.r;
    }
    Vec3 v0, v1, v2;
    if (!tri_world_verts(l.mesh_id, l.tri_id, l.inst_id, time, v0, v1, v2)) return 0.0;
    return 0.5 * len(cross(v1 - v0, v2 - v0));
}

bool World::light_sample_surface(const Light& l, double time, Rng& rng, Vec3& pos, Vec3& nrm,
                                 double& area) const {  // :242-272
    if (l.is_sphere) {
        if (l.idx >= spheres.size()) return false;
        const Sphere& s = spheres[l.idx];
        double u = rng.next_f64();
        double v = rng.next_f64();
        double z = 1.0 - 2.0 * u;
        double r = std::sqrt(rmax(1.0 - z * z, 0.0));
        double phi = TAU * v;
        Vec3 dir(r * std::cos(phi), z, r * std::sin(phi));
        pos = s.c + dir * s.r;
        nrm = dir;
        area = 4.0 * PI * s.r * s.r;
        return true;
    }
    Vec3 v0w, v1w, v2w;
    if (!tri_world_verts(l.mesh_id, l.tri_id, l.inst_id, time, v0w, v1w, v2w)) return false;
    double u = rng.next_f64();
    double v = rng.next_f64();
    double su = std::sqrt(u);
    double b0 = 1.0 - su;
    double b1 = v * su;
    double b2 = 1.0 - b0 - b1;
    pos = v0w * b0 + v1w * b1 + v2w * b2;
    Vec3 nn = cross(v1w - v0w, v2w - v0w);
    area = 0.5 * len(nn);
    nrm = area > 0.0 ? nn / (2.0 * area) : Vec3(0.0, 1.0, 0.0);
    return true;
}

void World::build_lights(const std::vector<Material>& mats, const std::vector<Material>* sampling) {  // :127-167
    lights.clear();
    light_cdf.clear();
    double total = 0.0;
    // test extension: selection weights from the sampling materials when given
    const std::vector<Material>& wm = sampling ? *sampling : mats;
    auto add = [&](const Light& light, Color emit, double area, size_t mat_id) {
        double weight = area * luminance(*material_emitted(wm[mat_id]));
        if (weight > 0.0) {
            total += weight;
            lights.push_back(LightInfo{light, emit, weight});
            light_cdf.push_back(total);
        }
    };
    auto emit_of = [&](size_t mat_id) -> std::optional<Color> {
        if (mat_id >= mats.size()) return std::nullopt;
        return material_emitted(mats[mat_id]);
    };
    for (size_t idx = 0; idx < spheres.size(); ++idx) {
        if (auto e = emit_of(spheres[idx].mat_id)) {
            Light l{true, idx, 0, 0, 0};
            add(l, *e, light_area(l, 0.5), spheres[idx].mat_id);
        }
    }
    for (size_t inst_id = 0; inst_id < instances.size(); ++inst_id) {
        const Instance& inst = instances[inst_id];
        if (inst.mesh_id >= meshes.size()) continue;
        const Mesh& mesh = meshes[inst.mesh_id];
        for (size_t tri_id = 0; tri_id < mesh.tris.size(); ++tri_id) {
            size_t mat_id = inst.mat_override ? *inst.mat_override : mesh.tris[tri_id].mat_id;
            if (auto e = emit_of(mat_id)) {
                Light l{false, 0, inst.mesh_id, tri_id, inst_id};
                add(l, *e, light_area(l, 0.5), mat_id);
            }
        }
    }
    light_total = total;
}

namespace {
size_t world_cdf_search(const std::vector<double>& cdf, double x) {                  // :324-336
    size_t lo = 0, hi = cdf.empty() ? 0 : cdf.size() - 1;
    while (lo + 1 < hi) {
        size_t mid = (lo + hi) / 2;
        if (cdf[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}
}  // namespace

std::optional<LightSample> World::sample_light(Rng& rng, double time, Vec3 p) const {  // :171-209
    if (light_total <= 0.0 || lights.empty()) return std::nullopt;
    double r = rng.next_f64() * light_total;
    size_t idx = std::min(world_cdf_search(light_cdf, r), lights.size() - 1);
    const LightInfo& info = lights[idx];
    double pdf_select = info.weight / light_total;
    Vec3 pos, normal;
    double area;
    if (!light_sample_surface(info.light, time, rng, pos, normal, area)) return std::nullopt;
    if (area <= 0.0) return std::nullopt;
    Vec3 to_light = pos - p;
    double dist2 = dot(to_light, to_light);
    if (dist2 <= 1e-12) return std::nullopt;
    double dist = std::sqrt(dist2);
    Vec3 wi = to_light / dist;
    double cos_light = rmax(dot(normal, -wi), 0.0);
    if (cos_light <= 0.0) return std::nullopt;
    double pdf_area = 1.0 / area;
    double pdf_omega = pdf_area * dist2 / cos_light;
    double pdf = pdf_select * pdf_omega;
    if (pdf <= 0.0) return std::nullopt;
    return LightSample{pos, normal, info.emit, pdf};
}

// ======================= src/integrator.rs ================================
namespace {
Color sky(Vec3 d) {                                                                   // :25-28
    double t = 0.5 * (d.y + 1.0);
    return (1.0 - t) * Vec3(0.9, 0.95, 1.0) + t * Vec3(0.6, 0.75, 1.0);
}
Color background(Vec3 d, const EnvMap* env) { return env ? env->sample(d) : sky(d); }  // :31-37
double mis_weight(double a, double b) {                                               // :221-225
    double a2 = a * a, b2 = b * b;
    return (a2 + b2 > 0.0) ? a2 / (a2 + b2) : 0.0;
}
Vec3 oriented_normal(Vec3 n, Vec3 d) { return dot(n, d) < 0.0 ? n : -n; }             // :138-140

Color nee_environment(const World& world, const EnvMap& env, const Material& mat, Color beta, Vec3 hit_p,
                      Vec3 n, const Ray& ray, Rng& rng, TraversalCounts* cnt) {       // :148-172
    Vec3 wi; Color li; double pdf_env;
    env.sample_dir(rng, wi, li, pdf_env);
    double c = rmax(dot(n, wi), 0.0);
    if (c <= 0.0 || pdf_env <= 0.0) return Color(0, 0, 0);
    Ray shadow{hit_p + RAY_EPSILON * wi, wi, ray.time};
    if (world.hit(shadow, RAY_EPSILON, RAY_T_MAX, cnt)) return Color(0, 0, 0);
    auto [f, pdf_bsdf] = material_eval(mat, norm(-ray.d), wi, n);
    double w = mis_weight(pdf_env, pdf_bsdf);
    return hadamard(hadamard(beta, f), li) * (c * w / pdf_env);
}

Color nee_area_light(const World& world, const Material& mat, Color beta, Vec3 hit_p, Vec3 n, const Ray& ray,
                     const LightSample& ls, TraversalCounts* cnt) {                   // :178-213
    Vec3 to_light = ls.position - hit_p;
    double dist2 = dot(to_light, to_light);
    double dist = std::sqrt(dist2);
    if (dist <= 1e-6) return Color(0, 0, 0);
    Vec3 wi = to_light / dist;
    double c = rmax(dot(n, wi), 0.0);
    if (c <= 0.0) return Color(0, 0, 0);
    Ray shadow{hit_p + RAY_EPSILON * wi, wi, ray.time};
    double tmax = rmax(dist - RAY_EPSILON, RAY_EPSILON);
    if (world.hit(shadow, RAY_EPSILON, tmax, cnt)) return Color(0, 0, 0);
    auto [f, pdf_bsdf] = material_eval(mat, norm(-ray.d), wi, n);
    if (ls.pdf <= 0.0) return Color(0, 0, 0);
    double w = mis_weight(ls.pdf, pdf_bsdf);
    return hadamard(hadamard(beta, f), ls.emit) * (c * w / ls.pdf);
}
}  // namespace

Color radiance(const World& world, const std::vector<Material>& mats, const EnvMap* env, Ray ray, Rng& rng,
               PathLimits limits, TraversalCounts* cnt) {  // :53-135
    Color acc(0, 0, 0);
    Color beta(1, 1, 1);
    double last_bsdf_pdf = 0.0;
    bool last_non_delta = false;
    for (size_t bounce = 0; bounce < limits.max_bounces; ++bounce) {
        auto hit = world.hit(ray, RAY_EPSILON, RAY_T_MAX, cnt);
        if (!hit) {
            Color contrib = hadamard(beta, background(ray.d, env));
            if (env && last_non_delta) {
                double pdf_env = env->pdf(ray.d);
                contrib = contrib * mis_weight(last_bsdf_pdf, pdf_env);
            }
            acc = acc + clamp_luminance(contrib, FIREFLY_CLAMP);
            break;
        }
        if (bounce >= limits.rr_start) {  // :89-95
            double p = rmax(rmin(rmax(rmax(beta.x, beta.y), beta.z), 0.95), 0.05);
            if (rng.next_f64() > p) break;
            beta = beta / p;
        }
        const Material& mat = mats[hit->mat_id];
        if (auto emit = material_emitted(mat)) {  // :100-104
            acc = acc + clamp_luminance(hadamard(beta, *emit), FIREFLY_CLAMP);
            break;
        }
        Vec3 n = oriented_normal(hit->n, ray.d);
        if (!material_is_delta(mat)) {  // :108-121
            if (env) acc = acc + nee_environment(world, *env, mat, beta, hit->p, n, ray, rng, cnt);
            if (auto ls = world.sample_light(rng, ray.time, hit->p))
                acc = acc + nee_area_light(world, mat, beta, hit->p, n, ray, *ls, cnt);
        }
        auto s = material_sample(mat, ray, *hit, rng);  // :124-132
        if (!s) break;
        last_bsdf_pdf = s->pdf;
        last_non_delta = !s->is_delta;
        beta = hadamard(beta, s->weight);
        ray = s->scattered;
    }
    return acc;
}

// ======================= src/render.rs ====================================
uint64_t interleave_bits(uint64_t v) {                                                // :291-299
    uint64_t x = v & 0x00000000ffffffffull;
    x = (x | (x << 16)) & 0x0000ffff0000ffffull;
    x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
    x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}
uint64_t morton2(size_t tx, size_t ty, size_t tiles_x, size_t tiles_y) {              // :284-288
    uint64_t x = std::min(tx, tiles_x == 0 ? 0 : tiles_x - 1);
    uint64_t y = std::min(ty, tiles_y == 0 ? 0 : tiles_y - 1);
    return interleave_bits(x) | (interleave_bits(y) << 1);
}

std::vector<Task> make_tasks(const RenderConfig& cfg) {                               // :75-100
    std::vector<Task> tasks;
    for (size_t y = 0; y < cfg.height; y += cfg.tile)
        for (size_t x = 0; x < cfg.width; x += cfg.tile)
            tasks.push_back(Task{0, x, y, std::min(x + cfg.tile, cfg.width), std::min(y + cfg.tile, cfg.height), 0,
                                 cfg.spp});
    if (cfg.morton_enabled) {
        size_t tiles_x = (cfg.width + cfg.tile - 1) / cfg.tile;
        size_t tiles_y = (cfg.height + cfg.tile - 1) / cfg.tile;
        // slice::sort_by_key is stable.
        std::stable_sort(tasks.begin(), tasks.end(), [&](const Task& a, const Task& b) {
            return morton2(a.x0 / cfg.tile, a.y0 / cfg.tile, tiles_x, tiles_y) <
                   morton2(b.x0 / cfg.tile, b.y0 / cfg.tile, tiles_x, tiles_y);
        });
    }
    for (size_t i = 0; i < tasks.size(); ++i) tasks[i].id = i;
    return tasks;
}

namespace {
// One tile task (render.rs:129-205).  Pixel values do not depend on the
// merge order (each pixel belongs to exactly one task), so results are
// written straight into the film.
// reseed > 0: at every sample s that is a multiple of reseed the pixel's RNG
// restarts from seed_for(x, y, s) ^ seed (the stream a task starting at s
// would draw), while the loop -- sums in sample order, one Welford over all
// samples -- stays the reference's.
void run_task(const Scene& scene, const RenderConfig& cfg, const Task& t, const Rect& out_rect, double* acc,
              double* acc_w, double* acc_sq, TraversalCounts* cnt, size_t reseed = 0) {
    const double inv_w = 1.0 / (double)cfg.width;
    const double inv_h = 1.0 / (double)cfg.height;
    PathLimits limits{cfg.max_bounces, cfg.rr_start};
    const EnvMap* env = scene.env ? &*scene.env : nullptr;
    for (size_t y = t.y0; y < t.y1; ++y) {
        for (size_t x = t.x0; x < t.x1; ++x) {
            Color c(0, 0, 0);
            Color c2(0, 0, 0);
            Rng rng(seed_for((uint32_t)x, (uint32_t)y, (uint32_t)t.sample_start) ^ cfg.seed);
            double wsum;
            if (cfg.adaptive_enabled) {  // :143-180
                size_t max_spp = std::max<size_t>(t.sample_end - t.sample_start, 1);
                size_t min_spp = std::min(std::max<size_t>(cfg.adaptive_min_spp, 1), max_spp);
                size_t n = 0;
                double mean = 0.0, m2 = 0.0;
                for (size_t s = t.sample_start; s < t.sample_end; ++s) {
                    if (reseed && s % reseed == 0) rng = Rng(seed_for((uint32_t)x, (uint32_t)y, (uint32_t)s) ^ cfg.seed);
                    double jx = rng.next_f64();
                    double jy = rng.next_f64();
                    double sx = ((double)x + jx) * inv_w * 2.0 - 1.0;
                    double sy = 1.0 - ((double)y + jy) * inv_h * 2.0;
                    Ray ray = scene.cam.ray(sx, sy, rng);
                    Color sample = radiance(scene.world, scene.mats, env, ray, rng, limits, cnt);
                    c = c + sample;
                    c2 = c2 + hadamard(sample, sample);
                    n += 1;
                    double lum = luminance(sample);
                    double delta = lum - mean;
                    mean += delta / (double)n;
                    double delta2 = lum - mean;
                    m2 += delta * delta2;
                    if (n >= min_spp) {
                        double var = n > 1 ? m2 / (double)(n - 1) : std::numeric_limits<double>::infinity();
                        double denom = rmax(std::fabs(mean), 1e-4);
                        double rel_std = std::sqrt(var) / denom;
                        if (rel_std < cfg.adaptive_threshold) break;
                    }
                }
                wsum = (double)n;
            } else {  // :181-191
                for (size_t s = t.sample_start; s < t.sample_end; ++s) {
                    if (reseed && s % reseed == 0) rng = Rng(seed_for((uint32_t)x, (uint32_t)y, (uint32_t)s) ^ cfg.seed);
                    double jx = rng.next_f64();
                    double jy = rng.next_f64();
                    double sx = ((double)x + jx) * inv_w * 2.0 - 1.0;
                    double sy = 1.0 - ((double)y + jy) * inv_h * 2.0;
                    Ray ray = scene.cam.ray(sx, sy, rng);
                    Color sample = radiance(scene.world, scene.mats, env, ray, rng, limits, cnt);
                    c = c + sample;
                    c2 = c2 + hadamard(sample, sample);
                }
                wsum = (double)(t.sample_end - t.sample_start);
            }
            // task.rs:42-45 idx(x, y, w), relative to the output rectangle
            size_t gi = (y - out_rect.y0) * (out_rect.x1 - out_rect.x0) + (x - out_rect.x0);
            acc[3 * gi + 0] = acc[3 * gi + 0] + c.x;
            acc[3 * gi + 1] = acc[3 * gi + 1] + c.y;
            acc[3 * gi + 2] = acc[3 * gi + 2] + c.z;
            acc_w[gi] += wsum;
            if (acc_sq) {
                acc_sq[3 * gi + 0] += c2.x;
                acc_sq[3 * gi + 1] += c2.y;
                acc_sq[3 * gi + 2] += c2.z;
            }
        }
    }
}
}  // namespace

void render(const Scene& scene, const RenderConfig& cfg, double* acc, double* acc_w, double* acc_sq, int threads,
            TraversalCounts* cnt, const Rect* rect, size_t sample_chunk, size_t reseed) {  // :42-278 (no checkpoints)
    Rect r = rect ? *rect : Rect{0, 0, cfg.width, cfg.height};
    size_t npx = (r.x1 - r.x0) * (r.y1 - r.y0);
    for (size_t i = 0; i < 3 * npx; ++i) acc[i] = 0.0;
    for (size_t i = 0; i < npx; ++i) acc_w[i] = 0.0;
    if (acc_sq)
        for (size_t i = 0; i < 3 * npx; ++i) acc_sq[i] = 0.0;
    std::vector<Task> tiles;
    for (const Task& t : make_tasks(cfg)) {  // clip the tile tasks to the rectangle
        Task c = t;
        c.x0 = std::max(t.x0, r.x0); c.x1 = std::min(t.x1, r.x1);
        c.y0 = std::max(t.y0, r.y0); c.y1 = std::min(t.y1, r.y1);
        if (c.x0 < c.x1 && c.y0 < c.y1) tiles.push_back(c);
    }
    // Sample-chunked tasks: chunk k of every tile, chunk by chunk.  Each chunk
    // renders into its own film, and the films are added in chunk order
    // below -- the task-id merge order of render.rs:226-241 for this list.
    const size_t n_chunks = (sample_chunk > 0 && sample_chunk < cfg.spp) ? (cfg.spp + sample_chunk - 1) / sample_chunk : 1;
    std::vector<Task> tasks;
    for (size_t k = 0; k < n_chunks; ++k)
        for (const Task& t : tiles) {
            Task c = t;
            if (n_chunks > 1) {
                c.sample_start = k * sample_chunk;
                c.sample_end = std::min(cfg.spp, (k + 1) * sample_chunk);
            }
            c.id = tasks.size();
            tasks.push_back(c);
        }
    std::vector<std::vector<double>> part_acc, part_w, part_sq;
    if (n_chunks > 1) {
        part_acc.assign(n_chunks, std::vector<double>(3 * npx, 0.0));
        part_w.assign(n_chunks, std::vector<double>(npx, 0.0));
        if (acc_sq) part_sq.assign(n_chunks, std::vector<double>(3 * npx, 0.0));
    }
    if (threads < 1) threads = 1;
    std::atomic<size_t> next{0};
    std::vector<TraversalCounts> counts((size_t)threads);
    auto worker = [&](int tid) {  // crossbeam worker loop (render.rs:132-205)
        for (;;) {
            size_t i = next.fetch_add(1);
            if (i >= tasks.size()) break;
            TraversalCounts* tc = cnt ? &counts[(size_t)tid] : nullptr;
            if (n_chunks > 1) {
                const size_t k = i / tiles.size();
                run_task(scene, cfg, tasks[i], r, part_acc[k].data(), part_w[k].data(),
                         acc_sq ? part_sq[k].data() : nullptr, tc);
            } else {
                run_task(scene, cfg, tasks[i], r, acc, acc_w, acc_sq, tc, reseed);
            }
        }
    };
    if (threads == 1) {
        worker(0);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t) pool.emplace_back(worker, t);
        for (auto& th : pool) th.join();
    }
    for (size_t k = 0; k < n_chunks && n_chunks > 1; ++k) {  // merge in task-id order (render.rs:226-241)
        for (size_t i = 0; i < 3 * npx; ++i) acc[i] = acc[i] + part_acc[k][i];
        for (size_t i = 0; i < npx; ++i) acc_w[i] += part_w[k][i];
        if (acc_sq)
            for (size_t i = 0; i < 3 * npx; ++i) acc_sq[i] += part_sq[k][i];
    }
    if (cnt) {
        for (const auto& c : counts) {
            cnt->world_hits += c.world_hits;
            cnt->node_pops += c.node_pops;
            cnt->node_box_tests += c.node_box_tests;
            cnt->tri_tests += c.tri_tests;
            cnt->sphere_tests += c.sphere_tests;
        }
    }
}

}  // namespace ref
