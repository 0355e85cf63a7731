// Host-side scene construction and flattening (see host_scene.hpp).
// Compiled with -ffp-contract=off for the host: every f64 quantity derived
// here feeds the f64 kernel, which must follow the reference's arithmetic.
#include "host_scene.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <future>
#include <limits>
#include <stdexcept>
#include <thread>

namespace tpt {

namespace {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr size_t kBins = 8;   // SAH_BINS (src/constants.rs:22)
constexpr size_t kLeaf = 4;   // LEAF_SIZE (src/constants.rs:24)

inline double dmax(double a, double b) { return std::fmax(a, b); }
inline double dmin(double a, double b) { return std::fmin(a, b); }
inline HVec sub(HVec a, HVec b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline HVec add(HVec a, HVec b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline HVec scale(HVec a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(HVec a, HVec b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline HVec cross(HVec a, HVec b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double length(HVec a) { return std::sqrt(dot(a, a)); }
inline HVec normalize(HVec a) {
    double l = dmax(length(a), 1e-30);
    return {a.x / l, a.y / l, a.z / l};
}
inline HVec load3(const double* p) { return {p[0], p[1], p[2]}; }
inline void store3(double* o, HVec v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }
inline double luma(const double* c) { return 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2]; }

// A box as six doubles; `grow`/`merge` use min/max, which are exact.
struct Box {
    double lo[3], hi[3];
    static Box none() {
        const double inf = std::numeric_limits<double>::infinity();
        return Box{{inf, inf, inf}, {-inf, -inf, -inf}};
    }
    void merge(const Box& b) {
        for (int k = 0; k < 3; ++k) { lo[k] = dmin(lo[k], b.lo[k]); hi[k] = dmax(hi[k], b.hi[k]); }
    }
    void grow(const double* p) {
        for (int k = 0; k < 3; ++k) { lo[k] = dmin(lo[k], p[k]); hi[k] = dmax(hi[k], p[k]); }
    }
    double half_area() const {  // the reference's 2*(xy+yz+zx) without the 2
        double ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
        return ex * ey + ey * ez + ez * ex;
    }
};

// Rust `f as usize` for the bin computation: saturating, NaN -> 0.
inline size_t bin_index(double cv, double minc, double inv_extent) {
    double f = (cv - minc) * inv_extent * (double)kBins;
    size_t b = (f > 0.0) ? (f >= 1.8446744073709552e19 ? SIZE_MAX : (size_t)f) : 0;
    return b >= kBins ? kBins - 1 : b;
}

}  // namespace

// ------------------------------------------------------------------------
// Reference BVH (src/bvh.rs:51-242).  Same split decisions and numbering as
// the reference's recursive build, done with an explicit stack (right range
// pushed first, so nodes come out in the same preorder) and a stable
// counting sort over the 8 bin keys in place of slice::sort_by_key.
HostBvh build_mesh_bvh(const double* positions, int64_t n_vertices, const int32_t* tri_idx, int64_t n_tris) {
    HostBvh out;
    const size_t nt = (size_t)n_tris;
    std::vector<Box> tbox(nt);
    std::vector<double> cen(3 * nt);
    for (size_t i = 0; i < nt; ++i) {
        Box b = Box::none();
        for (int k = 0; k < 3; ++k) {
            int32_t vi = tri_idx[3 * i + k];
            if (vi < 0 || vi >= n_vertices) throw std::runtime_error("triangle vertex index out of range");
            b.grow(positions + 3 * (size_t)vi);
        }
        // Aabb::from_points pads by 1e-9 (geometry.rs:70-80); the static
        // triangle's open/close boxes are equal, so their union is this box.
        for (int k = 0; k < 3; ++k) { b.lo[k] = b.lo[k] - 1e-9; b.hi[k] = b.hi[k] + 1e-9; }
        tbox[i] = b;
        for (int k = 0; k < 3; ++k) cen[3 * i + k] = (b.lo[k] + b.hi[k]) * 0.5;
    }
    out.indices.resize(nt);
    for (size_t i = 0; i < nt; ++i) out.indices[i] = (int64_t)i;
    if (nt == 0) return out;

    std::vector<int64_t>& ord = out.indices;
    std::vector<int64_t> scratch(nt);
    std::vector<uint8_t> bin_of(nt);
    struct Job { size_t start, end; int64_t parent; int side; int depth; };
    std::vector<Job> jobs;
    jobs.push_back(Job{0, nt, -1, 0, 1});
    while (!jobs.empty()) {
        Job j = jobs.back();
        jobs.pop_back();
        const size_t n = j.end - j.start;
        Box bbox = Box::none(), cbox = Box::none();
        for (size_t k = j.start; k < j.end; ++k) {
            size_t t = (size_t)ord[k];
            bbox.merge(tbox[t]);
            cbox.grow(&cen[3 * t]);
        }
        const int64_t node = (int64_t)(out.left_right.size() / 2);
        for (int k = 0; k < 3; ++k) out.bbox.push_back(bbox.lo[k]);
        for (int k = 0; k < 3; ++k) out.bbox.push_back(bbox.hi[k]);
        out.left_right.push_back(-1); out.left_right.push_back(-1);
        out.start_count.push_back(0); out.start_count.push_back(0);
        if (j.parent >= 0) out.left_right[2 * (size_t)j.parent + (size_t)j.side] = (int32_t)node;
        out.max_depth = std::max(out.max_depth, j.depth);
        if (n <= kLeaf) {
            out.start_count[2 * (size_t)node] = (uint32_t)j.start;
            out.start_count[2 * (size_t)node + 1] = (uint32_t)n;
            continue;
        }
        double ext[3] = {cbox.hi[0] - cbox.lo[0], cbox.hi[1] - cbox.lo[1], cbox.hi[2] - cbox.lo[2]};
        int axis = (ext[0] >= ext[1] && ext[0] >= ext[2]) ? 0 : (ext[1] >= ext[2] ? 1 : 2);
        size_t mid = j.start + n / 2;
        if (n >= kBins * 2) {
            double minc = cbox.lo[axis], maxc = cbox.hi[axis];
            double extent = maxc - minc;
            if (extent > 1e-12) {
                double inv_extent = 1.0 / extent;
                Box bbin[kBins];
                size_t cnt[kBins] = {0};
                for (size_t b = 0; b < kBins; ++b) bbin[b] = Box::none();
                for (size_t k = j.start; k < j.end; ++k) {
                    size_t t = (size_t)ord[k];
                    size_t b = bin_index(cen[3 * t + (size_t)axis], minc, inv_extent);
                    bin_of[t] = (uint8_t)b;
                    bbin[b].merge(tbox[t]);
                    cnt[b] += 1;
                }
                // Prefix boxes from the left and from the right (bvh.rs:137-157).
                Box lbox[kBins], rbox[kBins];
                size_t lcnt[kBins], rcnt[kBins];
                Box acc = Box::none();
                size_t acc_n = 0;
                for (size_t i = 0; i < kBins; ++i) {
                    if (cnt[i] > 0) { acc.merge(bbin[i]); acc_n += cnt[i]; }
                    lbox[i] = acc; lcnt[i] = acc_n;
                }
                acc = Box::none(); acc_n = 0;
                for (size_t i = kBins; i-- > 0;) {
                    if (cnt[i] > 0) { acc.merge(bbin[i]); acc_n += cnt[i]; }
                    rbox[i] = acc; rcnt[i] = acc_n;
                }
                double best = std::numeric_limits<double>::infinity();
                size_t split = 0;
                for (size_t i = 0; i + 1 < kBins; ++i) {
                    size_t lc = lcnt[i], rc = rcnt[i + 1];
                    if (lc == 0 || rc == 0) continue;
                    double la = 2.0 * lbox[i].half_area();
                    double ra = 2.0 * rbox[i + 1].half_area();
                    double cost = la * (double)lc + ra * (double)rc;
                    if (cost < best) { best = cost; split = i + 1; }
                }
                if (std::isfinite(best)) {
                    // Stable counting sort of the range by bin key.
                    size_t off[kBins];
                    size_t run = 0;
                    for (size_t b = 0; b < kBins; ++b) { off[b] = run; run += cnt[b]; }
                    for (size_t k = j.start; k < j.end; ++k) {
                        int64_t t = ord[k];
                        scratch[j.start + off[bin_of[(size_t)t]]++] = t;
                    }
                    std::copy(scratch.begin() + (ptrdiff_t)j.start, scratch.begin() + (ptrdiff_t)j.end,
                              ord.begin() + (ptrdiff_t)j.start);
                    size_t left_total = 0;
                    for (size_t b = 0; b < split; ++b) left_total += cnt[b];
                    if (left_total > 0 && left_total < n) mid = j.start + left_total;
                }
            }
        }
        jobs.push_back(Job{mid, j.end, node, 1, j.depth + 1});
        jobs.push_back(Job{j.start, mid, node, 0, j.depth + 1});
    }
    return out;
}

// ------------------------------------------------------------------------
namespace {

void make_camera(const tpt_camera_desc& d, CameraF64& c) {  // src/ray.rs:36-86
    HVec eye = load3(d.eye), target = load3(d.target), up = load3(d.up);
    double theta = d.fov_y_deg * (kPi / 180.0);
    c.half_h = std::tan(theta * 0.5);
    c.half_w = d.aspect * c.half_h;
    HVec w = normalize(sub(eye, target));
    HVec u = normalize(cross(up, w));
    HVec v = cross(w, u);
    store3(c.o, eye); store3(c.u, u); store3(c.v, v); store3(c.w, w);
    if (d.kind == TPT_CAMERA_LOOK_AT_DOF) {
        c.lens_radius = 0.5 * dmax(d.aperture, 0.0);
        c.focus_dist = dmax(d.focus_dist, 1e-6);
    } else {
        c.lens_radius = 0.0;
        c.focus_dist = length(sub(eye, target));
    }
    c.shutter_open = 0.0;
    c.shutter_close = 1.0;
}

// Transform::from_affine (src/transform.rs:24-27) with Mat3::invert
// (src/math.rs:151-169) and transpose.
void make_instance(const tpt_instance_desc& d, InstanceF64& x) {
    const double* m = d.linear;
    auto M = [&](int r, int c) { return m[3 * r + c]; };
    double det = M(0, 0) * (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1)) - M(0, 1) * (M(1, 0) * M(2, 2) - M(1, 2) * M(2, 0)) +
                 M(0, 2) * (M(1, 0) * M(2, 1) - M(1, 1) * M(2, 0));
    double id = 1.0 / det;
    double r[9];
    r[0] = (M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1)) * id;
    r[1] = (M(0, 2) * M(2, 1) - M(0, 1) * M(2, 2)) * id;
    r[2] = (M(0, 1) * M(1, 2) - M(0, 2) * M(1, 1)) * id;
    r[3] = (M(1, 2) * M(2, 0) - M(1, 0) * M(2, 2)) * id;
    r[4] = (M(0, 0) * M(2, 2) - M(0, 2) * M(2, 0)) * id;
    r[5] = (M(0, 2) * M(1, 0) - M(0, 0) * M(1, 2)) * id;
    r[6] = (M(1, 0) * M(2, 1) - M(1, 1) * M(2, 0)) * id;
    r[7] = (M(0, 1) * M(2, 0) - M(0, 0) * M(2, 1)) * id;
    r[8] = (M(0, 0) * M(1, 1) - M(0, 1) * M(1, 0)) * id;
    for (int i = 0; i < 9; ++i) { x.a[i] = m[i]; x.a_inv[i] = r[i]; }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) x.nmat[3 * i + j] = r[3 * j + i];
    for (int i = 0; i < 3; ++i) x.t[i] = d.translation[i];
    x.mesh_id = (int32_t)d.mesh_id;
    x.mat_override = (int32_t)d.mat_override;
}

HVec apply_point(const InstanceF64& x, HVec p) {  // src/transform.rs:75-77
    const double* a = x.a;
    HVec r{a[0] * p.x + a[1] * p.y + a[2] * p.z, a[3] * p.x + a[4] * p.y + a[5] * p.z,
           a[6] * p.x + a[7] * p.y + a[8] * p.z};
    return add(r, load3(x.t));
}

bool is_emitter(const std::vector<tpt_material>& mats, int64_t id) {
    return id >= 0 && id < (int64_t)mats.size() && mats[(size_t)id].kind == TPT_MAT_DIFFUSE_LIGHT;
}

// Triangle::vertices_at(time) for a static triangle, then the instance
// transform (src/world.rs:276-292).
void tri_world(const HostScene& hs, const InstanceF64& inst, int64_t tri, double time, HVec v[3]) {
    const HostScene::Mesh& m = hs.meshes[(size_t)inst.mesh_id];
    for (int k = 0; k < 3; ++k) {
        HVec p = load3(&m.pos[3 * (size_t)m.idx[3 * (size_t)tri + (size_t)k]]);
        HVec q = add(scale(p, 1.0 - time), scale(p, time));
        v[k] = apply_point(inst, q);
    }
}

}  // namespace

// World::build_lights (src/world.rs:127-167): spheres, then per instance per
// triangle; weight = area at time 0.5 x luminance of the emission.
void build_lights(HostScene& hs) {
    hs.lights.clear();
    hs.light_cdf.clear();
    double total = 0.0;
    auto add_light = [&](const HostLight& l, double area) {
        double weight = area * luma(hs.smats[(size_t)l.mat].rgb);
        if (weight > 0.0) {
            total += weight;
            HostLight k = l;
            k.weight = weight;
            hs.lights.push_back(k);
            hs.light_cdf.push_back(total);
        }
    };
    for (size_t s = 0; s < hs.spheres.size(); ++s) {
        if (!is_emitter(hs.smats, hs.spheres[s].mat_id)) continue;
        HostLight l{};
        l.is_sphere = 1;
        l.mat = hs.spheres[s].mat_id;
        l.sphere = (int64_t)s;
        const double* e = hs.mats[(size_t)hs.spheres[s].mat_id].rgb;
        l.emit[0] = e[0]; l.emit[1] = e[1]; l.emit[2] = e[2];
        double r = hs.spheres[s].radius;
        add_light(l, 4.0 * kPi * r * r);
    }
    for (size_t ii = 0; ii < hs.instances.size(); ++ii) {
        const InstanceF64& inst = hs.instances[ii];
        const HostScene::Mesh& m = hs.meshes[(size_t)inst.mesh_id];
        for (size_t t = 0; t < m.mat.size(); ++t) {
            int64_t mid = inst.mat_override >= 0 ? inst.mat_override : m.mat[t];
            if (!is_emitter(hs.smats, mid)) continue;
            HostLight l{};
            l.is_sphere = 0;
            l.mat = mid;
            l.mesh = inst.mesh_id; l.tri = (int64_t)t; l.inst = (int64_t)ii;
            const double* e = hs.mats[(size_t)mid].rgb;
            l.emit[0] = e[0]; l.emit[1] = e[1]; l.emit[2] = e[2];
            HVec v[3];
            tri_world(hs, inst, (int64_t)t, 0.5, v);
            add_light(l, 0.5 * length(cross(sub(v[1], v[0]), sub(v[2], v[0]))));
        }
    }
    hs.light_total = total;
}

void set_materials(HostScene& hs, const tpt_material* mats, const tpt_material* sampling, size_t n) {
    if (n != hs.mats.size()) throw std::runtime_error("set_materials: material count differs from the scene's");
    if (!mats) throw std::runtime_error("set_materials: null materials");
    for (size_t i = 0; i < n; ++i) {
        if (mats[i].kind != hs.mats[i].kind || (sampling && sampling[i].kind != hs.mats[i].kind))
            throw std::runtime_error("set_materials: a material changes kind");
    }
    hs.mats.assign(mats, mats + n);
    if (sampling) hs.smats.assign(sampling, sampling + n);
    else hs.smats = hs.mats;
    build_lights(hs);
}

void build_host_scene(const tpt_scene_desc& d, HostScene& hs, const MeshBvhBuilder& bvh) {
    if (d.n_materials < 0 || d.n_spheres < 0 || d.n_meshes < 0 || d.n_instances < 0)
        throw std::runtime_error("negative element count");
    if ((d.n_materials && !d.materials) || (d.n_spheres && !d.spheres) || (d.n_meshes && !d.meshes) ||
        (d.n_instances && !d.instances))
        throw std::runtime_error("null array with non-zero count");
    make_camera(d.camera, hs.cam);
    hs.mats.assign(d.materials, d.materials + d.n_materials);
    hs.smats = hs.mats;
    for (const tpt_material& m : hs.mats)
        if (m.kind < TPT_MAT_LAMBERT || m.kind > TPT_MAT_DIFFUSE_LIGHT) throw std::runtime_error("unknown material kind");
    hs.spheres.assign(d.spheres, d.spheres + d.n_spheres);
    for (const tpt_sphere& s : hs.spheres)
        if (s.mat_id < 0 || s.mat_id >= d.n_materials) throw std::runtime_error("sphere mat_id out of range");
    hs.meshes.resize((size_t)d.n_meshes);
    for (int64_t i = 0; i < d.n_meshes; ++i) {
        const tpt_mesh_desc& md = d.meshes[i];
        if (md.n_tris < 0 || md.n_vertices < 0 || (md.n_tris && (!md.indices || !md.mat_ids || !md.positions)))
            throw std::runtime_error("bad mesh description");
        if (md.n_tris >= (1ll << 27)) throw std::runtime_error("mesh has too many triangles");
        HostScene::Mesh& m = hs.meshes[(size_t)i];
        m.pos.assign(md.positions, md.positions + 3 * md.n_vertices);
        m.idx.assign(md.indices, md.indices + 3 * md.n_tris);
        m.mat.assign(md.mat_ids, md.mat_ids + md.n_tris);
        for (int32_t mid : m.mat)
            if (mid < 0 || mid >= d.n_materials) throw std::runtime_error("triangle mat_id out of range");
        m.bvh = bvh ? bvh(md) : build_mesh_bvh(md.positions, md.n_vertices, md.indices, md.n_tris);
    }
    hs.instances.resize((size_t)d.n_instances);
    for (int64_t i = 0; i < d.n_instances; ++i) {
        const tpt_instance_desc& id = d.instances[i];
        if (id.mesh_id < 0 || id.mesh_id >= d.n_meshes) throw std::runtime_error("instance mesh_id out of range");
        if (id.mat_override >= d.n_materials) throw std::runtime_error("instance mat_override out of range");
        make_instance(id, hs.instances[(size_t)i]);
    }

    build_lights(hs);

    // EnvMap::from_pixels (src/env.rs:61-89).
    hs.env_kind = d.env.kind;
    if (d.env.kind == TPT_ENV_MAP) {
        if (d.env.width <= 0 || d.env.height <= 0 || !d.env.pixels) throw std::runtime_error("bad env map");
        const size_t w = (size_t)d.env.width, h = (size_t)d.env.height;
        hs.env_w = d.env.width; hs.env_h = d.env.height;
        hs.env_data.assign(d.env.pixels, d.env.pixels + 3 * w * h);
        hs.env_row_cdf.assign(h + 1, 0.0);
        hs.env_col_cdf.assign(h * (w + 1), 0.0);
        double tot = 0.0;
        for (size_t y = 0; y < h; ++y) {
            double th0 = kPi * (double)y / (double)h;
            double th1 = kPi * (double)(y + 1) / (double)h;
            double rw = dmax(std::cos(th0) - std::cos(th1), 0.0);
            double row = 0.0;
            for (size_t x = 0; x < w; ++x) {
                row += dmax(luma(&hs.env_data[3 * (y * w + x)]), 0.0) * rw;
                hs.env_col_cdf[y * (w + 1) + x + 1] = row;
            }
            tot += row;
            hs.env_row_cdf[y + 1] = tot;
        }
        hs.env_total = tot;
    } else if (d.env.kind != TPT_ENV_NONE) {
        throw std::runtime_error("unknown env kind");
    }
}

// ------------------------------------------------------------------------
void flatten_plain_materials(const HostScene& hs, std::vector<MaterialF64>& mats, std::vector<LightF64>& lights) {
    mats.clear();
    lights.clear();
    for (const tpt_material& m : hs.mats) {
        MaterialF64 o{};
        o.kind = m.kind; o.c[0] = m.rgb[0]; o.c[1] = m.rgb[1]; o.c[2] = m.rgb[2]; o.p = m.param;
        mats.push_back(o);
    }
    for (const HostLight& l : hs.lights) {
        LightF64 o{};
        o.is_sphere = l.is_sphere;
        o.sphere = (int32_t)l.sphere;
        o.inst = (int32_t)l.inst;
        if (!l.is_sphere) {
            const HostScene::Mesh& m = hs.meshes[(size_t)l.mesh];
            for (int k = 0; k < 3; ++k) {
                const double* p = &m.pos[3 * (size_t)m.idx[3 * (size_t)l.tri + (size_t)k]];
                o.v[3 * k] = p[0]; o.v[3 * k + 1] = p[1]; o.v[3 * k + 2] = p[2];
            }
        }
        o.emit[0] = l.emit[0]; o.emit[1] = l.emit[1]; o.emit[2] = l.emit[2];
        o.weight = l.weight;
        lights.push_back(o);
    }
}

void flatten_plain(const HostScene& hs, PlainImage& img) {
    for (const HostScene::Mesh& m : hs.meshes) {
        MeshF64 me{(int32_t)img.nodes.size(), (int32_t)(m.bvh.left_right.size() / 2), (int32_t)img.tris.size(),
                   (int32_t)m.mat.size()};
        const size_t nn = m.bvh.left_right.size() / 2;
        for (size_t i = 0; i < nn; ++i) {
            NodeF64 n{};
            for (int k = 0; k < 3; ++k) { n.bmin[k] = m.bvh.bbox[6 * i + (size_t)k]; n.bmax[k] = m.bvh.bbox[6 * i + 3 + (size_t)k]; }
            n.left = m.bvh.left_right[2 * i]; n.right = m.bvh.left_right[2 * i + 1];
            n.start = m.bvh.start_count[2 * i]; n.count = m.bvh.start_count[2 * i + 1];
            img.nodes.push_back(n);
        }
        for (int64_t t : m.bvh.indices) {
            TriF64 tr{};
            for (int k = 0; k < 3; ++k) {
                const double* p = &m.pos[3 * (size_t)m.idx[3 * (size_t)t + (size_t)k]];
                double* dst = k == 0 ? tr.v0 : (k == 1 ? tr.v1 : tr.v2);
                dst[0] = p[0]; dst[1] = p[1]; dst[2] = p[2];
            }
            tr.mat = m.mat[(size_t)t];
            tr.orig = (int32_t)t;
            img.tris.push_back(tr);
        }
        img.meshes.push_back(me);
    }
    img.instances = hs.instances;
    for (const tpt_sphere& s : hs.spheres) {
        SphereF64 o{};
        o.c[0] = s.center[0]; o.c[1] = s.center[1]; o.c[2] = s.center[2];
        o.r = s.radius; o.mat = (int32_t)s.mat_id;
        img.spheres.push_back(o);
    }
    flatten_plain_materials(hs, img.mats, img.lights);
    img.light_cdf = hs.light_cdf;
    img.env_data = hs.env_data;
    img.env_row_cdf = hs.env_row_cdf;
    img.env_col_cdf = hs.env_col_cdf;
}

// ------------------------------------------------------------------------
namespace {

float f_down(double d) {  // largest float <= d
    float f = (float)d;
    if ((double)f > d) f = std::nextafter(f, -std::numeric_limits<float>::infinity());
    return f;
}
float f_up(double d) {  // smallest float >= d
    float f = (float)d;
    if ((double)f < d) f = std::nextafter(f, std::numeric_limits<float>::infinity());
    return f;
}
int32_t fbits_i(int32_t i) { return i; }
float as_float(int32_t i) { float f; std::memcpy(&f, &i, 4); return f; }

// Converts one BVH in the reference layout (preorder, leaves inline) into
// child-pair BVH2 nodes: interior nodes only, each holding both children's
// boxes.  leaf_ref(start, count) encodes a leaf's primitive range.  Every
// child of an interior node is a node or a leaf (the traversal tests no
// child for TPT_REF_NONE): a leaf without primitives becomes the leaf code
// of first 2, count 0, which tests nothing and differs from the traversal's
// exit markers (first 0 and 1, count 0); a missing child is an error.
template <class LeafRef>
int32_t emit_bvh2(const std::vector<double>& bbox, const std::vector<int32_t>& lr, const std::vector<uint32_t>& sc,
                  std::vector<BvhNode2>& nodes, LeafRef&& leaf_ref) {
    const size_t nn = lr.size() / 2;
    if (nn == 0) return TPT_REF_NONE;
    auto is_leaf = [&](size_t i) { return lr[2 * i] == -1 && lr[2 * i + 1] == -1; };
    std::vector<int32_t> gpu_index(nn, -1);
    const int32_t base = (int32_t)nodes.size();
    int32_t next = base;
    for (size_t i = 0; i < nn; ++i)
        if (!is_leaf(i)) gpu_index[i] = next++;
    auto ref_of = [&](int32_t child) -> int32_t {
        if (child < 0) throw std::runtime_error("BVH interior node without two children");
        size_t c = (size_t)child;
        if (is_leaf(c)) return sc[2 * c + 1] == 0 ? make_leaf_ref(2u, 0u) : leaf_ref(sc[2 * c], sc[2 * c + 1]);
        return gpu_index[c];
    };
    nodes.resize((size_t)next);
    for (size_t i = 0; i < nn; ++i) {
        if (is_leaf(i)) continue;
        BvhNode2& g = nodes[(size_t)gpu_index[i]];
        const double* a = &bbox[6 * (size_t)lr[2 * i]];
        const double* b = &bbox[6 * (size_t)lr[2 * i + 1]];
        g.lx = make_float4(f_down(a[0]), f_up(a[3]), f_down(a[1]), f_up(a[4]));
        g.rx = make_float4(f_down(b[0]), f_up(b[3]), f_down(b[1]), f_up(b[4]));
        g.zz = make_float4(f_down(a[2]), f_up(a[5]), f_down(b[2]), f_up(b[5]));
        g.refs = make_int4(ref_of(lr[2 * i]), ref_of(lr[2 * i + 1]), 0, 0);
    }
    if (is_leaf(0)) return sc[1] == 0 ? TPT_REF_NONE : leaf_ref(sc[0], sc[1]);
    return base;
}

// Top-level BVH over the world's spheres and mesh instances (the reference
// tests instances and then spheres linearly, src/world.rs:86-118; the
// closest hit is the same).  Each node splits where the surface-area
// heuristic is cheapest: over the three axes, the primitives sorted by box
// centre, every split position k weighed by area(left box) * k +
// area(right box) * (n - k).  Leaves hold one instance or one sphere; two
// spheres share a leaf only when splitting them costs more, a node visit
// weighed as one sphere test (as in the FP32 mesh trees).  Against leaves
// of two spheres always, this took the 1080p mesh + env frame from 3.247 to
// 3.383 G paths/s.  order lists the top primitives in leaf order (>= 0 sphere
// index, < 0 ~instance index).  (Against the median split this tree was
// built with before, it cuts the top-level node visits of the 1080p mesh +
// env frame's camera rays by 14%: 7.8 instead of 9.1 per ray.)
void build_top_bvh(const std::vector<Box>& boxes, const std::vector<int64_t>& ids, std::vector<double>& bbox,
                   std::vector<int32_t>& lr, std::vector<uint32_t>& sc, std::vector<int64_t>& order, int& depth) {
    const size_t n = boxes.size();
    std::vector<size_t> perm(n);
    for (size_t i = 0; i < n; ++i) perm[i] = i;
    depth = 0;
    order.clear();
    if (n == 0) return;
    auto centre = [&](size_t i, int k) { return 0.5 * (boxes[i].lo[k] + boxes[i].hi[k]); };
    struct Job { size_t s, e; int64_t parent; int side; int depth; };
    std::vector<Job> jobs{{0, n, -1, 0, 1}};
    while (!jobs.empty()) {
        Job j = jobs.back();
        jobs.pop_back();
        Box b = Box::none();
        bool has_instance = false;
        for (size_t k = j.s; k < j.e; ++k) {
            size_t i = perm[k];
            b.merge(boxes[i]);
            has_instance |= ids[i] < 0;
        }
        int64_t node = (int64_t)(lr.size() / 2);
        for (int k = 0; k < 3; ++k) bbox.push_back(b.lo[k]);
        for (int k = 0; k < 3; ++k) bbox.push_back(b.hi[k]);
        lr.push_back(-1); lr.push_back(-1); sc.push_back(0); sc.push_back(0);
        if (j.parent >= 0) lr[2 * (size_t)j.parent + (size_t)j.side] = (int32_t)node;
        depth = std::max(depth, j.depth);
        size_t cnt = j.e - j.s;
        if (cnt == 1) {
            sc[2 * (size_t)node] = (uint32_t)j.s;
            sc[2 * (size_t)node + 1] = (uint32_t)cnt;
            continue;
        }
        // SAH sweep: prefix (left) and suffix (right) box areas per axis
        auto area = [](const Box& x) {
            const double dx = x.hi[0] - x.lo[0], dy = x.hi[1] - x.lo[1], dz = x.hi[2] - x.lo[2];
            return 2.0 * (dx * dy + dy * dz + dz * dx);
        };
        double best_cost = std::numeric_limits<double>::infinity();
        int best_axis = 0;
        size_t best_k = cnt / 2;
        std::vector<size_t> order_ax(cnt);
        std::vector<double> right(cnt + 1);
        for (int axis = 0; axis < 3; ++axis) {
            for (size_t k = 0; k < cnt; ++k) order_ax[k] = perm[j.s + k];
            std::stable_sort(order_ax.begin(), order_ax.end(),
                             [&](size_t a, size_t c) { return centre(a, axis) < centre(c, axis); });
            Box rb = Box::none();
            right[cnt] = 0.0;
            for (size_t k = cnt; k-- > 0;) {
                rb.merge(boxes[order_ax[k]]);
                right[k] = area(rb);
            }
            Box lb = Box::none();
            for (size_t k = 1; k < cnt; ++k) {
                lb.merge(boxes[order_ax[k - 1]]);
                const double cost = area(lb) * (double)k + right[k] * (double)(cnt - k);
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = axis;
                    best_k = k;
                }
            }
        }
        if (cnt == 2 && !has_instance && 2.0 <= 1.0 + best_cost / area(b)) {
            sc[2 * (size_t)node] = (uint32_t)j.s;
            sc[2 * (size_t)node + 1] = (uint32_t)cnt;
            continue;
        }
        std::stable_sort(perm.begin() + (ptrdiff_t)j.s, perm.begin() + (ptrdiff_t)j.e,
                         [&](size_t a, size_t c) { return centre(a, best_axis) < centre(c, best_axis); });
        const size_t mid = j.s + best_k;
        jobs.push_back(Job{mid, j.e, node, 1, j.depth + 1});
        jobs.push_back(Job{j.s, mid, node, 0, j.depth + 1});
    }
    order.resize(n);
    for (size_t k = 0; k < n; ++k) order[k] = ids[perm[k]];
}

}  // namespace

void flatten_fp32_materials(const HostScene& hs, std::vector<MaterialF32>& mats, std::vector<LightF32>& lights,
                            std::vector<float>& light_cdf) {
    mats.clear();
    lights.clear();
    light_cdf.clear();
    for (size_t i = 0; i < hs.mats.size(); ++i) {
        const tpt_material& m = hs.mats[i];
        MaterialF32 o{};
        o.c = make_float4((float)m.rgb[0], (float)m.rgb[1], (float)m.rgb[2], (float)m.param);
        o.kind = m.kind;
        o.s_param = (float)hs.smats[i].param;
        mats.push_back(o);
    }
    // Light table: world-space geometry, pdf_select = weight / total.
    for (size_t i = 0; i < hs.lights.size(); ++i) {
        const HostLight& l = hs.lights[i];
        LightF32 o{};
        o.is_sphere = l.is_sphere;
        o.mat = (int32_t)l.mat;
        if (l.is_sphere) {
            const tpt_sphere& s = hs.spheres[(size_t)l.sphere];
            o.p0 = make_float4((float)s.center[0], (float)s.center[1], (float)s.center[2], (float)s.radius);
        } else {
            HVec v[3];
            tri_world(hs, hs.instances[(size_t)l.inst], l.tri, 0.0, v);
            o.p0 = make_float4((float)v[0].x, (float)v[0].y, (float)v[0].z, 0.0f);
            o.p1 = make_float4((float)v[1].x, (float)v[1].y, (float)v[1].z, 0.0f);
            o.p2 = make_float4((float)v[2].x, (float)v[2].y, (float)v[2].z, 0.0f);
        }
        o.emit = make_float4((float)l.emit[0], (float)l.emit[1], (float)l.emit[2], (float)(l.weight / hs.light_total));
        lights.push_back(o);
        light_cdf.push_back((float)(hs.light_cdf[i] / hs.light_total));
    }
}

// The FP32 forms walk their own mesh trees (build_fp32_mesh_bvh);
// TPT_FP32_TREE=reference makes them walk the reference's tree instead.
void flatten_fp32(const HostScene& hs, Fp32Image& img) {
    int max_depth = 0;
    const char* tree_setting = std::getenv("TPT_FP32_TREE");
    const bool reference_tree = tree_setting && std::strcmp(tree_setting, "reference") == 0;
    for (const HostScene::Mesh& m : hs.meshes) {
        HostBvh own;
        if (!reference_tree)
            own = build_fp32_mesh_bvh(m.pos.data(), (int64_t)(m.pos.size() / 3), m.idx.data(), (int64_t)m.mat.size());
        const HostBvh& tree = reference_tree ? m.bvh : own;
        MeshF32 me{};
        me.tri_offset = (int32_t)img.tris.size();
        me.n_tris = (int32_t)m.mat.size();
        const int32_t toff = me.tri_offset;
        me.root_ref = emit_bvh2(tree.bbox, tree.left_right, tree.start_count, img.nodes,
                                [&](uint32_t start, uint32_t count) { return make_leaf_ref((uint32_t)toff + start, count); });
        for (int64_t t : tree.indices) {
            const double* p0 = &m.pos[3 * (size_t)m.idx[3 * (size_t)t]];
            const double* p1 = &m.pos[3 * (size_t)m.idx[3 * (size_t)t + 1]];
            const double* p2 = &m.pos[3 * (size_t)m.idx[3 * (size_t)t + 2]];
            TriF32 tr;
            tr.v0 = make_float4((float)p0[0], (float)p0[1], (float)p0[2], as_float(fbits_i(m.mat[(size_t)t])));
            tr.e1 = make_float4((float)(p1[0] - p0[0]), (float)(p1[1] - p0[1]), (float)(p1[2] - p0[2]),
                                as_float((int32_t)t));
            tr.e2 = make_float4((float)(p2[0] - p0[0]), (float)(p2[1] - p0[1]), (float)(p2[2] - p0[2]), 0.0f);
            img.tris.push_back(tr);
        }
        max_depth = std::max(max_depth, tree.max_depth);
        img.meshes.push_back(me);
    }
    for (const InstanceF64& x : hs.instances) {
        InstanceF32 o{};
        const double* ai = x.a_inv;
        double tt[3] = {ai[0] * x.t[0] + ai[1] * x.t[1] + ai[2] * x.t[2], ai[3] * x.t[0] + ai[4] * x.t[1] + ai[5] * x.t[2],
                        ai[6] * x.t[0] + ai[7] * x.t[1] + ai[8] * x.t[2]};
        for (int r = 0; r < 3; ++r) {
            o.w2o[r] = make_float4((float)ai[3 * r], (float)ai[3 * r + 1], (float)ai[3 * r + 2], (float)(-tt[r]));
            o.nrm[r] = make_float4((float)x.nmat[3 * r], (float)x.nmat[3 * r + 1], (float)x.nmat[3 * r + 2], 0.0f);
        }
        // World box: the 8 corners of the mesh root box under p' = A p + t.
        const HostScene::Mesh& m = hs.meshes[(size_t)x.mesh_id];
        Box wb = Box::none();
        if (!m.bvh.bbox.empty()) {
            const double* rb = &m.bvh.bbox[0];
            for (int c = 0; c < 8; ++c) {
                HVec p{(c & 1) ? rb[3] : rb[0], (c & 2) ? rb[4] : rb[1], (c & 4) ? rb[5] : rb[2]};
                HVec q = apply_point(x, p);
                double qq[3] = {q.x, q.y, q.z};
                wb.grow(qq);
            }
        } else {
            for (int k = 0; k < 3; ++k) { wb.lo[k] = 1.0; wb.hi[k] = -1.0; }
        }
        // Pad by a relative margin: the FP32 ray transform rounds.
        double pad = 1e-5 * std::max({std::fabs(wb.lo[0]), std::fabs(wb.lo[1]), std::fabs(wb.lo[2]), std::fabs(wb.hi[0]),
                                      std::fabs(wb.hi[1]), std::fabs(wb.hi[2]), 1.0});
        bool identity = true;
        for (int r = 0; r < 3; ++r) {
            const float row[4] = {o.w2o[r].x, o.w2o[r].y, o.w2o[r].z, o.w2o[r].w};
            for (int c = 0; c < 4; ++c) identity = identity && row[c] == (c == r ? 1.0f : 0.0f);
        }
        o.wbox_min = make_float4(f_down(wb.lo[0] - pad), f_down(wb.lo[1] - pad), f_down(wb.lo[2] - pad),
                                 as_float((int32_t)x.mesh_id | (identity ? kInstIdentity : 0)));
        o.wbox_max = make_float4(f_up(wb.hi[0] + pad), f_up(wb.hi[1] + pad), f_up(wb.hi[2] + pad),
                                 as_float(x.mat_override));
        img.instances.push_back(o);
    }
    // Top-level BVH over spheres and instances, appended after the mesh
    // nodes.  Sphere leaves index the sphere array, which is stored in leaf
    // order; instance leaves carry the instance index with count 7.
    std::vector<Box> top_boxes;
    std::vector<int64_t> top_ids;
    for (size_t si = 0; si < hs.spheres.size(); ++si) {
        const tpt_sphere& s = hs.spheres[si];
        double r = std::fabs(s.radius);
        top_boxes.push_back(Box{{s.center[0] - r, s.center[1] - r, s.center[2] - r},
                                {s.center[0] + r, s.center[1] + r, s.center[2] + r}});
        top_ids.push_back((int64_t)si);
    }
    for (size_t ii = 0; ii < img.instances.size(); ++ii) {
        const InstanceF32& o = img.instances[ii];
        if (o.wbox_min.x > o.wbox_max.x) continue;  // empty mesh
        top_boxes.push_back(Box{{o.wbox_min.x, o.wbox_min.y, o.wbox_min.z}, {o.wbox_max.x, o.wbox_max.y, o.wbox_max.z}});
        top_ids.push_back(~(int64_t)ii);
    }
    std::vector<double> tb;
    std::vector<int32_t> tlr;
    std::vector<uint32_t> tsc;
    std::vector<int64_t> torder;
    int sdepth = 0;
    build_top_bvh(top_boxes, top_ids, tb, tlr, tsc, torder, sdepth);
    img.top_node_begin = (int32_t)img.nodes.size();
    std::vector<int32_t> sphere_slot(torder.size(), -1);
    for (size_t k = 0; k < torder.size(); ++k) {
        if (torder[k] < 0) continue;
        const tpt_sphere& s = hs.spheres[(size_t)torder[k]];
        SphereF32 o{};
        o.cr = make_float4((float)s.center[0], (float)s.center[1], (float)s.center[2], (float)s.radius);
        o.mat = (int32_t)s.mat_id;
        o.orig = (int32_t)torder[k];
        sphere_slot[k] = (int32_t)img.spheres.size();
        img.spheres.push_back(o);
    }
    img.top_root = emit_bvh2(tb, tlr, tsc, img.nodes, [&](uint32_t start, uint32_t count) {
        if (torder[start] < 0) return make_leaf_ref((uint32_t)~torder[start], 7u);  // one instance
        return make_leaf_ref((uint32_t)sphere_slot[start], count);
    });
    // stack: top-level path + the exit marker + the deepest mesh path
    img.max_stack = sdepth + 1 + max_depth + 1;
    flatten_fp32_materials(hs, img.mats, img.lights, img.light_cdf);
    if (hs.env_kind == TPT_ENV_MAP) {
        const size_t w = (size_t)hs.env_w, h = (size_t)hs.env_h;
        img.env_texels.resize(w * h);
        img.env_row_cdf.resize(h + 1);
        img.env_col_cdf.resize(h * (w + 1));
        for (size_t y = 0; y < h; ++y) {
            double th0 = kPi * (double)y / (double)h, th1 = kPi * (double)(y + 1) / (double)h;
            double rw = dmax(std::cos(th0) - std::cos(th1), 0.0);
            double row_sum = hs.env_col_cdf[y * (w + 1) + w];
            for (size_t x = 0; x < w; ++x) {
                const double* c = &hs.env_data[3 * (y * w + x)];
                double pdf_uv = 0.0;
                if (hs.env_total > 0.0) pdf_uv = (dmax(luma(c), 0.0) * rw / hs.env_total) * (double)w * (double)h;
                img.env_texels[y * w + x] = make_float4((float)c[0], (float)c[1], (float)c[2], (float)pdf_uv);
                img.env_col_cdf[y * (w + 1) + x] =
                    row_sum > 0.0 ? (float)(hs.env_col_cdf[y * (w + 1) + x] / row_sum) : 0.0f;
            }
            img.env_col_cdf[y * (w + 1) + w] = 1.0f;
            img.env_row_cdf[y] = hs.env_total > 0.0 ? (float)(hs.env_row_cdf[y] / hs.env_total) : 0.0f;
        }
        img.env_row_cdf[h] = 1.0f;
    }
}

namespace {
// Rebases a BVH2 child reference of a scene appended at the given offsets:
// interior node index, or a leaf's first primitive (triangle in a mesh
// tree, sphere slot in the top-level tree, instance for count 7).
int32_t rebase_ref(int32_t ref, bool top_tree, int32_t node_base, int32_t tri_base, int32_t sphere_base,
                   int32_t inst_base) {
    if (ref == TPT_REF_NONE || ref == ~0) return ref;
    if (ref >= 0) return ref + node_base;
    const uint32_t code = (uint32_t)(~ref);
    const uint32_t first = code >> 3, count = code & 7u;
    uint32_t nf = first;
    if (count == 7u) nf = first + (uint32_t)inst_base;
    else if (top_tree) nf = first + (uint32_t)sphere_base;
    else nf = first + (uint32_t)tri_base;
    if (nf >= (1u << 28)) throw std::runtime_error("batch too large for 28-bit leaf references");
    return ~(int32_t)((nf << 3) | count);
}
}  // namespace

void merge_scenes(const std::vector<const HostScene*>& scenes, BatchImage& out) {
    Fp32Image& F = out.fp;
    F = Fp32Image{};
    out.lights64.clear();
    out.inst64.clear();
    out.spheres64.clear();
    out.scenes.clear();
    int max_stack = 0;
    // The scenes' images (each building its FP32 mesh trees) are made in
    // parallel, then appended in scene order.
    std::vector<Fp32Image> images(scenes.size());
    {
        const size_t workers = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), scenes.size()));
        std::atomic<size_t> next{0};
        std::vector<std::future<void>> pool;
        for (size_t w = 0; w < workers; ++w)
            pool.push_back(std::async(std::launch::async, [&] {
                for (size_t i; (i = next++) < scenes.size();) flatten_fp32(*scenes[i], images[i]);
            }));
        for (std::future<void>& f : pool) f.get();
    }
    for (size_t si = 0; si < scenes.size(); ++si) {
        const HostScene& hs = *scenes[si];
        Fp32Image& img = images[si];
        PlainImage pl;
        flatten_plain_materials(hs, pl.mats, pl.lights);
        const int32_t node_base = (int32_t)F.nodes.size(), tri_base = (int32_t)F.tris.size();
        const int32_t sphere_base = (int32_t)F.spheres.size(), inst_base = (int32_t)F.instances.size();
        const int32_t mesh_base = (int32_t)F.meshes.size(), mat_base = (int32_t)F.mats.size();
        const int32_t light_base = (int32_t)F.lights.size();
        const int32_t sphere64_base = (int32_t)out.spheres64.size(), inst64_base = (int32_t)out.inst64.size();
        for (size_t k = 0; k < img.nodes.size(); ++k) {
            BvhNode2 n = img.nodes[k];
            const bool top = (int32_t)k >= img.top_node_begin;
            n.refs.x = rebase_ref(n.refs.x, top, node_base, tri_base, sphere_base, inst_base);
            n.refs.y = rebase_ref(n.refs.y, top, node_base, tri_base, sphere_base, inst_base);
            F.nodes.push_back(n);
        }
        for (TriF32 t : img.tris) {
            int32_t m;
            std::memcpy(&m, &t.v0.w, 4);
            t.v0.w = as_float(m + mat_base);
            F.tris.push_back(t);
        }
        for (MeshF32 m : img.meshes) {
            m.tri_offset += tri_base;
            m.root_ref = rebase_ref(m.root_ref, false, node_base, tri_base, sphere_base, inst_base);
            F.meshes.push_back(m);
        }
        for (InstanceF32 o : img.instances) {
            int32_t mesh, ov;
            std::memcpy(&mesh, &o.wbox_min.w, 4);
            std::memcpy(&ov, &o.wbox_max.w, 4);
            o.wbox_min.w = as_float(mesh + mesh_base);
            o.wbox_max.w = as_float(ov >= 0 ? ov + mat_base : ov);
            F.instances.push_back(o);
        }
        for (SphereF32 o : img.spheres) {
            o.mat += mat_base;
            o.orig += sphere64_base;
            F.spheres.push_back(o);
        }
        for (const MaterialF32& m : img.mats) F.mats.push_back(m);
        for (LightF32 l : img.lights) {
            l.mat += mat_base;
            F.lights.push_back(l);
        }
        for (float c : img.light_cdf) F.light_cdf.push_back(c);
        for (LightF64 l : pl.lights) {
            l.sphere += sphere64_base;
            l.inst += inst64_base;
            out.lights64.push_back(l);
        }
        for (InstanceF64 x : hs.instances) {
            x.mesh_id += mesh_base;
            if (x.mat_override >= 0) x.mat_override += mat_base;
            out.inst64.push_back(x);
        }
        for (const tpt_sphere& sp : hs.spheres) {
            SphereF64 o{};
            o.c[0] = sp.center[0]; o.c[1] = sp.center[1]; o.c[2] = sp.center[2];
            o.r = sp.radius;
            o.mat = (int32_t)sp.mat_id + mat_base;
            out.spheres64.push_back(o);
        }
        BatchScene b{};
        b.top_root = rebase_ref(img.top_root, true, node_base, tri_base, sphere_base, inst_base);
        const CameraF64& c = hs.cam;
        b.cam.o = make_float3((float)c.o[0], (float)c.o[1], (float)c.o[2]);
        b.cam.u = make_float3((float)c.u[0], (float)c.u[1], (float)c.u[2]);
        b.cam.v = make_float3((float)c.v[0], (float)c.v[1], (float)c.v[2]);
        b.cam.w = make_float3((float)c.w[0], (float)c.w[1], (float)c.w[2]);
        b.cam.half_h = (float)c.half_h;
        b.cam.half_w = (float)c.half_w;
        b.cam.lens_radius = (float)c.lens_radius;
        b.cam.focus_dist = (float)c.focus_dist;
        b.env_kind = hs.env_kind;
        b.env_w = hs.env_w;
        b.env_h = hs.env_h;
        b.env_has_cdf = hs.env_total > 0.0;
        b.env_tex_off = F.env_texels.size();
        b.env_row_off = F.env_row_cdf.size();
        b.env_col_off = F.env_col_cdf.size();
        F.env_texels.insert(F.env_texels.end(), img.env_texels.begin(), img.env_texels.end());
        F.env_row_cdf.insert(F.env_row_cdf.end(), img.env_row_cdf.begin(), img.env_row_cdf.end());
        F.env_col_cdf.insert(F.env_col_cdf.end(), img.env_col_cdf.begin(), img.env_col_cdf.end());
        b.light_begin = light_base;
        b.n_lights = (int32_t)img.lights.size();
        b.mat_begin = mat_base;
        b.n_mats = (int32_t)img.mats.size();
        out.scenes.push_back(b);
        max_stack = std::max(max_stack, img.max_stack);
    }
    F.max_stack = max_stack;
    F.top_root = TPT_REF_NONE;
}

}  // namespace tpt
