// ORACLE -- test infrastructure only (see ref_model.hpp).
// C ABI over the f64 restatement: builds the reference Scene from the same
// flattened tpt_scene_desc the product takes, and wraps the reference
// functions that the reference's own unit tests exercise.
#include "oracle.h"

#include <memory>
#include <stdexcept>
#include <string>

#include "ref_model.hpp"

using namespace ref;

namespace {
thread_local std::string g_err;

Vec3 v3(const double* p) { return Vec3(p[0], p[1], p[2]); }
void put3(double* o, Vec3 v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }

Material to_material(const tpt_material& m) {
    Material r;
    switch (m.kind) {
        case TPT_MAT_LAMBERT: r.kind = MatKind::Lambert; break;
        case TPT_MAT_METAL: r.kind = MatKind::Metal; break;
        case TPT_MAT_DIELECTRIC: r.kind = MatKind::Dielectric; break;
        case TPT_MAT_GGX: r.kind = MatKind::Ggx; break;
        case TPT_MAT_SUBSURFACE: r.kind = MatKind::Subsurface; break;
        case TPT_MAT_DIFFUSE_LIGHT: r.kind = MatKind::DiffuseLight; break;
        default: throw std::runtime_error("unknown material kind");
    }
    r.c = v3(m.rgb);
    r.p = m.param;
    return r;
}

Camera to_camera(const tpt_camera_desc& c) {
    if (c.kind == TPT_CAMERA_LOOK_AT_DOF)
        return Camera::look_at_dof(v3(c.eye), v3(c.target), v3(c.up), c.fov_y_deg, c.aspect, c.focus_dist,
                                   c.aperture);
    return Camera::look_at(v3(c.eye), v3(c.target), v3(c.up), c.fov_y_deg, c.aspect);
}

std::optional<EnvMap> to_env(const tpt_env_desc& e) {
    if (e.kind != TPT_ENV_MAP) return std::nullopt;
    if (e.width <= 0 || e.height <= 0 || !e.pixels) throw std::runtime_error("bad env map");
    std::vector<Color> data((size_t)e.width * (size_t)e.height);
    for (size_t i = 0; i < data.size(); ++i) data[i] = v3(e.pixels + 3 * i);
    return EnvMap::from_pixels((size_t)e.width, (size_t)e.height, std::move(data));
}

std::vector<Triangle> to_tris(const tpt_mesh_desc& m) {
    std::vector<Triangle> tris((size_t)m.n_tris);
    for (int64_t i = 0; i < m.n_tris; ++i) {
        int32_t a = m.indices[3 * i], b = m.indices[3 * i + 1], c = m.indices[3 * i + 2];
        if (a < 0 || b < 0 || c < 0 || a >= m.n_vertices || b >= m.n_vertices || c >= m.n_vertices)
            throw std::runtime_error("triangle index out of range");
        tris[(size_t)i] = Triangle::new_static(v3(m.positions + 3 * a), v3(m.positions + 3 * b),
                                               v3(m.positions + 3 * c), (size_t)m.mat_ids[i]);
    }
    return tris;
}

std::unique_ptr<Scene> to_scene(const tpt_scene_desc& d) {
    auto s = std::make_unique<Scene>();
    s->cam = to_camera(d.camera);
    for (int64_t i = 0; i < d.n_materials; ++i) s->mats.push_back(to_material(d.materials[i]));
    for (int64_t i = 0; i < d.n_spheres; ++i) {
        const tpt_sphere& sp = d.spheres[i];
        if (sp.mat_id < 0 || sp.mat_id >= d.n_materials) throw std::runtime_error("sphere mat_id out of range");
        s->world.spheres.push_back(Sphere{v3(sp.center), sp.radius, (size_t)sp.mat_id});
    }
    for (int64_t i = 0; i < d.n_meshes; ++i) {
        Mesh m;
        m.tris = to_tris(d.meshes[i]);
        for (const Triangle& t : m.tris)
            if (t.mat_id >= (size_t)d.n_materials) throw std::runtime_error("triangle mat_id out of range");
        m.bvh = Bvh::build(m.tris);  // Mesh::new (world.rs:29-32)
        s->world.meshes.push_back(std::move(m));
    }
    for (int64_t i = 0; i < d.n_instances; ++i) {
        const tpt_instance_desc& in = d.instances[i];
        Mat3 a{{{in.linear[0], in.linear[1], in.linear[2]},
                {in.linear[3], in.linear[4], in.linear[5]},
                {in.linear[6], in.linear[7], in.linear[8]}}};
        Instance inst;
        inst.mesh_id = (size_t)in.mesh_id;
        inst.xform = Transform::from_affine(a, v3(in.translation));
        if (in.mat_override >= 0) {
            if (in.mat_override >= d.n_materials) throw std::runtime_error("mat_override out of range");
            inst.mat_override = (size_t)in.mat_override;
        }
        s->world.instances.push_back(inst);
    }
    s->env = to_env(d.env);
    s->world.build_lights(s->mats);
    return s;
}

RenderConfig to_cfg(const tpt_render_config& c) {
    if (c.width <= 0 || c.height <= 0 || c.spp <= 0 || c.tile <= 0) throw std::runtime_error("bad render config");
    if (c.row_step > 0) throw std::runtime_error("row shards are not rendered by the oracle (use a rect)");
    RenderConfig r;
    r.width = (size_t)c.width; r.height = (size_t)c.height; r.spp = (size_t)c.spp;
    r.max_bounces = (size_t)std::max(c.max_bounces, 0); r.rr_start = (size_t)std::max(c.rr_start, 0);
    r.tile = (size_t)c.tile;
    r.adaptive_enabled = c.adaptive_enabled != 0;
    r.adaptive_min_spp = (size_t)std::max(c.adaptive_min_spp, 0);
    r.adaptive_threshold = c.adaptive_threshold;
    r.morton_enabled = c.morton_enabled != 0;
    r.seed = c.seed;
    return r;
}

void copy_counts(const TraversalCounts& t, oracle_counts* o) {
    if (!o) return;
    o->world_hits = t.world_hits; o->node_pops = t.node_pops; o->node_box_tests = t.node_box_tests;
    o->tri_tests = t.tri_tests; o->sphere_tests = t.sphere_tests;
}

template <class F>
int guarded(F&& f) {
    try {
        g_err.clear();
        return f();
    } catch (const std::exception& e) {
        g_err = e.what();
        return TPT_ERR_INVALID;
    }
}
}  // namespace

extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

int oracle_scene_create(const tpt_scene_desc* desc, void** out) {
    return guarded([&] {
        if (!desc || !out) throw std::runtime_error("null argument");
        *out = to_scene(*desc).release();
        return TPT_OK;
    });
}

void oracle_scene_destroy(void* scene) { delete static_cast<Scene*>(scene); }

int oracle_scene_set_materials(void* scene, const tpt_material* mats, const tpt_material* sampling, int64_t n) {
    return guarded([&] {
        if (!scene || !mats) throw std::runtime_error("null argument");
        Scene& s = *static_cast<Scene*>(scene);
        if (n != (int64_t)s.mats.size()) throw std::runtime_error("material count differs");
        std::vector<Material> m, sm;
        for (int64_t i = 0; i < n; ++i) {
            m.push_back(to_material(mats[i]));
            if (m.back().kind != s.mats[(size_t)i].kind) throw std::runtime_error("material changes kind");
        }
        if (sampling) {
            for (int64_t i = 0; i < n; ++i) {
                sm.push_back(to_material(sampling[i]));
                if (sm.back().kind != m[(size_t)i].kind) throw std::runtime_error("material changes kind");
                m[(size_t)i].sp = sm.back().p;
            }
        }
        s.mats = m;
        s.world.build_lights(s.mats, sampling ? &sm : nullptr);
        return TPT_OK;
    });
}

int oracle_scene_render(void* scene, const tpt_render_config* cfg, const int32_t* rect, double* acc,
                        double* acc_w, double* acc_sq, int threads, oracle_counts* counts) {
    return oracle_scene_render_tasks(scene, cfg, rect, 0, acc, acc_w, acc_sq, threads, counts);
}

int oracle_scene_render_tasks(void* scene, const tpt_render_config* cfg, const int32_t* rect, int sample_chunk,
                              double* acc, double* acc_w, double* acc_sq, int threads, oracle_counts* counts) {
    return oracle_scene_render_streams(scene, cfg, rect, sample_chunk, 0, acc, acc_w, acc_sq, threads, counts);
}

int oracle_scene_render_streams(void* scene, const tpt_render_config* cfg, const int32_t* rect, int sample_chunk,
                                int reseed, double* acc, double* acc_w, double* acc_sq, int threads,
                                oracle_counts* counts) {
    return guarded([&] {
        if (!scene || !cfg || !acc || !acc_w) throw std::runtime_error("null argument");
        if (sample_chunk < 0 || reseed < 0) throw std::runtime_error("negative sample_chunk or reseed");
        if (sample_chunk > 0 && reseed > 0) throw std::runtime_error("sample_chunk and reseed are exclusive");
        RenderConfig rc = to_cfg(*cfg);
        TraversalCounts tc;
        Rect r{0, 0, rc.width, rc.height};
        if (rect) {
            if (rect[0] < 0 || rect[1] < 0 || rect[2] > cfg->width || rect[3] > cfg->height || rect[0] >= rect[2] ||
                rect[1] >= rect[3])
                throw std::runtime_error("bad rect");
            r = Rect{(size_t)rect[0], (size_t)rect[1], (size_t)rect[2], (size_t)rect[3]};
        }
        render(*static_cast<Scene*>(scene), rc, acc, acc_w, acc_sq, threads, counts ? &tc : nullptr, &r,
               (size_t)sample_chunk, (size_t)reseed);
        copy_counts(tc, counts);
        return TPT_OK;
    });
}

// output.rs:96-102 resolve_pixels: acc[i] / max(acc_w[i], 1), per channel.
void oracle_resolve_pixels(int64_t n, const double* acc, const double* acc_w, double* out) {
    for (int64_t i = 0; i < n; ++i) {
        const double w = rmax(acc_w[i], 1.0);
        out[3 * i] = acc[3 * i] / w;
        out[3 * i + 1] = acc[3 * i + 1] / w;
        out[3 * i + 2] = acc[3 * i + 2] / w;
    }
}

int oracle_render(const tpt_scene_desc* desc, const tpt_render_config* cfg, double* acc, double* acc_w,
                  double* acc_sq, int threads, oracle_counts* counts) {
    void* s = nullptr;
    int rc = oracle_scene_create(desc, &s);
    if (rc != TPT_OK) return rc;
    rc = oracle_scene_render(s, cfg, nullptr, acc, acc_w, acc_sq, threads, counts);
    oracle_scene_destroy(s);
    return rc;
}

void oracle_rng_u32(uint64_t seed, int n, uint32_t* out) {
    Rng r(seed);
    for (int i = 0; i < n; ++i) out[i] = r.next_u32();
}
void oracle_rng_f64(uint64_t seed, int n, double* out) {
    Rng r(seed);
    for (int i = 0; i < n; ++i) out[i] = r.next_f64();
}
uint64_t oracle_seed_for(uint32_t px, uint32_t py, uint32_t s) { return seed_for(px, py, s); }
uint64_t oracle_interleave_bits(uint64_t v) { return interleave_bits(v); }

int oracle_tile_order(int w, int h, int tile, int morton, int32_t* out) {
    RenderConfig c;
    c.width = (size_t)w; c.height = (size_t)h; c.tile = (size_t)tile; c.morton_enabled = morton != 0; c.spp = 1;
    std::vector<Task> t = make_tasks(c);
    if (out)
        for (size_t i = 0; i < t.size(); ++i) {
            out[4 * i] = (int32_t)t[i].x0; out[4 * i + 1] = (int32_t)t[i].y0;
            out[4 * i + 2] = (int32_t)t[i].x1; out[4 * i + 3] = (int32_t)t[i].y1;
        }
    return (int)t.size();
}

int64_t oracle_bvh_build(const tpt_mesh_desc* mesh, double* bbox, int32_t* lr, uint32_t* sc, int64_t* indices) {
    try {
        std::vector<Triangle> tris = to_tris(*mesh);
        Bvh b = Bvh::build(tris);
        for (size_t i = 0; i < b.nodes.size(); ++i) {
            const BvhNode& n = b.nodes[i];
            if (bbox) {
                bbox[6 * i + 0] = n.bbox.min.x; bbox[6 * i + 1] = n.bbox.min.y; bbox[6 * i + 2] = n.bbox.min.z;
                bbox[6 * i + 3] = n.bbox.max.x; bbox[6 * i + 4] = n.bbox.max.y; bbox[6 * i + 5] = n.bbox.max.z;
            }
            if (lr) { lr[2 * i] = n.left; lr[2 * i + 1] = n.right; }
            if (sc) { sc[2 * i] = n.start; sc[2 * i + 1] = n.count; }
        }
        if (indices)
            for (size_t i = 0; i < b.indices.size(); ++i) indices[i] = (int64_t)b.indices[i];
        return (int64_t)b.nodes.size();
    } catch (const std::exception& e) {
        g_err = e.what();
        return TPT_ERR_INVALID;
    }
}

int oracle_material_sample(const tpt_material* m, const double ray_o[3], const double ray_d[3], double time,
                           double hit_t, const double hit_p[3], const double hit_n[3], uint64_t* rng_state,
                           double out[11]) {
    Material mat = to_material(*m);
    Ray r{v3(ray_o), v3(ray_d), time};
    Hit h{hit_t, v3(hit_p), v3(hit_n), 0};
    Rng rng(1);
    rng.state = *rng_state;
    auto s = material_sample(mat, r, h, rng);
    *rng_state = rng.state;
    if (!s) return 0;
    put3(out, s->scattered.o);
    put3(out + 3, s->scattered.d);
    put3(out + 6, s->weight);
    out[9] = s->pdf;
    out[10] = s->is_delta ? 1.0 : 0.0;
    return 1;
}

void oracle_material_eval(const tpt_material* m, const double wo[3], const double wi[3], const double n[3],
                          double out[4]) {
    auto [f, pdf] = material_eval(to_material(*m), v3(wo), v3(wi), v3(n));
    put3(out, f);
    out[3] = pdf;
}

void oracle_material_eval_n(const tpt_material* m, const double wo[3], const double* wi, const double n[3],
                            int64_t count, double* out) {
    const Material mat = to_material(*m);
    for (int64_t i = 0; i < count; ++i) {
        auto [f, pdf] = material_eval(mat, v3(wo), v3(wi + 3 * i), v3(n));
        put3(out + 4 * i, f);
        out[4 * i + 3] = pdf;
    }
}

void oracle_material_classify(const tpt_material* m, int32_t out[2]) {
    const Material mat = to_material(*m);
    out[0] = material_is_delta(mat) ? 1 : 0;
    out[1] = material_emitted(mat).has_value() ? 1 : 0;
}

void oracle_transform(int n_ops, const int32_t* kinds, const double* params, int mode, const double p[3],
                      double out[3], double a_t_out[12]) {
    Transform acc = Transform::identity();
    for (int i = 0; i < n_ops; ++i) {
        const double* q = params + 5 * i;
        Transform op;
        switch (kinds[i]) {
            case 0: op = Transform::translate(Vec3(q[0], q[1], q[2])); break;
            case 1: op = Transform::scale(Vec3(q[0], q[1], q[2])); break;
            case 2: op = Transform::rotate(Vec3(q[0], q[1], q[2]), q[3]); break;
            default: op = Transform::legacy(Vec3(q[0], q[1], q[2]), q[3], q[4]); break;
        }
        acc = acc.compose(op);
    }
    Vec3 r = mode == 0 ? acc.apply_point(v3(p)) : (mode == 1 ? acc.apply_point_inv(v3(p)) : acc.apply_normal(v3(p)));
    put3(out, r);
    if (a_t_out) {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) a_t_out[3 * i + j] = acc.a.m[i][j];
        put3(a_t_out + 9, acc.t);
    }
}

int oracle_sample_light(const tpt_scene_desc* desc, uint64_t* rng_state, double time, const double p[3],
                        double out[10], double* light_total_out, int64_t* n_lights_out) {
    return guarded([&] {
        auto s = to_scene(*desc);
        if (light_total_out) *light_total_out = s->world.light_total;
        if (n_lights_out) *n_lights_out = (int64_t)s->world.lights.size();
        Rng rng(1);
        rng.state = *rng_state;
        auto ls = s->world.sample_light(rng, time, v3(p));
        *rng_state = rng.state;
        if (!ls) return 0;
        put3(out, ls->position); put3(out + 3, ls->normal); put3(out + 6, ls->emit);
        out[9] = ls->pdf;
        return 1;
    });
}

void oracle_camera_ray(const tpt_camera_desc* cam, double sx, double sy, uint64_t* rng_state, double out[7]) {
    Camera c = to_camera(*cam);
    Rng rng(1);
    rng.state = *rng_state;
    Ray r = c.ray(sx, sy, rng);
    *rng_state = rng.state;
    put3(out, r.o); put3(out + 3, r.d); out[6] = r.time;
}

int oracle_env_eval(const tpt_env_desc* env, const double dir[3], double out[4]) {
    return guarded([&] {
        auto e = to_env(*env);
        if (!e) throw std::runtime_error("env kind must be TPT_ENV_MAP");
        put3(out, e->sample(v3(dir)));
        out[3] = e->pdf(v3(dir));
        return TPT_OK;
    });
}

int oracle_env_sample_dir(const tpt_env_desc* env, uint64_t* rng_state, double out[7]) {
    return guarded([&] {
        auto e = to_env(*env);
        if (!e) throw std::runtime_error("env kind must be TPT_ENV_MAP");
        Rng rng(1);
        rng.state = *rng_state;
        Vec3 d; Color c; double pdf;
        e->sample_dir(rng, d, c, pdf);
        *rng_state = rng.state;
        put3(out, d); put3(out + 3, c); out[6] = pdf;
        return TPT_OK;
    });
}

int oracle_radiance(const tpt_scene_desc* desc, const tpt_render_config* cfg, int x, int y, uint64_t* rng_state,
                    double out[3]) {
    return guarded([&] {
        auto s = to_scene(*desc);
        RenderConfig rc = to_cfg(*cfg);
        Rng rng(1);
        rng.state = *rng_state;
        double inv_w = 1.0 / (double)rc.width, inv_h = 1.0 / (double)rc.height;
        double jx = rng.next_f64(), jy = rng.next_f64();
        double sx = ((double)x + jx) * inv_w * 2.0 - 1.0;
        double sy = 1.0 - ((double)y + jy) * inv_h * 2.0;
        Ray ray = s->cam.ray(sx, sy, rng);
        Color c = radiance(s->world, s->mats, s->env ? &*s->env : nullptr, ray, rng,
                           PathLimits{rc.max_bounces, rc.rr_start}, nullptr);
        *rng_state = rng.state;
        put3(out, c);
        return TPT_OK;
    });
}

}  // extern "C"
