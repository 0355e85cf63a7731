/* ORACLE -- test infrastructure only.  C ABI of the CPU f64 restatement of
 * tinypt's path integrator (ref_model.hpp).  Loaded by tests/, by the smoke
 * check and by bench.py's CPU-baseline leg; never by the product. */
#ifndef TINYPT_ORACLE_H
#define TINYPT_ORACLE_H

#include <stdint.h>
#include "../include/tinypt_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_counts {
    uint64_t world_hits;      /* World::hit calls (closest + shadow rays)    */
    uint64_t node_pops;       /* BVH nodes popped (own box re-test)          */
    uint64_t node_box_tests;  /* slab tests incl. both children per interior */
    uint64_t tri_tests;       /* Triangle::hit calls                         */
    uint64_t sphere_tests;    /* Sphere::hit calls                           */
} oracle_counts;

/* Builds the reference Scene (meshes, BVHs, lights, env CDF) once. */
int oracle_scene_create(const tpt_scene_desc* desc, void** out);
void oracle_scene_destroy(void* scene);
/* Replaces the scene's materials (same count and kinds).  sampling, when not
 * NULL, gives the GGX alpha of the sampler and pdfs and the light-selection
 * weights (detached sampling, for finite-difference derivative checks). */
int oracle_scene_set_materials(void* scene, const tpt_material* mats, const tpt_material* sampling, int64_t n);
/* render() on a built scene; rect = NULL for the full film, else
 * {x0, y0, x1, y1}: only that sub-rectangle is rendered (same per-pixel RNG
 * streams) and outputs hold (x1-x0)*(y1-y0) pixels. */
int oracle_scene_render(void* scene, const tpt_render_config* cfg, const int32_t* rect, double* acc,
                        double* acc_w, double* acc_sq, int threads, oracle_counts* counts);

/* Same, with every tile task's samples cut into tasks of sample_chunk samples
 * (the reference worker's Task { sample_start, sample_end }, each seeded from
 * seed_for(x, y, sample_start); results merged in task-id order, chunk by
 * chunk).  sample_chunk = 0 is the reference's own task list. */
int oracle_scene_render_tasks(void* scene, const tpt_render_config* cfg, const int32_t* rect, int sample_chunk,
                              double* acc, double* acc_w, double* acc_sq, int threads, oracle_counts* counts);

/* The reference's task list and per-pixel loop (sums in sample order, one
 * Welford statistic for adaptive sampling) with each pixel's RNG restarted
 * from seed_for(x, y, s) ^ seed at every sample s that is a multiple of
 * reseed (reseed > 0; sample_chunk must then be 0). */
int oracle_scene_render_streams(void* scene, const tpt_render_config* cfg, const int32_t* rect, int sample_chunk,
                                int reseed, double* acc, double* acc_w, double* acc_sq, int threads,
                                oracle_counts* counts);

/* output.rs resolve_pixels: out[3i+c] = acc[3i+c] / max(acc_w[i], 1). */
void oracle_resolve_pixels(int64_t n, const double* acc, const double* acc_w, double* out);

/* render() over a flattened scene; acc_sq and counts may be NULL. */
int oracle_render(const tpt_scene_desc* desc, const tpt_render_config* cfg, double* acc, double* acc_w,
                  double* acc_sq, int threads, oracle_counts* counts);

/* rng.rs */
void oracle_rng_u32(uint64_t seed, int n, uint32_t* out);
void oracle_rng_f64(uint64_t seed, int n, double* out);
uint64_t oracle_seed_for(uint32_t px, uint32_t py, uint32_t s);
/* render.rs */
uint64_t oracle_interleave_bits(uint64_t v);
int oracle_tile_order(int w, int h, int tile, int morton, int32_t* x0y0x1y1);
/* bvh.rs: same output layout as tpt_bvh_build_host */
int64_t oracle_bvh_build(const tpt_mesh_desc* mesh, double* bbox, int32_t* left_right, uint32_t* start_count,
                         int64_t* indices);

/* material.rs sample(): out = o[3], d[3], weight[3], pdf, is_delta; returns
 * 1 for Some, 0 for None.  rng_state is advanced in place. */
int oracle_material_sample(const tpt_material* m, const double ray_o[3], const double ray_d[3], double time,
                           double hit_t, const double hit_p[3], const double hit_n[3], uint64_t* rng_state,
                           double out[11]);
/* material.rs eval(): out = f[3], pdf */
void oracle_material_eval(const tpt_material* m, const double wo[3], const double wi[3], const double n[3],
                          double out[4]);

/* eval() of `count` directions wi (count x 3): out = count x (f[3], pdf) */
void oracle_material_eval_n(const tpt_material* m, const double wo[3], const double* wi, const double n[3],
                            int64_t count, double* out);
/* material.rs is_delta() and emitted().is_some(): out = {is_delta, emits} */
void oracle_material_classify(const tpt_material* m, int32_t out[2]);

/* transform.rs: ops are applied as acc = acc.compose(op) in order.
 * op kinds: 0 translate(xyz), 1 scale(xyz), 2 rotate(axis xyz, deg), 3
 * legacy new(t xyz, rot_y_deg, s).  params: 5 doubles per op.
 * mode: 0 apply_point, 1 apply_point_inv, 2 apply_normal.
 * Also returns A (9) and t (3) of the composed transform in a_t_out. */
void oracle_transform(int n_ops, const int32_t* kinds, const double* params, int mode, const double p[3],
                      double out[3], double a_t_out[12]);

/* world.rs sample_light over a scene: out = position[3], normal[3], emit[3],
 * pdf; returns 1 for Some.  light_total_out receives World.light_total. */
int oracle_sample_light(const tpt_scene_desc* desc, uint64_t* rng_state, double time, const double p[3],
                        double out[10], double* light_total_out, int64_t* n_lights_out);

/* ray.rs Camera::ray: out = o[3], d[3], time */
void oracle_camera_ray(const tpt_camera_desc* cam, double sx, double sy, uint64_t* rng_state, double out[7]);

/* env.rs: sample(dir) -> rgb, pdf(dir), sample_dir -> dir, rgb, pdf */
int oracle_env_eval(const tpt_env_desc* env, const double dir[3], double out_rgb_pdf[4]);
int oracle_env_sample_dir(const tpt_env_desc* env, uint64_t* rng_state, double out[7]);

/* One path: radiance() for a given camera sample (pixel x, y; RNG state is
 * taken and returned in rng_state).  out = rgb. */
int oracle_radiance(const tpt_scene_desc* desc, const tpt_render_config* cfg, int x, int y, uint64_t* rng_state,
                    double out[3]);

const char* oracle_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
