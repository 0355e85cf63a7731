/*
 * tinypt_cuda.h -- C ABI of the B200 (sm_100a) path integrator.
 *
 * This is the drop-in boundary for tinypt's per-sample path integrator.  The
 * reference exposes the path as a Rust library API, not as an FFI:
 *
 *   render(scene: &Scene, config: &RenderConfig, ckpt_file: &str)
 *       -> io::Result<RenderOutput { acc: Vec<Color>, acc_w: Vec<f64> }>
 *                                                    (src/render.rs:42, :34-39)
 *   radiance(&World, &[Material], Option<&EnvMap>, Ray, &mut Rng, PathLimits)
 *                                                    (src/integrator.rs:53-60)
 *   Scene { cam, world, mats, env }                  (src/scene.rs:14-23)
 *
 * The entry points below are what a Rust `extern "C"` block would bind in
 * place of those calls.  The Scene is passed once, flattened into plain
 * arrays (tpt_scene_desc), and owned by an opaque handle on the device.
 *
 * Conventions
 *   - Every function returns TPT_OK (0) or a negative TPT_ERR_* code; the
 *     message of the last failure on the calling thread is tpt_last_error().
 *   - The caller owns every output buffer.  Host pointers are plain host
 *     memory; the *_device variants take device pointers.
 *   - One handle uses one CUDA stream; a handle is not re-entrant.  Several
 *     handles may render concurrently from different host threads.
 *   - A handle lives on the device that was current when it was created.
 *     Each call makes that device current for its work and restores the
 *     caller's current device before it returns.
 *   - All reference arithmetic is f64.  TPT_MODE_PLAIN_F64 keeps it; the
 *     wavefront mode traces and shades in FP32 and accumulates in f64.
 */
#ifndef TINYPT_CUDA_H
#define TINYPT_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define TPT_OK               0
#define TPT_ERR_INVALID     -1  /* bad argument or malformed scene          */
#define TPT_ERR_CUDA        -2  /* a CUDA runtime call failed               */
#define TPT_ERR_ALLOC       -3  /* device or host allocation failed         */
#define TPT_ERR_UNSUPPORTED -4  /* valid request this build does not serve  */
#define TPT_ERR_DEVICE      -5  /* a kernel reported an error flag
                                   (stack overflow, queue overflow, bounded
                                   wait gave up); the context stays usable  */

/* ---- scene description (src/material.rs:30-43) ------------------------ */
enum {
    TPT_MAT_LAMBERT       = 0,  /* Lambert { albedo }                    */
    TPT_MAT_METAL         = 1,  /* Metal { albedo }                      */
    TPT_MAT_DIELECTRIC    = 2,  /* Dielectric { ior, absorption }        */
    TPT_MAT_GGX           = 3,  /* Ggx { albedo, alpha }                 */
    TPT_MAT_SUBSURFACE    = 4,  /* Subsurface { albedo, scatter_dist }   */
    TPT_MAT_DIFFUSE_LIGHT = 5   /* DiffuseLight { emit }                 */
};

typedef struct tpt_material {
    int32_t kind;               /* TPT_MAT_*                                   */
    int32_t reserved;
    double  rgb[3];             /* albedo | absorption (Dielectric) | emit     */
    double  param;              /* ior | alpha (Ggx) | scatter_dist | unused   */
} tpt_material;

/* Sphere { c, r, mat_id }  (src/geometry.rs:26-34) */
typedef struct tpt_sphere {
    double  center[3];
    double  radius;
    int64_t mat_id;
} tpt_sphere;

/* A static triangle mesh (Mesh::new over Triangle::new_static,
 * src/world.rs:20-33, src/geometry.rs:199-210).  The BVH is built by the
 * library with the reference's binned-SAH rules (src/bvh.rs:51-242). */
typedef struct tpt_mesh_desc {
    const double*  positions;   /* n_vertices x 3                              */
    int64_t        n_vertices;
    const int32_t* indices;     /* n_tris x 3, 0-based vertex indices          */
    const int32_t* mat_ids;     /* n_tris, Triangle.mat_id                     */
    int64_t        n_tris;
} tpt_mesh_desc;

/* Instance { mesh_id, xform, mat_override }  (src/world.rs:39-46).
 * xform is Transform::from_affine(A, t): p' = A p + t  (src/transform.rs:24) */
typedef struct tpt_instance_desc {
    int64_t mesh_id;
    double  linear[9];          /* A, row-major                               */
    double  translation[3];     /* t                                          */
    int64_t mat_override;       /* -1 = None                                  */
} tpt_instance_desc;

/* Camera::look_at / Camera::look_at_dof  (src/ray.rs:36-86) */
enum { TPT_CAMERA_LOOK_AT = 0, TPT_CAMERA_LOOK_AT_DOF = 1 };
typedef struct tpt_camera_desc {
    int32_t kind;
    int32_t reserved;
    double  eye[3];
    double  target[3];
    double  up[3];
    double  fov_y_deg;
    double  aspect;
    double  focus_dist;         /* LOOK_AT_DOF only                           */
    double  aperture;           /* LOOK_AT_DOF only; lens radius = aperture/2 */
} tpt_camera_desc;

/* Option<EnvMap>  (src/env.rs:20-33; None -> sky(), src/integrator.rs:25-37) */
enum { TPT_ENV_NONE = 0, TPT_ENV_MAP = 1 };
typedef struct tpt_env_desc {
    int32_t       kind;
    int32_t       width;
    int32_t       height;
    int32_t       reserved;
    const double* pixels;       /* width*height*3 linear RGB; row 0 is theta=0 */
} tpt_env_desc;

typedef struct tpt_scene_desc {
    tpt_camera_desc          camera;
    const tpt_sphere*        spheres;   int64_t n_spheres;
    const tpt_mesh_desc*     meshes;    int64_t n_meshes;
    const tpt_instance_desc* instances; int64_t n_instances;
    const tpt_material*      materials; int64_t n_materials;
    tpt_env_desc             env;
} tpt_scene_desc;

/* ---- render configuration (RenderConfig, src/config.rs:5-46) ---------- */
enum {
    TPT_MODE_PLAIN_F64     = 0, /* one thread per pixel, reference f64 math   */
    TPT_MODE_WAVEFRONT_FP32 = 1 /* FP32 wavefront queues, f64 accumulation    */
};

typedef struct tpt_render_config {
    int32_t  width;
    int32_t  height;
    int32_t  spp;
    int32_t  max_bounces;       /* PathLimits.max_bounces                      */
    int32_t  rr_start;          /* PathLimits.rr_start                         */
    int32_t  tile;              /* tile edge in pixels (task partition)        */
    int32_t  adaptive_enabled;
    int32_t  adaptive_min_spp;
    double   adaptive_threshold;
    int32_t  morton_enabled;
    int32_t  mode;              /* TPT_MODE_*; TPT_MODE_WAVEFRONT_FP32 takes
                                   max_bounces <= 255 and, when a pixel's samples
                                   are one task (allocation-free renders,
                                   TPT_ADAPTIVE_ROUNDS=0), spp <= 524287;
                                   beyond: TPT_ERR_UNSUPPORTED               */
    uint64_t seed;
    /* Row sharding (no counterpart in the reference, whose workers split the
     * film into tiles inside one process): row_step <= 0 renders the whole
     * film.  Otherwise only rows y = row_begin + k*row_step (k = 0, 1, ...,
     * y < height) are rendered, each pixel with the same RNG stream as in
     * the whole-film render, and the output film holds just those rows,
     * compacted in order: n_rows = ceil((height - row_begin) / row_step)
     * rows of width pixels.  One GPU of N takes row_begin = rank,
     * row_step = N. */
    int32_t  row_begin;
    int32_t  row_step;
} tpt_render_config;

typedef struct tpt_stats {
    double   render_ms;         /* device time of the render (CUDA events)     */
    uint64_t paths;             /* camera samples finished (sum of acc_w)      */
    uint64_t rays_closest;      /* closest-hit traces: camera + extension      */
    uint64_t rays_shadow;       /* occlusion traces (NEE shadow rays)          */
    uint64_t iterations;        /* wavefront iterations (0 for PLAIN_F64)      */
    int32_t  device_flags;      /* TPT_FLAG_* raised by kernels                */
    int32_t  profile;           /* in: 1 = per-stage timing + traversal counts
                                   (wavefront only; slower, for profiling)   */
    /* Filled when profile == 1.  Stages: 0 extend, 1 shade, 2 shadow,
     * 3 regen.  Traversal counts are per stage 0 (closest hit) and 2
     * (occlusion): interior BVH2 nodes visited, triangles tested, spheres
     * tested, instance boxes tested. */
    double   stage_ms[4];
    uint64_t stage_launches[4];
    uint64_t nodes_visited[2];
    uint64_t tris_tested[2];
    uint64_t spheres_tested[2];
    uint64_t instances_tested[2];
    /* tpt_render_backward*: sum over pixels of dL/dimage . image, the image
     * being the one the adjoint's own paths estimate (the linearised loss;
     * its finite differences check the gradient with the same paths). */
    double   adjoint_linear;
    /* Filled when profile == 1 (wavefront).  node_steps: warp-wide steps of
     * the traversal's node loop per stage (0 closest hit, 1 occlusion);
     * nodes_visited / (32 * node_steps) is the fraction of lanes busy per
     * step.  camera_fast: samples whose camera ray left the scene and that
     * the closest-hit kernel finished in place. */
    uint64_t node_steps[2];
    uint64_t camera_fast;
    /* Filled when profile == 1 (wavefront): leaf visits (leaves, instance
     * entries and exits) per trace kind and the warp-wide steps they took;
     * warp-wide steps of the camera-miss fast path (camera_fast / (32 *
     * fast_steps) = its lanes busy). */
    uint64_t leaf_visits[2];
    uint64_t leaf_steps[2];
    uint64_t fast_steps;
    /* Wavefront renders: the samples per pool task the render ran with
     * (task k of a pixel draws Rng::new(seed_for(x, y, k * task_spp) ^
     * seed)) and its path slots in flight (after any halving for room). */
    int32_t  task_spp;
    int32_t  pool_slots;
    /* Wavefront renders, batch renders and adjoint (backward) renders
     * through pinhole cameras, adaptive ones excepted: samples of the
     * pixels whose every camera ray leaves the scene -- a conservative
     * frustum test against the top-level boxes -- which a coherent kernel
     * renders with the same draws and arithmetic instead of tracing them
     * (TPT_SKY_CULL=0 turns the test off; the film is the same either way).
     * They count in paths (and, forward, in rays_closest). */
    uint64_t sky_samples;
    /* Wavefront renders: the kernels the render launched (the device-side
     * loop's kernel nodes included). */
    uint64_t kernel_launches;
} tpt_stats;

#define TPT_FLAG_STACK_OVERFLOW 0x1  /* traversal stack limit reached        */
#define TPT_FLAG_QUEUE_OVERFLOW 0x2  /* a wavefront queue overflowed         */
#define TPT_FLAG_ITER_LIMIT     0x4  /* iteration bound reached              */

/* ---- entry points ------------------------------------------------------ */

/* Builds the per-mesh BVHs on the host (reference node order), flattens the
 * scene into device arrays and uploads it to the current CUDA device.
 * Replaces Scene construction + Mesh::new (src/world.rs:29-32) and
 * World::build_lights (src/world.rs:127-167). */
int tpt_scene_create(const tpt_scene_desc* desc, void** out_scene);

/* Frees every device allocation owned by the handle. */
void tpt_scene_destroy(void* scene);

/* render() (src/render.rs:42): writes acc (width*height*3 f64, linear RGB
 * sums) and acc_w (width*height f64, sample counts) to HOST memory.
 * stats may be NULL. */
int tpt_render(void* scene, const tpt_render_config* config,
               double* acc, double* acc_w, tpt_stats* stats);

/* Same as tpt_render with DEVICE output pointers (no host copies).  acc_sq
 * (width*height*3 f64, per-channel sums of squared sample radiance) may be
 * NULL; when given, it holds the second moments for per-pixel variance. */
int tpt_render_device(void* scene, const tpt_render_config* config,
                      double* d_acc, double* d_acc_w, double* d_acc_sq,
                      tpt_stats* stats);

/* Allocation-free render.  No counterpart in the reference (whose render()
 * allocates its film and thread pool on every call).  For callers that must
 * not allocate device memory while rendering -- a process whose own
 * allocator reserves the GPU at start-up, or a frame loop that cannot take
 * the device-wide synchronisation of cudaMalloc/cudaFree.  Renders in
 * TPT_MODE_WAVEFRONT_FP32 (config->mode is ignored) into the caller's DEVICE
 * buffers d_acc (width*height*3 f64) and d_acc_w (width*height f64).
 *
 * Scratch (path state, queues, counters) lives in one file-scope device array
 * of 5,128,704 bytes (about 5.1 MB) that every GPU loading the library holds
 * until exit; films larger than 16384 pixels are rejected with
 * TPT_ERR_INVALID.  The call
 * makes no cudaMalloc/cudaFree and creates no graph, event or stream.
 * The first call on a device looks up the array's device address (once per
 * device); make that first call before any stream capture.  Under CUDA's
 * lazy module loading (the default) that first call may also be when the
 * array is placed in device memory, so make it before the caller's own
 * allocator takes the GPU's free memory.  All calls share
 * the array: calls that overlap on the GPU race and must be serialised by
 * the caller.  stats may be NULL; its profile field is ignored. */
int tpt_render_device_noalloc(void* scene, const tpt_render_config* config, double* d_acc, double* d_acc_w,
                              tpt_stats* stats);

/* ---- differentiation --------------------------------------------------
 * No counterpart in the reference, which renders only.  The parameters are
 * 4 per material, in material order: rgb[0..2] (Lambert/Metal/Ggx/
 * Subsurface albedo, Dielectric absorption, DiffuseLight emission) and
 * param (Ggx alpha; the gradient of Dielectric ior and Subsurface
 * scatter_dist is reported as 0). */

/* Number of materials of the scene (the gradient has 4 entries each);
 * -1 for a NULL handle. */
int64_t tpt_scene_material_count(void* scene);

/* Replaces Scene.mats (src/scene.rs:14-23) in place: same count, same kinds;
 * the light table (World::build_lights, src/world.rs:127-167) is rebuilt.
 * sampling_materials, when not NULL, are the materials the samplers use --
 * the GGX alpha of the VNDF sampler and of every pdf (sample weights, MIS)
 * and the light-selection weights -- while BSDF values and emission come
 * from materials.  This holds sampling fixed while the evaluated parameters
 * move, the quantity tpt_render_backward differentiates, so finite
 * differences of tpt_render_forward can check it.  With sampling materials
 * that differ from materials only the FP32 form renders (PLAIN_F64 returns
 * TPT_ERR_UNSUPPORTED). */
int tpt_scene_set_materials(void* scene, const tpt_material* materials,
                            const tpt_material* sampling_materials,
                            int64_t n_materials);

/* Forward render for a loss: renders like tpt_render_device (config->mode
 * selects the form) and resolves acc / max(acc_w, 1) (src/output.rs:96-102)
 * into d_image (width*height*3 float, DEVICE). */
int tpt_render_forward_device(void* scene, const tpt_render_config* config,
                              float* d_image, tpt_stats* stats);
/* Same with a HOST image. */
int tpt_render_forward(void* scene, const tpt_render_config* config,
                       float* image, tpt_stats* stats);

/* Adjoint render: path-replay backpropagation.  Given dL/dimage
 * (width*height*3 float, the gradient of a loss with respect to the
 * resolved image), writes d_grad[4*n_materials] (f64, overwritten) =
 * dL/dparameters of the image the config renders, estimated with
 * config->spp samples per pixel seeded by config->seed (use a seed other
 * than the forward render's for an estimate independent of it).  Sampling
 * is detached (directions, light choices, pdfs, MIS and Russian-roulette
 * probabilities held fixed); each path is regenerated from its PCG32 seed,
 * traced once to total its adjoint-weighted radiance and once more to
 * distribute it, so nothing is stored per path.  FP32 form only
 * (config->mode must be WAVEFRONT_FP32); adaptive sampling must be off. */
int tpt_render_backward_device(void* scene, const tpt_render_config* config,
                               const float* d_dL_dimage, double* d_grad,
                               tpt_stats* stats);
/* Same with HOST dL/dimage and gradient. */
int tpt_render_backward(void* scene, const tpt_render_config* config,
                        const float* dL_dimage, double* grad,
                        tpt_stats* stats);

/* ---- batch renders ----------------------------------------------------
 * No counterpart in the reference, which renders one scene per process.
 * Many scenes, and films of uneven size and spp, render in ONE wavefront
 * loop (one graph launch): the scenes' device arrays are merged, each job
 * walks its own scene's top-level BVH with its own camera, env map and
 * lights, and one task pool spans all jobs.  Each job's film is identical
 * to what tpt_render_device writes for that scene and config with the same
 * tuning (per-pixel RNG streams do not depend on the batch). */

typedef struct tpt_batch_job {
    int32_t            scene;   /* index into the batch's scenes             */
    int32_t            reserved;
    tpt_render_config  config;  /* mode must be WAVEFRONT_FP32, adaptive off  */
    double*            d_acc;   /* DEVICE film: film pixels x 3 f64          */
    double*            d_acc_w; /* DEVICE sample counts: film pixels f64     */
} tpt_batch_job;

/* Wavefront schedule parameters (0 = the library default). */
typedef struct tpt_tuning {
    int32_t pool_slots;         /* paths in flight (default 64 Mi)            */
    int32_t task_spp;           /* samples per pool task (default 8)          */
    int32_t trace_chunk;        /* leaf visits between lane refills (def. 4)  */
    int32_t shade_ctas;         /* resident blocks per SM the shading kernel is
                                   compiled for: 4 or 8 (default 4)          */
} tpt_tuning;

/* Builds every scene's BVHs and uploads them merged (one handle). */
int tpt_batch_create(const tpt_scene_desc* scenes, int64_t n_scenes, void** out_batch);
void tpt_batch_destroy(void* batch);

/* Renders all jobs.  A job of at least 16 Mi paths (film pixels x spp;
 * TPT_BATCH_ALONE_PATHS overrides, 0 = none) keeps the GPU busy on its own
 * and renders alone with the single-render schedule, its film equal to
 * tpt_render_device's; the others share one wavefront loop under tuning
 * (NULL: the defaults).  stats (nullable) receives the totals of the batch. */
int tpt_batch_render_device(void* batch, const tpt_batch_job* jobs, int64_t n_jobs,
                            const tpt_tuning* tuning, tpt_stats* stats);

/* Autotuner: times short renders of the same jobs at reduced spp over a
 * set of schedules (pool size, then task length, then refill chunk, each
 * chosen with the others fixed, then the shading variant; 13 trials at
 * most, a warm-up included) and writes the fastest to *best (jobs that
 * render alone take their own schedule in every trial);
 * trial_ms (nullable, n_trials entries) receives each trial's time.
 * Returns the number of trials run, or a negative error code. */
int tpt_batch_autotune(void* batch, const tpt_batch_job* jobs, int64_t n_jobs,
                       tpt_tuning* best, double* trial_ms, int32_t n_trials);

/* ---- scene ingestion and image files (host only, no GPU work) ---------- */

/* Loads a Mitsuba XML scene (the subset of src/mitsuba.rs:137-595: film,
 * sampler, integrator, perspective sensor, sphere/rectangle/cube/disk/obj
 * shapes with transforms, diffuse/conductor/roughconductor/dielectric/
 * twosided bsdfs, area emitters, envmap (.hdr) and constant scene
 * emitters; OBJ meshes as src/obj_loader.rs).  film/sampler/integrator
 * values overwrite config's width, height, spp, max_bounces and rr_start.
 * *out_loaded owns the description; warnings are kept, not printed. */
int tpt_scene_load_xml(const char* path, tpt_render_config* config, void** out_loaded);
/* The built-in scene (src/scene.rs:26-95) for config's film aspect;
 * env_path (NULL: procedural sky) names a Radiance .hdr env map. */
int tpt_scene_default(const tpt_render_config* config, const char* env_path, void** out_loaded);
const tpt_scene_desc* tpt_loaded_desc(void* loaded);
int64_t tpt_loaded_warning_count(void* loaded);
const char* tpt_loaded_warning(void* loaded, int64_t index);
void tpt_loaded_destroy(void* loaded);

/* Writes linear RGB pixels (width*height*3 f64, row 0 at the top) in the
 * format the path's extension selects (src/output.rs:59-132): .exr ->
 * ACEScg float32; .hdr -> Radiance RGBE; otherwise PPM (P3) after exposure
 * (x 2^exposure), tonemap (0 none, 1 ACES fitted) and sRGB encoding. */
int tpt_write_image(const char* path, int32_t width, int32_t height, const double* rgb, double exposure,
                    int32_t tonemap);
/* Reads a Radiance .hdr (src/hdr.rs:20-60) into rgb (width*height*3 f64,
 * row 0 at the top).  rgb = NULL: only *width and *height are set. */
int tpt_read_hdr(const char* path, int32_t* width, int32_t* height, double* rgb);

/* ---- checkpoints (src/checkpoint.rs, HYPCKPT v1) ----------------------
 * Tasks are the film's tiles in the reference's order (tile edge
 * config->tile, Morton order when config->morton_enabled; render.rs:75-100);
 * next_id counts the tiles merged into the film. */
int tpt_checkpoint_save(const char* path, uint64_t scene_hash, int32_t width, int32_t height, uint64_t next_id,
                        const double* acc, const double* acc_w);
/* 1 and the film when the file matches (magic, version, hash, size); 0
 * when it is absent or does not match; a negative code on a bad file. */
int tpt_checkpoint_load(const char* path, uint64_t scene_hash, int32_t width, int32_t height, uint64_t* next_id,
                        double* acc, double* acc_w);
/* The film's tiles in task order (x0, y0, x1, y1 each; NULL: count only). */
int64_t tpt_film_tiles(int32_t width, int32_t height, int32_t tile, int32_t morton, int32_t* x0y0x1y1);
/* render() with a checkpoint file (src/render.rs:42-72, :250-272): resumes
 * from ckpt_path when it matches -- tiles before its next_id come from the
 * file, the others from this render -- and leaves the final checkpoint
 * (next_id = all tiles) there.  HOST film outputs like tpt_render.  As in
 * the reference, a checkpoint that cannot be read (truncated, unreadable)
 * is ignored like an absent one, and a failed final save is reported on
 * stderr while the call still returns the film. */
int tpt_render_resume(void* scene, const tpt_render_config* config, const char* ckpt_path, uint64_t scene_hash,
                      double* acc, double* acc_w, tpt_stats* stats);

/* Host-side helpers with no GPU work (usable on a machine without a GPU). */

/* Builds one mesh's BVH with the reference rules and copies it out:
 * bbox[6*n] (min xyz, max xyz), left_right[2*n], start_count[2*n] and the
 * leaf triangle order indices[n_tris].  Returns the node count, or a
 * negative error code.  Pass NULL outputs to query the node count only.
 * Mirrors Bvh::build (src/bvh.rs:51-242). */
int64_t tpt_bvh_build_host(const tpt_mesh_desc* mesh, double* bbox,
                           int32_t* left_right, uint32_t* start_count,
                           int64_t* indices);

/* The same BVH as tpt_bvh_build_host -- node for node, bit for bit --
 * built on the current CUDA device: triangle boxes, per-node box and bin
 * reductions and the stable partition by bin run as kernels, the per-node
 * SAH choice (8 bins, src/bvh.rs:99-176) on the host from the reduced bins,
 * nodes of at most 1024 triangles one per thread; nodes are numbered in
 * preorder like Bvh::build (src/bvh.rs:51-242).  Same outputs and NULL
 * convention as tpt_bvh_build_host; TPT_ERR_ALLOC when the device has no
 * room for the build's arrays, TPT_ERR_CUDA when another CUDA call fails.
 * tpt_scene_create and tpt_batch_create use this builder for meshes of
 * 32768 triangles or more (TPT_BVH_BUILD=host|device overrides). */
int64_t tpt_bvh_build_device(const tpt_mesh_desc* mesh, double* bbox,
                             int32_t* left_right, uint32_t* start_count,
                             int64_t* indices);

/* The mesh tree the FP32 forms walk (host, no GPU work): binned SAH over
 * the three axes, 16 bins, leaves of 1 to 6 triangles chosen by cost (a
 * node visit weighed as one triangle test), the triangle boxes of
 * tpt_bvh_build_host.  Same outputs and NULL convention as
 * tpt_bvh_build_host; nodes in preorder, root first.  The plain f64 form
 * keeps the reference's tree. */
int64_t tpt_bvh_build_fp32(const tpt_mesh_desc* mesh, double* bbox,
                           int32_t* left_right, uint32_t* start_count,
                           int64_t* indices);

/* Message of the last error on the calling thread ("" when none). */
const char* tpt_last_error(void);

/* Library version string. */
const char* tpt_version(void);

/* Measurement helper, no counterpart in the reference: streams a device
 * buffer of `bytes` (1 MiB .. 16 GiB) `reps` times with 16-byte loads that
 * bypass L1, on the current device, and writes the read bandwidth in GB/s
 * (CUDA events).  A buffer of at most half the L2 (64 MB on B200) gives the
 * L2 read bandwidth the traversal's roofline is quoted against; one larger
 * than L2 gives HBM read bandwidth.  Allocates and frees its buffer. */
int tpt_probe_read_bandwidth(int64_t bytes, int reps, double* gbs_out);

#ifdef __cplusplus
}
#endif

#endif /* TINYPT_CUDA_H */
