// Rust FFI declarations of include/tinypt_cuda.h, one for one: add to the
// tinypt crate as src/cuda.rs (with the build.rs link lines) to call the
// B200 integrator from render()'s callers.  Struct fields follow the C
// structs' order and types; tests/test_abi_layout.py checks both against
// the header.
use std::os::raw::{c_char, c_double, c_int, c_void};

#[repr(C)] pub struct TptMaterial { pub kind: i32, pub reserved: i32, pub rgb: [f64; 3], pub param: f64 }
#[repr(C)] pub struct TptSphere { pub center: [f64; 3], pub radius: f64, pub mat_id: i64 }
#[repr(C)] pub struct TptMeshDesc {
    pub positions: *const f64, pub n_vertices: i64,
    pub indices: *const i32, pub mat_ids: *const i32, pub n_tris: i64,
}
#[repr(C)] pub struct TptInstanceDesc { pub mesh_id: i64, pub linear: [f64; 9], pub translation: [f64; 3], pub mat_override: i64 }
#[repr(C)] pub struct TptCameraDesc {
    pub kind: i32, pub reserved: i32, pub eye: [f64; 3], pub target: [f64; 3], pub up: [f64; 3],
    pub fov_y_deg: f64, pub aspect: f64, pub focus_dist: f64, pub aperture: f64,
}
#[repr(C)] pub struct TptEnvDesc { pub kind: i32, pub width: i32, pub height: i32, pub reserved: i32, pub pixels: *const f64 }
#[repr(C)] pub struct TptSceneDesc {
    pub camera: TptCameraDesc,
    pub spheres: *const TptSphere, pub n_spheres: i64,
    pub meshes: *const TptMeshDesc, pub n_meshes: i64,
    pub instances: *const TptInstanceDesc, pub n_instances: i64,
    pub materials: *const TptMaterial, pub n_materials: i64,
    pub env: TptEnvDesc,
}
#[repr(C)] pub struct TptRenderConfig {
    pub width: i32, pub height: i32, pub spp: i32, pub max_bounces: i32, pub rr_start: i32, pub tile: i32,
    pub adaptive_enabled: i32, pub adaptive_min_spp: i32, pub adaptive_threshold: f64,
    pub morton_enabled: i32, pub mode: i32, pub seed: u64,
    pub row_begin: i32, pub row_step: i32,   // row shard; row_step = 0: the whole film
}
#[repr(C)] pub struct TptBatchJob { pub scene: i32, pub reserved: i32, pub config: TptRenderConfig,
                                  pub d_acc: *mut f64, pub d_acc_w: *mut f64 }
#[repr(C)] #[derive(Default)] pub struct TptTuning { pub pool_slots: i32, pub task_spp: i32, pub trace_chunk: i32,
                                                     pub shade_ctas: i32 }
#[repr(C)] #[derive(Default)] pub struct TptStats {
    pub render_ms: f64, pub paths: u64, pub rays_closest: u64, pub rays_shadow: u64, pub iterations: u64,
    pub device_flags: i32, pub profile: i32, pub stage_ms: [f64; 4], pub stage_launches: [u64; 4],
    pub nodes_visited: [u64; 2], pub tris_tested: [u64; 2], pub spheres_tested: [u64; 2], pub instances_tested: [u64; 2],
    pub adjoint_linear: f64, pub node_steps: [u64; 2], pub camera_fast: u64,
    pub leaf_visits: [u64; 2], pub leaf_steps: [u64; 2], pub fast_steps: u64, pub task_spp: i32, pub pool_slots: i32,
    pub sky_samples: u64, pub kernel_launches: u64,
}

extern "C" {
    pub fn tpt_scene_create(desc: *const TptSceneDesc, out_scene: *mut *mut c_void) -> c_int;
    pub fn tpt_scene_destroy(scene: *mut c_void);
    pub fn tpt_render(scene: *mut c_void, cfg: *const TptRenderConfig,
                      acc: *mut c_double, acc_w: *mut c_double, stats: *mut TptStats) -> c_int;
    pub fn tpt_render_device(scene: *mut c_void, cfg: *const TptRenderConfig, d_acc: *mut c_double,
                             d_acc_w: *mut c_double, d_acc_sq: *mut c_double, stats: *mut TptStats) -> c_int;
    pub fn tpt_render_device_noalloc(scene: *mut c_void, cfg: *const TptRenderConfig, d_acc: *mut c_double,
                                     d_acc_w: *mut c_double, stats: *mut TptStats) -> c_int;
    pub fn tpt_scene_material_count(scene: *mut c_void) -> i64;
    pub fn tpt_scene_set_materials(scene: *mut c_void, mats: *const TptMaterial,
                                   sampling_mats: *const TptMaterial, n: i64) -> c_int;
    pub fn tpt_render_forward(scene: *mut c_void, cfg: *const TptRenderConfig, image: *mut f32,
                              stats: *mut TptStats) -> c_int;
    pub fn tpt_render_forward_device(scene: *mut c_void, cfg: *const TptRenderConfig, d_image: *mut f32,
                                     stats: *mut TptStats) -> c_int;
    pub fn tpt_render_backward(scene: *mut c_void, cfg: *const TptRenderConfig, dl_dimage: *const f32,
                               grad: *mut f64, stats: *mut TptStats) -> c_int;
    pub fn tpt_render_backward_device(scene: *mut c_void, cfg: *const TptRenderConfig, d_dl_dimage: *const f32,
                                      d_grad: *mut f64, stats: *mut TptStats) -> c_int;
    pub fn tpt_batch_create(scenes: *const TptSceneDesc, n: i64, out: *mut *mut c_void) -> c_int;
    pub fn tpt_batch_destroy(batch: *mut c_void);
    pub fn tpt_batch_render_device(batch: *mut c_void, jobs: *const TptBatchJob, n_jobs: i64,
                                   tuning: *const TptTuning, stats: *mut TptStats) -> c_int;
    pub fn tpt_batch_autotune(batch: *mut c_void, jobs: *const TptBatchJob, n_jobs: i64, best: *mut TptTuning,
                              trial_ms: *mut f64, n_trials: i32) -> c_int;
    pub fn tpt_scene_load_xml(path: *const c_char, cfg: *mut TptRenderConfig, out_loaded: *mut *mut c_void) -> c_int;
    pub fn tpt_scene_default(cfg: *const TptRenderConfig, env_path: *const c_char,
                             out_loaded: *mut *mut c_void) -> c_int;
    pub fn tpt_loaded_desc(loaded: *mut c_void) -> *const TptSceneDesc;
    pub fn tpt_loaded_warning_count(loaded: *mut c_void) -> i64;
    pub fn tpt_loaded_warning(loaded: *mut c_void, index: i64) -> *const c_char;
    pub fn tpt_loaded_destroy(loaded: *mut c_void);
    pub fn tpt_write_image(path: *const c_char, width: i32, height: i32, rgb: *const f64, exposure: f64,
                           tonemap: i32) -> c_int;
    pub fn tpt_read_hdr(path: *const c_char, width: *mut i32, height: *mut i32, rgb: *mut f64) -> c_int;
    pub fn tpt_checkpoint_save(path: *const c_char, scene_hash: u64, width: i32, height: i32, next_id: u64,
                               acc: *const f64, acc_w: *const f64) -> c_int;
    pub fn tpt_checkpoint_load(path: *const c_char, scene_hash: u64, width: i32, height: i32, next_id: *mut u64,
                               acc: *mut f64, acc_w: *mut f64) -> c_int;
    pub fn tpt_film_tiles(width: i32, height: i32, tile: i32, morton: i32, x0y0x1y1: *mut i32) -> i64;
    pub fn tpt_render_resume(scene: *mut c_void, cfg: *const TptRenderConfig, ckpt_path: *const c_char,
                             scene_hash: u64, acc: *mut f64, acc_w: *mut f64, stats: *mut TptStats) -> c_int;
    pub fn tpt_bvh_build_host(mesh: *const TptMeshDesc, bbox: *mut f64, left_right: *mut i32,
                              start_count: *mut u32, indices: *mut i64) -> i64;
    pub fn tpt_bvh_build_device(mesh: *const TptMeshDesc, bbox: *mut f64, left_right: *mut i32,
                                start_count: *mut u32, indices: *mut i64) -> i64;
    pub fn tpt_bvh_build_fp32(mesh: *const TptMeshDesc, bbox: *mut f64, left_right: *mut i32,
                              start_count: *mut u32, indices: *mut i64) -> i64;
    pub fn tpt_last_error() -> *const c_char;
    pub fn tpt_version() -> *const c_char;
    pub fn tpt_probe_read_bandwidth(bytes: i64, reps: c_int, gbs_out: *mut f64) -> c_int;
}
