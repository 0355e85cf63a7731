"""ctypes mirror of include/tinypt_cuda.h and the loader of the sm_100a library.

The library is loaded from this package directory only (it is built in-tree
by ``tinypt_b200.build``).  There is no CPU fallback: if the library is
missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libtinypt_cuda.so"

TPT_OK = 0
TPT_ERR_INVALID = -1
TPT_ERR_CUDA = -2
TPT_ERR_ALLOC = -3
TPT_ERR_UNSUPPORTED = -4
TPT_ERR_DEVICE = -5

TPT_MAT_LAMBERT, TPT_MAT_METAL, TPT_MAT_DIELECTRIC, TPT_MAT_GGX, TPT_MAT_SUBSURFACE, TPT_MAT_DIFFUSE_LIGHT = range(6)
TPT_CAMERA_LOOK_AT, TPT_CAMERA_LOOK_AT_DOF = 0, 1
TPT_ENV_NONE, TPT_ENV_MAP = 0, 1
TPT_MODE_PLAIN_F64, TPT_MODE_WAVEFRONT_FP32 = 0, 1

TPT_FLAG_STACK_OVERFLOW = 0x1
TPT_FLAG_QUEUE_OVERFLOW = 0x2
TPT_FLAG_ITER_LIMIT = 0x4

D3 = C.c_double * 3


class tpt_material(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("rgb", D3), ("param", C.c_double)]


class tpt_sphere(C.Structure):
    _fields_ = [("center", D3), ("radius", C.c_double), ("mat_id", C.c_int64)]


class tpt_mesh_desc(C.Structure):
    _fields_ = [
        ("positions", C.POINTER(C.c_double)),
        ("n_vertices", C.c_int64),
        ("indices", C.POINTER(C.c_int32)),
        ("mat_ids", C.POINTER(C.c_int32)),
        ("n_tris", C.c_int64),
    ]


class tpt_instance_desc(C.Structure):
    _fields_ = [
        ("mesh_id", C.c_int64),
        ("linear", C.c_double * 9),
        ("translation", D3),
        ("mat_override", C.c_int64),
    ]


class tpt_camera_desc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("reserved", C.c_int32),
        ("eye", D3),
        ("target", D3),
        ("up", D3),
        ("fov_y_deg", C.c_double),
        ("aspect", C.c_double),
        ("focus_dist", C.c_double),
        ("aperture", C.c_double),
    ]


class tpt_env_desc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("reserved", C.c_int32),
        ("pixels", C.POINTER(C.c_double)),
    ]


class tpt_scene_desc(C.Structure):
    _fields_ = [
        ("camera", tpt_camera_desc),
        ("spheres", C.POINTER(tpt_sphere)),
        ("n_spheres", C.c_int64),
        ("meshes", C.POINTER(tpt_mesh_desc)),
        ("n_meshes", C.c_int64),
        ("instances", C.POINTER(tpt_instance_desc)),
        ("n_instances", C.c_int64),
        ("materials", C.POINTER(tpt_material)),
        ("n_materials", C.c_int64),
        ("env", tpt_env_desc),
    ]


class tpt_render_config(C.Structure):
    _fields_ = [
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("spp", C.c_int32),
        ("max_bounces", C.c_int32),
        ("rr_start", C.c_int32),
        ("tile", C.c_int32),
        ("adaptive_enabled", C.c_int32),
        ("adaptive_min_spp", C.c_int32),
        ("adaptive_threshold", C.c_double),
        ("morton_enabled", C.c_int32),
        ("mode", C.c_int32),
        ("seed", C.c_uint64),
        ("row_begin", C.c_int32),
        ("row_step", C.c_int32),
    ]


class tpt_stats(C.Structure):
    _fields_ = [
        ("render_ms", C.c_double),
        ("paths", C.c_uint64),
        ("rays_closest", C.c_uint64),
        ("rays_shadow", C.c_uint64),
        ("iterations", C.c_uint64),
        ("device_flags", C.c_int32),
        ("profile", C.c_int32),
        ("stage_ms", C.c_double * 4),
        ("stage_launches", C.c_uint64 * 4),
        ("nodes_visited", C.c_uint64 * 2),
        ("tris_tested", C.c_uint64 * 2),
        ("spheres_tested", C.c_uint64 * 2),
        ("instances_tested", C.c_uint64 * 2),
        ("adjoint_linear", C.c_double),
        ("node_steps", C.c_uint64 * 2),
        ("camera_fast", C.c_uint64),
        ("leaf_visits", C.c_uint64 * 2),
        ("leaf_steps", C.c_uint64 * 2),
        ("fast_steps", C.c_uint64),
        ("task_spp", C.c_int32),
        ("pool_slots", C.c_int32),
        ("sky_samples", C.c_uint64),
        ("kernel_launches", C.c_uint64),
    ]


class tpt_batch_job(C.Structure):
    _fields_ = [
        ("scene", C.c_int32),
        ("reserved", C.c_int32),
        ("config", tpt_render_config),
        ("d_acc", C.c_void_p),
        ("d_acc_w", C.c_void_p),
    ]


class tpt_tuning(C.Structure):
    _fields_ = [("pool_slots", C.c_int32), ("task_spp", C.c_int32), ("trace_chunk", C.c_int32),
                ("shade_ctas", C.c_int32)]


# Every exported symbol with its signature (restype, argtypes).
SIGNATURES = {
    "tpt_scene_create": (C.c_int, [C.POINTER(tpt_scene_desc), C.POINTER(C.c_void_p)]),
    "tpt_scene_destroy": (None, [C.c_void_p]),
    "tpt_render": (
        C.c_int,
        [C.c_void_p, C.POINTER(tpt_render_config), C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(tpt_stats)],
    ),
    "tpt_render_device": (
        C.c_int,
        [
            C.c_void_p,
            C.POINTER(tpt_render_config),
            C.c_void_p,
            C.c_void_p,
            C.c_void_p,
            C.POINTER(tpt_stats),
        ],
    ),
    "tpt_render_device_noalloc": (
        C.c_int,
        [C.c_void_p, C.POINTER(tpt_render_config), C.c_void_p, C.c_void_p, C.POINTER(tpt_stats)],
    ),
    "tpt_scene_material_count": (C.c_int64, [C.c_void_p]),
    "tpt_scene_load_xml": (C.c_int, [C.c_char_p, C.POINTER(tpt_render_config), C.POINTER(C.c_void_p)]),
    "tpt_scene_default": (C.c_int, [C.POINTER(tpt_render_config), C.c_char_p, C.POINTER(C.c_void_p)]),
    "tpt_loaded_desc": (C.POINTER(tpt_scene_desc), [C.c_void_p]),
    "tpt_loaded_warning_count": (C.c_int64, [C.c_void_p]),
    "tpt_loaded_warning": (C.c_char_p, [C.c_void_p, C.c_int64]),
    "tpt_loaded_destroy": (None, [C.c_void_p]),
    "tpt_write_image": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, C.POINTER(C.c_double), C.c_double, C.c_int32]),
    "tpt_checkpoint_save": (
        C.c_int,
        [C.c_char_p, C.c_uint64, C.c_int32, C.c_int32, C.c_uint64, C.POINTER(C.c_double), C.POINTER(C.c_double)],
    ),
    "tpt_checkpoint_load": (
        C.c_int,
        [C.c_char_p, C.c_uint64, C.c_int32, C.c_int32, C.POINTER(C.c_uint64), C.POINTER(C.c_double),
         C.POINTER(C.c_double)],
    ),
    "tpt_film_tiles": (C.c_int64, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "tpt_render_resume": (
        C.c_int,
        [C.c_void_p, C.POINTER(tpt_render_config), C.c_char_p, C.c_uint64, C.POINTER(C.c_double),
         C.POINTER(C.c_double), C.POINTER(tpt_stats)],
    ),
    "tpt_read_hdr": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "tpt_batch_create": (C.c_int, [C.POINTER(tpt_scene_desc), C.c_int64, C.POINTER(C.c_void_p)]),
    "tpt_batch_destroy": (None, [C.c_void_p]),
    "tpt_batch_render_device": (
        C.c_int,
        [C.c_void_p, C.POINTER(tpt_batch_job), C.c_int64, C.POINTER(tpt_tuning), C.POINTER(tpt_stats)],
    ),
    "tpt_batch_autotune": (
        C.c_int,
        [C.c_void_p, C.POINTER(tpt_batch_job), C.c_int64, C.POINTER(tpt_tuning), C.POINTER(C.c_double), C.c_int32],
    ),
    "tpt_scene_set_materials": (
        C.c_int,
        [C.c_void_p, C.POINTER(tpt_material), C.POINTER(tpt_material), C.c_int64],
    ),
    "tpt_render_forward_device": (C.c_int, [C.c_void_p, C.POINTER(tpt_render_config), C.c_void_p, C.POINTER(tpt_stats)]),
    "tpt_render_forward": (
        C.c_int,
        [C.c_void_p, C.POINTER(tpt_render_config), C.POINTER(C.c_float), C.POINTER(tpt_stats)],
    ),
    "tpt_render_backward_device": (
        C.c_int,
        [C.c_void_p, C.POINTER(tpt_render_config), C.c_void_p, C.c_void_p, C.POINTER(tpt_stats)],
    ),
    "tpt_render_backward": (
        C.c_int,
        [C.c_void_p, C.POINTER(tpt_render_config), C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(tpt_stats)],
    ),
    "tpt_bvh_build_host": (
        C.c_int64,
        [
            C.POINTER(tpt_mesh_desc),
            C.POINTER(C.c_double),
            C.POINTER(C.c_int32),
            C.POINTER(C.c_uint32),
            C.POINTER(C.c_int64),
        ],
    ),
    "tpt_bvh_build_device": (
        C.c_int64,
        [
            C.POINTER(tpt_mesh_desc),
            C.POINTER(C.c_double),
            C.POINTER(C.c_int32),
            C.POINTER(C.c_uint32),
            C.POINTER(C.c_int64),
        ],
    ),
    "tpt_bvh_build_fp32": (
        C.c_int64,
        [
            C.POINTER(tpt_mesh_desc),
            C.POINTER(C.c_double),
            C.POINTER(C.c_int32),
            C.POINTER(C.c_uint32),
            C.POINTER(C.c_int64),
        ],
    ),
    "tpt_last_error": (C.c_char_p, []),
    "tpt_version": (C.c_char_p, []),
    "tpt_probe_read_bandwidth": (C.c_int, [C.c_int64, C.c_int, C.POINTER(C.c_double)]),
}

_lib = None


class TinyptError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"tinypt error {code}: {message}")
        self.code = code


def lib() -> C.CDLL:
    """Loads libtinypt_cuda.so from the package directory (raises if absent)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m tinypt_b200.build` (nvcc, sm_100a). "
                "There is no CPU fallback."
            )
        handle = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(code: int) -> None:
    if code != TPT_OK:
        msg = lib().tpt_last_error().decode(errors="replace")
        raise TinyptError(code, msg)
