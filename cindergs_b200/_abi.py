"""ctypes binding of the C ABI in ``include/cgs.h`` (libcindergs.so).

The library is the only compute path: there is no Python or CPU fallback. A
missing library raises :class:`CgsLibraryMissing`; a failing call raises
:class:`CgsError` carrying the status code and ``cgs_last_error``.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libcindergs.so")

CGS_OK = 0
CGS_E_ARG = -1
CGS_E_OOM = -2
CGS_E_CUDA = -3
CGS_E_TIMEOUT = -4
CGS_E_CAPACITY = -5
CGS_E_STATE = -6
ERROR_NAMES = {
    CGS_E_ARG: "CGS_E_ARG", CGS_E_OOM: "CGS_E_OOM", CGS_E_CUDA: "CGS_E_CUDA",
    CGS_E_TIMEOUT: "CGS_E_TIMEOUT", CGS_E_CAPACITY: "CGS_E_CAPACITY", CGS_E_STATE: "CGS_E_STATE",
}

CGS_SH_F32 = 0
CGS_SH_F16 = 1

BUF_DEFORMED_POS = 1
BUF_DEFORMED_COV = 2
BUF_DEFORMED_OPA = 3
BUF_SPLIT_META = 4
BUF_SPLAT_ATTRS = 5
BUF_EXTENTS = 6
BUF_TILE_OFFSETS = 7
BUF_SORTED_KEYS = 8
BUF_SORTED_IDS = 9
BUF_TILE_RANGES = 10
BUF_TET_JACOBIANS = 11
BUF_TET_ROTATIONS = 12
BUF_TET_STRETCH = 13
BUF_MVC_ROTATIONS = 14

# Every function include/cgs.h declares, with (restype, argtypes).
_vp = ctypes.c_void_p
_u32 = ctypes.c_uint32
_u64 = ctypes.c_uint64
_i32 = ctypes.c_int32
_int = ctypes.c_int


class CgsCamera(ctypes.Structure):
    """cgs_camera: the 96-byte CameraUniforms block (render/camera.rs:9-36)."""
    _fields_ = [("view", ctypes.c_float * 16), ("focal_x", ctypes.c_float),
                ("focal_y", ctypes.c_float), ("principal_x", ctypes.c_float),
                ("principal_y", ctypes.c_float), ("viewport_width", ctypes.c_float),
                ("viewport_height", ctypes.c_float), ("near_plane", ctypes.c_float),
                ("pad", ctypes.c_float)]


class CgsCompositor(ctypes.Structure):
    """cgs_compositor: the 48-byte CompositorUniforms block (rasterizer/mod.rs:16-37)."""
    _fields_ = [("screen_width", _u32), ("screen_height", _u32), ("tiles_x", _u32),
                ("tiles_y", _u32), ("background", ctypes.c_float * 4),
                ("camera_position", ctypes.c_float * 3), ("sh_degree", _u32)]


class CgsFrameParams(ctypes.Structure):
    _fields_ = [("strain_split_threshold", ctypes.c_float), ("mip_filter_3d_var", ctypes.c_float),
                ("min_opacity", ctypes.c_float), ("min_radius_px", ctypes.c_float),
                ("profile_stages", _i32), ("force_stage3", _i32), ("write_f32", _i32),
                ("radix_bits", _i32), ("entry_sort", _i32), ("tile_shape", _i32)]


class CgsStageTimings(ctypes.Structure):
    _fields_ = [("stage1_deform_ms", ctypes.c_double), ("stage2_project_ms", ctypes.c_double),
                ("stage3_bin_sort_ms", ctypes.c_double), ("stage4_composite_ms", ctypes.c_double),
                ("stage1_skipped", _i32), ("stage3_cached", _i32),
                ("used_hardware_timestamps", _i32), ("used_64bit_keys", _i32),
                ("active_gaussians", _u64), ("surviving_gaussians", _u64),
                ("total_tile_entries", _u64)]


SORT_AUTO, SORT_RADIX, SORT_TRANSPOSE = 0, 1, 2
TILE_16X16, TILE_8X8, TILE_32X16 = 0, 1, 2
TILE_SHAPES = {TILE_16X16: (16, 16), TILE_8X8: (8, 8), TILE_32X16: (32, 16)}
FIELD_PER_FRAME = 1

KERNEL_NAMES = ["clear", "tet_transforms", "deform", "project", "bin", "entry_sort",
                "tile_ranges", "composite", "splat_sort", "mvc", "field"]
KERNEL_COUNT = len(KERNEL_NAMES)


class CgsViewsStats(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_double), ("total_tile_entries", _u64), ("graph_replayed", _u32),
                ("graph_captured", _u32), ("views_rerendered", _u32), ("pad", _u32)]


class CgsKernelProfile(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_double * KERNEL_COUNT), ("alg_bytes", _u64 * KERNEL_COUNT),
                ("launches", _u32 * KERNEL_COUNT), ("alg_flops", _u64 * KERNEL_COUNT)]


class CgsSpringCage(ctypes.Structure):
    """cgs_spring_cage: one spring-driven cage's vertex range, parameters and planes."""
    _fields_ = [("stiffness", ctypes.c_float), ("damping", ctypes.c_float),
                ("mass", ctypes.c_float), ("first_vertex", _u32), ("num_vertices", _u32),
                ("first_plane", _u32), ("num_planes", _u32), ("pad", _u32)]


class CgsCollisionPlane(ctypes.Structure):
    """cgs_collision_plane (CollisionPlane, dynamics.rs:4-14)."""
    _fields_ = [("normal", ctypes.c_float * 3), ("offset", ctypes.c_float),
                ("restitution", ctypes.c_float), ("friction", ctypes.c_float),
                ("pad", ctypes.c_float * 2)]


class CgsLaunchShape(ctypes.Structure):
    """cgs_launch_shape: block sizes of the frame's kernels (0 = default)."""
    _fields_ = [("project_threads", _u32), ("bin_blocks_per_sm", _u32),
                ("ranges_blocks", _u32), ("pad", _u32)]


assert ctypes.sizeof(CgsSpringCage) == 32 and ctypes.sizeof(CgsCollisionPlane) == 32
assert ctypes.sizeof(CgsCamera) == 96
assert ctypes.sizeof(CgsCompositor) == 48

SIGNATURES = {
    "cgs_ctx_create": (_int, [_int, _vp, ctypes.POINTER(_vp)]),
    "cgs_ctx_destroy": (_int, [_vp]),
    "cgs_last_error": (ctypes.c_char_p, [_vp]),
    "cgs_ctx_synchronize": (_int, [_vp]),
    "cgs_ctx_device_bytes": (_int, [_vp, ctypes.POINTER(_u64)]),
    "cgs_version": (ctypes.c_char_p, []),
    "cgs_ctx_set_device_budget": (_int, [_vp, _u64]),
    "cgs_ctx_set_launch_shape": (_int, [_vp, ctypes.POINTER(CgsLaunchShape)]),
    "cgs_ctx_wait_drill": (_int, [_vp, _u32, ctypes.POINTER(_u32)]),
    "cgs_scene_upload": (_int, [_vp, _u64, _vp, _vp, _vp, _vp, _i32]),
    "cgs_tet_cages_upload": (_int, [_vp, _u32, _vp, _vp, _u32, _vp, _vp]),
    "cgs_cage_vertices_update": (_int, [_vp, _vp, _u32]),
    "cgs_bind_tets": (_int, [_vp, _u32, _vp, _vp, _u32, _vp, _i32, _vp, _vp, _vp, _vp]),
    "cgs_execute_frame": (_int, [_vp, ctypes.POINTER(CgsCamera), ctypes.POINTER(CgsCompositor),
                                 ctypes.POINTER(CgsFrameParams),
                                 ctypes.POINTER(CgsStageTimings)]),
    "cgs_readback_rgba8": (_int, [_vp, _vp, _u32, _u32]),
    "cgs_readback_rgba_f32": (_int, [_vp, _vp, _u32, _u32]),
    "cgs_readback_rgba8_async": (_i32, [_vp, _vp, _u32, _u32, ctypes.POINTER(_u64)]),
    "cgs_readback_wait": (_i32, [_vp, _u64]),
    "cgs_framebuffer_device": (_int, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_u32)]),
    "cgs_invalidate_stage3": (_int, [_vp]),
    "cgs_invalidate": (_int, [_vp]),
    "cgs_read_frame_buffer": (_int, [_vp, _i32, _vp, _u64, ctypes.POINTER(_u64)]),
    "cgs_kernel_profile_read": (_int, [_vp, ctypes.POINTER(CgsKernelProfile)]),
    "cgs_kernel_profile_reset": (_int, [_vp]),
    "cgs_kernel_name": (ctypes.c_char_p, [_i32]),
    "cgs_mvc_cage_upload": (_i32, [_vp, _u32, _vp, _u32, _vp]),
    "cgs_mvc_vertices_update": (_i32, [_vp, _vp, _u32]),
    "cgs_mvc_bind": (_i32, [_vp, ctypes.POINTER(_u32)]),
    "cgs_mvc_weights": (_i32, [_vp, _u64, _vp, _vp]),
    "cgs_mvc_read_bindings": (_i32, [_vp, _u64, _vp, _vp, ctypes.POINTER(_u64)]),
    "cgs_scene_upload_quantized": (_i32, [_vp, _u64, _vp, _vp, _vp, _vp, _u32]),
    "cgs_execute_views": (_i32, [_vp, _u32, _vp, _vp, _vp, _vp, _i32,
                                 ctypes.POINTER(CgsViewsStats)]),
    "cgs_mvc_field_create": (_i32, [_vp, _u64]),
    "cgs_mvc_field_layout": (_i32, [_vp, _vp, _vp, _vp]),
    "cgs_mvc_field_params": (_i32, [_vp, _vp, _vp]),
    "cgs_mvc_field_train": (_i32, [_vp, _u64, _vp, _vp, _u32, _u32, ctypes.c_float, ctypes.c_float,
                                   _u64, _vp]),
    "cgs_mvc_field_grads": (_i32, [_vp, _u64, _vp, _vp, ctypes.c_float, _vp, _vp]),
    "cgs_mvc_field_eval": (_i32, [_vp, _u64, _vp, _vp]),
    "cgs_mvc_field_infer": (_i32, [_vp, _u64, _vp, _i32, _vp]),
    "cgs_mvc_bind_learned": (_i32, [_vp, ctypes.c_float, _u32, ctypes.POINTER(_u32),
                                    ctypes.POINTER(_u32)]),
    "cgs_sh_rotate": (_i32, [_vp, _u64, _vp, _u32, _vp, _vp, _u32]),
    "cgs_springs_upload": (_i32, [_vp, _u32, _vp, _u32, _vp, _u32, _vp, _vp, _vp, _vp]),
    "cgs_springs_step": (_i32, [_vp, ctypes.c_float, _u32]),
    "cgs_springs_impulse": (_i32, [_vp, ctypes.c_float]),
    "cgs_springs_read": (_i32, [_vp, _vp, _vp]),
    "cgs_export_deformed": (_i32, [_vp, _u32, _u64, _vp, _vp, _vp, _vp, ctypes.POINTER(_u64)]),
    "cgs_scan_u32": (_int, [_vp, _vp, _vp, _u64, ctypes.POINTER(_u64)]),
    "cgs_sort_pairs_u32": (_int, [_vp, _vp, _vp, _u64, _u32, _i32]),
    "cgs_sort_pairs_u64": (_int, [_vp, _vp, _vp, _vp, _u64, _u32, _i32]),
    "cgs_sort_pairs_u32_noalloc": (_int, [_vp, _vp, _u64, _u32, _i32, _vp]),
}


class CgsLibraryMissing(RuntimeError):
    pass


class CgsError(RuntimeError):
    def __init__(self, code: int, func: str, message: str):
        self.code = code
        name = ERROR_NAMES.get(code, str(code))
        super().__init__(f"{func} failed with {name}: {message}")


_lib = None


def load(path: str | None = None):
    """Loads libcindergs.so (building it first is the caller's job)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("CINDERGS_LIB", LIB_PATH)
    if not os.path.exists(p):
        raise CgsLibraryMissing(
            f"{p} not found: build it with `python -m cindergs_b200.build` "
            "(the CUDA library is required; there is no CPU fallback)")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(code: int, func: str, ctx=None) -> None:
    if code != CGS_OK:
        msg = load().cgs_last_error(ctx).decode() if ctx else "(no context)"
        raise CgsError(code, func, msg)
