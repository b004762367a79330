//! Raw declarations of the C ABI in `include/cgs.h` (libcindergs, sm_100a),
//! one `extern "C"` item per exported function, and the `#[repr(C)]` structs
//! those functions take. The safe layer that replaces the CubeCL backend's
//! `GpuPipelineState` (render/gpu_state.rs:538-626) is `pipeline`.
//!
//! Every function returns `CGS_OK` (0) or a negative `CGS_E_*` status;
//! `cgs_last_error(ctx)` holds the message. "d_" pointers are device memory
//! of the context's GPU, all other pointers host memory borrowed for the call.
#![allow(non_camel_case_types)]

use std::os::raw::{c_char, c_int, c_void};

pub mod pipeline;

pub const CGS_OK: c_int = 0;
pub const CGS_E_ARG: c_int = -1;
pub const CGS_E_OOM: c_int = -2;
pub const CGS_E_CUDA: c_int = -3;
pub const CGS_E_TIMEOUT: c_int = -4;
pub const CGS_E_CAPACITY: c_int = -5;
pub const CGS_E_STATE: c_int = -6;

pub const CGS_SH_F32: i32 = 0;
pub const CGS_SH_F16: i32 = 1;

pub const CGS_TILE_16X16: i32 = 0;
pub const CGS_TILE_8X8: i32 = 1;
pub const CGS_TILE_32X16: i32 = 2;

pub const CGS_SORT_AUTO: i32 = 0;
pub const CGS_SORT_RADIX: i32 = 1;
pub const CGS_SORT_TRANSPOSE: i32 = 2;

pub const CGS_FIELD_PER_FRAME: u32 = 1;

pub const CGS_K_CLEAR: i32 = 0;
pub const CGS_K_TET_TRANSFORMS: i32 = 1;
pub const CGS_K_DEFORM: i32 = 2;
pub const CGS_K_PROJECT: i32 = 3;
pub const CGS_K_BIN: i32 = 4;
pub const CGS_K_ENTRY_SORT: i32 = 5;
pub const CGS_K_TILE_RANGES: i32 = 6;
pub const CGS_K_COMPOSITE: i32 = 7;
pub const CGS_K_SPLAT_SORT: i32 = 8;
pub const CGS_K_MVC: i32 = 9;
pub const CGS_K_FIELD: i32 = 10;
pub const CGS_KERNEL_COUNT: usize = 11;

pub const CGS_BUF_DEFORMED_POS: i32 = 1;
pub const CGS_BUF_DEFORMED_COV: i32 = 2;
pub const CGS_BUF_DEFORMED_OPA: i32 = 3;
pub const CGS_BUF_SPLIT_META: i32 = 4;
pub const CGS_BUF_SPLAT_ATTRS: i32 = 5;
pub const CGS_BUF_EXTENTS: i32 = 6;
pub const CGS_BUF_TILE_OFFSETS: i32 = 7;
pub const CGS_BUF_SORTED_KEYS: i32 = 8;
pub const CGS_BUF_SORTED_IDS: i32 = 9;
pub const CGS_BUF_TILE_RANGES: i32 = 10;
pub const CGS_BUF_TET_JACOBIANS: i32 = 11;
pub const CGS_BUF_TET_ROTATIONS: i32 = 12;
pub const CGS_BUF_TET_STRETCH: i32 = 13;
pub const CGS_BUF_MVC_ROTATIONS: i32 = 14;

pub const CGS_NOALLOC_SORT_MAX_PAIRS: u64 = 1048576;

/// Opaque context: one device, one stream, all device memory.
#[repr(C)]
pub struct cgs_ctx {
    _opaque: [u8; 0],
}

/// CameraUniforms (render/camera.rs:9-36), 96 bytes.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct cgs_camera {
    pub view: [f32; 16],
    pub focal_x: f32,
    pub focal_y: f32,
    pub principal_x: f32,
    pub principal_y: f32,
    pub viewport_width: f32,
    pub viewport_height: f32,
    pub near_plane: f32,
    pub pad: f32,
}

/// CompositorUniforms (render/rasterizer/mod.rs:16-37), 48 bytes.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct cgs_compositor {
    pub screen_width: u32,
    pub screen_height: u32,
    pub tiles_x: u32,
    pub tiles_y: u32,
    pub background: [f32; 4],
    pub camera_position: [f32; 3],
    pub sh_degree: u32,
}

/// The scalar arguments of execute_frame_gpu (render/gpu_state.rs:613-626)
/// and the library's output options.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct cgs_frame_params {
    pub strain_split_threshold: f32,
    pub mip_filter_3d_var: f32,
    pub min_opacity: f32,
    pub min_radius_px: f32,
    pub profile_stages: i32,
    pub force_stage3: i32,
    pub write_f32: i32,
    pub radix_bits: i32,
    pub entry_sort: i32,
    pub tile_shape: i32,
}

/// GpuStageTimings (render/gpu_state.rs:513-534).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct cgs_stage_timings {
    pub stage1_deform_ms: f64,
    pub stage2_project_ms: f64,
    pub stage3_bin_sort_ms: f64,
    pub stage4_composite_ms: f64,
    pub stage1_skipped: i32,
    pub stage3_cached: i32,
    pub used_hardware_timestamps: i32,
    pub used_64bit_keys: i32,
    pub active_gaussians: u64,
    pub surviving_gaussians: u64,
    pub total_tile_entries: u64,
}

/// One spring-driven cage (deformation/dynamics.rs:75-131).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct cgs_spring_cage {
    pub stiffness: f32,
    pub damping: f32,
    pub mass: f32,
    pub first_vertex: u32,
    pub num_vertices: u32,
    pub first_plane: u32,
    pub num_planes: u32,
    pub pad: u32,
}

/// CollisionPlane (deformation/dynamics.rs:4-33).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct cgs_collision_plane {
    pub normal: [f32; 3],
    pub offset: f32,
    pub restitution: f32,
    pub friction: f32,
    pub pad: [f32; 2],
}

/// Launch shapes of the frame's kernels (cgs_ctx_set_launch_shape).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct cgs_launch_shape {
    pub project_threads: u32,
    pub bin_blocks_per_sm: u32,
    pub ranges_blocks: u32,
    pub pad: u32,
}

/// Statistics of one cgs_execute_views step.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct cgs_views_stats {
    pub ms: f64,
    pub total_tile_entries: u64,
    pub graph_replayed: u32,
    pub graph_captured: u32,
    pub views_rerendered: u32,
    pub pad: u32,
}

/// Per-kernel device time, launches, algorithmic bytes and tensor flops.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct cgs_kernel_profile {
    pub ms: [f64; CGS_KERNEL_COUNT],
    pub alg_bytes: [u64; CGS_KERNEL_COUNT],
    pub launches: [u32; CGS_KERNEL_COUNT],
    pub alg_flops: [u64; CGS_KERNEL_COUNT],
}

#[link(name = "cindergs")]
extern "C" {
    // ---- context (GpuCompute::acquire, render/gpu.rs:70-113)
    pub fn cgs_ctx_create(device: c_int, stream: *mut c_void, out_ctx: *mut *mut cgs_ctx) -> c_int;
    pub fn cgs_ctx_destroy(ctx: *mut cgs_ctx) -> c_int;
    pub fn cgs_last_error(ctx: *const cgs_ctx) -> *const c_char;
    pub fn cgs_ctx_synchronize(ctx: *mut cgs_ctx) -> c_int;
    pub fn cgs_ctx_device_bytes(ctx: *const cgs_ctx, out_bytes: *mut u64) -> c_int;
    pub fn cgs_version() -> *const c_char;
    pub fn cgs_ctx_set_launch_shape(ctx: *mut cgs_ctx, shape: *const cgs_launch_shape) -> c_int;
    pub fn cgs_ctx_set_device_budget(ctx: *mut cgs_ctx, bytes: u64) -> c_int;
    pub fn cgs_ctx_wait_drill(ctx: *mut cgs_ctx, polls: u32, out_gave_up: *mut u32) -> c_int;

    // ---- scene residency (GpuSceneState, render/gpu_state.rs:95-343)
    pub fn cgs_scene_upload(ctx: *mut cgs_ctx, n: u64, pos: *const f32, cov: *const f32,
                            opa: *const f32, sh: *const c_void, sh_format: i32) -> c_int;
    pub fn cgs_scene_upload_quantized(ctx: *mut cgs_ctx, n: u64, pos: *const f32,
                                      cov_f16x2: *const u32, opa: *const f32,
                                      sh_f16x2: *const u32, sh_degree: u32) -> c_int;
    pub fn cgs_tet_cages_upload(ctx: *mut cgs_ctx, num_tets: u32, elems: *const u32,
                                inv_dm: *const f32, num_verts: u32, bind_tet: *const u32,
                                bind_w: *const f32) -> c_int;
    pub fn cgs_cage_vertices_update(ctx: *mut cgs_ctx, verts: *const f32, num_verts: u32) -> c_int;

    // ---- cage springs on the device (deformation/dynamics.rs)
    pub fn cgs_springs_upload(ctx: *mut cgs_ctx, num_cages: u32, cages: *const cgs_spring_cage,
                              num_planes: u32, planes: *const cgs_collision_plane,
                              num_verts: u32, rest: *const f32, current: *const f32,
                              velocity: *const f32, pinned: *const u8) -> c_int;
    pub fn cgs_springs_step(ctx: *mut cgs_ctx, dt: f32, steps: u32) -> c_int;
    pub fn cgs_springs_impulse(ctx: *mut cgs_ctx, magnitude: f32) -> c_int;
    pub fn cgs_springs_read(ctx: *mut cgs_ctx, current: *mut f32, velocity: *mut f32) -> c_int;

    // ---- tet binding (TetMesh::bind_point, deformation/mod.rs:263-310)
    pub fn cgs_bind_tets(ctx: *mut cgs_ctx, num_tets: u32, elems: *const u32, inv_dm: *const f32,
                         num_verts: u32, rest_verts: *const f32, use_bounds: i32,
                         bmin: *const f32, bmax: *const f32, bind_tet: *mut u32,
                         bind_w: *mut f32) -> c_int;

    // ---- polygon cage, mean value coordinates (deformation/mvc.rs)
    pub fn cgs_mvc_cage_upload(ctx: *mut cgs_ctx, num_verts: u32, rest_verts: *const f32,
                               num_tris: u32, tris: *const u32) -> c_int;
    pub fn cgs_mvc_vertices_update(ctx: *mut cgs_ctx, verts: *const f32, num_verts: u32) -> c_int;
    pub fn cgs_mvc_bind(ctx: *mut cgs_ctx, out_bound: *mut u32) -> c_int;
    pub fn cgs_mvc_weights(ctx: *mut cgs_ctx, n: u64, d_points: *const f32,
                           d_weights: *mut f32) -> c_int;
    pub fn cgs_mvc_read_bindings(ctx: *mut cgs_ctx, max_slots: u64, gaussian: *mut u32,
                                 wg: *mut f32, out_slots: *mut u64) -> c_int;

    // ---- learned MVC weight field (no counterpart in the crate)
    pub fn cgs_mvc_field_create(ctx: *mut cgs_ctx, seed: u64) -> c_int;
    pub fn cgs_mvc_field_layout(ctx: *mut cgs_ctx, offsets: *mut u32, total: *mut u32,
                                enc: *mut f32) -> c_int;
    pub fn cgs_mvc_field_params(ctx: *mut cgs_ctx, dst: *mut f32, src: *const f32) -> c_int;
    pub fn cgs_mvc_field_train(ctx: *mut cgs_ctx, n: u64, d_points: *const f32,
                               d_weights: *const f32, steps: u32, batch: u32, lr: f32,
                               lambda: f32, seed: u64, out_loss: *mut f32) -> c_int;
    pub fn cgs_mvc_field_grads(ctx: *mut cgs_ctx, n: u64, d_points: *const f32,
                               d_weights: *const f32, lambda: f32, grads: *mut f32,
                               out_loss: *mut f32) -> c_int;
    pub fn cgs_mvc_field_eval(ctx: *mut cgs_ctx, n: u64, d_points: *const f32,
                              d_weights: *mut f32) -> c_int;
    pub fn cgs_mvc_field_infer(ctx: *mut cgs_ctx, n: u64, d_points: *const f32, use_rest: i32,
                               d_out: *mut f32) -> c_int;
    pub fn cgs_mvc_bind_learned(ctx: *mut cgs_ctx, threshold: f32, flags: u32,
                                out_bound: *mut u32, out_fallback: *mut u32) -> c_int;

    // ---- frame (GpuPipelineState, render/gpu_state.rs:538-1243)
    pub fn cgs_execute_frame(ctx: *mut cgs_ctx, camera: *const cgs_camera,
                             comp: *const cgs_compositor, params: *const cgs_frame_params,
                             timings: *mut cgs_stage_timings) -> c_int;
    pub fn cgs_execute_views(ctx: *mut cgs_ctx, num_views: u32, cameras: *const cgs_camera,
                             comps: *const cgs_compositor, params: *const cgs_frame_params,
                             d_rgba8: *const *mut u32, use_graph: i32,
                             stats: *mut cgs_views_stats) -> c_int;
    pub fn cgs_readback_rgba8(ctx: *mut cgs_ctx, dst: *mut u8, width: u32, height: u32) -> c_int;
    pub fn cgs_readback_rgba8_async(ctx: *mut cgs_ctx, dst: *mut u8, width: u32, height: u32,
                                    ticket: *mut u64) -> c_int;
    pub fn cgs_readback_wait(ctx: *mut cgs_ctx, ticket: u64) -> c_int;
    pub fn cgs_readback_rgba_f32(ctx: *mut cgs_ctx, dst: *mut f32, width: u32, height: u32) -> c_int;
    pub fn cgs_framebuffer_device(ctx: *mut cgs_ctx, d_rgba8: *mut *mut c_void,
                                  row_pitch_px: *mut u32) -> c_int;
    pub fn cgs_kernel_profile_read(ctx: *mut cgs_ctx, out: *mut cgs_kernel_profile) -> c_int;
    pub fn cgs_kernel_profile_reset(ctx: *mut cgs_ctx) -> c_int;
    pub fn cgs_kernel_name(id: i32) -> *const c_char;
    pub fn cgs_invalidate_stage3(ctx: *mut cgs_ctx) -> c_int;
    pub fn cgs_invalidate(ctx: *mut cgs_ctx) -> c_int;
    pub fn cgs_read_frame_buffer(ctx: *mut cgs_ctx, which: i32, dst: *mut c_void, dst_bytes: u64,
                                 out_bytes: *mut u64) -> c_int;

    // ---- SH coefficient rotation and deformed-scene export
    pub fn cgs_sh_rotate(ctx: *mut cgs_ctx, n: u64, d_sh: *mut f32, num_rotations: u32,
                         d_rotations: *const f32, d_index: *const u32, degree: u32) -> c_int;
    pub fn cgs_export_deformed(ctx: *mut cgs_ctx, sh_degree: u32, capacity: u64, pos: *mut f32,
                               cov: *mut f32, opa: *mut f32, sh: *mut f32,
                               out_count: *mut u64) -> c_int;

    // ---- stage primitives on device memory (render/kernels/scan.rs, radix_sort.rs)
    pub fn cgs_scan_u32(ctx: *mut cgs_ctx, d_in: *const u32, d_out: *mut u32, n: u64,
                        total: *mut u64) -> c_int;
    pub fn cgs_sort_pairs_u32(ctx: *mut cgs_ctx, d_keys: *mut u32, d_vals: *mut u32, n: u64,
                              key_bits: u32, digit_bits: i32) -> c_int;
    pub fn cgs_sort_pairs_u64(ctx: *mut cgs_ctx, d_tiles: *mut u32, d_depths: *mut u32,
                              d_ids: *mut u32, n: u64, tile_bits: u32, digit_bits: i32) -> c_int;

    // ---- allocation-free pair sort (no counterpart in the reference)
    pub fn cgs_sort_pairs_u32_noalloc(d_keys: *mut u32, d_vals: *mut u32, n: u64, key_bits: u32,
                                      digit_bits: i32, stream: *mut c_void) -> c_int;
}

#[cfg(test)]
mod layout {
    use super::*;
    use std::mem::size_of;

    #[test]
    fn struct_sizes_match_the_header() {
        assert_eq!(size_of::<cgs_camera>(), 96);
        assert_eq!(size_of::<cgs_compositor>(), 48);
        assert_eq!(size_of::<cgs_frame_params>(), 40);
        assert_eq!(size_of::<cgs_stage_timings>(), 72);
        assert_eq!(size_of::<cgs_spring_cage>(), 32);
        assert_eq!(size_of::<cgs_collision_plane>(), 32);
        assert_eq!(size_of::<cgs_views_stats>(), 32);
    }
}
