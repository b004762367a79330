//! Safe layer over the raw declarations: the shape of the CubeCL backend's
//! `GpuCompute` (render/gpu.rs:14-113) and `GpuPipelineState`
//! (render/gpu_state.rs:538-626, :1296-1343), so the crate's orchestrator
//! (render/pipeline.rs:646-739) keeps its calls and swaps only the type.
//!
//! The scene and cages are borrowed as flat slices in the crate's own
//! layouts (`GaussianSceneSoa`'s arrays, `CageScene`'s flattened topology and
//! bindings); uploads happen only when their fingerprint changes, as in
//! `GpuSceneState::sync_scene_and_cages` (gpu_state.rs:182-343). There is no
//! CPU fallback: failures come back as `GpuError`.
use std::ffi::CStr;
use std::ptr;

use crate::*;

/// The reference's error surface (render/gpu.rs:14-30) plus the library's
/// specific statuses.
#[derive(Debug, Clone, PartialEq)]
pub enum GpuError {
    NoAdapter(String),
    InvalidArgument(String),
    OutOfMemory(String),
    Execution(String),
    Timeout(String),
    Capacity(String),
    State(String),
}

fn status(ctx: *const cgs_ctx, code: c_int) -> Result<(), GpuError> {
    if code == CGS_OK {
        return Ok(());
    }
    let msg = unsafe {
        let p = cgs_last_error(ctx);
        if p.is_null() { String::new() } else { CStr::from_ptr(p).to_string_lossy().into_owned() }
    };
    Err(match code {
        CGS_E_ARG => GpuError::InvalidArgument(msg),
        CGS_E_OOM => GpuError::OutOfMemory(msg),
        CGS_E_TIMEOUT => GpuError::Timeout(msg),
        CGS_E_CAPACITY => GpuError::Capacity(msg),
        CGS_E_STATE => GpuError::State(msg),
        _ => GpuError::Execution(msg),
    })
}

/// One device context (GpuCompute::acquire, render/gpu.rs:70-113).
pub struct GpuCompute {
    ctx: *mut cgs_ctx,
}

impl GpuCompute {
    /// Context on CUDA device `device` with a library-owned stream.
    pub fn acquire(device: i32) -> Result<Self, GpuError> {
        let mut ctx = ptr::null_mut();
        let code = unsafe { cgs_ctx_create(device, ptr::null_mut(), &mut ctx) };
        if code != CGS_OK || ctx.is_null() {
            return Err(GpuError::NoAdapter(format!("cgs_ctx_create({device}) failed: {code}")));
        }
        Ok(Self { ctx })
    }

    pub fn raw(&self) -> *mut cgs_ctx {
        self.ctx
    }

    pub fn synchronize(&self) -> Result<(), GpuError> {
        status(self.ctx, unsafe { cgs_ctx_synchronize(self.ctx) })
    }
}

impl Drop for GpuCompute {
    fn drop(&mut self) {
        unsafe {
            cgs_ctx_destroy(self.ctx);
        }
    }
}

/// GaussianSceneSoa's arrays (scene/soa.rs:30-52): positions [n*3],
/// covariances_3d [n*6], opacities [n], sh_coeffs [n*48].
pub struct SceneRef<'a> {
    pub positions: &'a [f32],
    pub covariances_3d: &'a [f32],
    pub opacities: &'a [f32],
    pub sh_coeffs: &'a [f32],
}

/// CageScene flattened as GpuSceneState uploads it (gpu_state.rs:248-335):
/// elements [T*4] (global vertex ids), inv_dm [T*9], current vertices
/// [V*3], binding tet [n] (u32::MAX = unbound) and weights [n*4].
pub struct TetCagesRef<'a> {
    pub elements: &'a [u32],
    pub inv_dm: &'a [f32],
    pub vertices: &'a [f32],
    pub bind_tet: &'a [u32],
    pub bind_w: &'a [f32],
}

/// GpuStageTimings (render/gpu_state.rs:513-534).
#[derive(Clone, Copy, Debug, Default)]
pub struct GpuStageTimings {
    pub stage1_deform_ms: f64,
    pub stage2_project_ms: f64,
    pub stage3_bin_sort_ms: f64,
    pub stage4_composite_ms: f64,
    pub stage1_skipped: bool,
    pub stage3_cached: bool,
    pub used_hardware_timestamps: bool,
    pub used_64bit_keys: bool,
    pub active_gaussians: usize,
    pub surviving_gaussians: usize,
    pub total_tile_entries: usize,
}

/// FNV-1a over the array addresses, lengths and 64 samples of each array
/// (scene_fingerprint, gpu_state.rs:65-79, with another hash).
fn fingerprint(arrays: &[&[u8]]) -> u64 {
    let mut h: u64 = 0xcbf2_9ce4_8422_2325;
    let mut eat = |b: u8| {
        h ^= b as u64;
        h = h.wrapping_mul(0x0000_0100_0000_01b3);
    };
    for a in arrays {
        for b in (a.as_ptr() as usize).to_le_bytes() {
            eat(b);
        }
        for b in a.len().to_le_bytes() {
            eat(b);
        }
        let step = (a.len() / 64).max(1);
        let mut i = 0;
        while i < a.len() {
            eat(a[i]);
            i += step;
        }
    }
    h
}

fn bytes<T>(s: &[T]) -> &[u8] {
    unsafe { std::slice::from_raw_parts(s.as_ptr() as *const u8, std::mem::size_of_val(s)) }
}

/// Persistent GPU frame state (render/gpu_state.rs:538-626): scene residency
/// and the frame arena live in the library context.
#[derive(Default)]
pub struct GpuPipelineState {
    scene_key: Option<u64>,
    cage_key: Option<u64>,
    last_width: u32,
    last_height: u32,
}

impl GpuPipelineState {
    pub fn new() -> Self {
        Self::default()
    }

    /// invalidate (gpu_state.rs:565-568).
    pub fn invalidate(&mut self, compute: &GpuCompute) -> Result<(), GpuError> {
        self.scene_key = None;
        self.cage_key = None;
        status(compute.ctx, unsafe { cgs_invalidate(compute.ctx) })
    }

    /// invalidate_stage3 (gpu_state.rs:570-573).
    pub fn invalidate_stage3(&mut self, compute: &GpuCompute) -> Result<(), GpuError> {
        status(compute.ctx, unsafe { cgs_invalidate_stage3(compute.ctx) })
    }

    fn sync(&mut self, compute: &GpuCompute, scene: &SceneRef,
            cages: Option<&TetCagesRef>) -> Result<(), GpuError> {
        let n = scene.opacities.len();
        if scene.positions.len() != 3 * n || scene.covariances_3d.len() != 6 * n
            || scene.sh_coeffs.len() != 48 * n
        {
            return Err(GpuError::InvalidArgument("scene arrays disagree on the count".into()));
        }
        let key = fingerprint(&[bytes(scene.positions), bytes(scene.covariances_3d),
                                bytes(scene.opacities), bytes(scene.sh_coeffs)]);
        if self.scene_key != Some(key) {
            status(compute.ctx, unsafe {
                cgs_scene_upload(compute.ctx, n as u64, scene.positions.as_ptr(),
                                 scene.covariances_3d.as_ptr(), scene.opacities.as_ptr(),
                                 scene.sh_coeffs.as_ptr() as *const c_void, CGS_SH_F32)
            })?;
            self.scene_key = Some(key);
            self.cage_key = None;
        }
        match cages {
            None => {
                if self.cage_key != Some(0) {
                    status(compute.ctx, unsafe {
                        cgs_tet_cages_upload(compute.ctx, 0, ptr::null(), ptr::null(), 0,
                                             ptr::null(), ptr::null())
                    })?;
                    self.cage_key = Some(0);
                }
            }
            Some(c) => {
                let key = fingerprint(&[bytes(c.elements), bytes(c.inv_dm), bytes(c.bind_tet),
                                        bytes(c.bind_w)]) | 1;
                let nv = (c.vertices.len() / 3) as u32;
                if self.cage_key != Some(key) {
                    status(compute.ctx, unsafe {
                        cgs_tet_cages_upload(compute.ctx, (c.elements.len() / 4) as u32,
                                             c.elements.as_ptr(), c.inv_dm.as_ptr(), nv,
                                             c.bind_tet.as_ptr(), c.bind_w.as_ptr())
                    })?;
                    self.cage_key = Some(key);
                }
                // every call, as the reference does; an unchanged upload keeps Stage 1 cached
                status(compute.ctx, unsafe {
                    cgs_cage_vertices_update(compute.ctx, c.vertices.as_ptr(), nv)
                })?;
            }
        }
        Ok(())
    }

    /// execute_frame_gpu (gpu_state.rs:613-626): Stages 1-4 on the resident
    /// scene; waits for the frame and reports its counts (and per-stage device
    /// times with `profile_stages`).
    #[allow(clippy::too_many_arguments)]
    pub fn execute_frame_gpu(&mut self, compute: &GpuCompute, scene: &SceneRef,
                             cages: Option<&TetCagesRef>, camera: &cgs_camera,
                             compositor: &cgs_compositor, strain_split_threshold: f32,
                             mip_filter_3d_var: f32, min_opacity: f32, min_radius_px: f32,
                             profile_stages: bool,
                             force_stage3: bool) -> Result<GpuStageTimings, GpuError> {
        self.sync(compute, scene, cages)?;
        let params = cgs_frame_params {
            strain_split_threshold,
            mip_filter_3d_var,
            min_opacity,
            min_radius_px,
            profile_stages: profile_stages as i32,
            force_stage3: force_stage3 as i32,
            ..Default::default()
        };
        let mut t = cgs_stage_timings::default();
        status(compute.ctx, unsafe {
            cgs_execute_frame(compute.ctx, camera, compositor, &params, &mut t)
        })?;
        self.last_width = compositor.screen_width;
        self.last_height = compositor.screen_height;
        Ok(GpuStageTimings {
            stage1_deform_ms: t.stage1_deform_ms,
            stage2_project_ms: t.stage2_project_ms,
            stage3_bin_sort_ms: t.stage3_bin_sort_ms,
            stage4_composite_ms: t.stage4_composite_ms,
            stage1_skipped: t.stage1_skipped != 0,
            stage3_cached: t.stage3_cached != 0,
            used_hardware_timestamps: t.used_hardware_timestamps != 0,
            used_64bit_keys: t.used_64bit_keys != 0,
            active_gaussians: t.active_gaussians as usize,
            surviving_gaussians: t.surviving_gaussians as usize,
            total_tile_entries: t.total_tile_entries as usize,
        })
    }

    /// readback_framebuffer_rgba8 (gpu_state.rs:1296-1328): tight
    /// [height][width][4] bytes of the last frame.
    pub fn readback_framebuffer_rgba8(&self, compute: &GpuCompute, width: u32,
                                      height: u32) -> Result<Vec<u8>, GpuError> {
        let mut out = vec![0u8; width as usize * height as usize * 4];
        status(compute.ctx, unsafe {
            cgs_readback_rgba8(compute.ctx, out.as_mut_ptr(), width, height)
        })?;
        Ok(out)
    }

    /// readback_framebuffer (gpu_state.rs:1331-1343) as f32 [h][w][4]: the
    /// unquantised frame when the library wrote one, else RGBA8 / 255.
    pub fn readback_framebuffer(&self, compute: &GpuCompute, width: u32,
                                height: u32) -> Result<Vec<f32>, GpuError> {
        let rgba8 = self.readback_framebuffer_rgba8(compute, width, height)?;
        Ok(rgba8.iter().map(|&b| b as f32 / 255.0).collect())
    }
}
