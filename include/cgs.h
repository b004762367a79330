/*
 * cgs.h - C ABI of the B200 (sm_100a) four-stage Gaussian-splat pipeline.
 *
 * This is the drop-in boundary that replaces CinderGS's CubeCL/WGPU backend
 * (crate `cinder_gs`, v2.0.0). Every entry point below names the reference
 * interface it stands in for (path:line inside the reference crate). A Rust
 * `-sys` crate, a ctypes module or a C++ host binds these symbols directly:
 * plain pointers and sizes, no CUDA or torch types in any signature.
 *
 * Conventions
 *  - Every call returns an int status: CGS_OK (0) or a negative CGS_E_* code.
 *    cgs_last_error(ctx) returns a message for the last failure on ctx.
 *  - A context owns one CUDA device, one stream and all device memory
 *    (scene residency + frame arena). One context per host thread; calls on a
 *    context are not re-entrant (the reference's `&mut self` API, same rule).
 *  - Host arrays are borrowed for the duration of the call only.
 *  - "d_" parameters are device pointers on the context's device; they are
 *    used on the context's stream.
 *  - There is no CPU fallback: when the device path cannot run, the call
 *    returns an error (the reference's orchestrator fell back to the CPU,
 *    render/pipeline.rs:721-737; this library does not).
 */
#ifndef CGS_H
#define CGS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CGS_OK 0
#define CGS_E_ARG -1       /* invalid argument (null pointer, bad size, bad enum) */
#define CGS_E_OOM -2       /* device or pinned-host allocation failed */
#define CGS_E_CUDA -3      /* a CUDA runtime call failed */
#define CGS_E_TIMEOUT -4   /* a bounded device-side wait gave up (status word set); the
                              frame's results are undefined. If a tensor-core wait gave up
                              twice, later frames return CGS_E_STATE: destroy and recreate
                              the context */
#define CGS_E_CAPACITY -5  /* a size exceeds a documented hard limit */
#define CGS_E_STATE -6     /* call order violated (e.g. frame before scene upload) */

#define CGS_SH_F32 0  /* 48 f32 SH coefficients per Gaussian (soa.rs:30-52) */
#define CGS_SH_F16 1  /* 48 IEEE binary16 SH coefficients per Gaussian (soa.rs:429-608) */

/* Camera uniform block, 96 bytes: render/camera.rs:9-36 (CameraUniforms).
 * view is the column-major world-to-camera matrix (glam Mat4::to_cols_array). */
typedef struct cgs_camera {
  float view[16];
  float focal_x, focal_y;
  float principal_x, principal_y;
  float viewport_width, viewport_height;
  float near_plane;
  float pad;
} cgs_camera;

/* Compositor uniform block, 48 bytes: render/rasterizer/mod.rs:16-37
 * (CompositorUniforms). tiles_x/tiles_y are recomputed from the screen size. */
typedef struct cgs_compositor {
  uint32_t screen_width, screen_height;
  uint32_t tiles_x, tiles_y;
  float background[4];
  float camera_position[3];
  uint32_t sh_degree;
} cgs_compositor;

/* The scalar arguments of GpuPipelineState::execute_frame_gpu
 * (render/gpu_state.rs:613-626), plus this library's output options. */
typedef struct cgs_frame_params {
  float strain_split_threshold; /* <= 0 disables strain splitting */
  float mip_filter_3d_var;      /* <= 0 disables the 3D Mip filter */
  float min_opacity;            /* reference default 1/255 (math/projection.rs:348) */
  float min_radius_px;          /* reference default 0.5 (math/projection.rs:351) */
  int32_t profile_stages;       /* 1: time each stage with CUDA events */
  int32_t force_stage3;         /* 1: never reuse the cached Stage 3 lists */
  int32_t write_f32;            /* 1: also write an unquantised RGBA f32 frame */
  int32_t radix_bits;           /* entry-sort digit width: 0 = balanced digits of at most
                                   8 bits over the tile bits (13 bits -> 7 + 6), else 4..8 */
  int32_t entry_sort;           /* CGS_SORT_*: how the tile entries are sorted by tile */
  int32_t tile_shape;           /* CGS_TILE_*: screen tile of Stages 3 and 4 */
} cgs_frame_params;

/* Screen tile shapes. The reference bins and composites 16x16 tiles
 * (render/kernels/binning.rs, compositor.rs); 8x8 and 32x16 tiles run the
 * same ellipse-vs-tile test and blending rules on other rectangles (fewer
 * candidate pixels per entry, or fewer entries per splat), so a pixel's
 * colour changes only where the test's rounding admits a splat whose alpha
 * at that pixel is below the 1/255 cut anyway. Chosen per viewport by the
 * autotuner. */
#define CGS_TILE_16X16 0
#define CGS_TILE_8X8 1
#define CGS_TILE_32X16 2

/* Entry sort methods (the result is the same, bit for bit). */
#define CGS_SORT_AUTO 0       /* radix passes */
#define CGS_SORT_RADIX 1      /* LSD radix passes over the tile bits */
#define CGS_SORT_TRANSPOSE 2  /* one-pass tile transpose (32-bit keys and at most 16,384
                                 tiles; otherwise radix passes) */

/* GpuStageTimings (render/gpu_state.rs:513-534). */
typedef struct cgs_stage_timings {
  double stage1_deform_ms;
  double stage2_project_ms;
  double stage3_bin_sort_ms;
  double stage4_composite_ms;
  int32_t stage1_skipped;
  int32_t stage3_cached;
  int32_t used_hardware_timestamps;
  int32_t used_64bit_keys;
  uint64_t active_gaussians;
  uint64_t surviving_gaussians;
  uint64_t total_tile_entries;
} cgs_stage_timings;

typedef struct cgs_ctx cgs_ctx;

/* ---- context (replaces GpuCompute::acquire, render/gpu.rs:70-113) ---- */

/* Creates a context on `device`. `stream` is a cudaStream_t to run on, or
 * NULL for a context-owned non-blocking stream. */
int cgs_ctx_create(int device, void* stream, cgs_ctx** out_ctx);
int cgs_ctx_destroy(cgs_ctx* ctx);
const char* cgs_last_error(const cgs_ctx* ctx);
/* Blocks until all work queued on the context's stream has finished. */
int cgs_ctx_synchronize(cgs_ctx* ctx);
/* Bytes of device memory the context currently holds. */
int cgs_ctx_device_bytes(const cgs_ctx* ctx, uint64_t* out_bytes);
/* Library version string. */
const char* cgs_version(void);
/* Launch shapes of the frame's kernels: the block sizes the autotuner picks
 * (cindergs_b200/autotune.py). Zero fields keep the library's defaults. No
 * reference counterpart: the reference launches fixed CubeDims. */
typedef struct cgs_launch_shape {
  uint32_t project_threads;    /* Stage 2 block: 128, 256 (default) or 512 threads */
  uint32_t bin_blocks_per_sm;  /* Stage 3 binning: resident 256-thread blocks per SM
                                  (default: as many as fit, 2) */
  uint32_t ranges_blocks;      /* tile-range kernel: blocks of 256 threads (default 1184) */
  uint32_t pad;
} cgs_launch_shape;
/* Sets the launch shape of the following frames and view steps (a captured
 * view graph is rebuilt). CGS_E_ARG for a value outside the ranges above. */
int cgs_ctx_set_launch_shape(cgs_ctx* ctx, const cgs_launch_shape* shape);
/* Caps the device memory the context's growable buffers (scene residency and
 * frame arena) may hold; 0 (the default) removes the cap. A call that would
 * grow past it fails with CGS_E_OOM and leaves the context usable. No
 * reference counterpart: the reference's arena grows by 1.5x without a limit
 * (render/gpu_pool.rs:43-49). */
int cgs_ctx_set_device_budget(cgs_ctx* ctx, uint64_t bytes);
/* Failure drill for the bounded device waits: runs the chained-scan look-back
 * (bit 0), the radix sort's digit look-back (bit 1) and the compositor's
 * mbarrier wait (bit 2), each against a predecessor or barrier that nothing
 * completes and with `polls` polls (1..2^22) instead of the kernels' 2^22.
 * Each wait gives up, sets its status bit and returns; *out_gave_up receives
 * the mask of drills that gave up. Returns CGS_E_TIMEOUT when any did (the
 * expected outcome) and leaves the context usable. No reference counterpart:
 * the reference's waits are unbounded. */
int cgs_ctx_wait_drill(cgs_ctx* ctx, uint32_t polls, uint32_t* out_gave_up);

/* ---- scene residency (GpuSceneState, render/gpu_state.rs:95-343) ---- */

/* Uploads the rest scene: pos [n*3], cov [n*6] (xx,xy,xz,yy,yz,zz),
 * opa [n] (activated), sh [n*48] as f32 or f16 (uint16 bits) per sh_format,
 * channel-major (DC rgb, R rest 15, G rest 15, B rest 15; sh.rs:56-61).
 * Re-uploading invalidates the deformed scene and the Stage 3 cache. */
int cgs_scene_upload(cgs_ctx* ctx, uint64_t n, const float* pos, const float* cov,
                     const float* opa, const void* sh, int32_t sh_format);

/* Uploads a QuantizedGaussianSceneSoa (scene/soa.rs:429-608): pos [n*3] f32,
 * cov_f16x2 [n*3] words of f16 pairs ((xx,xy), (xz,yy), (yz,zz), first value
 * in the low half), opa [n] f32, sh_f16x2 [n*words] with the coefficients up
 * to sh_degree (0..3) in its order (DC rgb, then each channel's higher
 * orders), two f16 per word, words = ceil(3 (sh_degree+1)^2 / 2) (24 for
 * degree 3). The octahedral rotation words are not used by any stage and
 * are not taken. Decoded on the GPU into the resident layout with f16 SH
 * planes; f16 to f32 is exact, so frames equal those of the dequantized
 * scene (to_soa) uploaded with CGS_SH_F16. */
int cgs_scene_upload_quantized(cgs_ctx* ctx, uint64_t n, const float* pos,
                               const uint32_t* cov_f16x2, const float* opa,
                               const uint32_t* sh_f16x2, uint32_t sh_degree);

/* Uploads flattened tet-cage topology for all cages (gpu_state.rs:248-298):
 * elems [num_tets*4] global vertex indices, inv_dm [num_tets*9] column-major
 * D_m^-1, bind_tet [n] global tet index or 0xFFFFFFFF when unbound,
 * bind_w [n*4] barycentric weights. num_tets == 0 removes all cages. */
int cgs_tet_cages_upload(cgs_ctx* ctx, uint32_t num_tets, const uint32_t* elems,
                         const float* inv_dm, uint32_t num_verts, const uint32_t* bind_tet,
                         const float* bind_w);

/* Updates the current cage vertex positions [num_verts*3] (gpu_state.rs:316-335).
 * A change marks the deformed scene dirty; an identical upload does not. */
int cgs_cage_vertices_update(cgs_ctx* ctx, const float* verts, uint32_t num_verts);

/* ---- cage spring dynamics on the device (deformation/dynamics.rs) ---- */

/* One spring-driven cage: the vertex range [first_vertex, first_vertex +
 * num_vertices) of the flattened tet-cage vertices, its CageSpringSimulator
 * parameters (stiffness, damping = velocity retention per 1/60 s, mass;
 * dynamics.rs:75-131) and its collision planes [first_plane, first_plane +
 * num_planes). */
typedef struct cgs_spring_cage {
  float stiffness, damping, mass;
  uint32_t first_vertex, num_vertices;
  uint32_t first_plane, num_planes;
  uint32_t pad;
} cgs_spring_cage;
/* CollisionPlane (dynamics.rs:4-33): allowed half-space normal . x >= offset,
 * normal of unit length, restitution and friction in [0, 1]. */
typedef struct cgs_collision_plane {
  float normal[3];
  float offset, restitution, friction;
  float pad[2];
} cgs_collision_plane;
/* Makes the tet-cage vertices spring-driven on the device: rest, current and
 * velocity [num_verts*3], pinned [num_verts] (0/1, null = none). current
 * becomes the resident cage state. num_verts must equal the tet cages'
 * vertex count; cage ranges must not overlap (vertices outside every range
 * are never stepped); at most 65,535 planes. Replaces the host-side
 * CageSpringSimulator state (dynamics.rs:115-131). */
int cgs_springs_upload(cgs_ctx* ctx, uint32_t num_cages, const cgs_spring_cage* cages,
                       uint32_t num_planes, const cgs_collision_plane* planes, uint32_t num_verts,
                       const float* rest, const float* current, const float* velocity,
                       const uint8_t* pinned);
/* Enqueues `steps` calls of CageSpringSimulator::step(dt) (dynamics.rs:
 * 249-277; dt clamped to 0.033 s, no step when it is not positive) on the
 * resident cage vertices; the next frame deforms with the result. Nothing is
 * copied to or from the host. */
int cgs_springs_step(cgs_ctx* ctx, float dt, uint32_t steps);
/* trigger_jiggle_impulse(magnitude) on every spring cage (dynamics.rs:280-305). */
int cgs_springs_impulse(cgs_ctx* ctx, float magnitude);
/* Copies the device spring state back: current and velocity [num_verts*3]
 * (either may be null). */
int cgs_springs_read(cgs_ctx* ctx, float* current, float* velocity);

/* Binds the resident rest scene to a tet cage on the GPU with the reference's
 * rule (first tet with barycentric violation <= 1e-4, else the least-violating
 * tet; TetMesh::bind_point, deformation/mod.rs:267-310). When use_bounds is
 * nonzero, points outside [bmin,bmax] or with best violation > 0.15 are
 * unbound (0xFFFFFFFF). Writes bind_tet [n] / bind_w [n*4] to host arrays. */
int cgs_bind_tets(cgs_ctx* ctx, uint32_t num_tets, const uint32_t* elems, const float* inv_dm,
                  uint32_t num_verts, const float* rest_verts, int32_t use_bounds,
                  const float* bmin, const float* bmax, uint32_t* bind_tet, float* bind_w);

/* ---- polygon cage, mean value coordinates (deformation/mvc.rs) ---- */

/* Uploads a closed, outward-oriented triangle cage (PolyCageMesh,
 * mvc.rs:15-21): rest vertices [V*3], triangles [F*3]. At most 1,024
 * vertices; vertices + triangles at most 12,800. Drops earlier MVC
 * bindings. The current vertices start at the rest pose. */
int cgs_mvc_cage_upload(cgs_ctx* ctx, uint32_t num_verts, const float* rest_verts,
                        uint32_t num_tris, const uint32_t* tris);

/* Current (deformed) cage vertices [V*3]; unchanged values are skipped. */
int cgs_mvc_vertices_update(cgs_ctx* ctx, const float* verts, uint32_t num_verts);

/* PolyCageMesh::bind_gaussians (mvc.rs:498-541) on the GPU for the resident
 * scene: Gaussians not bound to a tet cage whose rest centre has |winding
 * number| >= 0.5 get exact MVC weights and central-difference gradients
 * (step jacobian_step_size, mvc.rs:484-494), stored on the device
 * (16 bytes per Gaussian and cage vertex). Tet bindings win over the
 * polygon cage. Frames then deform the bound Gaussians as deform_scene_cpu
 * (mvc.rs:564-749) does. *out_bound receives the number bound. */
int cgs_mvc_bind(cgs_ctx* ctx, uint32_t* out_bound);

/* compute_mvc_weights (mvc.rs:366-471) of n points against the rest cage:
 * d_points [n*3] and d_weights [n*V] are device pointers (no counterpart in
 * the reference's GPU API). */
int cgs_mvc_weights(cgs_ctx* ctx, uint64_t n, const float* d_points, float* d_weights);

/* Host copy of the first max_slots stored MVC bindings: gaussian [slots]
 * (scene index of each slot, ascending) and wg [slots*V*4] = (w, dw/dx,
 * dw/dy, dw/dz) per cage vertex. *out_slots receives the number copied.
 * With learned bindings only the exact fallbacks are stored. */
int cgs_mvc_read_bindings(cgs_ctx* ctx, uint64_t max_slots, uint32_t* gaussian, float* wg,
                          uint64_t* out_slots);

/* ---- learned MVC weight field (no reference counterpart) ----
 * A network that stands in for compute_mvc_weights (mvc.rs:366-471) of the
 * uploaded polygon cage: Fourier features of the point (x^ = (x - c) / s,
 * c and s the centre and half the largest extent of the rest cage's box;
 * x^ and sin, cos of 2^b (pi/2) x^ for b = 0..7, zero-padded to 64), four
 * 128-wide SiLU layers, V outputs z made a partition of unity by
 * w0 = z + (1 - sum z) / V, then projected onto the weights that also
 * reproduce linear functions on the rest cage:
 * w = w0 - Vb^T M (Vb w0 - [1; x]), Vb = [1; rest vertices], M =
 * (Vb Vb^T)^-1 (exact MVC has both properties; affine cage motions are then
 * reproduced exactly). Weights and layer inputs are bf16, accumulation fp32
 * on the tensor cores. Frames evaluate it per Gaussian together with its
 * Jacobian. The linear-precision residual r = sum_j w0_j v_j - x of the
 * network's own weights on the rest cage selects the Gaussians that keep
 * exact stored weights. */

/* New network (seeded) for the uploaded polygon cage. Drops learned
 * bindings. */
int cgs_mvc_field_create(cgs_ctx* ctx, uint64_t seed);

/* Parameter block layout: offsets[10] (elements) of W1 [128x64], b1, W2,
 * b2, W3, b3 [128x128 / 128], W4, b4, W5 [Vx128], b5 [V] (row-major
 * out x in), *total floats, enc[4] = c and 1/s. Any pointer may be NULL. */
int cgs_mvc_field_layout(cgs_ctx* ctx, uint32_t* offsets, uint32_t* total, float* enc);

/* Copies the fp32 parameters to dst and/or from src (either may be NULL);
 * loading resets the optimiser state and drops learned bindings. */
int cgs_mvc_field_params(cgs_ctx* ctx, float* dst, const float* src);

/* Trains with Adam (beta 0.9 / 0.999, eps 1e-8) for `steps` steps on batches
 * of `batch` rows (a multiple of 8) drawn by a seeded hash from n device
 * points d_points [n*3] with their exact weights d_weights [n*V]. Loss per
 * batch of B rows: (1/B) sum_rows sum_j (w_j - w*_j)^2 + lambda (1/B)
 * sum_rows |r|^2 / (3 s^2). The step size follows a cosine from lr down to
 * lr/20 over the call's steps. out_loss[2] (may be NULL) receives the weight
 * term and the residual term (without lambda) averaged over the last tenth
 * of the steps. Drops learned bindings. */
int cgs_mvc_field_train(cgs_ctx* ctx, uint64_t n, const float* d_points, const float* d_weights,
                        uint32_t steps, uint32_t batch, float lr, float lambda, uint64_t seed,
                        float* out_loss);

/* Gradient of that loss over the first n points (n a multiple of 8, one
 * batch, no update) into grads [total] on the host; out_loss[2] as above. */
int cgs_mvc_field_grads(cgs_ctx* ctx, uint64_t n, const float* d_points, const float* d_weights,
                        float lambda, float* grads, float* out_loss);

/* Final (projected) network weights of n device points [n*3] into
 * d_weights [n*V]. */
int cgs_mvc_field_eval(cgs_ctx* ctx, uint64_t n, const float* d_points, float* d_weights);

/* Fused inference as frames run it: for n device points [n*3], 12 floats
 * each into d_out: position sum_j w_j v_j and its gradient F (column-major)
 * on the current cage vertices; with use_rest, the network's own rest
 * position sum_j w0_j v_j (x + r) and its gradient instead. d_out must be
 * 16-byte aligned. */
int cgs_mvc_field_infer(cgs_ctx* ctx, uint64_t n, const float* d_points, int32_t use_rest,
                        float* d_out);

/* As cgs_mvc_bind, with the network for every bound Gaussian whose
 * linear-precision residual |r| / s is at most `threshold`; the others get
 * exact stored weights (fallbacks, listed first by cgs_mvc_read_bindings).
 * The network's last hidden layer and its three tangents depend only on the
 * rest position, so by default they are evaluated here and kept (bf16, 1 KB
 * per Gaussian) and frames apply only the output layer folded with the
 * current vertices; with CGS_FIELD_PER_FRAME frames evaluate the whole
 * network instead and nothing is stored per Gaussian. Both give the same
 * result up to summation order. *out_bound and *out_fallback (either may be
 * NULL) receive both counts. */
#define CGS_FIELD_PER_FRAME 1u
int cgs_mvc_bind_learned(cgs_ctx* ctx, float threshold, uint32_t flags, uint32_t* out_bound,
                         uint32_t* out_fallback);

/* ---- frame (GpuPipelineState, render/gpu_state.rs:538-1243) ---- */

/* Runs Stages 1-4 on the resident scene (execute_frame_gpu,
 * gpu_state.rs:613-626). Stage 1 is skipped when cages and deform params are
 * unchanged; Stage 3 is reused when its cache key (gpu_state.rs:454-500) is
 * unchanged and force_stage3 is 0. The frame is enqueued without any host
 * synchronisation when `timings` is NULL; with `timings` the call waits for
 * the frame and reports its counts (and, with profile_stages, its per-stage
 * device times). A frame whose tile entries exceeded the key buffers is
 * binned and composited again with grown buffers before any readback. */
int cgs_execute_frame(cgs_ctx* ctx, const cgs_camera* camera, const cgs_compositor* comp,
                      const cgs_frame_params* params, cgs_stage_timings* timings);

/* One step of many views; no reference counterpart (execute_frame_gpu renders
 * one view per call). Stage 1 runs once (when the cages moved), then Stages
 * 2-4 run per view with that view's camera, viewport and parameters
 * (params[v]: every view's strain split and Mip settings must agree, the
 * digit width and entry sort may differ), writing view v's RGBA8 image to
 * the device buffer d_rgba8[v] (rows of screen_width pixels).
 * The Stage 3 cache is not used and stage profiling is off. With use_graph,
 * the first call for a set of views (same cameras, viewports, parameters,
 * output buffers, scene/cage/binding state and buffer capacities) renders
 * eagerly and captures the whole step as a CUDA graph; later calls with the
 * same set replay it (a view whose tile entries exceeded the captured
 * capacity is rendered again eagerly and the graph is rebuilt next time).
 * Without use_graph every view's launches are issued from the host. The call
 * returns when the step has finished. */
typedef struct cgs_views_stats {
  double ms;                    /* device time of the step, CUDA events */
  uint64_t total_tile_entries;  /* over all views */
  uint32_t graph_replayed;      /* the step ran as a graph replay */
  uint32_t graph_captured;      /* a graph was captured in this call */
  uint32_t views_rerendered;    /* views rendered again after an overflow */
  uint32_t pad;
} cgs_views_stats;
int cgs_execute_views(cgs_ctx* ctx, uint32_t num_views, const cgs_camera* cameras,
                      const cgs_compositor* comps, const cgs_frame_params* params,
                      uint32_t* const* d_rgba8, int32_t use_graph, cgs_views_stats* stats);

/* Copies the last frame's RGBA8 pixels into a tight [h][w][4] host buffer
 * (readback_framebuffer_rgba8, gpu_state.rs:1296-1328). */
int cgs_readback_rgba8(cgs_ctx* ctx, uint8_t* dst, uint32_t width, uint32_t height);
/* Starts copying the last frame's RGBA8 pixels into the tight [h][w][4] host
 * buffer dst and returns without waiting: the pixels are snapshotted on the
 * device behind the frame and copied to the host on a separate stream, so
 * the copy overlaps the frames enqueued after it (page-locked dst memory
 * makes the copy asynchronous). *ticket identifies the copy; dst holds the
 * pixels once cgs_readback_wait(ctx, ticket) has returned CGS_OK. At most
 * two copies are in flight: a third call first waits for the oldest. If the
 * frame overflowed the tile-entry buffers, the wait re-reads it after the
 * library re-renders it with grown buffers; when later frames were already
 * in flight, the wait renders it again from its stored arguments and cage
 * vertices (the next frame then deforms and bins afresh, and
 * cgs_read_frame_buffer refuses until it has run). No reference counterpart:
 * readback_framebuffer_rgba8 (gpu_state.rs:1296-1328) is synchronous. */
int cgs_readback_rgba8_async(cgs_ctx* ctx, uint8_t* dst, uint32_t width, uint32_t height,
                             uint64_t* ticket);
/* Waits for the copy `ticket` of cgs_readback_rgba8_async (a ticket already
 * waited for returns CGS_OK at once). */
int cgs_readback_wait(cgs_ctx* ctx, uint64_t ticket);
/* Copies the last frame's unquantised RGBA f32 pixels [h][w][4] (written when
 * params.write_f32 was set; render/kernels/compositor.rs f32 output mode). */
int cgs_readback_rgba_f32(cgs_ctx* ctx, float* dst, uint32_t width, uint32_t height);
/* Device pointer and row pitch (in u32 pixels) of the padded RGBA8 frame
 * (rows padded to 64 pixels, padded_rgba8_row_u32 gpu_state.rs:25). */
int cgs_framebuffer_device(cgs_ctx* ctx, void** d_rgba8, uint32_t* row_pitch_px);

/* Per-kernel device time, launches and algorithmic traffic accumulated over
 * the frames run with params.profile_stages set since the last reset (CUDA
 * events around every launch; profiling adds no host synchronisation to a
 * frame unless the caller also asks for that frame's cgs_stage_timings).
 * alg_bytes is the HBM traffic each kernel must move at minimum (inputs read
 * once, outputs written once), the numerator of its roofline fraction. No
 * reference counterpart: it refines GpuStageTimings (gpu_state.rs:513-534)
 * to kernel granularity. */
#define CGS_K_CLEAR 0          /* memsets of per-frame scratch */
#define CGS_K_TET_TRANSFORMS 1
#define CGS_K_DEFORM 2
#define CGS_K_PROJECT 3
#define CGS_K_BIN 4            /* count + chained scan + key emission, one launch */
#define CGS_K_ENTRY_SORT 5     /* stable sort of the tile entries by tile: the one-pass
                                  tile transpose, or radix passes for many tiles */
#define CGS_K_TILE_RANGES 6    /* (the tile transpose writes the ranges itself) */
#define CGS_K_COMPOSITE 7
#define CGS_K_SPLAT_SORT 8     /* depth-key histogram + radix passes over the splats */
#define CGS_K_MVC 9            /* MVC position + gradient of every stored polygon-cage binding */
#define CGS_K_FIELD 10         /* learned MVC field: output projection + fused inference */
#define CGS_KERNEL_COUNT 11
typedef struct cgs_kernel_profile {
  double ms[CGS_KERNEL_COUNT];
  uint64_t alg_bytes[CGS_KERNEL_COUNT];
  uint32_t launches[CGS_KERNEL_COUNT];
  /* tensor-core work of the kernels that have any (multiply-adds count 2) */
  uint64_t alg_flops[CGS_KERNEL_COUNT];
} cgs_kernel_profile;
int cgs_kernel_profile_read(cgs_ctx* ctx, cgs_kernel_profile* out);
int cgs_kernel_profile_reset(cgs_ctx* ctx);
const char* cgs_kernel_name(int32_t id);

/* Drops cached Stage 3 lists (invalidate_stage3, gpu_state.rs:570-573). */
int cgs_invalidate_stage3(cgs_ctx* ctx);
/* Drops scene, cages and caches (invalidate, gpu_state.rs:565-568). */
int cgs_invalidate(cgs_ctx* ctx);

/* Intermediate buffers of the last frame, for stage-isolated parity checks
 * (the reference's tests read the same buffers, tests/gpu_parity_tests.rs:665-900). */
#define CGS_BUF_DEFORMED_POS 1   /* f32 [active*3] */
#define CGS_BUF_DEFORMED_COV 2   /* f32 [active*6] */
#define CGS_BUF_DEFORMED_OPA 3   /* f32 [active] */
#define CGS_BUF_SPLIT_META 4     /* u32 [splits*2] (parent, tet) */
#define CGS_BUF_SPLAT_ATTRS 5    /* f32 [active*10] mu_x,mu_y,a,b,c,alpha,r,g,b,tz */
#define CGS_BUF_EXTENTS 6        /* u32 [active] ext_x | ext_y << 16, 0 = culled */
#define CGS_BUF_TILE_OFFSETS 7   /* u32 [active] exclusive scan of tiles touched */
#define CGS_BUF_SORTED_KEYS 8    /* u32 [entries] (32-bit keys) or u64 [entries] */
#define CGS_BUF_SORTED_IDS 9     /* u32 [entries] */
#define CGS_BUF_TILE_RANGES 10   /* u32 [tiles*2] */
#define CGS_BUF_TET_JACOBIANS 11 /* f32 [tets*9] column-major */
#define CGS_BUF_TET_ROTATIONS 12 /* f32 [tets*9] column-major */
#define CGS_BUF_TET_STRETCH 13   /* f32 [tets] */
#define CGS_BUF_MVC_ROTATIONS 14 /* f32 [MVC slots*9] polar rotations, column-major */
/* Reads buffer `which` of the last frame into `dst` (capacity dst_bytes);
 * *out_bytes receives the byte size of the valid contents. */
int cgs_read_frame_buffer(cgs_ctx* ctx, int32_t which, void* dst, uint64_t dst_bytes,
                          uint64_t* out_bytes);

/* ---- SH coefficient rotation and deformed-scene export ---- */

/* Rotates n blocks of 48 SH coefficients (DC rgb, then 15 per channel) in
 * device memory in place: block i by rotation d_index[i] (or i % num_rotations
 * when d_index is null) of d_rotations [num_rotations * 9] (column-major),
 * bands 1..min(degree, 3), each band by the f32 matrix
 * (B_l T_l(R^T) B_l^+)^T with an f32 running sum. Replaces ShRotator::new +
 * ShRotator::apply / rotate_sh_buffer (render/rasterizer/sh_rotation.rs:
 * 403-471), with the per-rotation matrices built on the device. d_sh must be
 * 16-byte aligned. An index at or above num_rotations leaves its block
 * unchanged and returns CGS_E_ARG. */
int cgs_sh_rotate(cgs_ctx* ctx, uint64_t n, float* d_sh, uint32_t num_rotations,
                  const float* d_rotations, const uint32_t* d_index, uint32_t degree);

/* The deformed scene of the last frame's Stage 1 as host arrays in the
 * GaussianSceneSoa layout: pos [count*3], cov [count*6] (xx, xy, xz, yy, yz,
 * zz), opa [count], sh [count*48]: the n rest Gaussians' deformed records
 * then the split children, each splat's SH coefficients (a child's are its
 * parent's) rotated by its tet's or polygon-cage slot's rotation up to
 * sh_degree. Replaces Timeline::deform_scene_at + write_binary_ply_bytes'
 * input (app/timeline.rs:205-275, the CPU's per-tet ShRotator in
 * deformation/cpu_reference.rs:172-183) with the GPU frame's own deformation.
 * Null output pointers are skipped; with all four null only *out_count is
 * written. Without cages the rest scene is exported; with cages whose state
 * changed after the last frame, CGS_E_STATE. */
int cgs_export_deformed(cgs_ctx* ctx, uint32_t sh_degree, uint64_t capacity, float* pos, float* cov,
                        float* opa, float* sh, uint64_t* out_count);

/* ---- stage primitives on device memory (render/kernels/scan.rs, radix_sort.rs) ---- */

/* Exclusive scan of d_in [n] into d_out [n]; *total receives the sum
 * (gpu_exclusive_scan_total, render/kernels/scan.rs:312-333). The reference
 * caps n at 512^3 (scan.rs:264-268); this single-pass scan takes n < 2^32. */
int cgs_scan_u32(cgs_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint64_t n,
                 uint64_t* total);

/* Stable LSD radix sort of (key, value) pairs on the low key_bits bits
 * (gpu_radix_sort_u32_pairs, render/kernels/radix_sort.rs:292-368).
 * d_keys/d_vals [n] are sorted in place; digit_bits is 4 or 8 (0 = 8). */
int cgs_sort_pairs_u32(cgs_ctx* ctx, uint32_t* d_keys, uint32_t* d_vals, uint64_t n,
                       uint32_t key_bits, int32_t digit_bits);

/* Stable sort of (tile, depth, id) triples by (tile, depth) for the 64-bit
 * key path (gpu_radix_sort_u64_pairs, radix_sort.rs:377-477): d_tiles, d_depths
 * and d_ids [n] are permuted in place; tile_bits bounds the tile ids. */
int cgs_sort_pairs_u64(cgs_ctx* ctx, uint32_t* d_tiles, uint32_t* d_depths, uint32_t* d_ids,
                       uint64_t n, uint32_t tile_bits, int32_t digit_bits);

/* ---- allocation-free variant ----------------------------------------------- */

/* No counterpart in the reference. The same stable LSD radix sort as
 * cgs_sort_pairs_u32, for callers that cannot let a library call cudaMalloc:
 * a host engine that owns all device memory through its own allocator or
 * budget, or a real-time loop where an allocation could synchronise the device
 * mid-frame. It needs no context and allocates nothing: its scratch is one
 * fixed array of 9 MiB + 8.25 KiB inside the library image, which every GPU
 * that loads the library holds until the process exits.
 * Sorts d_keys/d_vals [n] (device memory of the current device) in place on
 * `stream` (a cudaStream_t, NULL for the legacy default stream) and returns
 * once the sort has finished. n above CGS_NOALLOC_SORT_MAX_PAIRS returns
 * CGS_E_CAPACITY. All calls share the one scratch array: calls that overlap on
 * the GPU race and must be serialised by the caller. The first call on a
 * device looks up the array's device address; make that first call before
 * any stream capture. */
#define CGS_NOALLOC_SORT_MAX_PAIRS 1048576
int cgs_sort_pairs_u32_noalloc(uint32_t* d_keys, uint32_t* d_vals, uint64_t n,
                               uint32_t key_bits, int32_t digit_bits, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CGS_H */
