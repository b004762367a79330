// Host-side launchers for the sm_100a kernels (one per .cu translation unit).
// All launchers enqueue on `stream` and return the launch error code.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace cgs {

// ---- Stage 1 (stage1_deform.cu) --------------------------------------------
struct DeformArgs {
  uint32_t n;                 // rest Gaussians
  uint32_t num_tets;
  const float* verts;         // [V*3] current cage vertices
  const uint4* elems;         // [T]
  const float* inv_dm;        // [T*9]
  float* tet_J;               // [T*9] out (column-major)
  float* tet_R;               // [T*9] out (column-major)
  float* tet_stretch;         // [T] out
  const uint32_t* bind_tet;   // [n]
  const float4* bind_w;       // [n]
  const float4* rest_pos;     // [n] xyz + opacity
  const float4* rest_cova;    // [n] xx, xy, xz, yy
  const float2* rest_covb;    // [n] yz, zz
  float4* def_pos;            // [2n]
  float4* def_cova;           // [2n]
  float2* def_covb;           // [2n]
  uint2* split_meta;          // [n] (parent, tet)
  uint32_t* split_count;      // persistent device word
  unsigned long long* status; // [ceil(n/256)] chained-scan status, zeroed
  FrameCounters* fc;
  float split_threshold;
  float mip;
  // MVC-bound Gaussians (bind_tet == kMvcBound): per slot the deformed
  // position and gradient (3 float4, k_mvc_jacobian) in, the polar rotation
  // (9 floats, column-major) out for Stage 2's SH directions
  const float4* mvc_xf;
  float* mvc_R;
  // 1: the deform launch also computes the tet transforms (its first blocks
  // take the tets; the Gaussian blocks wait for them), instead of a separate
  // launch_tet_transforms
  uint32_t fuse_tets;
};
// FrameCounters::tile_ctr slot counting the finished tet blocks of a fused
// deform launch.
constexpr int kTetsDoneCtr = 8;
cudaError_t launch_tet_transforms(const DeformArgs& a, cudaStream_t s);

// ---- MVC (stage1_mvc.cu) -----------------------------------------------------
// bind_tet value of a Gaussian bound to the polygon (MVC) cage; its bind_w.x
// holds the bits of its MVC slot.
constexpr uint32_t kMvcBound = 0xFFFFFFFEu;
struct MvcCage {
  uint32_t V, F;
  const float4* verts;      // [V] rest (binding) or current vertices
  const uint4* tris;        // [F] outward triangles
  const uint32_t* vf_off;   // [V + 1] incident faces per vertex (CSR)
  const uint32_t* vf_list;  // face << 2 | corner, ascending faces per vertex
};
bool mvc_cage_fits(uint32_t V, uint32_t F);
cudaError_t launch_mvc_weights(const MvcCage& c, uint32_t n, const float* pts, float* w,
                               cudaStream_t s);
cudaError_t launch_mvc_inside(const MvcCage& c, uint32_t n, const float4* rest_pos,
                              const uint32_t* bind_tet, uint32_t* flag, cudaStream_t s);
cudaError_t launch_mvc_compact(uint32_t n, const uint32_t* flag, const uint32_t* slot_of,
                               uint32_t* bind_tet, float4* bind_w, uint32_t* list, cudaStream_t s);
cudaError_t launch_mvc_bind_weights(const MvcCage& c, uint32_t nb, const uint32_t* list,
                                    const float4* rest_pos, float h, float4* wg, cudaStream_t s);
cudaError_t launch_mvc_jacobian(uint32_t V, const float4* verts, uint32_t nb, const float4* wg,
                                float4* xf, cudaStream_t s);
// Linear-precision residual |x' - x| / s at each listed rest position, where
// x' (xf, 3 float4 per slot) is the learned field's position on the rest
// cage; flag = residual > threshold.
cudaError_t launch_mvc_residual(uint32_t nb, const uint32_t* list, const float4* rest_pos,
                                const float4* xf, float inv_scale, float threshold, float* resid,
                                uint32_t* flag, cudaStream_t s);

// ---- learned MVC field (mvc_field.cu) ------------------------------------------
constexpr int kFieldBands = 8;
constexpr int kFieldIn = 64;    // 3 + 6 * bands, zero-padded
constexpr int kFieldHid = 128;
constexpr int kEpiF32 = 0, kEpiBias = 1, kEpiBiasSilu = 2;
// per-frame projection: Pc (128 x 3), pc (3), A3 (3 x 3)
constexpr int kFieldProj = 3 * kFieldHid + 3 + 9;
struct FieldMat {  // M = (Vb Vb^T)^-1, row-major 4 x 4
  float m[16];
};

struct FieldNet {  // device pointers into one parameter block
  const __nv_bfloat16 *W1b, *W2b, *W3b, *W4b, *W5b;
  const float *b1, *b2, *b3, *b4, *b5;
};
struct GemmArgs {  // C = A B^T (+ bias), D = bf16(silu(C)); tcgen05 (mvc_field_tc.cu)
  const __nv_bfloat16* A;
  const __nv_bfloat16* B;
  uint32_t M, N, K, lda, ldb;
  float* C;
  uint32_t ldc;
  const float* bias;
  __nv_bfloat16* D;
  uint32_t ldd;
  uint32_t* status;      // kStatusBarrierTimeout / kStatusPoisoned on a failed wait, or null
  float* ws;             // split-K partial sums (F32 epilogue), or null: no split
  size_t ws_floats;
};
struct FieldBatch {
  const float* points;   // [n*3]
  const float* target;   // [n*V] exact weights or null
  uint32_t n, V, B, ldw;
  uint32_t seed;         // 0: rows r % n in order
  const float* enc;      // [4] centre xyz, 1/s
  float* x;              // [B*3]
  float* wt;             // [B*ldw]
  __nv_bfloat16* a0;     // [B*64]
};
struct FieldLoss {
  const float* z;        // [B*ldz]
  const float* wt;       // [B*ldw]
  const float* x;        // [B*3]
  const float4* verts;   // [V] rest vertices
  uint32_t B, V, ldz, ldw;
  float lambda, s2;
  float M[16];           // (Vb Vb^T)^-1 of the rest cage
  float* dz;             // [B*ldz]
  __nv_bfloat16* dzb;    // [B*ldz]
  float* loss;           // [2] accumulated (weight term, residual term)
};
struct FieldInfer {
  FieldNet net;
  const float* enc;      // [4]
  const float* proj;     // [kFieldProj]
  const uint32_t* gauss; // item -> point index, or null (identity)
  const float4* points4; // rest positions (xyz), or null
  const float* points3;  // packed xyz when points4 is null
  uint32_t first, count, out_first;
  float4* xf;            // [(out_first + count) * 3]
  // cached codes [count][4][128] bf16 and the items' rest positions
  // [count]: written by launch_field_infer when codes is set (instead of
  // xf), read by launch_field_apply
  __nv_bfloat16* codes;
  float4* code_pos;
  uint32_t* status;      // kStatusBarrierTimeout when a bounded wait gave up, or null
};
cudaError_t launch_field_gather(const FieldBatch& b, cudaStream_t s);
cudaError_t launch_gemm_nt(const GemmArgs& g, int epi, cudaStream_t s);
cudaError_t launch_transpose_f32(const float* in, uint32_t R, uint32_t C, uint32_t ldi,
                                 __nv_bfloat16* out, uint32_t ldo, cudaStream_t s);
cudaError_t launch_transpose_bf16(const __nv_bfloat16* in, uint32_t R, uint32_t C, uint32_t ldi,
                                  __nv_bfloat16* out, uint32_t ldo, cudaStream_t s);
cudaError_t launch_field_loss(const FieldLoss& l, cudaStream_t s);
cudaError_t launch_silu_back(uint32_t n, const float* da, const float* pre, float* dpre,
                             __nv_bfloat16* dpreb, cudaStream_t s);
cudaError_t launch_colsum(const float* g, uint32_t B, uint32_t N, uint32_t ld, float* out,
                          cudaStream_t s);
cudaError_t launch_adam(uint32_t n, float* p, const float* g, float* m, float* v,
                        __nv_bfloat16* pb, float lr, float b1, float b2, float eps, float c1,
                        float c2, cudaStream_t s);
// verts null: the network's own rest position (no linear-precision
// projection); otherwise the projected weights on current vertices verts.
cudaError_t launch_field_project(const FieldNet& net, uint32_t V, const float4* rest,
                                 const float4* verts, const float* M, float* proj,
                                 cudaStream_t s);
cudaError_t launch_field_infer(const FieldInfer& fi, cudaStream_t s);
// The same on the tcgen05 tensor cores (mvc_field_tc.cu).
cudaError_t launch_field_infer_tc(const FieldInfer& fi, cudaStream_t s);
// Output layer over cached codes (needs codes, points4): position + gradient.
cudaError_t launch_field_apply(const FieldInfer& fi, cudaStream_t s);

cudaError_t launch_deform(const DeformArgs& a, cudaStream_t s);

struct BindArgs {
  uint32_t n;
  uint32_t num_tets;
  const float4* points;   // [n] xyz (+ unused w)
  const float* tet_x0;    // [T*3] rest position of each tet's first vertex
  const float* inv_dm;    // [T*9]
  int use_bounds;
  float bmin[3], bmax[3];
  uint32_t* bind_tet;     // [n] out
  float4* bind_w;         // [n] out
};
cudaError_t launch_bind(const BindArgs& a, cudaStream_t s);

// ---- Stage 2 (stage2_project.cu) -------------------------------------------
struct ProjectArgs {
  uint32_t threads;           // block size: 128, 256 (0) or 512
  const float4* pos;          // [max_n] xyz + opacity
  const float4* cova;         // [max_n]
  const float2* covb;         // [max_n]
  const void* sh;             // SH planes: f32 -> float4 [12][sh_stride]; f16 -> uint4 [6][sh_stride]
  int sh_f16;
  uint32_t sh_stride;         // plane stride (rest Gaussian count)
  const uint32_t* bind_tet;   // [n_rest] or null
  const float4* bind_w;       // [n_rest] (MVC slot bits in .x for kMvcBound) or null
  const float* tet_R;         // [T*9] or null
  uint32_t num_tets;
  const float* mvc_R;         // [MVC slots * 9] or null
  const uint2* split_meta;    // [n_rest] or null
  const uint32_t* split_count;  // device word or null (no splitting)
  uint32_t n_rest;
  uint32_t max_n;             // grid covers max_n splats
  float cam[24];
  float cam_pos[3];
  float mip, min_opacity, min_radius;
  uint32_t sh_degree;
  SplatRec* out;              // [max_n]
  FrameCounters* fc;
  // Stage 3's per-splat depth keys and slot ids (null when the frame reuses
  // an earlier frame's Stage 3): 32-bit keys get the quantised depth of the
  // packed (tile, depth) key, 64-bit keys the raw depth bits; culled splats
  // get 0xFFFFFFFF, which sorts after every visible depth.
  uint32_t* depth_keys;       // [max_n]
  uint32_t* depth_ids;        // [max_n]
  int key64;
  uint32_t depth_base_bits;   // near-plane exponent bits (32-bit keys)
  uint32_t depth_bits;        // depth bits in a 32-bit key
};
cudaError_t launch_project(const ProjectArgs& a, cudaStream_t s);

// QuantizedGaussianSceneSoa words (f16 covariance pairs, degree-trimmed f16
// SH) into the resident layout with f16 SH planes.
cudaError_t launch_scene_decode_quantized(uint32_t n, const float* pos, const uint32_t* cov_words,
                                          const float* opa, const uint32_t* sh_words,
                                          uint32_t sh_degree, float4* out_pos, float4* out_cova,
                                          float2* out_covb, void* out_sh, cudaStream_t s);
// Rest-scene layout conversion from the reference's interleaved SoA.
cudaError_t launch_scene_layout(uint32_t n, const float* pos, const float* cov, const float* opa,
                                const void* sh, int sh_f16, float4* out_pos, float4* out_cova,
                                float2* out_covb, void* out_sh, cudaStream_t s);

// ---- Stage 3 (stage3_bin.cu) -------------------------------------------------
struct BinArgs {
  const SplatRec* recs;
  // Splats in depth-key order (the stable radix sort of Stage 2's depth keys):
  // slot s of the binning grid is splat order_ids[s] with depth key
  // order_keys[s]; its entries are emitted in this order.
  const uint32_t* order_keys;
  const uint32_t* order_ids;
  const uint32_t* split_count;  // null when no splitting
  uint32_t n_rest;
  uint32_t max_n;
  uint32_t width, height, tiles_x, tiles_y;
  uint32_t tile_w_log2, tile_h_log2;  // screen tile shape (8x8, 16x16 or 32x16 pixels)
  // per slot (depth order): the first entry (direct mode), or the tile count
  // that a scan turns into the first entry in place (record mode)
  uint32_t* offsets;            // [max_n]
  // direct mode: look-back words of the 32-slot tiles' hit counts, zeroed
  unsigned long long* lookback; // [ceil(max_n/32)]
  // record mode: staging start and records of each 32-slot tile and group
  uint32_t* tile_stage;
  uint32_t* tile_count;
  uint32_t blocks_per_sm;       // resident blocks per SM of the count kernel (0: all that fit)
  FrameCounters* fc;
  int key64;
  uint32_t depth_bits;          // depth bits in a 32-bit key
  // record mode: the staged records; direct mode: the entries in depth order
  uint32_t* stage_keys;
  uint32_t* keys;               // 32-bit: packed keys; 64-bit: tile ids
  uint32_t* depths;             // 64-bit: raw depth bits
  uint32_t* ids;
  uint32_t* hist;               // [passes][1 << radix_bits] tile-digit histograms, zeroed
  uint32_t radix_bits;
  uint32_t tile_bits;           // tile id bits (the entry sort's key bits)
  uint32_t entry_cap;           // capacity of every entry buffer
  // Record mode (the tile transpose): stage one word per hit, tile << 5 |
  // slot lane, instead of keys and ids; no histograms. Each 32-slot tile
  // stages one run per group of 2^group_shift screen tiles, so tile_stage /
  // tile_count are [ceil(max_n/32)][groups].
  int records;
  uint32_t groups;              // <= 8
  uint32_t group_shift;
};
// Counts each slot's tiles and, in direct mode, writes the scanned offsets,
// the entry total (fc->entries) and every entry at its place in depth order
// and accumulates the tile-digit histograms (k_bin_count, one launch); in
// record mode it stages one record per hit and leaves the per-slot counts
// for a scan (launch_scan_u32).
cudaError_t launch_bin_count(const BinArgs& a, cudaStream_t s);
// Tile transpose (the entry sort when the tiles fit shared memory): a
// one-pass stable counting sort of the staged records by tile. Chunk k is the
// 32-slot tiles [k * chunk_wtiles, (k + 1) * chunk_wtiles); warp w of a chunk
// block owns the w-th eighth of them.
struct TransposeArgs {
  const uint32_t* records;      // staged tile << 5 | slot lane
  const uint32_t* tile_stage;   // [num_wtiles][groups] staging start of each run
  const uint32_t* tile_count;   // [num_wtiles][groups] records of each run
  const uint32_t* order_ids;    // slot -> splat index
  uint32_t num_wtiles;
  uint32_t chunk_wtiles;        // multiple of 8, at most 2040
  uint32_t num_chunks;
  uint32_t num_tiles;           // screen tiles
  uint32_t groups;              // tile groups (runs per 32-slot tile)
  uint32_t group_tiles;         // screen tiles per group (a power of two)
  uint32_t* cmat;               // [num_tiles][num_chunks] counts -> first entries (in place)
  uint32_t* totals;             // [num_tiles] entries per tile, zeroed
  const uint32_t* tile_base;    // [num_tiles] exclusive scan of totals
  uint32_t* ranges;             // [num_tiles] (start, end), (0, 0) when empty
  uint32_t* ids_out;            // [capacity] sorted splat indices
  uint32_t capacity;
  uint32_t* status_word;
};
constexpr uint32_t kTransposeGroupTiles = 2048;  // screen tiles per group (2^11)
cudaError_t launch_chunk_counts(const TransposeArgs& a, cudaStream_t s);
cudaError_t launch_column_scan(const TransposeArgs& a, cudaStream_t s);
cudaError_t launch_chunk_place(const TransposeArgs& a, cudaStream_t s);

// Per-tile [start, end) from sorted words: tile = word >> shift, over
// min(*n_ptr, capacity) words. ranges zeroed.
// Turns the last sort pass's range words (complemented first entries, ends)
// into [first, end) per screen tile; empty tiles stay (0, 0).
cudaError_t launch_ranges_fixup(uint32_t* ranges, uint32_t num_tiles, cudaStream_t s);
cudaError_t launch_tile_ranges(const uint32_t* sorted, uint32_t shift, const uint32_t* n_ptr,
                               uint32_t capacity, uint32_t total_tiles, uint32_t* ranges,
                               uint32_t blocks, cudaStream_t s);
// Generic exclusive scan of n u32 (chained scan); total -> *d_total.
cudaError_t launch_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* d_total,
                            unsigned long long* status, uint32_t* tile_ctr, uint32_t* status_word,
                            cudaStream_t s);
uint32_t scan_tiles(uint32_t n);

// ---- radix sort (radix_sort.cu) ----------------------------------------------
struct SortArgs {
  uint32_t* keys[2];     // ping-pong key buffers
  uint32_t* vals[2];     // ping-pong payload word 0
  uint32_t* vals2[2];    // ping-pong payload word 1 (null for one-word payloads)
  const uint32_t* n_ptr; // device element count (may exceed capacity -> capacity flag)
  uint32_t capacity;     // elements the buffers hold; grid is sized for it
  uint32_t first_bit;    // lowest key bit to sort on
  uint32_t num_bits;     // bits to sort on (from first_bit)
  uint32_t radix_bits;   // digit width, 4..8
  uint32_t* hist;        // [passes][radix] counts of the digits, filled before the passes
                         // (each block of a pass scans its pass's counts)
  // optional: the last pass also finds the [first, end) entries of every
  // screen tile (key >> tile_shift) into ranges[2 t], ranges[2 t + 1]
  // (zeroed before the sort; finish with launch_ranges_fixup)
  uint32_t* ranges = nullptr;
  uint32_t tile_shift = 0;
  uint32_t num_tiles = 0;
  void* status;          // [passes][tiles][radix] zeroed look-back words (when status2 is null)
  void* status2[2];      // optional: two [tiles][radix] look-back buffers used
                         // alternately; each pass clears the one it does not
                         // use for the next pass, so no per-frame memset is needed
  int* parity;           // in/out: buffer index the next pass uses (with status2)
  // look-back words of 64 bits (any 32-bit count; required above 2^30
  // elements) instead of 32 bits (counts below 2^30)
  bool wide_lookback = false;
  // words per tile that each pass clears in the status2 buffer it does not
  // use (0: the radix). A pair shared by sorts of different digit widths sets
  // the widest radix (256), so that a narrow sort leaves no stale word for a
  // later wide one to read.
  uint32_t lb_stride = 0;
  uint32_t* tile_ctr;    // [passes] zeroed
  uint32_t* status_word;
  int src;               // index of the buffer holding the input
  // bit p: pass p finds the lanes sharing a digit with one ballot per digit
  // bit (a fixed cost) instead of __match_any_sync (cheap when a warp's keys
  // share few digits, expensive when they are all different)
  uint32_t ballot_mask = ~0u;
  // bit p: pass p uses shared-memory peer masks instead (one atomicOr and
  // one warp barrier per key: cheapest for many distinct 8-bit digits)
  uint32_t smem_mask = 0u;
};
// Wait drills (cgs_ctx_wait_drill): each runs one of the library's bounded
// device waits against a predecessor or barrier that nothing completes, with
// `limit` polls, so that it gives up and sets its status bit in *status_word.
// The look-back arrays must hold two zeroed tiles.
cudaError_t launch_drill_chained_scan(unsigned long long* status, uint32_t* status_word,
                                      uint32_t limit, cudaStream_t s);
cudaError_t launch_drill_digit_lookback(const uint32_t* status, uint32_t radix,
                                        uint32_t* status_word, uint32_t limit, cudaStream_t s);
cudaError_t launch_drill_mbarrier(uint32_t* status_word, uint32_t limit, cudaStream_t s);
// Runs the passes; returns in *out_src the index of the buffer with the result.
cudaError_t run_radix_sort(const SortArgs& a, int* out_src, cudaStream_t s);
cudaError_t launch_histogram(const uint32_t* keys, const uint32_t* n_ptr, uint32_t capacity,
                             uint32_t first_bit, uint32_t num_bits, uint32_t radix_bits,
                             uint32_t* hist, cudaStream_t s);
uint32_t sort_tiles(uint32_t capacity);
uint32_t sort_passes(uint32_t num_bits, uint32_t radix_bits);

// ---- Cage springs (springs.cu) -----------------------------------------------
struct SpringCageDev {
  float kim;        // stiffness / max(mass, 0.001)
  float gamma;      // velocity factor exp(-c dt) of one step
  float dt;         // min(dt, 0.033); a step is skipped unless > 0
  float pad;
  float cx, cy, cz; // rest centroid (jiggle impulse)
  uint32_t planes;  // first plane | count << 16
};
struct SpringArgs {
  uint32_t V, num_cages, steps;
  const float4* rest;          // [V] xyz + cage index bits (>= num_cages: no cage)
  float4* vel;                 // [V]
  const uint8_t* pinned;       // [V]
  float* verts;                // [V*3] the resident cage vertices, stepped in place
  const SpringCageDev* cages;  // [num_cages]
  const float4* planes;        // [2 per plane] (nx, ny, nz, offset), (restitution, friction, -, -)
};
cudaError_t launch_springs_step(const SpringArgs& a, cudaStream_t s);
cudaError_t launch_springs_impulse(const SpringArgs& a, float magnitude, cudaStream_t s);

// ---- SH coefficient rotation and export (sh_rotate.cu) ------------------------
// Floats per rotation in the band-matrix table: M1 (9), M2 (25), M3 (49), pad.
constexpr uint32_t kShRotStride = 84;
struct ExportArgs {
  uint32_t n_rest;            // rest Gaussians (splats at or above are split children)
  uint32_t first, count;      // the chunk of splats to write
  const float4* pos;          // [first + count] xyz + opacity (deformed or rest)
  const float4* cova;         // xx, xy, xz, yy
  const float2* covb;         // yz, zz
  const void* sh;             // resident SH planes (f32 [12][sh_stride] or f16 [6][sh_stride])
  int sh_f16;
  uint32_t sh_stride;
  const uint32_t* bind_tet;   // [n_rest] or null (no rotation)
  const float4* bind_w;       // [n_rest] (MVC slot bits in .x)
  const uint2* split_meta;    // [children] (parent, tet)
  uint32_t num_tets;          // table rows [0, num_tets) are tet rotations
  int mvc;                    // table rows num_tets + slot are MVC rotations
  const float* table;         // [rotations * kShRotStride] or null
  uint32_t degree;
  float* out_pos;             // [count * 3] or null
  float* out_cov;             // [count * 6] or null
  float* out_opa;             // [count] or null
  float* out_sh;              // [count * 48] or null
};
size_t sh_basis_bytes();
cudaError_t launch_sh_basis(void* basis, cudaStream_t s);
cudaError_t launch_sh_rotators(uint32_t count, const float* rot, const void* basis, uint32_t degree,
                               float* table, cudaStream_t s);
cudaError_t launch_sh_apply(uint64_t n, float* sh, const float* table, uint32_t num_rot,
                            const uint32_t* index, uint32_t degree, uint32_t* bad, cudaStream_t s);
cudaError_t launch_export(const ExportArgs& a, cudaStream_t s);

// ---- Stage 4 (stage4_composite.cu) -------------------------------------------
struct CompositeArgs {
  const SplatRec* recs;
  const uint32_t* sorted_ids;
  const uint32_t* ranges;
  uint32_t width, height, tiles_x, tiles_y;
  uint32_t tile_w_log2, tile_h_log2;  // screen tile shape: 8x8, 16x16 or 32x16 pixels
  uint32_t pitch_px;        // RGBA8 row pitch in pixels
  float bg[4];
  uint32_t* out_rgba8;
  float4* out_f32;          // null when not requested
  FrameCounters* fc;
  uint32_t num_recs;        // splat records (ids at or above are rejected)
  uint32_t num_entries;     // sorted ids (ranges beyond are clamped)
};
cudaError_t launch_composite(const CompositeArgs& a, cudaStream_t s);

}  // namespace cgs
