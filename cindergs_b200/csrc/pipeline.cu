// Context, device residency, frame orchestration and the C ABI (include/cgs.h).
//
// Mirrors GpuPipelineState { GpuSceneState, GpuFrameArena }
// (render/gpu_state.rs:95-1343): the rest scene and cage topology stay
// resident and are re-uploaded only when the caller uploads them again; cage
// vertices are compared with the last upload so a stationary cage skips
// Stage 1; Stage 3's sorted lists are reused while the Stage 3 cache key
// (deform generation, camera, viewport, filter parameters) is unchanged;
// intermediate buffers grow by 1.5x and never shrink (gpu_pool.rs:43-49).
//
// A frame is enqueued with no host synchronisation inside it (the reference
// reads three counters back in the middle of every frame,
// gpu_state.rs:1020-1035). The tile-entry count is only known on the device,
// so the key buffers are sized from the counts of earlier frames with 30%
// headroom; every frame copies its counters to pinned host memory and is
// checked once its completion event has fired. A frame whose entries
// overflowed the buffers is binned and composited again with grown buffers if
// it is still the latest frame (so a readback never sees a truncated frame),
// otherwise it is reported by the next synchronising call. Status bits set by
// bounded device waits are reported as CGS_E_TIMEOUT.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cgs.h"
#include "field.h"
#include "kernels.h"

using namespace cgs;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;  // bytes
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  template <typename T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

// calculate_exponential_growth (render/gpu_pool.rs:43-49), in bytes.
size_t grow(size_t current, size_t needed) {
  if (needed <= current) return current;
  size_t scaled = (size_t)std::ceil((double)current * 1.5);
  size_t v = scaled > needed ? scaled : needed;
  return v < 256 ? 256 : v;
}

struct Stage3Key {
  uint64_t deform_generation = ~0ull;
  uint32_t view[16] = {};
  uint32_t fx = 0, fy = 0, cx = 0, cy = 0, near_bits = 0;
  uint32_t width = 0, height = 0;
  uint32_t mip = 0, min_opa = 0, min_rad = 0;
  uint32_t radix_bits = 0;
  bool operator==(const Stage3Key& o) const { return std::memcmp(this, &o, sizeof(*this)) == 0; }
};

uint32_t fbits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
float bitsf(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// Everything Stages 3 and 4 of one frame need, kept so that a frame whose
// tile entries overflowed the key buffers can be binned and composited again.
struct FrameDesc {
  uint32_t W = 0, H = 0, tiles_x = 0, tiles_y = 0, total_tiles = 0, pitch = 0;
  uint32_t tile_lw = 4, tile_lh = 4;  // log2 of the screen tile's width and height
  uint32_t n = 0, max_n = 0;
  bool split_possible = false, key64 = false, write_f32 = false;
  uint32_t tile_bits = 0, depth_bits = 0, sort_bits = 0, radix_bits = 8, depth_base_bits = 0;
  int entry_sort = CGS_SORT_AUTO;
  float bg[4] = {0, 0, 0, 1};
  uint32_t* out_rgba8 = nullptr;  // Stage 4 target when not the context's framebuffer
  uint32_t out_pitch = 0;         // its row pitch in pixels
};

// Per-frame counters copied to pinned host memory at the end of the frame.
struct HostCounters {
  FrameCounters fc;
  uint32_t split;
  uint32_t pad[3];
};

constexpr int kRing = 4;          // frames that may be in flight unchecked
constexpr int kMaxMarks = 24;     // profiled launches per frame

// Scratch layout of a frame (one memset): counters | deform look-back |
// binning look-back | radix histograms | radix tile counters.
// Screen tiles up to which the entries are sorted by the one-pass tile
// transpose (its per-chunk tile counts fit shared memory); beyond, by radix
// passes.
constexpr uint32_t kTransposeMaxTiles = 8 * kTransposeGroupTiles;

struct ScratchLayout {
  size_t def, bin, btile, hist, rtiles, shist, ttot, tbase, tscan, bytes;
  ScratchLayout(uint32_t n, uint32_t mn) {
    def = 256;
    bin = def + ((size_t)(n + 255) / 256) * 8 + 256;      // offsets scan look-back
    btile = bin + ((size_t)(mn + 4095) / 4096) * 8 + 256;  // staging start / count per 32 slots
    hist = btile + ((size_t)(mn + 31) / 32) * 8 * 8 + 256;  // (x 8 tile groups)
    rtiles = hist + 8 * 256 * 4;  // [0, 32): entry passes; [32, 40): splat passes
    shist = rtiles + 256;         // splat depth-key histograms, 4 passes x 256
    ttot = shist + 4 * 256 * 4;   // tile transpose: entries per screen tile
    tbase = ttot + (size_t)kTransposeMaxTiles * 4;   // first entry per screen tile
    tscan = tbase + (size_t)kTransposeMaxTiles * 4;  // look-back of that scan
    bytes = tscan + ((kTransposeMaxTiles + 4095) / 4096) * 8 + 256;
  }
};
constexpr uint32_t kSplatSortTileCtr = 32;

}  // namespace

struct cgs_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  // rest scene
  uint32_t n = 0;
  bool scene_ready = false;
  int sh_f16 = 0;
  DevBuf rest_pos, rest_cova, rest_covb, rest_sh;
  // cages
  uint32_t num_tets = 0, num_verts = 0;
  bool has_cages = false;
  DevBuf tet_elems, tet_inv_dm, cage_verts, bind_tet, bind_w;
  std::vector<float> last_verts;
  // polygon (MVC) cage: topology, rest and current vertices, exact bindings
  uint32_t mvc_V = 0, mvc_F = 0, mvc_nb = 0;
  bool mvc_ready = false;
  float mvc_h = 0.0f;
  DevBuf mvc_rest, mvc_verts, mvc_tris, mvc_vf_off, mvc_vf_list, mvc_list, mvc_wg, mvc_xf, mvc_R;
  std::vector<float> mvc_last_verts;
  // learned MVC field; with learned bindings the slots [0, mvc_nfb) keep
  // exact stored weights (the residual fallbacks), [mvc_nfb, mvc_nb) are
  // evaluated by the network every frame
  FieldState field;
  bool field_ready = false, mvc_learned = false;
  bool mvc_cached = false;  // learned slots keep the network's codes (1 KB each)
  uint32_t mvc_nfb = 0;
  DevBuf mvc_codes, mvc_code_pos;
  uint32_t mvc_nwg() const { return mvc_learned ? mvc_nfb : mvc_nb; }  // stored slots
  void mvc_unbind() {
    mvc_nb = 0;
    mvc_nfb = 0;
    mvc_learned = false;
    mvc_cached = false;
  }
  // Field inference over the learned slots: rest positions in, position and
  // gradient into mvc_xf at the same slots.
  FieldInfer field_infer_args(const float* proj) const {
    FieldInfer fi{};
    fi.net = field.net();
    fi.enc = field.enc_d.as<float>();
    fi.proj = proj;
    fi.gauss = mvc_list.as<uint32_t>();
    fi.points4 = rest_pos.as<float4>();
    fi.first = mvc_nfb;
    fi.count = mvc_nb - mvc_nfb;
    fi.out_first = mvc_nfb;
    fi.xf = mvc_xf.as<float4>();
    fi.codes = nullptr;
    fi.code_pos = nullptr;
    fi.status = field.status.as<uint32_t>();
    return fi;
  }
  bool deform_on() const { return has_cages || mvc_nb > 0; }
  MvcCage mvc_cage(bool rest) const {
    MvcCage c;
    c.V = mvc_V;
    c.F = mvc_F;
    c.verts = rest ? mvc_rest.as<float4>() : mvc_verts.as<float4>();
    c.tris = mvc_tris.as<uint4>();
    c.vf_off = mvc_vf_off.as<uint32_t>();
    c.vf_list = mvc_vf_list.as<uint32_t>();
    return c;
  }
  bool verts_uploaded = false;
  bool deformed_valid = false;
  uint64_t deform_generation = 1;
  uint32_t last_split_bits = 0xFFFFFFFFu, last_mip_bits = 0xFFFFFFFFu;
  // arena
  DevBuf tet_J, tet_R, tet_S, def_pos, def_cova, def_covb, split_meta, persist;
  DevBuf recs, offsets, scratch, ranges, keys[2], ids[2], depths[2], radix_lb[2];
  DevBuf fb_rgba8, fb_f32;
  DevBuf prim[4];  // scratch for the stand-alone scan/sort entry points
  // SH coefficient rotation (cgs_sh_rotate, cgs_export_deformed): the band
  // bases (built once), the per-rotation band matrices and the export chunk
  DevBuf sh_basis, sh_table, sh_stage;
  bool sh_basis_ready = false;
  // device cage springs (cgs_springs_*): per-vertex rest (+ cage index),
  // velocity and pin; per-cage parameters and planes
  DevBuf spr_rest, spr_vel, spr_pin, spr_cages, spr_planes;
  std::vector<cgs_spring_cage> spr_host;
  std::vector<float> spr_centroid;  // 3 per cage
  uint32_t spr_V = 0;
  bool spr_ready = false;
  // splat depth sort (Stage 3): keys/ids ping-pong and look-back pair
  DevBuf skeys[2], sids[2], splat_lb[2];
  uint32_t splat_cap = 0;  // slots those buffers hold; fixed between reallocations
  int splat_parity = 0;
  int s3_order_src = 0;    // buffer holding the latest Stage 3's splat order
  bool s3_transpose = false;  // the latest Stage 3 sorted by the tile transpose
  DevBuf cmat;             // tile transpose: [tiles][chunks] counts / first entries
  uint32_t entry_cap = 0;       // capacity of the key/id buffers (entries)
  uint32_t radix_lb_tiles = 0;  // tiles the radix look-back buffers cover
  uint32_t radix_lb_bits = 0;
  int radix_parity = 0;
  HostCounters* h_ring = nullptr;  // pinned [kRing]
  // Buffer reallocations and state changes (uploads, bindings), for the
  // validity of captured graphs, which hold device pointers and launch shapes.
  uint64_t alloc_epoch = 0, state_epoch = 0;
  // multi-view steps (cgs_execute_views)
  HostCounters* h_views = nullptr;  // pinned [views_cap]
  uint32_t views_cap = 0;
  cudaGraphExec_t views_exec = nullptr;
  std::vector<unsigned char> views_key;
  int views_radix_parity = 0, views_splat_parity = 0;  // host parities after a replay
  cudaEvent_t views_ev[2] = {};
  // Pinned staging of the per-frame uploads (cage vertices): a copy from
  // pageable memory synchronises the stream before it starts, one from a
  // pinned slot is enqueued behind the frames in flight. A slot is refilled
  // once the copy that last read it has completed (its event).
  struct UploadRing {
    void* p[kRing] = {};
    size_t cap[kRing] = {};
    cudaEvent_t ev[kRing] = {};
    bool pending[kRing] = {};
    int next = 0;
  } up;
  uint32_t* h_misc = nullptr;      // pinned scratch for the primitives
  // Stage 3 cache
  bool s3_valid = false;
  Stage3Key s3_key;
  uint32_t s3_entries = 0, s3_surviving = 0, s3_active = 0;
  int s3_key64 = 0, s3_src = 0;
  uint32_t s3_depth_bits = 0;
  // last frame
  FrameDesc last_desc;
  uint32_t last_w = 0, last_h = 0, last_pitch = 0, last_active = 0, last_tiles = 0;
  bool last_f32 = false, frame_done = false;
  int latest_slot = -1;
  uint64_t frame_seq = 0;        // frames enqueued by cgs_execute_frame
  uint64_t rerun_count = 0;      // Stage 3/4 re-runs after an entry overflow
  uint64_t rerun_seq = 0;        // frame number of the latest re-run
  // Asynchronous RGBA8 readbacks (cgs_readback_rgba8_async): a device
  // snapshot of the framebuffer per slot, copied to the host on rb_stream.
  struct Readback {
    DevBuf stage;
    cudaEvent_t ready = nullptr, done = nullptr;
    uint64_t ticket = 0, frame_seq = 0, reruns = 0;
    uint8_t* dst = nullptr;
    uint32_t W = 0, H = 0;
    int frame_slot = -1;
    bool pending = false;
  } rb[2];
  cudaStream_t rb_stream = nullptr;
  uint64_t rb_tickets = 0;
  // in-flight frames
  struct Pending {
    uint64_t seq = 0;  // frame number (cgs_execute_frame calls)
    bool used = false, stage3_ran = false, profiled = false, need_deform = false;
    bool split_possible = false, key64 = false;
    uint32_t n = 0, cap = 0, sort_passes = 0, splat_passes = 0, total_tiles = 0, W = 0, H = 0;
    uint32_t bin_launches = 0, sort_launches = 0;
    bool write_f32 = false;
    cudaEvent_t done = nullptr;
    cudaEvent_t kev[2 * kMaxMarks] = {};
    int kid[kMaxMarks] = {};
    int kcount = 0;
    // what it takes to render the frame again after its tile entries
    // overflowed while later frames were in flight: its arguments and the
    // cage vertices it deformed with (device snapshots)
    cgs_camera cam{};
    cgs_compositor comp{};
    cgs_frame_params params{};
    DevBuf verts_snap, mvc_snap;
    size_t verts_bytes = 0, mvc_bytes = 0;
    bool overflowed = false;
  } ring[kRing];
  // The arena holds an earlier frame's intermediates (a re-render), not the
  // last frame's, until the next frame.
  bool arena_rerendered = false;
  int next_slot = 0;
  int cur = -1;              // slot of the frame being enqueued
  bool kprof = false;
  cgs_kernel_profile kp_acc{};
  int sticky = CGS_OK;       // error found while checking an older frame
  bool poisoned = false;     // kStatusPoisoned seen: frames refuse to run
  std::string sticky_msg;

  void kbegin(int id) {
    if (!kprof || cur < 0) return;
    Pending& p = ring[cur];
    if (p.kcount >= kMaxMarks) return;
    p.kid[p.kcount] = id;
    cudaEventRecord(p.kev[2 * p.kcount], stream);
  }
  void kend() {
    if (!kprof || cur < 0) return;
    Pending& p = ring[cur];
    if (p.kcount >= kMaxMarks) return;
    cudaEventRecord(p.kev[2 * p.kcount + 1], stream);
    ++p.kcount;
  }

  int fail(int code, const std::string& msg) {
    err = msg;
    return code;
  }
  int cuda_fail(cudaError_t e, const char* what) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return CGS_E_CUDA;
  }
  // Device bytes the arena may hold (cgs_ctx_set_device_budget; 0 = no
  // limit) and the bytes its growable buffers hold now.
  uint64_t budget = 0, held = 0;
  cgs_launch_shape shape{};  // cgs_ctx_set_launch_shape (zeros: defaults)
  int ensure(DevBuf& b, size_t bytes, const char* what) {
    if (bytes <= b.cap && b.p) return CGS_OK;
    size_t nb = grow(b.cap, bytes);
    if (budget && held - b.cap + nb > budget)
      return fail(CGS_E_OOM, std::string("device memory budget of ") + std::to_string(budget) +
                                 " bytes exceeded by " + what + " (" + std::to_string(nb) +
                                 " bytes with " + std::to_string(held - b.cap) + " held)");
    if (b.p) {
      cudaStreamSynchronize(stream);
      cudaFree(b.p);
      held -= b.cap;
      b.p = nullptr;
      b.cap = 0;
    }
    ++alloc_epoch;
    cudaError_t e = cudaMalloc(&b.p, nb);
    if (e != cudaSuccess) {
      b.p = nullptr;
      return fail(CGS_E_OOM, std::string("device allocation failed for ") + what + " (" +
                                 std::to_string(nb) + " bytes): " + cudaGetErrorString(e));
    }
    b.cap = nb;
    held += nb;
    return CGS_OK;
  }
  int take_sticky() {
    if (sticky == CGS_OK) return CGS_OK;
    const int s = sticky;
    sticky = CGS_OK;
    return fail(s, sticky_msg);
  }
};

#define CGS_CUDA(call, what)                 \
  do {                                       \
    cudaError_t e_ = (call);                 \
    if (e_ != cudaSuccess) return ctx->cuda_fail(e_, what); \
  } while (0)
#define CGS_TRY(call)          \
  do {                         \
    int r_ = (call);           \
    if (r_ != CGS_OK) return r_; \
  } while (0)

namespace {

// Key buffers and radix look-back buffers for `cap` entries.
int ensure_entry_buffers(cgs_ctx* ctx, uint32_t cap, bool key64, uint32_t radix_bits) {
  const size_t ecap = cap ? cap : 1;
  for (int k = 0; k < 2; ++k) {
    CGS_TRY(ctx->ensure(ctx->keys[k], ecap * 4, "sort keys"));
    CGS_TRY(ctx->ensure(ctx->ids[k], ecap * 4, "sort values"));
    if (key64) CGS_TRY(ctx->ensure(ctx->depths[k], ecap * 4, "sort depths"));
  }
  const uint32_t tiles = sort_tiles((uint32_t)ecap);
  if (tiles != ctx->radix_lb_tiles || radix_bits != ctx->radix_lb_bits || !ctx->radix_lb[0].p) {
    const size_t bytes = (size_t)tiles * (1u << radix_bits) * 8;  // 64-bit look-back words
    for (int k = 0; k < 2; ++k) {
      CGS_TRY(ctx->ensure(ctx->radix_lb[k], bytes, "radix look-back"));
      CGS_CUDA(cudaMemsetAsync(ctx->radix_lb[k].p, 0, bytes, ctx->stream), "clear look-back");
    }
    ctx->radix_lb_tiles = tiles;
    ctx->radix_lb_bits = radix_bits;
    ctx->radix_parity = 0;
  }
  return CGS_OK;
}

// Depth-key buffers and look-back pair of the splat sort for `mn` slots. The
// capacity (and so the sort's grid) only changes on reallocation, when both
// look-back buffers are cleared: the passes clear the buffer they do not use
// over the whole grid, which keeps them clean only while the grid is fixed.
int ensure_splat_buffers(cgs_ctx* ctx, uint32_t mn) {
  if (mn <= ctx->splat_cap && ctx->splat_lb[0].p) return CGS_OK;
  const uint64_t want = std::max<uint64_t>((uint64_t)mn + mn / 4, 4096);
  const uint32_t cap = (uint32_t)std::min<uint64_t>((want + 4095) / 4096 * 4096, 0xFFFFF000ull);
  for (int k = 0; k < 2; ++k) {
    CGS_TRY(ctx->ensure(ctx->skeys[k], (size_t)cap * 4, "splat depth keys"));
    CGS_TRY(ctx->ensure(ctx->sids[k], (size_t)cap * 4, "splat order"));
  }
  const size_t bytes = (size_t)sort_tiles(cap) * 256 * 4;
  for (int k = 0; k < 2; ++k) {
    CGS_TRY(ctx->ensure(ctx->splat_lb[k], bytes, "splat sort look-back"));
    CGS_CUDA(cudaMemsetAsync(ctx->splat_lb[k].p, 0, bytes, ctx->stream), "clear look-back");
  }
  ctx->splat_cap = cap;
  ctx->splat_parity = 0;
  return CGS_OK;
}

// Enqueues Stage 3 for `d` with the current key-buffer capacity:
//   1. stable radix sort of Stage 2's per-splat depth keys (skipped with
//      `sort_splats` false: a re-run of the same frame reuses its order);
//   2. binning in that order (k_bin): entries leave ordered by depth;
//   3. stable radix sort of the entries on their tile bits only;
//   4. tile ranges.
// *result_src receives the buffer holding the sorted lists; *passes and
// *splat_passes the number of radix passes over entries and splats.
int enqueue_stage3(cgs_ctx* ctx, const FrameDesc& d, const ScratchLayout& L, int* result_src,
                   uint32_t* passes, uint32_t* splat_passes, bool sort_splats,
                   uint32_t* bin_launches = nullptr, uint32_t* sort_launches = nullptr) {
  cudaStream_t s = ctx->stream;
  char* sc = ctx->scratch.as<char>();
  FrameCounters* fc = (FrameCounters*)sc;
  uint32_t* d_split = ctx->persist.as<uint32_t>();
  uint32_t* d_hist = (uint32_t*)(sc + L.hist);
  uint32_t* rtiles = (uint32_t*)(sc + L.rtiles);
  const bool transpose =
      d.entry_sort == CGS_SORT_TRANSPOSE && !d.key64 && d.total_tiles <= kTransposeMaxTiles;
  ctx->s3_transpose = transpose;
  if (!transpose) {
    ctx->kbegin(CGS_K_CLEAR);
    CGS_CUDA(cudaMemsetAsync(ctx->ranges.p, 0, (size_t)d.total_tiles * 8, s), "clear ranges");
    ctx->kend();
  }
  const uint32_t dbits = d.key64 ? 32u : d.depth_bits;
  *splat_passes = 0;
  if (sort_splats) {
    uint32_t* shist = (uint32_t*)(sc + L.shist);
    ctx->kbegin(CGS_K_SPLAT_SORT);
    // balanced digits of at most 8 bits (19 depth bits -> 7 + 6 + 6)
    const uint32_t spp = (dbits + 7) / 8, srb = std::max(4u, (dbits + spp - 1) / spp);
    CGS_CUDA(launch_histogram(ctx->skeys[0].as<uint32_t>(), &fc->active, ctx->splat_cap, 0, dbits,
                              srb, shist, s),
             "splat histogram");
    SortArgs so{};
    so.keys[0] = ctx->skeys[0].as<uint32_t>();
    so.keys[1] = ctx->skeys[1].as<uint32_t>();
    so.vals[0] = ctx->sids[0].as<uint32_t>();
    so.vals[1] = ctx->sids[1].as<uint32_t>();
    so.n_ptr = &fc->active;
    so.capacity = ctx->splat_cap;
    so.first_bit = 0;
    so.num_bits = dbits;
    so.radix_bits = srb;
    so.hist = shist;
    // depth digits of splats in index order are spread over all values
    so.smem_mask = ~0u;
    so.status2[0] = ctx->splat_lb[0].p;
    so.status2[1] = ctx->splat_lb[1].p;
    so.parity = &ctx->splat_parity;
    // the digit width follows the frame's depth bits (8 at 360p, 7 at 1080p):
    // clear the full 256-word stride so a narrower sort leaves no stale words
    so.lb_stride = 256;
    so.tile_ctr = rtiles + kSplatSortTileCtr;
    so.status_word = &fc->status;
    so.src = 0;
    CGS_CUDA(run_radix_sort(so, &ctx->s3_order_src, s), "splat sort");
    ctx->kend();
    *splat_passes = sort_passes(dbits, srb);
  }
  BinArgs b{};
  b.blocks_per_sm = ctx->shape.bin_blocks_per_sm;
  b.recs = ctx->recs.as<SplatRec>();
  b.order_keys = ctx->skeys[ctx->s3_order_src].as<uint32_t>();
  b.order_ids = ctx->sids[ctx->s3_order_src].as<uint32_t>();
  b.split_count = d.split_possible ? d_split : nullptr;
  b.n_rest = d.n;
  b.max_n = d.max_n;
  b.width = d.W;
  b.height = d.H;
  b.tiles_x = d.tiles_x;
  b.tiles_y = d.tiles_y;
  b.tile_w_log2 = d.tile_lw;
  b.tile_h_log2 = d.tile_lh;
  b.offsets = ctx->offsets.as<uint32_t>();
  b.tile_stage = (uint32_t*)(sc + L.btile);
  b.tile_count = b.tile_stage + (size_t)8 * ((d.max_n + 31) / 32);
  b.fc = fc;
  b.key64 = d.key64;
  b.depth_bits = d.depth_bits;
  b.stage_keys = ctx->keys[1].as<uint32_t>();
  b.keys = ctx->keys[0].as<uint32_t>();
  b.depths = d.key64 ? ctx->depths[0].as<uint32_t>() : nullptr;
  b.ids = ctx->ids[0].as<uint32_t>();
  b.hist = d_hist;
  b.radix_bits = d.radix_bits;
  b.tile_bits = d.tile_bits;
  b.entry_cap = ctx->entry_cap;
  b.records = transpose ? 1 : 0;
  b.group_shift = 11;  // kTransposeGroupTiles = 2^11
  b.groups = transpose ? (d.total_tiles + kTransposeGroupTiles - 1) / kTransposeGroupTiles : 1u;
  // Direct mode (radix path): one launch counts, scans (look-back over the
  // 32-slot tiles) and writes every entry at its place in depth order. The
  // tile transpose stages records and then scans the per-slot counts in place
  // (first entries, entry total).
  const uint32_t nwt = (d.max_n + 31) / 32;
  b.lookback = reinterpret_cast<unsigned long long*>(b.tile_stage + 2 * (size_t)nwt);
  ctx->kbegin(CGS_K_BIN);
  CGS_CUDA(launch_bin_count(b, s), "bin count launch");
  if (transpose) {
    CGS_CUDA(launch_scan_u32(b.offsets, b.offsets, d.max_n, &fc->entries,
                             (unsigned long long*)(sc + L.bin), &fc->tile_ctr[3], &fc->status, s),
             "offsets scan launch");
  }
  ctx->kend();
  if (bin_launches) *bin_launches = transpose ? 2u : 1u;
  if (transpose) {
    // one-pass stable counting sort of the staged records by tile
    const uint32_t target = 296;  // chunks: two per SM
    uint32_t m = 8 * ((nwt + 8 * target - 1) / (8 * target));
    m = std::min<uint32_t>(std::max<uint32_t>(m, 8u), 2040u);
    TransposeArgs ta{};
    ta.records = ctx->keys[1].as<uint32_t>();
    ta.tile_stage = b.tile_stage;
    ta.tile_count = b.tile_count;
    ta.order_ids = b.order_ids;
    ta.num_wtiles = nwt;
    ta.chunk_wtiles = m;
    ta.num_chunks = (nwt + m - 1) / m;
    ta.num_tiles = d.total_tiles;
    ta.groups = b.groups;
    ta.group_tiles = kTransposeGroupTiles;
    CGS_TRY(ctx->ensure(ctx->cmat, (size_t)d.total_tiles * ta.num_chunks * 4, "tile transpose counts"));
    ta.cmat = ctx->cmat.as<uint32_t>();
    ta.totals = (uint32_t*)(sc + L.ttot);
    ta.tile_base = (uint32_t*)(sc + L.tbase);
    ta.ranges = ctx->ranges.as<uint32_t>();
    ta.ids_out = ctx->ids[0].as<uint32_t>();
    ta.capacity = ctx->entry_cap;
    ta.status_word = &fc->status;
    *passes = 0;
    ctx->kbegin(CGS_K_ENTRY_SORT);
    CGS_CUDA(launch_chunk_counts(ta, s), "chunk counts launch");
    CGS_CUDA(launch_scan_u32(ta.totals, (uint32_t*)(sc + L.tbase), d.total_tiles, &fc->tile_ctr[5],
                             (unsigned long long*)(sc + L.tscan), &fc->tile_ctr[4], &fc->status, s),
             "tile totals scan launch");
    CGS_CUDA(launch_column_scan(ta, s), "column scan launch");
    CGS_CUDA(launch_chunk_place(ta, s), "chunk place launch");
    ctx->kend();
    if (sort_launches) *sort_launches = 4;
    *result_src = 0;
    return CGS_OK;
  }
  const uint32_t* n_ptr = &fc->entries;
  *passes = sort_passes(d.tile_bits, d.radix_bits);
  // Entries arrive in (depth, splat) order; a stable sort on the tile bits
  // (above the depth bits of a 32-bit key, or the whole tile word of the
  // 64-bit layout, whose depth word travels as a second payload) completes
  // the (tile, depth, splat) order.
  SortArgs sa{};
  sa.keys[0] = ctx->keys[0].as<uint32_t>();
  sa.keys[1] = ctx->keys[1].as<uint32_t>();
  sa.vals[0] = ctx->ids[0].as<uint32_t>();
  sa.vals[1] = ctx->ids[1].as<uint32_t>();
  if (d.key64) {
    sa.vals2[0] = ctx->depths[0].as<uint32_t>();
    sa.vals2[1] = ctx->depths[1].as<uint32_t>();
  }
  sa.n_ptr = n_ptr;
  sa.capacity = ctx->entry_cap;
  sa.first_bit = d.key64 ? 0u : d.depth_bits;
  sa.num_bits = d.tile_bits;
  sa.radix_bits = d.radix_bits;
  sa.status2[0] = ctx->radix_lb[0].p;
  sa.status2[1] = ctx->radix_lb[1].p;
  // 64-bit look-back words only when the buffers may hold more than 2^30
  // entries (32-bit words carry 30-bit counts); the width follows the
  // capacity, whose every change clears the look-back buffers
  sa.wide_lookback = ctx->entry_cap > (1u << 30);
  sa.parity = &ctx->radix_parity;
  sa.tile_ctr = rtiles;
  sa.status_word = &fc->status;
  sa.hist = d_hist;
  // the last pass finds the tile ranges (the ranges were zeroed above)
  const bool pass_ranges = *passes > 0;
  if (pass_ranges) {
    sa.ranges = ctx->ranges.as<uint32_t>();
    sa.tile_shift = d.key64 ? 0u : d.depth_bits;
    sa.num_tiles = d.total_tiles;
  }
  sa.src = 0;
  // The entries' first digit (the low tile bits) differs from lane to lane,
  // so that pass ranks with shared-memory peer masks (measured faster than
  // per-bit ballots: 0.310 vs 0.329 ms for both passes at 26M entries);
  // after it a warp's keys mostly share their higher digits, which
  // __match_any_sync groups more cheaply.
  sa.ballot_mask = 1u;
  sa.smem_mask = 1u;
  ctx->kbegin(CGS_K_ENTRY_SORT);
  CGS_CUDA(run_radix_sort(sa, result_src, s), "radix sort");
  if (sort_launches) *sort_launches = *passes;  // one onesweep launch per pass
  ctx->kend();
  ctx->kbegin(CGS_K_TILE_RANGES);
  if (pass_ranges)
    CGS_CUDA(launch_ranges_fixup(ctx->ranges.as<uint32_t>(), d.total_tiles, s), "ranges fix-up");
  else
    CGS_CUDA(launch_tile_ranges(ctx->keys[*result_src].as<uint32_t>(), d.key64 ? 0u : d.depth_bits,
                                n_ptr, ctx->entry_cap, d.total_tiles, ctx->ranges.as<uint32_t>(),
                                ctx->shape.ranges_blocks, s),
             "ranges launch");
  ctx->kend();
  return CGS_OK;
}

int enqueue_stage4(cgs_ctx* ctx, const FrameDesc& d, int result_src) {
  char* sc = ctx->scratch.as<char>();
  CompositeArgs c{};
  c.recs = ctx->recs.as<SplatRec>();
  c.sorted_ids = ctx->ids[result_src].as<uint32_t>();
  c.ranges = ctx->ranges.as<uint32_t>();
  c.width = d.W;
  c.height = d.H;
  c.tiles_x = d.tiles_x;
  c.tiles_y = d.tiles_y;
  c.tile_w_log2 = d.tile_lw;
  c.tile_h_log2 = d.tile_lh;
  c.pitch_px = d.out_rgba8 ? d.out_pitch : d.pitch;
  std::memcpy(c.bg, d.bg, 16);
  c.out_rgba8 = d.out_rgba8 ? d.out_rgba8 : ctx->fb_rgba8.as<uint32_t>();
  c.out_f32 = d.write_f32 ? ctx->fb_f32.as<float4>() : nullptr;
  c.fc = (FrameCounters*)sc;
  c.num_recs = d.max_n ? d.max_n : 1u;
  c.num_entries = ctx->entry_cap;
  ctx->kbegin(CGS_K_COMPOSITE);
  CGS_CUDA(launch_composite(c, ctx->stream), "composite launch");
  ctx->kend();
  return CGS_OK;
}

// Re-runs Stages 3 and 4 of the latest frame after its entries overflowed the
// key buffers (capacity already grown), synchronously.
int rerun_stage34(cgs_ctx* ctx, uint32_t entries) {
  const FrameDesc& d = ctx->last_desc;
  ctx->entry_cap = (uint32_t)std::min<uint64_t>((uint64_t)entries + entries / 4 + 4096, (uint64_t)kMaxEntryCap);
  CGS_TRY(ensure_entry_buffers(ctx, ctx->entry_cap, d.key64, d.radix_bits));
  const ScratchLayout L(d.n, d.max_n ? d.max_n : 1u);
  char* sc = ctx->scratch.as<char>();
  // keep fc->surviving and fc->active (Stage 2's words); clear the Stage 3 words
  CGS_CUDA(cudaMemsetAsync(sc + 8, 0, sizeof(FrameCounters) - 8, ctx->stream), "clear counters");
  CGS_CUDA(cudaMemsetAsync(sc + L.bin, 0, L.bytes - L.bin, ctx->stream), "clear scratch");
  const bool kp = ctx->kprof;
  const int cur = ctx->cur;
  ctx->kprof = false;
  ctx->cur = -1;
  int src = 0;
  uint32_t passes = 0, splat_passes = 0;
  int rc = enqueue_stage3(ctx, d, L, &src, &passes, &splat_passes, false);
  if (rc == CGS_OK) rc = enqueue_stage4(ctx, d, src);
  ctx->kprof = kp;
  ctx->cur = cur;
  CGS_TRY(rc);
  CGS_CUDA(cudaMemcpyAsync(&ctx->h_ring[ctx->latest_slot].fc, sc, sizeof(FrameCounters),
                           cudaMemcpyDeviceToHost, ctx->stream), "read counters");
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "stage 3 re-run");
  ctx->s3_src = src;
  ++ctx->rerun_count;
  ctx->rerun_seq = ctx->ring[ctx->latest_slot].seq;
  const FrameCounters& f = ctx->h_ring[ctx->latest_slot].fc;
  if (f.status & kStatusCapacity) return ctx->fail(CGS_E_CAPACITY, "tile entries still exceed the grown buffers");
  return CGS_OK;
}

// Checks frame slot `k` once it has finished: status bits, capacity, Stage 3
// cache bookkeeping and the kernel profile. `block` waits for it.
int check_slot(cgs_ctx* ctx, int k, bool block) {
  cgs_ctx::Pending& p = ctx->ring[k];
  if (!p.used) return CGS_OK;
  if (block) {
    CGS_CUDA(cudaEventSynchronize(p.done), "frame completion");
  } else {
    const cudaError_t q = cudaEventQuery(p.done);
    if (q == cudaErrorNotReady) return CGS_OK;
    if (q != cudaSuccess) return ctx->cuda_fail(q, "frame completion");
  }
  p.used = false;
  const HostCounters& h = ctx->h_ring[k];
  uint32_t entries = h.fc.entries;
  uint32_t status = h.fc.status;
  if (status & (kStatusLookbackTimeout | kStatusBarrierTimeout)) {
    ctx->sticky = CGS_E_TIMEOUT;
    ctx->sticky_msg = "a bounded device-side wait gave up during a frame";
  }
  if (status & kStatusPoisoned) ctx->poisoned = true;
  if (p.stage3_ran && (status & kStatusCapacity || entries > p.cap)) {
    if (k == ctx->latest_slot) {
      CGS_TRY(rerun_stage34(ctx, entries));
      entries = ctx->h_ring[k].fc.entries;
    } else {
      // a later frame is in flight: its pixels are rendered again if a
      // readback waits for them (rerender_slot); the buffers grow now
      p.overflowed = true;
      ctx->entry_cap = std::max(ctx->entry_cap,
                                (uint32_t)std::min<uint64_t>((uint64_t)entries * 13 / 10 + 4096, (uint64_t)kMaxEntryCap));
    }
  } else if (p.stage3_ran && entries > ctx->entry_cap / 10 * 8) {
    // keep 25% headroom for the next frames
    ctx->entry_cap = (uint32_t)std::min<uint64_t>((uint64_t)entries * 13 / 10 + 4096, (uint64_t)kMaxEntryCap);
  }
  if (k == ctx->latest_slot) {
    if (p.stage3_ran) {
      ctx->s3_entries = entries;
      ctx->s3_surviving = h.fc.surviving;
      ctx->s3_active = p.n + (p.split_possible ? h.split : 0u);
    }
    ctx->last_active = p.n + (p.split_possible ? h.split : 0u);
  }
  if (p.profiled) {
    cgs_kernel_profile& kp = ctx->kp_acc;
    for (int c = 0; c < p.kcount; ++c) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, p.kev[2 * c], p.kev[2 * c + 1]);
      kp.ms[p.kid[c]] += ms;
      kp.launches[p.kid[c]] += p.kid[c] == CGS_K_ENTRY_SORT   ? p.sort_launches
                               : p.kid[c] == CGS_K_SPLAT_SORT ? 1u + p.splat_passes
                               : p.kid[c] == CGS_K_BIN        ? p.bin_launches
                                                              : 1u;
    }
    const uint64_t A = p.n + (p.split_possible ? h.split : 0u);
    const uint64_t S = h.fc.surviving, E = p.stage3_ran ? entries : 0, T = ctx->num_tets;
    const uint64_t shb = ctx->sh_f16 ? 96 : 192;
    if (p.need_deform && ctx->mvc_nwg()) {
      // stored bindings: (w, grad w) per cage vertex in, position + F out
      kp.alg_bytes[CGS_K_MVC] += (uint64_t)ctx->mvc_nwg() * ((uint64_t)ctx->mvc_V * 16 + 48);
    }
    if (p.need_deform && ctx->mvc_learned && ctx->mvc_nb > ctx->mvc_nfb) {
      // learned slots: slot -> Gaussian, rest position in, position + F out;
      // four streams (value and three tangents) through the hidden layers
      const uint64_t L = ctx->mvc_nb - ctx->mvc_nfb;
      if (ctx->mvc_cached) {
        // cached code (value + 3 tangents, 128 bf16 each) in
        kp.alg_bytes[CGS_K_FIELD] += L * (16 + 48 + 4 * kFieldHid * 2);
      } else {
        kp.alg_bytes[CGS_K_FIELD] += L * (4 + 16 + 48);
        kp.alg_flops[CGS_K_FIELD] +=
            L * 4 * 2 * ((uint64_t)kFieldIn * kFieldHid + 3ull * kFieldHid * kFieldHid);
      }
    }
    if (p.need_deform) {
      // tet transforms (fused into the deform launch): 16 B elements + 36 B
      // D_m^-1 + 48 B corner vertices in, J, R (36 B each) and sigma_1 out
      kp.alg_bytes[CGS_K_DEFORM] += T * (16 + 36 + 48 + 76) + (uint64_t)p.n * 60 + A * 40 +
                                    (A - p.n) * 8;
    }
    kp.alg_bytes[CGS_K_PROJECT] += A * 40 + S * (shb + 48) + (A - S) * 16 + (p.stage3_ran ? A * 8 : 0);
    if (p.stage3_ran) {
      kp.alg_bytes[CGS_K_SPLAT_SORT] += A * 4 + (uint64_t)p.splat_passes * A * 16;
      kp.alg_bytes[CGS_K_BIN] += A * 44 + E * (p.key64 ? 12 : 8);
      if (p.sort_passes) {
        kp.alg_bytes[CGS_K_ENTRY_SORT] += (uint64_t)p.sort_passes * E * (p.key64 ? 24 : 16);
        kp.alg_bytes[CGS_K_TILE_RANGES] += E * 4 + (uint64_t)p.total_tiles * 8;
      } else {
        // tile transpose: records read twice (counts, placement), splat
        // index gathered and written once
        kp.alg_bytes[CGS_K_ENTRY_SORT] += E * 16 + (uint64_t)p.total_tiles * 8;
      }
    }
    // The compositor stops a tile once every pixel has saturated, so its
    // algorithmic traffic is the records it actually gathered (48 B + the
    // 4-byte id each), the ranges and the framebuffer.
    kp.alg_bytes[CGS_K_COMPOSITE] += (uint64_t)h.fc.fetched * 52 + (uint64_t)p.total_tiles * 8 +
                                     (uint64_t)p.W * p.H * (p.write_f32 ? 20 : 4);
  }
  return CGS_OK;
}

int drain(cgs_ctx* ctx, bool block) {
  for (int i = 1; i <= kRing; ++i) {
    const int k = (ctx->next_slot + i - 1) % kRing;  // oldest first
    CGS_TRY(check_slot(ctx, k, block));
  }
  return CGS_OK;
}

// Enqueues a host -> device copy of `bytes` through the next pinned upload
// slot; fill(slot) writes the bytes into the slot.
template <typename Fill>
int staged_upload(cgs_ctx* ctx, void* dst, size_t bytes, Fill fill, const char* what) {
  auto& r = ctx->up;
  const int k = r.next;
  r.next = (k + 1) % kRing;
  if (r.pending[k]) {
    CGS_CUDA(cudaEventSynchronize(r.ev[k]), what);
    r.pending[k] = false;
  }
  if (r.cap[k] < bytes) {
    if (r.p[k]) cudaFreeHost(r.p[k]);
    r.p[k] = nullptr;
    r.cap[k] = 0;
    CGS_CUDA(cudaHostAlloc(&r.p[k], bytes, cudaHostAllocDefault), what);
    r.cap[k] = bytes;
  }
  if (!r.ev[k]) CGS_CUDA(cudaEventCreateWithFlags(&r.ev[k], cudaEventDisableTiming), what);
  fill(r.p[k]);
  CGS_CUDA(cudaMemcpyAsync(dst, r.p[k], bytes, cudaMemcpyHostToDevice, ctx->stream), what);
  CGS_CUDA(cudaEventRecord(r.ev[k], ctx->stream), what);
  r.pending[k] = true;
  return CGS_OK;
}

}  // namespace

#pragma GCC visibility push(default)
extern "C" {

const char* cgs_version(void) { return "cindergs_b200 0.1.0 (sm_100a)"; }

int cgs_ctx_create(int device, void* stream, cgs_ctx** out_ctx) {
  if (!out_ctx) return CGS_E_ARG;
  *out_ctx = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return CGS_E_CUDA;
  if (device < 0 || device >= ndev) return CGS_E_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return CGS_E_CUDA;
  cgs_ctx* ctx = new cgs_ctx();
  ctx->device = device;
  if (stream) {
    ctx->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete ctx;
      return CGS_E_CUDA;
    }
    ctx->own_stream = true;
  }
  if (cudaMallocHost(&ctx->h_ring, kRing * sizeof(HostCounters)) != cudaSuccess ||
      cudaMallocHost(&ctx->h_misc, 64) != cudaSuccess) {
    delete ctx;
    return CGS_E_OOM;
  }
  std::memset(ctx->h_ring, 0, kRing * sizeof(HostCounters));
  for (auto& p : ctx->ring) {
    if (cudaEventCreateWithFlags(&p.done, cudaEventDisableTiming) != cudaSuccess) {
      delete ctx;
      return CGS_E_CUDA;
    }
    for (auto& e : p.kev)
      if (cudaEventCreate(&e) != cudaSuccess) {
        delete ctx;
        return CGS_E_CUDA;
      }
  }
  // persistent words: [0] split count
  if (ctx->ensure(ctx->persist, 256, "persistent words") != CGS_OK ||
      cudaMemset(ctx->persist.p, 0, 256) != cudaSuccess) {
    delete ctx;
    return CGS_E_OOM;
  }
  *out_ctx = ctx;
  return CGS_OK;
}

int cgs_ctx_destroy(cgs_ctx* ctx) {
  if (!ctx) return CGS_E_ARG;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto& p : ctx->ring) {
    if (p.done) cudaEventDestroy(p.done);
    for (auto& e : p.kev)
      if (e) cudaEventDestroy(e);
  }
  if (ctx->h_ring) cudaFreeHost(ctx->h_ring);
  if (ctx->h_misc) cudaFreeHost(ctx->h_misc);
  for (int k = 0; k < kRing; ++k) {
    if (ctx->up.p[k]) cudaFreeHost(ctx->up.p[k]);
    if (ctx->up.ev[k]) cudaEventDestroy(ctx->up.ev[k]);
  }
  if (ctx->rb_stream) {
    cudaStreamSynchronize(ctx->rb_stream);
    cudaStreamDestroy(ctx->rb_stream);
  }
  for (auto& r : ctx->rb) {
    if (r.ready) cudaEventDestroy(r.ready);
    if (r.done) cudaEventDestroy(r.done);
  }
  if (ctx->views_exec) cudaGraphExecDestroy(ctx->views_exec);
  if (ctx->h_views) cudaFreeHost(ctx->h_views);
  for (auto& e : ctx->views_ev)
    if (e) cudaEventDestroy(e);
  cudaStream_t s = ctx->stream;
  bool own = ctx->own_stream;
  delete ctx;
  if (own) cudaStreamDestroy(s);
  return CGS_OK;
}

const char* cgs_last_error(const cgs_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int cgs_ctx_synchronize(cgs_ctx* ctx) {
  if (!ctx) return CGS_E_ARG;
  cudaSetDevice(ctx->device);
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
  CGS_TRY(drain(ctx, true));
  return ctx->take_sticky();
}

int cgs_ctx_set_launch_shape(cgs_ctx* ctx, const cgs_launch_shape* shape) {
  if (!ctx || !shape) return CGS_E_ARG;
  const uint32_t t = shape->project_threads;
  if (t != 0 && t != 128 && t != 256 && t != 512)
    return ctx->fail(CGS_E_ARG, "project_threads must be 0, 128, 256 or 512");
  if (shape->bin_blocks_per_sm > 8) return ctx->fail(CGS_E_ARG, "bin_blocks_per_sm must be <= 8");
  if (shape->ranges_blocks > 65535) return ctx->fail(CGS_E_ARG, "ranges_blocks must be <= 65535");
  ctx->shape = *shape;
  ++ctx->state_epoch;  // launch shapes are part of a captured view graph
  return CGS_OK;
}

int cgs_ctx_set_device_budget(cgs_ctx* ctx, uint64_t bytes) {
  if (!ctx) return CGS_E_ARG;
  ctx->budget = bytes;
  return CGS_OK;
}

// Each drill's scratch: two tiles of 64-bit chained-scan words, two tiles of
// 256 digit words and the status word, zeroed, in a buffer of its own.
int cgs_ctx_wait_drill(cgs_ctx* ctx, uint32_t polls, uint32_t* out_gave_up) {
  if (!ctx) return CGS_E_ARG;
  if (polls == 0 || polls > kSpinLimit) return ctx->fail(CGS_E_ARG, "polls must be in [1, 2^22]");
  cudaSetDevice(ctx->device);
  CGS_TRY(drain(ctx, true));
  const size_t bytes = 2 * sizeof(unsigned long long) + 2 * 256 * sizeof(uint32_t) + 16;
  DevBuf buf;
  CGS_CUDA(cudaMalloc(&buf.p, 3 * bytes), "drill scratch");
  CGS_CUDA(cudaMemsetAsync(buf.p, 0, 3 * bytes, ctx->stream), "clear drill scratch");
  uint32_t gave_up = 0;
  for (int k = 0; k < 3; ++k) {
    char* base = buf.as<char>() + k * bytes;
    unsigned long long* scan_status = (unsigned long long*)base;
    uint32_t* digits = (uint32_t*)(base + 2 * sizeof(unsigned long long));
    uint32_t* word = digits + 2 * 256;
    cudaError_t e = k == 0   ? launch_drill_chained_scan(scan_status, word, polls, ctx->stream)
                    : k == 1 ? launch_drill_digit_lookback(digits, 256, word, polls, ctx->stream)
                             : launch_drill_mbarrier(word, polls, ctx->stream);
    CGS_CUDA(e, "drill launch");
    uint32_t w = 0;
    CGS_CUDA(cudaMemcpyAsync(&w, word, 4, cudaMemcpyDeviceToHost, ctx->stream), "drill status");
    CGS_CUDA(cudaStreamSynchronize(ctx->stream), "drill");
    const uint32_t want = k == 2 ? kStatusBarrierTimeout : kStatusLookbackTimeout;
    if (w & want) gave_up |= 1u << k;
  }
  if (out_gave_up) *out_gave_up = gave_up;
  if (gave_up) return ctx->fail(CGS_E_TIMEOUT, "bounded device waits gave up (drill mask " +
                                                   std::to_string(gave_up) + ")");
  return CGS_OK;
}

int cgs_ctx_device_bytes(const cgs_ctx* ctx, uint64_t* out) {
  if (!ctx || !out) return CGS_E_ARG;
  const DevBuf* bufs[] = {&ctx->rest_pos, &ctx->rest_cova, &ctx->rest_covb, &ctx->rest_sh,
                          &ctx->tet_elems, &ctx->tet_inv_dm, &ctx->cage_verts, &ctx->bind_tet,
                          &ctx->bind_w, &ctx->tet_J, &ctx->tet_R, &ctx->tet_S, &ctx->def_pos,
                          &ctx->def_cova, &ctx->def_covb, &ctx->split_meta, &ctx->persist,
                          &ctx->recs, &ctx->offsets, &ctx->scratch, &ctx->ranges, &ctx->keys[0],
                          &ctx->keys[1], &ctx->ids[0], &ctx->ids[1], &ctx->depths[0],
                          &ctx->depths[1], &ctx->radix_lb[0], &ctx->radix_lb[1], &ctx->fb_rgba8,
                          &ctx->fb_f32, &ctx->prim[0], &ctx->prim[1], &ctx->prim[2],
                          &ctx->prim[3]};
  uint64_t t = 0;
  for (auto* b : bufs) t += b->cap;
  *out = t;
  return CGS_OK;
}

int cgs_scene_upload(cgs_ctx* ctx, uint64_t n, const float* pos, const float* cov,
                     const float* opa, const void* sh, int32_t sh_format) {
  if (ctx) ++ctx->state_epoch;
  if (!ctx) return CGS_E_ARG;
  if (sh_format != CGS_SH_F32 && sh_format != CGS_SH_F16)
    return ctx->fail(CGS_E_ARG, "sh_format must be CGS_SH_F32 or CGS_SH_F16");
  if (n >= (1ull << 30)) return ctx->fail(CGS_E_CAPACITY, "scene exceeds 2^30 Gaussians");
  if (n > 0 && (!pos || !cov || !opa || !sh)) return ctx->fail(CGS_E_ARG, "null scene array");
  cudaSetDevice(ctx->device);
  ctx->scene_ready = false;  // until the new scene is resident (a failed growth loses the old one)
  const size_t shb = (size_t)n * 48 * (sh_format == CGS_SH_F16 ? 2 : 4);
  const size_t nn = n ? n : 1;
  CGS_TRY(ctx->ensure(ctx->rest_pos, nn * 16, "rest positions"));
  CGS_TRY(ctx->ensure(ctx->rest_cova, nn * 16, "rest covariances"));
  CGS_TRY(ctx->ensure(ctx->rest_covb, nn * 8, "rest covariances"));
  CGS_TRY(ctx->ensure(ctx->rest_sh, shb ? shb : 16, "rest SH"));
  if (n > 0) {
    // Stage the interleaved arrays, then convert to the resident layout.
    void* stage = nullptr;
    const size_t pb = (size_t)n * 12, cb = (size_t)n * 24, ob = (size_t)n * 4;
    const size_t ofs_c = (pb + 255) & ~(size_t)255, ofs_o = ofs_c + ((cb + 255) & ~(size_t)255),
                 ofs_s = ofs_o + ((ob + 255) & ~(size_t)255);
    CGS_CUDA(cudaMalloc(&stage, ofs_s + shb), "cudaMalloc scene staging");
    char* st = (char*)stage;
    cudaError_t e = cudaMemcpyAsync(st, pos, pb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(st + ofs_c, cov, cb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(st + ofs_o, opa, ob, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(st + ofs_s, sh, shb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
      e = launch_scene_layout((uint32_t)n, (const float*)st, (const float*)(st + ofs_c),
                              (const float*)(st + ofs_o), st + ofs_s, sh_format == CGS_SH_F16,
                              ctx->rest_pos.as<float4>(), ctx->rest_cova.as<float4>(),
                              ctx->rest_covb.as<float2>(), ctx->rest_sh.p, ctx->stream);
    cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    cudaFree(stage);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "scene upload");
    if (e2 != cudaSuccess) return ctx->cuda_fail(e2, "scene upload");
  }
  ctx->n = (uint32_t)n;
  ctx->sh_f16 = sh_format == CGS_SH_F16;
  ctx->scene_ready = true;
  ctx->deformed_valid = false;
  ctx->deform_generation++;
  ctx->s3_valid = false;
  ctx->has_cages = false;  // cage bindings refer to the previous scene
  ctx->spr_ready = false;
  ctx->num_tets = 0;
  ctx->mvc_unbind();
  return CGS_OK;
}

int cgs_scene_upload_quantized(cgs_ctx* ctx, uint64_t n, const float* pos,
                               const uint32_t* cov_f16x2, const float* opa,
                               const uint32_t* sh_f16x2, uint32_t sh_degree) {
  if (ctx) ++ctx->state_epoch;
  if (!ctx) return CGS_E_ARG;
  if (sh_degree > 3) return ctx->fail(CGS_E_ARG, "sh_degree must be 0..3");
  if (n >= (1ull << 30)) return ctx->fail(CGS_E_CAPACITY, "scene exceeds 2^30 Gaussians");
  if (n > 0 && (!pos || !cov_f16x2 || !opa || !sh_f16x2))
    return ctx->fail(CGS_E_ARG, "null scene array");
  cudaSetDevice(ctx->device);
  ctx->scene_ready = false;  // until the new scene is resident (a failed growth loses the old one)
  const size_t nn = n ? n : 1;
  const size_t bases = sh_degree == 0 ? 1 : (sh_degree == 1 ? 4 : (sh_degree == 2 ? 9 : 16));
  const size_t words = (bases * 3 + 1) / 2;
  CGS_TRY(ctx->ensure(ctx->rest_pos, nn * 16, "rest positions"));
  CGS_TRY(ctx->ensure(ctx->rest_cova, nn * 16, "rest covariances"));
  CGS_TRY(ctx->ensure(ctx->rest_covb, nn * 8, "rest covariances"));
  CGS_TRY(ctx->ensure(ctx->rest_sh, nn * 96, "rest SH"));
  if (n > 0) {
    void* stage = nullptr;
    const size_t pb = (size_t)n * 12, cb = (size_t)n * 12, ob = (size_t)n * 4,
                 sb = (size_t)n * words * 4;
    const size_t ofs_c = (pb + 255) & ~(size_t)255, ofs_o = ofs_c + ((cb + 255) & ~(size_t)255),
                 ofs_s = ofs_o + ((ob + 255) & ~(size_t)255);
    CGS_CUDA(cudaMalloc(&stage, ofs_s + sb), "cudaMalloc scene staging");
    char* st = (char*)stage;
    cudaError_t e = cudaMemcpyAsync(st, pos, pb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(st + ofs_c, cov_f16x2, cb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(st + ofs_o, opa, ob, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(st + ofs_s, sh_f16x2, sb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
      e = launch_scene_decode_quantized((uint32_t)n, (const float*)st, (const uint32_t*)(st + ofs_c),
                                        (const float*)(st + ofs_o), (const uint32_t*)(st + ofs_s),
                                        sh_degree, ctx->rest_pos.as<float4>(),
                                        ctx->rest_cova.as<float4>(), ctx->rest_covb.as<float2>(),
                                        ctx->rest_sh.p, ctx->stream);
    cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    cudaFree(stage);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "quantized scene upload");
    if (e2 != cudaSuccess) return ctx->cuda_fail(e2, "quantized scene upload");
  }
  ctx->n = (uint32_t)n;
  ctx->sh_f16 = 1;
  ctx->scene_ready = true;
  ctx->deformed_valid = false;
  ctx->deform_generation++;
  ctx->s3_valid = false;
  ctx->has_cages = false;
  ctx->spr_ready = false;
  ctx->num_tets = 0;
  ctx->mvc_unbind();
  return CGS_OK;
}

int cgs_tet_cages_upload(cgs_ctx* ctx, uint32_t num_tets, const uint32_t* elems,
                         const float* inv_dm, uint32_t num_verts, const uint32_t* bind_tet,
                         const float* bind_w) {
  if (ctx) ++ctx->state_epoch;
  if (!ctx) return CGS_E_ARG;
  if (!ctx->scene_ready) return ctx->fail(CGS_E_STATE, "upload the scene before the cages");
  cudaSetDevice(ctx->device);
  if (num_tets == 0) {
    // Tet-bound Gaussians fall back to the rest pose (their tet index is now
    // out of range); polygon-cage bindings stay valid.
    if (ctx->has_cages) {
      ctx->deform_generation++;
      ctx->deformed_valid = false;
    }
    ctx->has_cages = false;
    ctx->spr_ready = false;
    ctx->num_tets = 0;
    ctx->s3_valid = false;
    return CGS_OK;
  }
  if (!elems || !inv_dm || !bind_tet || !bind_w || num_verts == 0)
    return ctx->fail(CGS_E_ARG, "null cage array or zero vertices");
  for (uint64_t i = 0; i < (uint64_t)num_tets * 4; ++i)
    if (elems[i] >= num_verts) return ctx->fail(CGS_E_ARG, "tet element index out of range");
  const uint32_t n = ctx->n;
  CGS_TRY(ctx->ensure(ctx->tet_elems, (size_t)num_tets * 16, "tet elements"));
  CGS_TRY(ctx->ensure(ctx->tet_inv_dm, (size_t)num_tets * 36, "tet inv_dm"));
  CGS_TRY(ctx->ensure(ctx->cage_verts, (size_t)num_verts * 12, "cage vertices"));
  CGS_TRY(ctx->ensure(ctx->bind_tet, (size_t)(n ? n : 1) * 4, "bindings"));
  CGS_TRY(ctx->ensure(ctx->bind_w, (size_t)(n ? n : 1) * 16, "binding weights"));
  CGS_CUDA(cudaMemcpyAsync(ctx->tet_elems.p, elems, (size_t)num_tets * 16, cudaMemcpyHostToDevice, ctx->stream), "upload elems");
  CGS_CUDA(cudaMemcpyAsync(ctx->tet_inv_dm.p, inv_dm, (size_t)num_tets * 36, cudaMemcpyHostToDevice, ctx->stream), "upload inv_dm");
  if (n) {
    CGS_CUDA(cudaMemcpyAsync(ctx->bind_tet.p, bind_tet, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream), "upload bindings");
    CGS_CUDA(cudaMemcpyAsync(ctx->bind_w.p, bind_w, (size_t)n * 16, cudaMemcpyHostToDevice, ctx->stream), "upload weights");
  }
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "cage upload");
  ctx->num_tets = num_tets;
  ctx->num_verts = num_verts;
  ctx->has_cages = true;
  ctx->spr_ready = false;
  ctx->mvc_unbind();  // the bindings were replaced: bind the polygon cage again
  ctx->verts_uploaded = false;
  ctx->last_verts.clear();
  ctx->deformed_valid = false;
  return CGS_OK;
}

int cgs_cage_vertices_update(cgs_ctx* ctx, const float* verts, uint32_t num_verts) {
  if (!ctx || !verts) return CGS_E_ARG;
  if (!ctx->has_cages) return ctx->fail(CGS_E_STATE, "no cages uploaded");
  if (num_verts != ctx->num_verts) return ctx->fail(CGS_E_ARG, "vertex count differs from the cage topology");
  const size_t cnt = (size_t)num_verts * 3;
  if (ctx->verts_uploaded && ctx->last_verts.size() == cnt &&
      std::memcmp(ctx->last_verts.data(), verts, cnt * 4) == 0)
    return CGS_OK;
  cudaSetDevice(ctx->device);
  CGS_TRY(staged_upload(ctx, ctx->cage_verts.p, cnt * 4,
                        [&](void* dst) { std::memcpy(dst, verts, cnt * 4); }, "upload vertices"));
  ctx->last_verts.assign(verts, verts + cnt);
  ctx->verts_uploaded = true;
  ctx->deformed_valid = false;
  return CGS_OK;
}

int cgs_mvc_cage_upload(cgs_ctx* ctx, uint32_t V, const float* rest, uint32_t F,
                        const uint32_t* tris) {
  if (ctx) ++ctx->state_epoch;
  if (!ctx || !rest || !tris) return CGS_E_ARG;
  if (V < 4 || F < 4) return ctx->fail(CGS_E_ARG, "a polygon cage needs at least 4 vertices and 4 triangles");
  if (!mvc_cage_fits(V, F)) return ctx->fail(CGS_E_CAPACITY, "polygon cage too large (1,024 vertices, 12,800 vertices + triangles)");
  for (uint32_t f = 0; f < F; ++f) {
    const uint32_t* t = tris + 3 * (size_t)f;
    if (t[0] >= V || t[1] >= V || t[2] >= V) return ctx->fail(CGS_E_ARG, "triangle index out of range");
    if (t[0] == t[1] || t[1] == t[2] || t[2] == t[0]) return ctx->fail(CGS_E_ARG, "degenerate triangle");
  }
  cudaSetDevice(ctx->device);
  // incident faces per vertex, ascending (the order the reference adds them in)
  std::vector<uint32_t> off(V + 1, 0), list(3 * (size_t)F);
  for (uint32_t f = 0; f < F; ++f)
    for (int k = 0; k < 3; ++k) ++off[tris[3 * (size_t)f + k] + 1];
  for (uint32_t j = 0; j < V; ++j) off[j + 1] += off[j];
  std::vector<uint32_t> fill(off.begin(), off.end() - 1);
  for (uint32_t f = 0; f < F; ++f)
    for (uint32_t k = 0; k < 3; ++k) list[fill[tris[3 * (size_t)f + k]]++] = (f << 2) | k;
  std::vector<float4> v4(V);
  for (uint32_t j = 0; j < V; ++j) v4[j] = make_float4(rest[3 * j], rest[3 * j + 1], rest[3 * j + 2], 0.0f);
  std::vector<uint4> t4(F);
  for (uint32_t f = 0; f < F; ++f) t4[f] = make_uint4(tris[3 * f], tris[3 * f + 1], tris[3 * f + 2], 0u);
  // jacobian_step_size (mvc.rs:484-494): 1e-3 of the bounding-box diagonal,
  // clamped to [1e-5, 1e-2]
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t j = 0; j < V; ++j)
    for (int k = 0; k < 3; ++k) {
      mn[k] = std::fmin(mn[k], rest[3 * j + k]);
      mx[k] = std::fmax(mx[k], rest[3 * j + k]);
    }
  const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
  const float diag = std::fmax(std::sqrt((dx * dx + dy * dy) + dz * dz), 1e-3f);
  ctx->mvc_h = std::fmin(std::fmax(diag * 1e-3f, 1e-5f), 1e-2f);
  CGS_TRY(ctx->ensure(ctx->mvc_rest, (size_t)V * 16, "mvc rest vertices"));
  CGS_TRY(ctx->ensure(ctx->mvc_verts, (size_t)V * 16, "mvc vertices"));
  CGS_TRY(ctx->ensure(ctx->mvc_tris, (size_t)F * 16, "mvc triangles"));
  CGS_TRY(ctx->ensure(ctx->mvc_vf_off, (size_t)(V + 1) * 4, "mvc incidence"));
  CGS_TRY(ctx->ensure(ctx->mvc_vf_list, (size_t)F * 12, "mvc incidence"));
  cudaStream_t s = ctx->stream;
  CGS_CUDA(cudaMemcpyAsync(ctx->mvc_rest.p, v4.data(), (size_t)V * 16, cudaMemcpyHostToDevice, s), "mvc upload");
  CGS_CUDA(cudaMemcpyAsync(ctx->mvc_verts.p, v4.data(), (size_t)V * 16, cudaMemcpyHostToDevice, s), "mvc upload");
  CGS_CUDA(cudaMemcpyAsync(ctx->mvc_tris.p, t4.data(), (size_t)F * 16, cudaMemcpyHostToDevice, s), "mvc upload");
  CGS_CUDA(cudaMemcpyAsync(ctx->mvc_vf_off.p, off.data(), (size_t)(V + 1) * 4, cudaMemcpyHostToDevice, s), "mvc upload");
  CGS_CUDA(cudaMemcpyAsync(ctx->mvc_vf_list.p, list.data(), (size_t)F * 12, cudaMemcpyHostToDevice, s), "mvc upload");
  CGS_CUDA(cudaStreamSynchronize(s), "mvc upload");
  ctx->mvc_V = V;
  ctx->mvc_F = F;
  ctx->mvc_ready = true;
  ctx->field_ready = false;  // the network belongs to the previous cage
  ctx->mvc_last_verts.assign(rest, rest + 3 * (size_t)V);
  if (ctx->mvc_nb) {
    ctx->mvc_unbind();
    ctx->deformed_valid = false;
    ctx->deform_generation++;
  }
  return CGS_OK;
}

int cgs_mvc_vertices_update(cgs_ctx* ctx, const float* verts, uint32_t V) {
  if (!ctx || !verts) return CGS_E_ARG;
  if (!ctx->mvc_ready) return ctx->fail(CGS_E_STATE, "no polygon cage uploaded");
  if (V != ctx->mvc_V) return ctx->fail(CGS_E_ARG, "vertex count differs from the polygon cage");
  const size_t cnt = (size_t)V * 3;
  if (ctx->mvc_last_verts.size() == cnt && std::memcmp(ctx->mvc_last_verts.data(), verts, cnt * 4) == 0)
    return CGS_OK;
  cudaSetDevice(ctx->device);
  CGS_TRY(staged_upload(ctx, ctx->mvc_verts.p, (size_t)V * 16, [&](void* dst) {
    float4* v4 = static_cast<float4*>(dst);
    for (uint32_t j = 0; j < V; ++j)
      v4[j] = make_float4(verts[3 * j], verts[3 * j + 1], verts[3 * j + 2], 0.0f);
  }, "mvc vertices"));
  ctx->mvc_last_verts.assign(verts, verts + cnt);
  if (ctx->mvc_nb) ctx->deformed_valid = false;
  return CGS_OK;
}

namespace {

// Learned bindings were made with the current network: a new or changed
// network drops them (the Gaussians fall back to their rest pose until bound
// again).
void field_changed(cgs_ctx* ctx) {
  ++ctx->state_epoch;
  if (!ctx->mvc_learned) return;
  ctx->mvc_unbind();
  ctx->deformed_valid = false;
  ctx->deform_generation++;
  ctx->s3_valid = false;
}

// PolyCageMesh::bind_gaussians (mvc.rs:498-541) over the resident scene:
// inside test, slots in index order, then either exact stored weights for
// every slot, or (learned) the network for the slots whose residual on the
// rest cage is at most `threshold` and exact weights for the others, which
// are renumbered to come first.
int mvc_bind(cgs_ctx* ctx, bool learned, float threshold, bool cache, uint32_t* out_bound,
             uint32_t* out_fallback) {
  if (!ctx) return CGS_E_ARG;
  ++ctx->state_epoch;
  if (!ctx->scene_ready) return ctx->fail(CGS_E_STATE, "no scene uploaded");
  if (!ctx->mvc_ready) return ctx->fail(CGS_E_STATE, "no polygon cage uploaded");
  if (learned && !ctx->field_ready) return ctx->fail(CGS_E_STATE, "no learned field created");
  if (learned && !(threshold >= 0.0f)) return ctx->fail(CGS_E_ARG, "threshold must be >= 0");
  cudaSetDevice(ctx->device);
  CGS_TRY(drain(ctx, true));
  cudaStream_t s = ctx->stream;
  const uint32_t n = ctx->n;
  if (!ctx->has_cages) {
    CGS_TRY(ctx->ensure(ctx->bind_tet, (size_t)(n ? n : 1) * 4, "bindings"));
    CGS_TRY(ctx->ensure(ctx->bind_w, (size_t)(n ? n : 1) * 16, "binding weights"));
    CGS_CUDA(cudaMemsetAsync(ctx->bind_tet.p, 0xFF, (size_t)(n ? n : 1) * 4, s), "clear bindings");
    CGS_CUDA(cudaMemsetAsync(ctx->bind_w.p, 0, (size_t)(n ? n : 1) * 16, s), "clear bindings");
  }
  ctx->mvc_unbind();
  uint32_t nb = 0, nfb = 0;
  if (n) {
    DevBuf flag, slot, tmp;
    const size_t scan_status = ((size_t)scan_tiles(n) + 1) * 8 + 64;
    CGS_CUDA(cudaMalloc(&flag.p, (size_t)n * 4), "mvc flags");
    flag.cap = (size_t)n * 4;
    CGS_CUDA(cudaMalloc(&slot.p, (size_t)n * 4 + scan_status), "mvc slots");
    slot.cap = (size_t)n * 4 + scan_status;
    char* sb = slot.as<char>() + (size_t)n * 4;
    uint32_t* words = (uint32_t*)(sb + scan_status - 64);
    uint32_t hw[4] = {};
    int rc = CGS_OK;
    cudaError_t e = cudaMemsetAsync(sb, 0, scan_status, s);
    const MvcCage rest = ctx->mvc_cage(true);
    if (e == cudaSuccess)
      e = launch_mvc_inside(rest, n, ctx->rest_pos.as<float4>(), ctx->bind_tet.as<uint32_t>(),
                            flag.as<uint32_t>(), s);
    if (e == cudaSuccess)
      e = launch_scan_u32(flag.as<uint32_t>(), slot.as<uint32_t>(), n, words,
                          (unsigned long long*)sb, words + 1, words + 2, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hw, words, 12, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && hw[2]) rc = ctx->fail(CGS_E_TIMEOUT, "mvc slot scan gave up waiting");
    nb = hw[0];
    if (e == cudaSuccess && rc == CGS_OK && nb) {
      if ((rc = ctx->ensure(ctx->mvc_list, (size_t)nb * 4, "mvc slots")) == CGS_OK &&
          (rc = ctx->ensure(ctx->mvc_xf, (size_t)nb * 48, "mvc position/gradient")) == CGS_OK &&
          (rc = ctx->ensure(ctx->mvc_R, (size_t)nb * 36, "mvc rotations")) == CGS_OK) {
        e = launch_mvc_compact(n, flag.as<uint32_t>(), slot.as<uint32_t>(),
                               ctx->bind_tet.as<uint32_t>(), ctx->bind_w.as<float4>(),
                               ctx->mvc_list.as<uint32_t>(), s);
        nfb = nb;
        if (learned && e == cudaSuccess) {
          // residual of the network on the rest cage; fallbacks get the first slots
          FieldState& f = ctx->field;
          ctx->mvc_nfb = 0;
          ctx->mvc_nb = nb;
          e = cudaMemsetAsync(f.status.p, 0, 4, s);
          if (e == cudaSuccess) e = f.project(nullptr, f.proj_rest.as<float>(), s);  // raw: sum_j w0_j v_j
          if (e == cudaSuccess) {
            FieldInfer fi = ctx->field_infer_args(f.proj_rest.as<float>());
            e = launch_field_infer(fi, s);
          }
          ctx->mvc_nb = 0;
          if (e == cudaSuccess)
            e = launch_mvc_residual(nb, ctx->mvc_list.as<uint32_t>(), ctx->rest_pos.as<float4>(),
                                    ctx->mvc_xf.as<float4>(), f.enc[3], threshold, nullptr,
                                    flag.as<uint32_t>(), s);
          if (e == cudaSuccess) e = cudaMemsetAsync(sb, 0, scan_status, s);
          if (e == cudaSuccess)
            e = launch_scan_u32(flag.as<uint32_t>(), slot.as<uint32_t>(), nb, words,
                                (unsigned long long*)sb, words + 1, words + 2, s);
          if (e == cudaSuccess) e = cudaMemcpyAsync(hw, words, 12, cudaMemcpyDeviceToHost, s);
          if (e == cudaSuccess) e = cudaStreamSynchronize(s);
          if (e == cudaSuccess && hw[2])
            rc = ctx->fail(CGS_E_TIMEOUT, "mvc fallback scan gave up waiting");
          nfb = hw[0];
          if (e == cudaSuccess && rc == CGS_OK) {
            e = cudaMalloc(&tmp.p, (size_t)nb * 4);
            if (e == cudaSuccess) {
              tmp.cap = (size_t)nb * 4;
              e = launch_mvc_reslot(nb, flag.as<uint32_t>(), slot.as<uint32_t>(), nfb,
                                    ctx->mvc_list.as<uint32_t>(), tmp.as<uint32_t>(),
                                    ctx->bind_w.as<float4>(), s);
            }
            if (e == cudaSuccess)
              e = cudaMemcpyAsync(ctx->mvc_list.p, tmp.p, (size_t)nb * 4,
                                  cudaMemcpyDeviceToDevice, s);
          }
        }
        if (learned && cache && e == cudaSuccess && rc == CGS_OK && nb > nfb) {
          // codes of the learned slots, in their new order
          rc = ctx->ensure(ctx->mvc_codes, (size_t)(nb - nfb) * 4 * kFieldHid * 2, "field codes");
          if (rc == CGS_OK)
            rc = ctx->ensure(ctx->mvc_code_pos, (size_t)(nb - nfb) * 16, "field code positions");
          if (rc == CGS_OK) {
            ctx->mvc_nb = nb;
            ctx->mvc_nfb = nfb;
            FieldInfer fi = ctx->field_infer_args(ctx->field.proj_rest.as<float>());
            fi.codes = ctx->mvc_codes.as<__nv_bfloat16>();
            fi.code_pos = ctx->mvc_code_pos.as<float4>();
            e = launch_field_infer(fi, s);
            ctx->mvc_nb = 0;
            ctx->mvc_nfb = 0;
          }
        }
        if (e == cudaSuccess && rc == CGS_OK && nfb) {
          rc = ctx->ensure(ctx->mvc_wg, (size_t)nfb * ctx->mvc_V * 16, "mvc bindings");
          if (rc == CGS_OK)
            e = launch_mvc_bind_weights(rest, nfb, ctx->mvc_list.as<uint32_t>(),
                                        ctx->rest_pos.as<float4>(), ctx->mvc_h,
                                        ctx->mvc_wg.as<float4>(), s);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (learned && e == cudaSuccess && rc == CGS_OK) {
          uint32_t fst = 0;
          e = cudaMemcpy(&fst, ctx->field.status.p, 4, cudaMemcpyDeviceToHost);
          if (e == cudaSuccess && (fst & kStatusPoisoned)) ctx->poisoned = true;
          if (e == cudaSuccess && fst)
            rc = ctx->fail(CGS_E_TIMEOUT, "field inference gave up waiting for the tensor cores");
        }
      }
    }
    if (rc != CGS_OK || e != cudaSuccess) {
      cudaStreamSynchronize(s);
      ctx->mvc_unbind();
      ctx->deformed_valid = false;
      ctx->deform_generation++;
      ctx->s3_valid = false;
      return rc != CGS_OK ? rc : ctx->cuda_fail(e, "mvc binding");
    }
  }
  ctx->mvc_nb = nb;
  ctx->mvc_learned = learned;
  ctx->mvc_cached = learned && cache;
  ctx->mvc_nfb = learned ? nfb : 0;
  ctx->deformed_valid = false;
  ctx->deform_generation++;
  ctx->s3_valid = false;
  if (out_bound) *out_bound = nb;
  if (out_fallback) *out_fallback = learned ? nfb : nb;
  return CGS_OK;
}

int field_check(cgs_ctx* ctx) {
  if (!ctx) return CGS_E_ARG;
  if (!ctx->mvc_ready) return ctx->fail(CGS_E_STATE, "no polygon cage uploaded");
  if (!ctx->field_ready) return ctx->fail(CGS_E_STATE, "no learned field created");
  cudaSetDevice(ctx->device);
  return drain(ctx, true);
}

}  // namespace

int cgs_mvc_bind(cgs_ctx* ctx, uint32_t* out_bound) {
  return mvc_bind(ctx, false, 0.0f, false, out_bound, nullptr);
}

int cgs_mvc_bind_learned(cgs_ctx* ctx, float threshold, uint32_t flags, uint32_t* out_bound,
                         uint32_t* out_fallback) {
  if (ctx && (flags & ~(uint32_t)CGS_FIELD_PER_FRAME))
    return ctx->fail(CGS_E_ARG, "unknown field binding flags");
  return mvc_bind(ctx, true, threshold, !(flags & CGS_FIELD_PER_FRAME), out_bound, out_fallback);
}

int cgs_mvc_field_create(cgs_ctx* ctx, uint64_t seed) {
  if (!ctx) return CGS_E_ARG;
  if (!ctx->mvc_ready) return ctx->fail(CGS_E_STATE, "no polygon cage uploaded");
  cudaSetDevice(ctx->device);
  CGS_TRY(drain(ctx, true));
  field_changed(ctx);
  std::vector<float> r4((size_t)ctx->mvc_V * 4);
  CGS_CUDA(cudaMemcpy(r4.data(), ctx->mvc_rest.p, r4.size() * 4, cudaMemcpyDeviceToHost),
           "field rest cage");
  ctx->field_ready = false;
  CGS_CUDA(ctx->field.init(ctx->mvc_V, r4.data(), seed, ctx->stream), "field init");
  ctx->field_ready = true;
  return CGS_OK;
}

int cgs_mvc_field_layout(cgs_ctx* ctx, uint32_t* offsets, uint32_t* total, float* enc) {
  CGS_TRY(field_check(ctx));
  if (offsets)
    for (int k = 0; k < kFieldParams; ++k) offsets[k] = ctx->field.off[k];
  if (total) *total = ctx->field.total();
  if (enc) std::memcpy(enc, ctx->field.enc, 16);
  return CGS_OK;
}

int cgs_mvc_field_params(cgs_ctx* ctx, float* dst, const float* src) {
  CGS_TRY(field_check(ctx));
  FieldState& f = ctx->field;
  const size_t bytes = (size_t)f.total() * 4;
  if (dst) CGS_CUDA(cudaMemcpy(dst, f.p32.p, bytes, cudaMemcpyDeviceToHost), "field params");
  if (src) {
    field_changed(ctx);
    cudaStream_t s = ctx->stream;
    CGS_CUDA(cudaMemcpyAsync(f.p32.p, src, bytes, cudaMemcpyHostToDevice, s), "field params");
    // bf16 copy: a 1 x total transpose is an elementwise conversion
    CGS_CUDA(launch_transpose_f32(f.p32.as<float>(), 1, f.total(), f.total(),
                                  f.pb.as<__nv_bfloat16>(), 1, s), "field params");
    CGS_CUDA(cudaMemsetAsync(f.m1.p, 0, bytes, s), "field params");
    CGS_CUDA(cudaMemsetAsync(f.m2.p, 0, bytes, s), "field params");
    CGS_CUDA(cudaStreamSynchronize(s), "field params");
    f.step = 0;
  }
  return CGS_OK;
}

// Waits for the field's stream and turns its status word into the call's
// result: a bounded wait for the tensor cores gave up (CGS_E_TIMEOUT), and if
// MMAs may still have been running when their tensor memory was released,
// the context is unusable from then on.
static int field_status(cgs_ctx* ctx, const char* what) {
  uint32_t fst = 0;
  CGS_CUDA(cudaMemcpyAsync(&fst, ctx->field.status.p, 4, cudaMemcpyDeviceToHost, ctx->stream), what);
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), what);
  if (fst & kStatusPoisoned) ctx->poisoned = true;
  if (fst) return ctx->fail(CGS_E_TIMEOUT, "gave up waiting for the tensor cores");
  return CGS_OK;
}

int cgs_mvc_field_train(cgs_ctx* ctx, uint64_t n, const float* d_points, const float* d_weights,
                        uint32_t steps, uint32_t batch, float lr, float lambda, uint64_t seed,
                        float* out_loss) {
  CGS_TRY(field_check(ctx));
  if (!d_points || !d_weights || n == 0) return ctx->fail(CGS_E_ARG, "no training points");
  if (n > 0xFFFFFFFFull) return ctx->fail(CGS_E_CAPACITY, "at most 2^32 - 1 points");
  if (batch == 0 || batch % 8) return ctx->fail(CGS_E_ARG, "batch must be a positive multiple of 8");
  if (!(lr > 0.0f) || !(lambda >= 0.0f)) return ctx->fail(CGS_E_ARG, "lr > 0 and lambda >= 0");
  field_changed(ctx);
  FieldState& f = ctx->field;
  cudaStream_t s = ctx->stream;
  const uint32_t tail = std::max<uint32_t>(1, steps / 10);
  CGS_CUDA(cudaMemsetAsync(f.loss.p, 0, 8, s), "field train");
  CGS_CUDA(cudaMemsetAsync(f.status.p, 0, 4, s), "field train");
  uint64_t st = seed ^ 0xD1B54A32D192ED03ull;
  for (uint32_t t = 0; t < steps; ++t) {
    if (t == steps - tail) CGS_CUDA(cudaMemsetAsync(f.loss.p, 0, 8, s), "field train");
    st += 0x9E3779B97F4A7C15ull;
    uint64_t z = st;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    const uint32_t bseed = (uint32_t)(z ^ (z >> 31)) | 1u;
    CGS_CUDA(f.forward(d_points, d_weights, (uint32_t)n, batch, bseed, ctx->mvc_rest.as<float4>(),
                       lambda, s), "field forward");
    CGS_CUDA(f.backward(batch, s), "field backward");
    const double c = 0.5 * (1.0 + std::cos(3.141592653589793 * (double)t / (double)steps));
    CGS_CUDA(f.adam(lr * (float)(0.05 + 0.95 * c), s), "field adam");
  }
  float hl[2] = {0.0f, 0.0f};
  CGS_CUDA(cudaMemcpyAsync(hl, f.loss.p, 8, cudaMemcpyDeviceToHost, s), "field train");
  CGS_TRY(field_status(ctx, "field training"));
  if (out_loss) {
    out_loss[0] = steps ? hl[0] / (float)tail : 0.0f;
    out_loss[1] = steps ? hl[1] / (float)tail : 0.0f;
  }
  return CGS_OK;
}

int cgs_mvc_field_grads(cgs_ctx* ctx, uint64_t n, const float* d_points, const float* d_weights,
                        float lambda, float* grads, float* out_loss) {
  CGS_TRY(field_check(ctx));
  if (!d_points || !d_weights || n == 0 || n % 8 || n > 0x7FFFFFFFull)
    return ctx->fail(CGS_E_ARG, "n must be a positive multiple of 8");
  FieldState& f = ctx->field;
  cudaStream_t s = ctx->stream;
  CGS_CUDA(cudaMemsetAsync(f.loss.p, 0, 8, s), "field grads");
  CGS_CUDA(cudaMemsetAsync(f.status.p, 0, 4, s), "field grads");
  CGS_CUDA(f.forward(d_points, d_weights, (uint32_t)n, (uint32_t)n, 0, ctx->mvc_rest.as<float4>(),
                     lambda, s), "field forward");
  CGS_CUDA(f.backward((uint32_t)n, s), "field backward");
  float hl[2];
  CGS_CUDA(cudaMemcpyAsync(hl, f.loss.p, 8, cudaMemcpyDeviceToHost, s), "field grads");
  CGS_TRY(field_status(ctx, "field gradients"));
  if (grads)
    CGS_CUDA(cudaMemcpy(grads, f.g32.p, (size_t)f.total() * 4, cudaMemcpyDeviceToHost),
             "field grads");
  if (out_loss) {
    out_loss[0] = hl[0];
    out_loss[1] = hl[1];
  }
  return CGS_OK;
}

int cgs_mvc_field_eval(cgs_ctx* ctx, uint64_t n, const float* d_points, float* d_weights) {
  CGS_TRY(field_check(ctx));
  if (n == 0) return CGS_OK;
  if (!d_points || !d_weights) return CGS_E_ARG;
  if (n > 0xFFFFFFFFull) return ctx->fail(CGS_E_CAPACITY, "at most 2^32 - 1 points");
  CGS_CUDA(cudaMemsetAsync(ctx->field.status.p, 0, 4, ctx->stream), "field eval");
  CGS_CUDA(ctx->field.eval((uint32_t)n, d_points, d_weights, ctx->stream), "field eval");
  return field_status(ctx, "field evaluation");
}

int cgs_mvc_field_infer(cgs_ctx* ctx, uint64_t n, const float* d_points, int32_t use_rest,
                        float* d_out) {
  CGS_TRY(field_check(ctx));
  if (n == 0) return CGS_OK;
  if (!d_points || !d_out) return CGS_E_ARG;
  if ((uintptr_t)d_out & 15) return ctx->fail(CGS_E_ARG, "d_out must be 16-byte aligned");
  if (n > 0xFFFFFFFFull) return ctx->fail(CGS_E_CAPACITY, "at most 2^32 - 1 points");
  FieldState& f = ctx->field;
  cudaStream_t s = ctx->stream;
  float* pr = use_rest ? f.proj_rest.as<float>() : f.proj.as<float>();
  CGS_CUDA(f.project(use_rest ? nullptr : ctx->mvc_verts.as<float4>(), pr, s),
           "field projection");
  FieldInfer fi{};
  fi.net = f.net();
  fi.enc = f.enc_d.as<float>();
  fi.proj = pr;
  fi.points3 = d_points;
  fi.count = (uint32_t)n;
  fi.xf = reinterpret_cast<float4*>(d_out);
  fi.status = f.status.as<uint32_t>();
  CGS_CUDA(cudaMemsetAsync(f.status.p, 0, 4, s), "field inference");
  CGS_CUDA(launch_field_infer(fi, s), "field inference");
  uint32_t fst = 0;
  CGS_CUDA(cudaMemcpyAsync(&fst, f.status.p, 4, cudaMemcpyDeviceToHost, s), "field inference");
  CGS_CUDA(cudaStreamSynchronize(s), "field inference");
  if (fst & kStatusPoisoned) ctx->poisoned = true;
  if (fst) return ctx->fail(CGS_E_TIMEOUT, "field inference gave up waiting for the tensor cores");
  return CGS_OK;
}

int cgs_mvc_weights(cgs_ctx* ctx, uint64_t n, const float* d_points, float* d_weights) {
  if (!ctx) return CGS_E_ARG;
  if (!ctx->mvc_ready) return ctx->fail(CGS_E_STATE, "no polygon cage uploaded");
  if (n == 0) return CGS_OK;
  if (!d_points || !d_weights) return CGS_E_ARG;
  if (n > 0xFFFFFFFFull) return ctx->fail(CGS_E_CAPACITY, "at most 2^32 - 1 points");
  cudaSetDevice(ctx->device);
  CGS_CUDA(launch_mvc_weights(ctx->mvc_cage(true), (uint32_t)n, d_points, d_weights, ctx->stream),
           "mvc weights launch");
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "mvc weights");
  return CGS_OK;
}

int cgs_mvc_read_bindings(cgs_ctx* ctx, uint64_t max_slots, uint32_t* gaussian, float* wg,
                          uint64_t* out_slots) {
  if (!ctx || !out_slots) return CGS_E_ARG;
  cudaSetDevice(ctx->device);
  CGS_TRY(drain(ctx, true));
  const uint64_t k = std::min<uint64_t>(max_slots, ctx->mvc_nwg());
  *out_slots = k;
  if (k == 0) return CGS_OK;
  const uint32_t V = ctx->mvc_V, nb = ctx->mvc_nwg();
  if (gaussian)
    CGS_CUDA(cudaMemcpy(gaussian, ctx->mvc_list.p, k * 4, cudaMemcpyDeviceToHost), "read mvc slots");
  if (wg) {
    // vertex-major on the device: row j holds every slot's entry for vertex j
    std::vector<float4> row(k);
    for (uint32_t j = 0; j < V; ++j) {
      CGS_CUDA(cudaMemcpy(row.data(), ctx->mvc_wg.as<float4>() + (size_t)j * nb, k * 16,
                          cudaMemcpyDeviceToHost), "read mvc bindings");
      for (uint64_t i = 0; i < k; ++i) std::memcpy(wg + 4 * ((size_t)i * V + j), &row[i], 16);
    }
  }
  return CGS_OK;
}

namespace {

// f32::min / f32::max: a NaN operand yields the other one.
float rmin(float a, float b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a < b ? a : b)); }
float rmax(float a, float b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a > b ? a : b)); }

// CageSpringSimulator::frame_damping (deformation/dynamics.rs:137-148), with
// the C library's logf / expf.
float spring_frame_damping(float damping, float dt) {
  float r = damping;
  if (r < 1.0e-4f) r = 1.0e-4f;
  if (r > 0.9999f) r = 0.9999f;
  const float c = -logf(r) * 60.0f;
  return expf(-c * dt);
}

SpringArgs spring_args(cgs_ctx* ctx, uint32_t steps) {
  SpringArgs a{};
  a.V = ctx->spr_V;
  a.num_cages = (uint32_t)ctx->spr_host.size();
  a.steps = steps;
  a.rest = ctx->spr_rest.as<float4>();
  a.vel = ctx->spr_vel.as<float4>();
  a.pinned = ctx->spr_pin.as<uint8_t>();
  a.verts = ctx->cage_verts.as<float>();
  a.cages = ctx->spr_cages.as<SpringCageDev>();
  a.planes = ctx->spr_planes.as<float4>();
  return a;
}

// Per-cage step constants for `dt`, uploaded through the pinned ring.
int spring_params(cgs_ctx* ctx, float dt) {
  const size_t nc = ctx->spr_host.size();
  std::vector<SpringCageDev> p(nc);
  const float dt_sim = rmin(dt, 0.033f);
  for (size_t c = 0; c < nc; ++c) {
    const cgs_spring_cage& h = ctx->spr_host[c];
    p[c].kim = h.stiffness * (1.0f / rmax(h.mass, 0.001f));
    p[c].gamma = dt_sim > 0.0f ? spring_frame_damping(h.damping, dt_sim) : 1.0f;
    p[c].dt = dt_sim > 0.0f ? dt_sim : 0.0f;
    p[c].cx = ctx->spr_centroid[3 * c];
    p[c].cy = ctx->spr_centroid[3 * c + 1];
    p[c].cz = ctx->spr_centroid[3 * c + 2];
    p[c].planes = h.first_plane | (h.num_planes << 16);
  }
  return staged_upload(ctx, ctx->spr_cages.p, nc * sizeof(SpringCageDev),
                       [&](void* dst) { std::memcpy(dst, p.data(), nc * sizeof(SpringCageDev)); },
                       "spring parameters");
}

}  // namespace

int cgs_springs_upload(cgs_ctx* ctx, uint32_t num_cages, const cgs_spring_cage* cages,
                       uint32_t num_planes, const cgs_collision_plane* planes, uint32_t num_verts,
                       const float* rest, const float* current, const float* velocity,
                       const uint8_t* pinned) {
  if (!ctx) return CGS_E_ARG;
  ctx->spr_ready = false;
  if (!ctx->has_cages) return ctx->fail(CGS_E_STATE, "no tet cages uploaded");
  if (num_verts != ctx->num_verts) return ctx->fail(CGS_E_ARG, "vertex count differs from the cage topology");
  if (num_cages == 0 || !cages || !rest || !current) return CGS_E_ARG;
  if (num_planes > 0xFFFFu || (num_planes && !planes)) return ctx->fail(CGS_E_ARG, "bad collision planes");
  std::vector<float4> r(num_verts), v(num_verts);
  std::vector<uint8_t> pin(num_verts, 0);
  for (uint32_t i = 0; i < num_verts; ++i) {
    r[i] = make_float4(rest[3 * i], rest[3 * i + 1], rest[3 * i + 2], bitsf(kInvalid));
    v[i] = velocity ? make_float4(velocity[3 * i], velocity[3 * i + 1], velocity[3 * i + 2], 0.0f)
                    : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (pinned) pin[i] = pinned[i] ? 1 : 0;
  }
  std::vector<float> centroid(3 * (size_t)num_cages, 0.0f);
  for (uint32_t c = 0; c < num_cages; ++c) {
    const cgs_spring_cage& h = cages[c];
    if ((uint64_t)h.first_vertex + h.num_vertices > num_verts)
      return ctx->fail(CGS_E_ARG, "spring cage vertex range outside the cage vertices");
    if ((uint64_t)h.first_plane + h.num_planes > num_planes)
      return ctx->fail(CGS_E_ARG, "spring cage plane range outside the planes");
    float s[3] = {0.0f, 0.0f, 0.0f};  // rest centroid, summed in vertex order
    for (uint32_t i = h.first_vertex; i < h.first_vertex + h.num_vertices; ++i) {
      if (fbits(r[i].w) != kInvalid)
        return ctx->fail(CGS_E_ARG, "spring cage vertex ranges overlap");
      r[i].w = bitsf(c);
      s[0] = s[0] + rest[3 * i];
      s[1] = s[1] + rest[3 * i + 1];
      s[2] = s[2] + rest[3 * i + 2];
    }
    for (int k = 0; k < 3; ++k)
      centroid[3 * c + k] = h.num_vertices ? s[k] / (float)h.num_vertices : 0.0f;
  }
  cudaSetDevice(ctx->device);
  CGS_TRY(ctx->ensure(ctx->spr_rest, (size_t)num_verts * 16, "spring rest"));
  CGS_TRY(ctx->ensure(ctx->spr_vel, (size_t)num_verts * 16, "spring velocities"));
  CGS_TRY(ctx->ensure(ctx->spr_pin, num_verts ? num_verts : 1, "spring pins"));
  CGS_TRY(ctx->ensure(ctx->spr_cages, (size_t)num_cages * sizeof(SpringCageDev), "spring cages"));
  CGS_TRY(ctx->ensure(ctx->spr_planes, (size_t)(num_planes ? num_planes : 1) * 32, "spring planes"));
  CGS_TRY(drain(ctx, true));
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "spring upload");
  CGS_CUDA(cudaMemcpy(ctx->spr_rest.p, r.data(), (size_t)num_verts * 16, cudaMemcpyHostToDevice), "spring rest");
  CGS_CUDA(cudaMemcpy(ctx->spr_vel.p, v.data(), (size_t)num_verts * 16, cudaMemcpyHostToDevice), "spring velocities");
  CGS_CUDA(cudaMemcpy(ctx->spr_pin.p, pin.data(), num_verts, cudaMemcpyHostToDevice), "spring pins");
  if (num_planes) {
    std::vector<float4> pl(2 * (size_t)num_planes);
    for (uint32_t q = 0; q < num_planes; ++q) {
      const cgs_collision_plane& h = planes[q];
      pl[2 * q] = make_float4(h.normal[0], h.normal[1], h.normal[2], h.offset);
      pl[2 * q + 1] = make_float4(h.restitution, h.friction, 0.0f, 0.0f);
    }
    CGS_CUDA(cudaMemcpy(ctx->spr_planes.p, pl.data(), pl.size() * 16, cudaMemcpyHostToDevice),
             "spring planes");
  }
  CGS_CUDA(cudaMemcpy(ctx->cage_verts.p, current, (size_t)num_verts * 12, cudaMemcpyHostToDevice),
           "spring positions");
  ctx->spr_host.assign(cages, cages + num_cages);
  ctx->spr_centroid = centroid;
  ctx->spr_V = num_verts;
  ctx->spr_ready = true;
  ctx->last_verts.assign(current, current + (size_t)num_verts * 3);
  ctx->verts_uploaded = true;
  ctx->deformed_valid = false;
  return CGS_OK;
}

int cgs_springs_step(cgs_ctx* ctx, float dt, uint32_t steps) {
  if (!ctx) return CGS_E_ARG;
  if (!ctx->spr_ready) return ctx->fail(CGS_E_STATE, "no device springs uploaded");
  if (steps == 0) return CGS_OK;
  cudaSetDevice(ctx->device);
  CGS_TRY(spring_params(ctx, dt));
  CGS_CUDA(launch_springs_step(spring_args(ctx, steps), ctx->stream), "springs launch");
  if (rmin(dt, 0.033f) > 0.0f) {
    ctx->last_verts.clear();  // the host copy no longer matches
    ctx->deformed_valid = false;
  }
  return CGS_OK;
}

int cgs_springs_impulse(cgs_ctx* ctx, float magnitude) {
  if (!ctx) return CGS_E_ARG;
  if (!ctx->spr_ready) return ctx->fail(CGS_E_STATE, "no device springs uploaded");
  cudaSetDevice(ctx->device);
  CGS_TRY(spring_params(ctx, 0.0f));
  CGS_CUDA(launch_springs_impulse(spring_args(ctx, 0), magnitude, ctx->stream), "impulse launch");
  return CGS_OK;
}

int cgs_springs_read(cgs_ctx* ctx, float* current, float* velocity) {
  if (!ctx) return CGS_E_ARG;
  if (!ctx->spr_ready) return ctx->fail(CGS_E_STATE, "no device springs uploaded");
  cudaSetDevice(ctx->device);
  CGS_TRY(drain(ctx, true));
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "springs read");
  const uint32_t V = ctx->spr_V;
  if (current)
    CGS_CUDA(cudaMemcpy(current, ctx->cage_verts.p, (size_t)V * 12, cudaMemcpyDeviceToHost),
             "read spring positions");
  if (velocity) {
    std::vector<float4> v(V);
    CGS_CUDA(cudaMemcpy(v.data(), ctx->spr_vel.p, (size_t)V * 16, cudaMemcpyDeviceToHost),
             "read spring velocities");
    for (uint32_t i = 0; i < V; ++i) {
      velocity[3 * i] = v[i].x;
      velocity[3 * i + 1] = v[i].y;
      velocity[3 * i + 2] = v[i].z;
    }
  }
  return CGS_OK;
}

int cgs_bind_tets(cgs_ctx* ctx, uint32_t num_tets, const uint32_t* elems, const float* inv_dm,
                  uint32_t num_verts, const float* rest_verts, int32_t use_bounds,
                  const float* bmin, const float* bmax, uint32_t* bind_tet, float* bind_w) {
  if (ctx) ++ctx->state_epoch;
  if (!ctx || !elems || !inv_dm || !rest_verts || !bind_tet || !bind_w) return CGS_E_ARG;
  if (!ctx->scene_ready) return ctx->fail(CGS_E_STATE, "upload the scene before binding");
  if (use_bounds && (!bmin || !bmax)) return ctx->fail(CGS_E_ARG, "bounds requested but null");
  cudaSetDevice(ctx->device);
  const uint32_t n = ctx->n;
  if (n == 0) return CGS_OK;
  std::vector<float> x0((size_t)num_tets * 3);
  for (uint32_t t = 0; t < num_tets; ++t) {
    const uint32_t v = elems[4 * (size_t)t];
    if (v >= num_verts) return ctx->fail(CGS_E_ARG, "tet element index out of range");
    std::memcpy(&x0[3 * (size_t)t], rest_verts + 3 * (size_t)v, 12);
  }
  void* d = nullptr;
  const size_t bx = (size_t)num_tets * 12, bm = (size_t)num_tets * 36;
  const size_t o_m = (bx + 255) & ~(size_t)255, o_t = o_m + ((bm + 255) & ~(size_t)255),
               o_w = o_t + (((size_t)n * 4 + 255) & ~(size_t)255);
  CGS_CUDA(cudaMalloc(&d, o_w + (size_t)n * 16 + 16), "cudaMalloc binding scratch");
  char* b = (char*)d;
  cudaError_t e = cudaSuccess;
  if (num_tets) {
    e = cudaMemcpyAsync(b, x0.data(), bx, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + o_m, inv_dm, bm, cudaMemcpyHostToDevice, ctx->stream);
  }
  BindArgs a{};
  a.n = n;
  a.num_tets = num_tets;
  a.points = ctx->rest_pos.as<float4>();
  a.tet_x0 = (const float*)b;
  a.inv_dm = (const float*)(b + o_m);
  a.use_bounds = use_bounds;
  for (int k = 0; k < 3; ++k) {
    a.bmin[k] = use_bounds ? bmin[k] : 0.0f;
    a.bmax[k] = use_bounds ? bmax[k] : 0.0f;
  }
  a.bind_tet = (uint32_t*)(b + o_t);
  a.bind_w = (float4*)(b + o_w);
  if (e == cudaSuccess) e = launch_bind(a, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(bind_tet, b + o_t, (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(bind_w, b + o_w, (size_t)n * 16, cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "binding");
  if (e2 != cudaSuccess) return ctx->cuda_fail(e2, "binding");
  return CGS_OK;
}

namespace {

// log2 of the screen tile's width and height for CGS_TILE_* (the reference's
// 16x16 for 0); false for an unknown shape.
bool tile_shape_log2(int32_t shape, uint32_t* lw, uint32_t* lh) {
  switch (shape) {
    case CGS_TILE_16X16: *lw = 4; *lh = 4; return true;
    case CGS_TILE_8X8: *lw = 3; *lh = 3; return true;
    case CGS_TILE_32X16: *lw = 5; *lh = 4; return true;
    default: return false;
  }
}

// How a frame is enqueued (cgs_execute_frame, cgs_execute_views).
struct FrameCtl {
  bool allow_cache = true;     // may reuse the cached Stage 3 lists
  bool force_stage1 = false;   // deform even when the deformed scene is current
  HostCounters* counters = nullptr;  // pinned destination of the frame's counters
  cudaEvent_t done = nullptr;        // recorded after the frame, if set
  uint32_t* out_rgba8 = nullptr;     // Stage 4 target (else the context's framebuffer)
  uint32_t out_pitch = 0;            // its row pitch in pixels
};
struct FrameInfo {
  FrameDesc d;
  bool cached = false, need_deform = false;
  uint32_t passes = 0, splat_passes = 0, bin_launches = 0, sort_launches = 0;
};

int check_frame_args(cgs_ctx* ctx, const cgs_camera* camera, const cgs_compositor* comp,
                     const cgs_frame_params* params) {
  if (!ctx || !camera || !comp || !params) return CGS_E_ARG;
  if (!ctx->scene_ready) return ctx->fail(CGS_E_STATE, "no scene uploaded");
  if (ctx->has_cages && !ctx->verts_uploaded)
    return ctx->fail(CGS_E_STATE, "cage vertices not uploaded");
  if (params->radix_bits != 0 && (params->radix_bits < 4 || params->radix_bits > 8))
    return ctx->fail(CGS_E_ARG, "radix_bits must be 0 or 4..8");
  if (params->entry_sort < CGS_SORT_AUTO || params->entry_sort > CGS_SORT_TRANSPOSE)
    return ctx->fail(CGS_E_ARG, "entry_sort must be one of CGS_SORT_*");
  uint32_t lw = 4, lh = 4;
  if (!tile_shape_log2(params->tile_shape, &lw, &lh))
    return ctx->fail(CGS_E_ARG, "tile_shape must be one of CGS_TILE_*");
  const uint32_t W = comp->screen_width ? comp->screen_width : 1u;
  const uint32_t H = comp->screen_height ? comp->screen_height : 1u;
  const uint32_t tiles_x = (W + (1u << lw) - 1) >> lw, tiles_y = (H + (1u << lh) - 1) >> lh;
  const uint64_t total_tiles64 = (uint64_t)tiles_x * tiles_y;
  if (total_tiles64 > 0xFFFFFFFFull / 2) return ctx->fail(CGS_E_CAPACITY, "viewport too large");
  if (W >= (1u << 22) || H >= (1u << 22))
    return ctx->fail(CGS_E_CAPACITY, "viewport wider or taller than 4,194,303 pixels");
  return CGS_OK;
}

// Enqueues one frame (Stages 1-4) on the context's stream without waiting
// for anything: buffers are grown here, so a frame being captured into a
// graph must find them large enough already.
int enqueue_frame(cgs_ctx* ctx, const cgs_camera* camera, const cgs_compositor* comp,
                  const cgs_frame_params* params, const FrameCtl& ctl, FrameInfo* fi) {
  cudaStream_t s = ctx->stream;
  const uint32_t W = comp->screen_width ? comp->screen_width : 1u;
  const uint32_t H = comp->screen_height ? comp->screen_height : 1u;
  FrameDesc d;
  tile_shape_log2(params->tile_shape, &d.tile_lw, &d.tile_lh);  // validated by the caller
  const uint32_t tiles_x = (W + (1u << d.tile_lw) - 1) >> d.tile_lw;
  const uint32_t tiles_y = (H + (1u << d.tile_lh) - 1) >> d.tile_lh;
  const uint64_t total_tiles64 = (uint64_t)tiles_x * tiles_y;
  d.W = W;
  d.H = H;
  d.tiles_x = tiles_x;
  d.tiles_y = tiles_y;
  d.total_tiles = (uint32_t)total_tiles64;
  d.pitch = (W + 63) / 64 * 64;
  d.radix_bits = (uint32_t)params->radix_bits;
  d.entry_sort = params->entry_sort;
  d.write_f32 = params->write_f32 != 0;
  std::memcpy(d.bg, comp->background, 16);
  if (W != ctx->last_w || H != ctx->last_h) ctx->s3_valid = false;

  if (ctl.out_rgba8) {
    d.out_rgba8 = ctl.out_rgba8;
    d.out_pitch = ctl.out_pitch;
  } else {
    CGS_TRY(ctx->ensure(ctx->fb_rgba8, (size_t)d.pitch * H * 4, "framebuffer"));
  }
  if (d.write_f32) CGS_TRY(ctx->ensure(ctx->fb_f32, (size_t)W * H * 16, "f32 framebuffer"));

  const uint32_t n = ctx->n;
  const bool has_cages = ctx->has_cages;   // tet cages
  const bool deform_on = ctx->deform_on();  // tet and/or polygon cage bindings
  const uint32_t split_bits = fbits(params->strain_split_threshold), mip_bits = fbits(params->mip_filter_3d_var);
  const bool params_changed = split_bits != ctx->last_split_bits || mip_bits != ctx->last_mip_bits;
  const bool need_deform =
      deform_on && (ctl.force_stage1 || !ctx->deformed_valid || params_changed);
  d.n = n;
  d.split_possible = deform_on && params->strain_split_threshold > 0.0f;
  d.max_n = d.split_possible ? 2 * n : n;
  const uint32_t mn = d.max_n ? d.max_n : 1u;
  d.key64 = d.total_tiles > 65535u;
  d.tile_bits = d.total_tiles <= 1 ? 1u : 32u - (uint32_t)__builtin_clz(d.total_tiles - 1);
  d.depth_bits = d.tile_bits >= 32 ? 0u : (32u - d.tile_bits < 28u ? 32u - d.tile_bits : 28u);
  d.sort_bits = d.tile_bits + d.depth_bits > 32 ? 32 : d.tile_bits + d.depth_bits;
  if (d.radix_bits == 0) {
    // balanced digits: the fewest passes of at most 8 bits over the tile bits,
    // split as evenly as possible (13 bits -> 7 + 6), at least 4 bits
    const uint32_t passes = (d.tile_bits + 7) / 8;
    d.radix_bits = std::max(4u, (d.tile_bits + passes - 1) / passes);
  }
  const float near_c = camera->near_plane > 1e-6f ? camera->near_plane : 1e-6f;
  d.depth_base_bits = fbits(near_c) & 0x7F800000u;

  const ScratchLayout L(n, mn);
  CGS_TRY(ctx->ensure(ctx->scratch, L.bytes, "frame scratch"));
  CGS_TRY(ctx->ensure(ctx->recs, (size_t)mn * sizeof(SplatRec), "splat records"));
  CGS_TRY(ctx->ensure(ctx->offsets, (size_t)mn * 4, "tile offsets"));
  CGS_TRY(ctx->ensure(ctx->ranges, (size_t)d.total_tiles * 8, "tile ranges"));
  char* sc = ctx->scratch.as<char>();
  FrameCounters* fc = (FrameCounters*)sc;
  uint32_t* d_split = ctx->persist.as<uint32_t>();
  if (has_cages) {
    CGS_TRY(ctx->ensure(ctx->tet_J, (size_t)ctx->num_tets * 36, "tet J"));
    CGS_TRY(ctx->ensure(ctx->tet_R, (size_t)ctx->num_tets * 36, "tet R"));
    CGS_TRY(ctx->ensure(ctx->tet_S, (size_t)ctx->num_tets * 4, "tet stretch"));
  }
  if (deform_on) {
    CGS_TRY(ctx->ensure(ctx->def_pos, (size_t)mn * 16, "deformed positions"));
    CGS_TRY(ctx->ensure(ctx->def_cova, (size_t)mn * 16, "deformed covariances"));
    CGS_TRY(ctx->ensure(ctx->def_covb, (size_t)mn * 8, "deformed covariances"));
    CGS_TRY(ctx->ensure(ctx->split_meta, (size_t)(n ? n : 1) * 8, "split meta"));
  }

  // Stage 3 cache key (gpu_state.rs:454-500). A hit needs the frame that
  // built the cache to have been checked.
  Stage3Key key;
  key.deform_generation = deform_on ? (need_deform ? ctx->deform_generation + 1 : ctx->deform_generation) : 0;
  for (int k = 0; k < 16; ++k) key.view[k] = fbits(camera->view[k]);
  key.fx = fbits(camera->focal_x);
  key.fy = fbits(camera->focal_y);
  key.cx = fbits(camera->principal_x);
  key.cy = fbits(camera->principal_y);
  key.near_bits = fbits(camera->near_plane);
  key.width = W;
  key.height = H;
  key.mip = mip_bits;
  key.min_opa = fbits(params->min_opacity);
  key.min_rad = fbits(params->min_radius_px);
  key.radix_bits = d.radix_bits | ((uint32_t)d.entry_sort << 8) | (d.tile_lw << 16) | (d.tile_lh << 20);
  bool cached = ctl.allow_cache && !params->force_stage3 && ctx->s3_valid && ctx->s3_key == key;
  if (cached) {
    CGS_TRY(drain(ctx, true));
    cached = ctx->s3_valid && ctx->s3_key == key;
  }
  if (!cached) {
    if (ctx->entry_cap == 0)
      ctx->entry_cap = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(32ull * mn, 1u << 20), (uint64_t)kMaxEntryCap);
    CGS_TRY(ensure_entry_buffers(ctx, ctx->entry_cap, d.key64, d.radix_bits));
    CGS_TRY(ensure_splat_buffers(ctx, mn));
  }

  ctx->kbegin(CGS_K_CLEAR);
  CGS_CUDA(cudaMemsetAsync(sc, 0, L.bytes, s), "clear frame scratch");
  ctx->kend();

  // ---------------- Stage 1
  if (need_deform) {
    DeformArgs da{};
    da.n = n;
    da.num_tets = ctx->num_tets;
    da.verts = ctx->cage_verts.as<float>();
    da.elems = ctx->tet_elems.as<uint4>();
    da.inv_dm = ctx->tet_inv_dm.as<float>();
    da.tet_J = ctx->tet_J.as<float>();
    da.tet_R = ctx->tet_R.as<float>();
    da.tet_stretch = ctx->tet_S.as<float>();
    da.bind_tet = ctx->bind_tet.as<uint32_t>();
    da.bind_w = ctx->bind_w.as<float4>();
    da.rest_pos = ctx->rest_pos.as<float4>();
    da.rest_cova = ctx->rest_cova.as<float4>();
    da.rest_covb = ctx->rest_covb.as<float2>();
    da.def_pos = ctx->def_pos.as<float4>();
    da.def_cova = ctx->def_cova.as<float4>();
    da.def_covb = ctx->def_covb.as<float2>();
    da.split_meta = ctx->split_meta.as<uint2>();
    da.split_count = d_split;
    da.status = (unsigned long long*)(sc + L.def);
    da.fc = fc;
    da.split_threshold = params->strain_split_threshold;
    da.mip = params->mip_filter_3d_var;
    if (!has_cages) da.num_tets = 0;
    if (ctx->mvc_nb) {
      da.mvc_xf = ctx->mvc_xf.as<float4>();
      da.mvc_R = ctx->mvc_R.as<float>();
      if (ctx->mvc_nwg()) {
        ctx->kbegin(CGS_K_MVC);
        CGS_CUDA(launch_mvc_jacobian(ctx->mvc_V, ctx->mvc_verts.as<float4>(), ctx->mvc_nwg(),
                                     ctx->mvc_wg.as<float4>(), ctx->mvc_xf.as<float4>(), s),
                 "mvc jacobian launch");
        ctx->kend();
      }
      if (ctx->mvc_learned && ctx->mvc_nb > ctx->mvc_nfb) {
        ctx->kbegin(CGS_K_FIELD);
        CGS_CUDA(ctx->field.project(ctx->mvc_verts.as<float4>(), ctx->field.proj.as<float>(), s),
                 "field projection launch");
        FieldInfer fi = ctx->field_infer_args(ctx->field.proj.as<float>());
        fi.status = &fc->status;
        if (ctx->mvc_cached) {
          fi.codes = ctx->mvc_codes.as<__nv_bfloat16>();
          fi.code_pos = ctx->mvc_code_pos.as<float4>();
          CGS_CUDA(launch_field_apply(fi, s), "field output layer launch");
        } else {
          CGS_CUDA(launch_field_infer(fi, s), "field inference launch");
        }
        ctx->kend();
      }
    }
    // the tet transforms run in the deform launch's first blocks
    da.fuse_tets = has_cages ? 1u : 0u;
    ctx->kbegin(CGS_K_DEFORM);
    CGS_CUDA(launch_deform(da, s), "deform launch");
    ctx->kend();
    ctx->deformed_valid = true;
    ctx->deform_generation++;
    ctx->last_split_bits = split_bits;
    ctx->last_mip_bits = mip_bits;
  }

  // ---------------- Stage 2
  ProjectArgs p{};
  p.threads = ctx->shape.project_threads;
  if (deform_on) {
    p.pos = ctx->def_pos.as<float4>();
    p.cova = ctx->def_cova.as<float4>();
    p.covb = ctx->def_covb.as<float2>();
    p.bind_tet = ctx->bind_tet.as<uint32_t>();
    p.bind_w = ctx->bind_w.as<float4>();
    p.tet_R = has_cages ? ctx->tet_R.as<float>() : nullptr;
    p.num_tets = has_cages ? ctx->num_tets : 0;
    p.mvc_R = ctx->mvc_nb ? ctx->mvc_R.as<float>() : nullptr;
    p.split_meta = ctx->split_meta.as<uint2>();
    p.split_count = d.split_possible ? d_split : nullptr;
  } else {
    p.pos = ctx->rest_pos.as<float4>();
    p.cova = ctx->rest_cova.as<float4>();
    p.covb = ctx->rest_covb.as<float2>();
  }
  p.sh = ctx->rest_sh.p;
  p.sh_f16 = ctx->sh_f16;
  p.sh_stride = n;
  p.n_rest = n;
  p.max_n = d.max_n;
  std::memcpy(p.cam, camera, 24 * sizeof(float));
  std::memcpy(p.cam_pos, comp->camera_position, 3 * sizeof(float));
  p.mip = deform_on ? 0.0f : params->mip_filter_3d_var;
  p.min_opacity = params->min_opacity;
  p.min_radius = params->min_radius_px;
  p.sh_degree = comp->sh_degree > 3 ? 3 : comp->sh_degree;
  p.out = ctx->recs.as<SplatRec>();
  p.fc = fc;
  if (!cached) {
    p.depth_keys = ctx->skeys[0].as<uint32_t>();
    p.depth_ids = ctx->sids[0].as<uint32_t>();
  }
  p.key64 = d.key64;
  p.depth_base_bits = d.depth_base_bits;
  p.depth_bits = d.depth_bits;
  ctx->kbegin(CGS_K_PROJECT);
  CGS_CUDA(launch_project(p, s), "project launch");
  ctx->kend();

  // ---------------- Stages 3 and 4
  int src = ctx->s3_src;
  uint32_t passes = 0, splat_passes = 0, bin_launches = 0, sort_launches = 0;
  if (!cached) {
    CGS_TRY(enqueue_stage3(ctx, d, L, &src, &passes, &splat_passes, true, &bin_launches,
                           &sort_launches));
    ctx->s3_valid = true;
    ctx->s3_key = key;
    ctx->s3_src = src;
    ctx->s3_key64 = d.key64;
    ctx->s3_depth_bits = d.depth_bits;
  }
  CGS_TRY(enqueue_stage4(ctx, d, src));
  CGS_CUDA(cudaMemcpyAsync(&ctl.counters->fc, fc, sizeof(FrameCounters), cudaMemcpyDeviceToHost, s),
           "read counters");
  CGS_CUDA(cudaMemcpyAsync(&ctl.counters->split, d_split, 4, cudaMemcpyDeviceToHost, s),
           "read split count");
  if (ctl.done) CGS_CUDA(cudaEventRecord(ctl.done, s), "frame event");
  fi->d = d;
  fi->cached = cached;
  fi->need_deform = need_deform;
  fi->passes = passes;
  fi->splat_passes = splat_passes;
  fi->bin_launches = bin_launches;
  fi->sort_launches = sort_launches;
  return CGS_OK;
}

}  // namespace

int cgs_execute_frame(cgs_ctx* ctx, const cgs_camera* camera, const cgs_compositor* comp,
                      const cgs_frame_params* params, cgs_stage_timings* timings) {
  CGS_TRY(check_frame_args(ctx, camera, comp, params));
  if (ctx->poisoned)
    return ctx->fail(CGS_E_STATE, "a tensor-core wait gave up twice in an earlier frame; the "
                                  "device state is undefined: destroy and recreate the context");
  cudaSetDevice(ctx->device);
  cgs_stage_timings tm{};
  const bool prof = params->profile_stages != 0;

  // Take a ring slot; the frame that used it last is checked first.
  const int slot = ctx->next_slot;
  CGS_TRY(check_slot(ctx, slot, true));
  CGS_TRY(drain(ctx, false));
  ctx->next_slot = (slot + 1) % kRing;

  cgs_ctx::Pending& P = ctx->ring[slot];
  P.kcount = 0;
  ctx->kprof = prof;
  ctx->cur = slot;
  FrameCtl ctl;
  ctl.counters = &ctx->h_ring[slot];
  ctl.done = P.done;
  FrameInfo fi;
  const int rc = enqueue_frame(ctx, camera, comp, params, ctl, &fi);
  if (rc != CGS_OK) {
    ctx->cur = -1;
    return rc;
  }
  const FrameDesc& d = fi.d;
  const bool cached = fi.cached, need_deform = fi.need_deform;
  const uint32_t n = d.n, W = d.W, H = d.H;
  const uint32_t passes = fi.passes, splat_passes = fi.splat_passes;
  const uint32_t bin_launches = fi.bin_launches, sort_launches = fi.sort_launches;
  P.used = true;
  P.seq = ++ctx->frame_seq;
  P.stage3_ran = !cached;
  P.profiled = prof;
  P.need_deform = need_deform;
  P.split_possible = d.split_possible;
  P.key64 = d.key64;
  P.n = n;
  P.cap = ctx->entry_cap;
  P.sort_passes = passes;
  P.splat_passes = splat_passes;
  P.bin_launches = bin_launches;
  P.sort_launches = sort_launches;
  P.total_tiles = d.total_tiles;
  P.W = W;
  P.H = H;
  P.write_f32 = d.write_f32;
  P.overflowed = false;
  P.cam = *camera;
  P.comp = *comp;
  P.params = *params;
  P.verts_bytes = P.mvc_bytes = 0;
  if (ctx->has_cages && ctx->cage_verts.p) {
    P.verts_bytes = (size_t)ctx->num_verts * 12;
    CGS_TRY(ctx->ensure(P.verts_snap, P.verts_bytes ? P.verts_bytes : 4, "frame vertex snapshot"));
    CGS_CUDA(cudaMemcpyAsync(P.verts_snap.p, ctx->cage_verts.p, P.verts_bytes,
                             cudaMemcpyDeviceToDevice, ctx->stream), "vertex snapshot");
  }
  if (ctx->mvc_nb > 0 && ctx->mvc_verts.p) {
    P.mvc_bytes = (size_t)ctx->mvc_V * 16;
    CGS_TRY(ctx->ensure(P.mvc_snap, P.mvc_bytes ? P.mvc_bytes : 4, "frame vertex snapshot"));
    CGS_CUDA(cudaMemcpyAsync(P.mvc_snap.p, ctx->mvc_verts.p, P.mvc_bytes,
                             cudaMemcpyDeviceToDevice, ctx->stream), "vertex snapshot");
  }
  ctx->arena_rerendered = false;
  ctx->cur = -1;
  ctx->latest_slot = slot;
  if (!cached) ctx->last_desc = d;
  ctx->last_w = W;
  ctx->last_h = H;
  ctx->last_pitch = d.pitch;
  ctx->last_f32 = d.write_f32;
  ctx->last_tiles = d.total_tiles;
  ctx->frame_done = true;

  tm.stage1_skipped = need_deform ? 0 : 1;
  tm.stage3_cached = cached ? 1 : 0;
  tm.used_64bit_keys = d.key64 ? 1 : 0;
  if (timings) {
    // Counts (and per-stage device times) need the frame to have finished.
    CGS_TRY(drain(ctx, true));
    CGS_TRY(ctx->take_sticky());
    const HostCounters& h = ctx->h_ring[slot];
    tm.total_tile_entries = ctx->s3_entries;
    tm.surviving_gaussians = h.fc.surviving;
    tm.active_gaussians = ctx->last_active;
    if (prof) {
      double ms[CGS_KERNEL_COUNT] = {};
      for (int c = 0; c < P.kcount; ++c) {
        float v = 0.0f;
        cudaEventElapsedTime(&v, P.kev[2 * c], P.kev[2 * c + 1]);
        ms[P.kid[c]] += v;
      }
      tm.stage1_deform_ms = ms[CGS_K_TET_TRANSFORMS] + ms[CGS_K_DEFORM];
      tm.stage2_project_ms = ms[CGS_K_PROJECT];
      tm.stage3_bin_sort_ms =
          ms[CGS_K_SPLAT_SORT] + ms[CGS_K_BIN] + ms[CGS_K_ENTRY_SORT] + ms[CGS_K_TILE_RANGES];
      tm.stage4_composite_ms = ms[CGS_K_COMPOSITE];
      tm.used_hardware_timestamps = 1;
    }
    *timings = tm;
  }
  return CGS_OK;
}

namespace {

// Reads the views' counters after the step has completed: bounded waits that
// gave up are errors; views whose entries exceeded the key buffers are
// listed (the capacity is grown for them and kept 30% above the largest
// count).
int check_views(cgs_ctx* ctx, uint32_t nv, const uint32_t* cap_used,
                std::vector<uint32_t>* overflowed, uint64_t* total_entries) {
  uint32_t most = 0;
  *total_entries = 0;
  overflowed->clear();
  for (uint32_t v = 0; v < nv; ++v) {
    const FrameCounters& fc = ctx->h_views[v].fc;
    if (fc.status & kStatusPoisoned) ctx->poisoned = true;
    if (fc.status & (kStatusLookbackTimeout | kStatusBarrierTimeout))
      return ctx->fail(CGS_E_TIMEOUT, "a bounded device-side wait gave up during a view");
    if ((fc.status & kStatusCapacity) || fc.entries > cap_used[v]) overflowed->push_back(v);
    most = std::max(most, fc.entries);
    *total_entries += fc.entries;
  }
  if (most > ctx->entry_cap / 10 * 8)
    ctx->entry_cap = (uint32_t)std::min<uint64_t>((uint64_t)most * 13 / 10 + 4096, (uint64_t)kMaxEntryCap);
  return CGS_OK;
}

int enqueue_view(cgs_ctx* ctx, const cgs_camera* cam, const cgs_compositor* comp,
                 const cgs_frame_params* params, uint32_t v, uint32_t* out, bool force_stage1,
                 uint32_t* cap_used) {
  FrameCtl ctl;
  ctl.allow_cache = false;
  ctl.force_stage1 = force_stage1;
  ctl.counters = &ctx->h_views[v];
  ctl.out_rgba8 = out;
  ctl.out_pitch = comp->screen_width ? comp->screen_width : 1u;
  FrameInfo fi;
  CGS_TRY(enqueue_frame(ctx, cam, comp, params, ctl, &fi));
  *cap_used = ctx->entry_cap;
  return CGS_OK;
}

// The views one by one (each view's launches issued from the host), then a
// wait and the counter check; overflowed views are rendered again with grown
// buffers.
int views_eager(cgs_ctx* ctx, uint32_t nv, const cgs_camera* cams, const cgs_compositor* comps,
                const cgs_frame_params* params, uint32_t* const* outs, uint32_t* rerendered,
                uint64_t* entries) {
  std::vector<uint32_t> cap(nv), over;
  for (uint32_t v = 0; v < nv; ++v)
    CGS_TRY(enqueue_view(ctx, &cams[v], &comps[v], &params[v], v, outs[v], false, &cap[v]));
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "views");
  CGS_TRY(check_views(ctx, nv, cap.data(), &over, entries));
  for (int round = 0; !over.empty() && round < 3; ++round) {
    for (uint32_t v : over) {
      CGS_TRY(enqueue_view(ctx, &cams[v], &comps[v], &params[v], v, outs[v], false, &cap[v]));
      ++*rerendered;
    }
    CGS_CUDA(cudaStreamSynchronize(ctx->stream), "views");
    CGS_TRY(check_views(ctx, nv, cap.data(), &over, entries));
  }
  if (!over.empty()) return ctx->fail(CGS_E_CAPACITY, "tile entries kept exceeding the key buffers");
  return CGS_OK;
}

void drop_views_graph(cgs_ctx* ctx) {
  if (ctx->views_exec) cudaGraphExecDestroy(ctx->views_exec);
  ctx->views_exec = nullptr;
  ctx->views_key.clear();
}

void put_bytes(std::vector<unsigned char>& k, const void* p, size_t bytes) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  k.insert(k.end(), b, b + bytes);
}

// Captures the step (Stage 1 of the first view, then every view) into a
// graph. The look-back buffers of both radix sorts are cleared at its start,
// so a replay does not depend on the alternation state the previous work
// left behind.
int capture_views(cgs_ctx* ctx, uint32_t nv, const cgs_camera* cams, const cgs_compositor* comps,
                  const cgs_frame_params* params, uint32_t* const* outs) {
  cudaStream_t s = ctx->stream;
  drop_views_graph(ctx);
  std::vector<uint32_t> cap(nv);
  cudaGraph_t g = nullptr;
  CGS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed), "begin capture");
  int rc = CGS_OK;
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
    if (ctx->radix_lb[k].p) e = cudaMemsetAsync(ctx->radix_lb[k].p, 0, ctx->radix_lb[k].cap, s);
    if (e == cudaSuccess && ctx->splat_lb[k].p)
      e = cudaMemsetAsync(ctx->splat_lb[k].p, 0, ctx->splat_lb[k].cap, s);
  }
  ctx->radix_parity = 0;
  ctx->splat_parity = 0;
  const uint64_t epoch = ctx->alloc_epoch;
  for (uint32_t v = 0; v < nv && rc == CGS_OK && e == cudaSuccess; ++v)
    rc = enqueue_view(ctx, &cams[v], &comps[v], &params[v], v, outs[v],
                      v == 0 && ctx->deform_on(), &cap[v]);
  const cudaError_t ee = cudaStreamEndCapture(s, &g);
  if (e == cudaSuccess) e = ee;
  if (rc == CGS_OK && e == cudaSuccess && ctx->alloc_epoch != epoch)
    rc = ctx->fail(CGS_E_STATE, "buffers grew while capturing the views");
  if (rc == CGS_OK && e == cudaSuccess) e = cudaGraphInstantiate(&ctx->views_exec, g, 0);
  if (g) cudaGraphDestroy(g);
  // Both look-back pairs clean again for whatever runs next, eagerly or as
  // the graph (nothing captured has run yet).
  for (int k = 0; k < 2; ++k) {
    if (ctx->radix_lb[k].p) cudaMemsetAsync(ctx->radix_lb[k].p, 0, ctx->radix_lb[k].cap, s);
    if (ctx->splat_lb[k].p) cudaMemsetAsync(ctx->splat_lb[k].p, 0, ctx->splat_lb[k].cap, s);
  }
  ctx->views_radix_parity = ctx->radix_parity;
  ctx->views_splat_parity = ctx->splat_parity;
  if (rc != CGS_OK || e != cudaSuccess) {
    ctx->views_exec = nullptr;
    return rc != CGS_OK ? rc : ctx->cuda_fail(e, "views capture");
  }
  return CGS_OK;
}

}  // namespace

int cgs_execute_views(cgs_ctx* ctx, uint32_t num_views, const cgs_camera* cameras,
                      const cgs_compositor* comps, const cgs_frame_params* params,
                      uint32_t* const* d_rgba8, int32_t use_graph, cgs_views_stats* stats) {
  if (!ctx || (num_views && (!cameras || !comps || !d_rgba8 || !params))) return CGS_E_ARG;
  for (uint32_t v = 0; v < num_views; ++v) {
    CGS_TRY(check_frame_args(ctx, &cameras[v], &comps[v], &params[v]));
    if (!d_rgba8[v] || ((uintptr_t)d_rgba8[v] & 3)) return ctx->fail(CGS_E_ARG, "view image pointer");
    if (fbits(params[v].strain_split_threshold) != fbits(params[0].strain_split_threshold) ||
        fbits(params[v].mip_filter_3d_var) != fbits(params[0].mip_filter_3d_var))
      return ctx->fail(CGS_E_ARG, "views must share the strain split and Mip settings");
  }
  cgs_views_stats st{};
  if (num_views == 0) {
    if (stats) *stats = st;
    return CGS_OK;
  }
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  CGS_TRY(drain(ctx, true));
  CGS_TRY(ctx->take_sticky());
  if (num_views > ctx->views_cap) {
    if (ctx->h_views) cudaFreeHost(ctx->h_views);
    ctx->h_views = nullptr;
    ctx->views_cap = 0;
    CGS_CUDA(cudaHostAlloc((void**)&ctx->h_views, (size_t)num_views * sizeof(HostCounters),
                           cudaHostAllocDefault), "view counters");
    ctx->views_cap = num_views;
    drop_views_graph(ctx);  // it wrote the old counters
  }
  for (auto& ev : ctx->views_ev)
    if (!ev) CGS_CUDA(cudaEventCreate(&ev), "views event");
  std::vector<cgs_frame_params> prm(params, params + num_views);
  for (auto& q : prm) {
    q.profile_stages = 0;
    q.write_f32 = 0;
    q.force_stage3 = 1;
  }
  ctx->kprof = false;
  ctx->cur = -1;

  auto key_of = [&]() {
    std::vector<unsigned char> k;
    put_bytes(k, &num_views, sizeof(num_views));
    put_bytes(k, cameras, num_views * sizeof(cgs_camera));
    put_bytes(k, comps, num_views * sizeof(cgs_compositor));
    put_bytes(k, prm.data(), num_views * sizeof(cgs_frame_params));
    put_bytes(k, d_rgba8, num_views * sizeof(uint32_t*));
    put_bytes(k, &ctx->alloc_epoch, sizeof(ctx->alloc_epoch));
    put_bytes(k, &ctx->state_epoch, sizeof(ctx->state_epoch));
    put_bytes(k, &ctx->entry_cap, sizeof(ctx->entry_cap));
    return k;
  };
  CGS_CUDA(cudaEventRecord(ctx->views_ev[0], s), "views event");
  if (use_graph && ctx->views_exec && ctx->views_key == key_of()) {
    CGS_CUDA(cudaGraphLaunch(ctx->views_exec, s), "views graph launch");
    CGS_CUDA(cudaEventRecord(ctx->views_ev[1], s), "views event");
    CGS_CUDA(cudaStreamSynchronize(s), "views");
    ctx->radix_parity = ctx->views_radix_parity;
    ctx->splat_parity = ctx->views_splat_parity;
    st.graph_replayed = 1;
    std::vector<uint32_t> cap(num_views, ctx->entry_cap), over;
    const uint32_t cap_before = ctx->entry_cap;
    CGS_TRY(check_views(ctx, num_views, cap.data(), &over, &st.total_tile_entries));
    if (!over.empty()) {
      // render the overflowed views again eagerly; the graph is rebuilt on
      // the next call (its capacity no longer matches)
      for (uint32_t v : over) {
        CGS_TRY(enqueue_view(ctx, &cameras[v], &comps[v], &prm[v], v, d_rgba8[v], false, &cap[v]));
        ++st.views_rerendered;
      }
      CGS_CUDA(cudaStreamSynchronize(s), "views");
      CGS_TRY(check_views(ctx, num_views, cap.data(), &over, &st.total_tile_entries));
      if (!over.empty()) return ctx->fail(CGS_E_CAPACITY, "tile entries exceeded the key buffers");
    }
    if (ctx->entry_cap != cap_before) drop_views_graph(ctx);
  } else {
    CGS_TRY(views_eager(ctx, num_views, cameras, comps, prm.data(), d_rgba8, &st.views_rerendered,
                        &st.total_tile_entries));
    CGS_CUDA(cudaEventRecord(ctx->views_ev[1], s), "views event");
    if (use_graph) {
      // grow the key buffers to the capacity the graph will be captured with
      bool key64 = false;
      for (uint32_t v = 0; v < num_views; ++v) {
        uint32_t lw = 4, lh = 4;
        tile_shape_log2(prm[v].tile_shape, &lw, &lh);
        const uint64_t W = comps[v].screen_width ? comps[v].screen_width : 1u;
        const uint64_t H = comps[v].screen_height ? comps[v].screen_height : 1u;
        key64 = key64 || ((W + (1u << lw) - 1) >> lw) * ((H + (1u << lh) - 1) >> lh) > 65535u;
      }
      CGS_TRY(ensure_entry_buffers(ctx, ctx->entry_cap, key64, ctx->radix_lb_bits ? ctx->radix_lb_bits : 8));
      CGS_TRY(capture_views(ctx, num_views, cameras, comps, prm.data(), d_rgba8));
      ctx->views_key = key_of();
      st.graph_captured = 1;
    }
    CGS_CUDA(cudaStreamSynchronize(s), "views");
  }
  float ms = 0.0f;
  CGS_CUDA(cudaEventElapsedTime(&ms, ctx->views_ev[0], ctx->views_ev[1]), "views time");
  st.ms = ms;
  // The deformed scene is current; Stage 3 lists and the framebuffer belong
  // to no single frame.
  ctx->deformed_valid = ctx->deform_on();
  ctx->s3_valid = false;
  ctx->frame_done = false;
  if (stats) *stats = st;
  return CGS_OK;
}

int cgs_readback_rgba8(cgs_ctx* ctx, uint8_t* dst, uint32_t width, uint32_t height) {
  if (!ctx || !dst) return CGS_E_ARG;
  if (!ctx->frame_done) return ctx->fail(CGS_E_STATE, "no frame rendered");
  if (width != ctx->last_w || height != ctx->last_h)
    return ctx->fail(CGS_E_ARG, "size differs from the last frame");
  cudaSetDevice(ctx->device);
  CGS_TRY(drain(ctx, true));
  CGS_CUDA(cudaMemcpy2DAsync(dst, (size_t)width * 4, ctx->fb_rgba8.p, (size_t)ctx->last_pitch * 4,
                             (size_t)width * 4, height, cudaMemcpyDeviceToHost, ctx->stream),
           "framebuffer readback");
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "framebuffer readback");
  return ctx->take_sticky();
}

namespace {

// Renders frame slot k again (Stages 1-4 from its stored arguments and cage
// vertex snapshots, with the grown key buffers) into out (rows of `pitch`
// pixels), synchronously; the current cage vertices are restored after, and
// the next frame deforms and bins afresh.
int rerender_slot(cgs_ctx* ctx, int k, uint32_t* out, uint32_t pitch) {
  cgs_ctx::Pending& p = ctx->ring[k];
  cudaStream_t s = ctx->stream;
  CGS_TRY(drain(ctx, true));  // every frame checked (a latest-frame re-run happens first)
  DevBuf save_t, save_m;
  if (p.verts_bytes) {
    CGS_CUDA(cudaMalloc(&save_t.p, p.verts_bytes), "vertex save");
    CGS_CUDA(cudaMemcpyAsync(save_t.p, ctx->cage_verts.p, p.verts_bytes, cudaMemcpyDeviceToDevice, s),
             "vertex save");
    CGS_CUDA(cudaMemcpyAsync(ctx->cage_verts.p, p.verts_snap.p, p.verts_bytes,
                             cudaMemcpyDeviceToDevice, s), "vertex restore");
  }
  if (p.mvc_bytes) {
    CGS_CUDA(cudaMalloc(&save_m.p, p.mvc_bytes), "vertex save");
    CGS_CUDA(cudaMemcpyAsync(save_m.p, ctx->mvc_verts.p, p.mvc_bytes, cudaMemcpyDeviceToDevice, s),
             "vertex save");
    CGS_CUDA(cudaMemcpyAsync(ctx->mvc_verts.p, p.mvc_snap.p, p.mvc_bytes,
                             cudaMemcpyDeviceToDevice, s), "vertex restore");
  }
  cgs_frame_params prm = p.params;
  prm.force_stage3 = 1;
  prm.profile_stages = 0;
  prm.write_f32 = 0;
  FrameCtl ctl;
  ctl.allow_cache = false;
  ctl.force_stage1 = true;
  ctl.counters = &ctx->h_ring[k];
  ctl.out_rgba8 = out;
  ctl.out_pitch = pitch;
  const bool kp = ctx->kprof;
  ctx->kprof = false;
  ctx->cur = -1;
  int rc = CGS_OK;
  for (int attempt = 0; attempt < 2; ++attempt) {
    FrameInfo fi;
    rc = enqueue_frame(ctx, &p.cam, &p.comp, &prm, ctl, &fi);
    if (rc != CGS_OK) break;
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      rc = ctx->fail(CGS_E_CUDA, "re-render of an earlier frame failed");
      break;
    }
    const FrameCounters& f = ctx->h_ring[k].fc;
    if (f.status & (kStatusLookbackTimeout | kStatusBarrierTimeout)) {
      rc = ctx->fail(CGS_E_TIMEOUT, "a bounded device-side wait gave up during a re-render");
      break;
    }
    if (!(f.status & kStatusCapacity) && f.entries <= ctx->entry_cap) break;
    ctx->entry_cap = (uint32_t)std::min<uint64_t>((uint64_t)f.entries * 13 / 10 + 4096,
                                                  (uint64_t)kMaxEntryCap);
    rc = ctx->fail(CGS_E_CAPACITY, "tile entries exceed the largest key buffers");
  }
  ctx->kprof = kp;
  if (p.verts_bytes)
    cudaMemcpyAsync(ctx->cage_verts.p, save_t.p, p.verts_bytes, cudaMemcpyDeviceToDevice, s);
  if (p.mvc_bytes)
    cudaMemcpyAsync(ctx->mvc_verts.p, save_m.p, p.mvc_bytes, cudaMemcpyDeviceToDevice, s);
  CGS_CUDA(cudaStreamSynchronize(s), "vertex restore");
  ctx->deformed_valid = false;
  ctx->s3_valid = false;
  ctx->arena_rerendered = true;
  p.overflowed = false;
  ++ctx->rerun_count;
  return rc;
}

}  // namespace

int cgs_readback_wait(cgs_ctx* ctx, uint64_t ticket) {
  if (!ctx) return CGS_E_ARG;
  cgs_ctx::Readback* r = nullptr;
  for (auto& x : ctx->rb)
    if (x.pending && x.ticket == ticket) r = &x;
  if (!r) {
    if (ticket == 0 || ticket > ctx->rb_tickets) return ctx->fail(CGS_E_ARG, "unknown readback ticket");
    return CGS_OK;  // finished and waited for already
  }
  cudaSetDevice(ctx->device);
  r->pending = false;
  CGS_CUDA(cudaEventSynchronize(r->done), "framebuffer readback");
  // The copied frame has finished; check its counters now if no call has
  // (an entry overflow re-renders the latest frame with grown buffers).
  cgs_ctx::Pending& p = ctx->ring[r->frame_slot];
  if (p.used && p.seq == r->frame_seq) CGS_TRY(check_slot(ctx, r->frame_slot, true));
  if (p.overflowed && p.seq == r->frame_seq) {
    // its entries overflowed while a later frame was in flight: render it
    // again into the snapshot buffer, then copy that
    CGS_TRY(rerender_slot(ctx, r->frame_slot, r->stage.as<uint32_t>(), r->W));
    CGS_CUDA(cudaMemcpyAsync(r->dst, r->stage.p, (size_t)r->W * r->H * 4, cudaMemcpyDeviceToHost,
                             ctx->stream), "framebuffer readback");
    CGS_CUDA(cudaStreamSynchronize(ctx->stream), "framebuffer readback");
    return ctx->take_sticky();
  }
  if (ctx->rerun_count != r->reruns && ctx->rerun_seq == r->frame_seq) {
    // re-rendered after the snapshot: copy again while it is the last frame
    if (ctx->latest_slot < 0 || ctx->ring[ctx->latest_slot].seq != r->frame_seq)
      return ctx->fail(CGS_E_CAPACITY,
                       "the frame was re-rendered after its readback began and is no longer the last frame");
    CGS_CUDA(cudaMemcpy2DAsync(r->dst, (size_t)r->W * 4, ctx->fb_rgba8.p, (size_t)ctx->last_pitch * 4,
                               (size_t)r->W * 4, r->H, cudaMemcpyDeviceToHost, ctx->stream),
             "framebuffer readback");
    CGS_CUDA(cudaStreamSynchronize(ctx->stream), "framebuffer readback");
  }
  return ctx->take_sticky();
}

int cgs_readback_rgba8_async(cgs_ctx* ctx, uint8_t* dst, uint32_t width, uint32_t height,
                             uint64_t* ticket) {
  if (!ctx || !dst || !ticket) return CGS_E_ARG;
  if (!ctx->frame_done || ctx->latest_slot < 0) return ctx->fail(CGS_E_STATE, "no frame rendered");
  if (width != ctx->last_w || height != ctx->last_h)
    return ctx->fail(CGS_E_ARG, "size differs from the last frame");
  cudaSetDevice(ctx->device);
  if (!ctx->rb_stream)
    CGS_CUDA(cudaStreamCreateWithFlags(&ctx->rb_stream, cudaStreamNonBlocking), "readback stream");
  const uint64_t t = ctx->rb_tickets + 1;
  cgs_ctx::Readback& r = ctx->rb[t & 1];
  if (r.pending) CGS_TRY(cgs_readback_wait(ctx, r.ticket));  // at most two in flight
  if (!r.ready) CGS_CUDA(cudaEventCreateWithFlags(&r.ready, cudaEventDisableTiming), "readback event");
  if (!r.done) CGS_CUDA(cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming), "readback event");
  const size_t bytes = (size_t)width * height * 4;
  CGS_TRY(ctx->ensure(r.stage, bytes ? bytes : 4, "readback snapshot"));
  // snapshot on the frame stream (the next frame may overwrite the
  // framebuffer), then the host copy on the readback stream
  CGS_CUDA(cudaMemcpy2DAsync(r.stage.p, (size_t)width * 4, ctx->fb_rgba8.p, (size_t)ctx->last_pitch * 4,
                             (size_t)width * 4, height, cudaMemcpyDeviceToDevice, ctx->stream),
           "framebuffer snapshot");
  CGS_CUDA(cudaEventRecord(r.ready, ctx->stream), "readback event");
  CGS_CUDA(cudaStreamWaitEvent(ctx->rb_stream, r.ready, 0), "readback event");
  CGS_CUDA(cudaMemcpyAsync(dst, r.stage.p, bytes, cudaMemcpyDeviceToHost, ctx->rb_stream),
           "framebuffer readback");
  CGS_CUDA(cudaEventRecord(r.done, ctx->rb_stream), "readback event");
  ctx->rb_tickets = t;
  r.ticket = t;
  r.frame_slot = ctx->latest_slot;
  r.frame_seq = ctx->ring[ctx->latest_slot].seq;
  r.reruns = ctx->rerun_count;
  r.dst = dst;
  r.W = width;
  r.H = height;
  r.pending = true;
  *ticket = t;
  return CGS_OK;
}

int cgs_readback_rgba_f32(cgs_ctx* ctx, float* dst, uint32_t width, uint32_t height) {
  if (!ctx || !dst) return CGS_E_ARG;
  if (!ctx->frame_done || !ctx->last_f32) return ctx->fail(CGS_E_STATE, "no f32 frame rendered");
  if (width != ctx->last_w || height != ctx->last_h)
    return ctx->fail(CGS_E_ARG, "size differs from the last frame");
  cudaSetDevice(ctx->device);
  CGS_TRY(drain(ctx, true));
  CGS_CUDA(cudaMemcpyAsync(dst, ctx->fb_f32.p, (size_t)width * height * 16, cudaMemcpyDeviceToHost, ctx->stream), "f32 readback");
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "f32 readback");
  return ctx->take_sticky();
}

int cgs_framebuffer_device(cgs_ctx* ctx, void** d_rgba8, uint32_t* row_pitch_px) {
  if (!ctx || !d_rgba8 || !row_pitch_px) return CGS_E_ARG;
  if (!ctx->frame_done) return ctx->fail(CGS_E_STATE, "no frame rendered");
  CGS_TRY(drain(ctx, true));
  *d_rgba8 = ctx->fb_rgba8.p;
  *row_pitch_px = ctx->last_pitch;
  return CGS_OK;
}

int cgs_invalidate_stage3(cgs_ctx* ctx) {
  if (!ctx) return CGS_E_ARG;
  ctx->s3_valid = false;
  return CGS_OK;
}

int cgs_invalidate(cgs_ctx* ctx) {
  if (ctx) ++ctx->state_epoch;
  if (!ctx) return CGS_E_ARG;
  ctx->s3_valid = false;
  ctx->scene_ready = false;
  ctx->has_cages = false;
  ctx->num_tets = 0;
  ctx->mvc_unbind();
  ctx->spr_ready = false;
  ctx->deformed_valid = false;
  ctx->verts_uploaded = false;
  ctx->last_verts.clear();
  ctx->deform_generation++;
  return CGS_OK;
}

int cgs_read_frame_buffer(cgs_ctx* ctx, int32_t which, void* dst, uint64_t dst_bytes,
                          uint64_t* out_bytes) {
  if (!ctx || !out_bytes) return CGS_E_ARG;
  if (!ctx->frame_done) return ctx->fail(CGS_E_STATE, "no frame rendered");
  if (ctx->arena_rerendered)
    return ctx->fail(CGS_E_STATE, "an earlier frame was rendered again since the last frame; "
                                  "its intermediates replaced the last frame's");
  cudaSetDevice(ctx->device);
  CGS_TRY(drain(ctx, true));
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "read frame buffer");
  const size_t active = ctx->last_active;
  const size_t splits = active > ctx->n ? active - ctx->n : 0;
  const size_t entries = ctx->s3_entries;
  std::vector<char> tmp;
  auto fetch = [&](const DevBuf& b, size_t bytes) -> int {
    tmp.resize(bytes);
    if (bytes == 0) return CGS_OK;
    if (!b.p || b.cap < bytes) return ctx->fail(CGS_E_STATE, "buffer not populated by the last frame");
    cudaError_t e = cudaMemcpy(tmp.data(), b.p, bytes, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? CGS_OK : ctx->cuda_fail(e, "buffer readback");
  };
  std::vector<char> out;
  switch (which) {
    case CGS_BUF_DEFORMED_POS:
    case CGS_BUF_DEFORMED_OPA: {
      if (!ctx->deform_on()) return ctx->fail(CGS_E_STATE, "no cages: no deformed scene");
      CGS_TRY(fetch(ctx->def_pos, active * 16));
      const float* f = (const float*)tmp.data();
      if (which == CGS_BUF_DEFORMED_POS) {
        out.resize(active * 12);
        float* o = (float*)out.data();
        for (size_t i = 0; i < active; ++i) {
          o[3 * i] = f[4 * i]; o[3 * i + 1] = f[4 * i + 1]; o[3 * i + 2] = f[4 * i + 2];
        }
      } else {
        out.resize(active * 4);
        float* o = (float*)out.data();
        for (size_t i = 0; i < active; ++i) o[i] = f[4 * i + 3];
      }
      break;
    }
    case CGS_BUF_DEFORMED_COV: {
      if (!ctx->deform_on()) return ctx->fail(CGS_E_STATE, "no cages: no deformed scene");
      CGS_TRY(fetch(ctx->def_cova, active * 16));
      std::vector<char> a = tmp;
      CGS_TRY(fetch(ctx->def_covb, active * 8));
      const float* fa = (const float*)a.data();
      const float* fb = (const float*)tmp.data();
      out.resize(active * 24);
      float* o = (float*)out.data();
      for (size_t i = 0; i < active; ++i) {
        for (int k = 0; k < 4; ++k) o[6 * i + k] = fa[4 * i + k];
        o[6 * i + 4] = fb[2 * i];
        o[6 * i + 5] = fb[2 * i + 1];
      }
      break;
    }
    case CGS_BUF_SPLIT_META:
      CGS_TRY(fetch(ctx->split_meta, splits * 8));
      out = tmp;
      break;
    case CGS_BUF_SPLAT_ATTRS:
    case CGS_BUF_EXTENTS: {
      CGS_TRY(fetch(ctx->recs, active * sizeof(SplatRec)));
      const SplatRec* r = (const SplatRec*)tmp.data();
      if (which == CGS_BUF_EXTENTS) {
        out.resize(active * 4);
        uint32_t* o = (uint32_t*)out.data();
        for (size_t i = 0; i < active; ++i) o[i] = fbits(r[i].cc.w);
      } else {
        out.assign(active * 40, 0);
        float* o = (float*)out.data();
        for (size_t i = 0; i < active; ++i) {
          if (fbits(r[i].cc.w) == 0) continue;
          const float v[10] = {r[i].geo.x, r[i].geo.y, r[i].geo.z, r[i].geo.w, r[i].cc.x,
                               r[i].cc.y,  r[i].rgb.x, r[i].rgb.y, r[i].rgb.z, r[i].cc.z};
          std::memcpy(o + 10 * i, v, 40);
        }
      }
      break;
    }
    case CGS_BUF_TILE_OFFSETS: {
      // The binning kernel scans the counts in depth order; the reference's
      // buffer is the scan in splat order, rebuilt here from the per-slot
      // offsets, the splat order and the entry total.
      const size_t sa = ctx->s3_active;
      CGS_TRY(fetch(ctx->offsets, sa * 4));
      const std::vector<char> off_b = tmp;
      CGS_TRY(fetch(ctx->sids[ctx->s3_order_src], sa * 4));
      const uint32_t* off = (const uint32_t*)off_b.data();
      const uint32_t* ord = (const uint32_t*)tmp.data();
      std::vector<uint32_t> cnt(sa, 0);
      for (size_t j = 0; j < sa; ++j) {
        const uint32_t next = j + 1 < sa ? off[j + 1] : (uint32_t)entries;
        if (ord[j] >= sa) return ctx->fail(CGS_E_STATE, "splat order out of range");
        cnt[ord[j]] = next - off[j];
      }
      out.resize(sa * 4);
      uint32_t* o = (uint32_t*)out.data();
      uint32_t run = 0;
      for (size_t i = 0; i < sa; ++i) {
        o[i] = run;
        run += cnt[i];
      }
      break;
    }
    case CGS_BUF_SORTED_KEYS:
      if (ctx->s3_transpose) {
        // The tile transpose sorts splat indices only; the 32-bit keys are
        // tile << depth_bits | depth key, from the ranges and the splat order.
        const size_t sa = ctx->s3_active;
        CGS_TRY(fetch(ctx->ranges, (size_t)ctx->last_tiles * 8));
        const std::vector<char> rg = tmp;
        CGS_TRY(fetch(ctx->sids[ctx->s3_order_src], sa * 4));
        const std::vector<char> ord = tmp;
        CGS_TRY(fetch(ctx->skeys[ctx->s3_order_src], sa * 4));
        const std::vector<char> dk = tmp;
        CGS_TRY(fetch(ctx->ids[ctx->s3_src], entries * 4));
        const uint32_t* r = (const uint32_t*)rg.data();
        const uint32_t* os = (const uint32_t*)ord.data();
        const uint32_t* ds = (const uint32_t*)dk.data();
        const uint32_t* ids = (const uint32_t*)tmp.data();
        std::vector<uint32_t> dq_of(sa, 0);
        for (size_t j = 0; j < sa; ++j)
          if (os[j] < sa) dq_of[os[j]] = ds[j];
        out.assign(entries * 4, 0);
        uint32_t* o = (uint32_t*)out.data();
        const uint32_t db = ctx->s3_depth_bits;
        for (uint32_t t = 0; t < ctx->last_tiles; ++t)
          for (uint32_t i = r[2 * t]; i < r[2 * t + 1] && i < entries; ++i)
            o[i] = (db >= 32 ? 0u : (t << db)) | (ids[i] < sa ? dq_of[ids[i]] : 0u);
      } else if (!ctx->s3_key64) {
        CGS_TRY(fetch(ctx->keys[ctx->s3_src], entries * 4));
        out = tmp;
      } else {
        CGS_TRY(fetch(ctx->keys[ctx->s3_src], entries * 4));
        std::vector<char> t = tmp;
        CGS_TRY(fetch(ctx->depths[ctx->s3_src], entries * 4));
        out.resize(entries * 8);
        uint64_t* o = (uint64_t*)out.data();
        for (size_t i = 0; i < entries; ++i)
          o[i] = ((uint64_t)((uint32_t*)t.data())[i] << 32) | ((uint32_t*)tmp.data())[i];
      }
      break;
    case CGS_BUF_SORTED_IDS:
      CGS_TRY(fetch(ctx->ids[ctx->s3_src], entries * 4));
      out = tmp;
      break;
    case CGS_BUF_TILE_RANGES:
      CGS_TRY(fetch(ctx->ranges, (size_t)ctx->last_tiles * 8));
      out = tmp;
      break;
    case CGS_BUF_TET_JACOBIANS:
      CGS_TRY(fetch(ctx->tet_J, (size_t)ctx->num_tets * 36));
      out = tmp;
      break;
    case CGS_BUF_TET_ROTATIONS:
      CGS_TRY(fetch(ctx->tet_R, (size_t)ctx->num_tets * 36));
      out = tmp;
      break;
    case CGS_BUF_MVC_ROTATIONS:
      CGS_TRY(fetch(ctx->mvc_R, (size_t)ctx->mvc_nb * 36));
      out = tmp;
      break;
    case CGS_BUF_TET_STRETCH:
      CGS_TRY(fetch(ctx->tet_S, (size_t)ctx->num_tets * 4));
      out = tmp;
      break;
    default:
      return ctx->fail(CGS_E_ARG, "unknown buffer id");
  }
  *out_bytes = out.size();
  if (dst) {
    if (dst_bytes < out.size()) return ctx->fail(CGS_E_ARG, "destination too small");
    std::memcpy(dst, out.data(), out.size());
  }
  return CGS_OK;
}

namespace {

// The band bases B_l and B_l^+ are constants: built on the device once.
int ensure_sh_basis(cgs_ctx* ctx) {
  if (ctx->sh_basis_ready) return CGS_OK;
  CGS_TRY(ctx->ensure(ctx->sh_basis, sh_basis_bytes(), "sh basis"));
  CGS_CUDA(launch_sh_basis(ctx->sh_basis.p, ctx->stream), "sh basis launch");
  ctx->sh_basis_ready = true;
  return CGS_OK;
}

}  // namespace

int cgs_sh_rotate(cgs_ctx* ctx, uint64_t n, float* d_sh, uint32_t num_rotations,
                  const float* d_rotations, const uint32_t* d_index, uint32_t degree) {
  if (!ctx) return CGS_E_ARG;
  if (n == 0 || degree == 0) return CGS_OK;
  if (!d_sh || !d_rotations || num_rotations == 0) return CGS_E_ARG;
  if (((uintptr_t)d_sh & 15u) != 0) return ctx->fail(CGS_E_ARG, "coefficients must be 16-byte aligned");
  cudaSetDevice(ctx->device);
  CGS_TRY(drain(ctx, true));
  const uint32_t deg = degree > 3 ? 3u : degree;
  CGS_TRY(ensure_sh_basis(ctx));
  CGS_TRY(ctx->ensure(ctx->sh_table, (size_t)num_rotations * kShRotStride * 4 + 64, "sh rotations"));
  uint32_t* bad = (uint32_t*)(ctx->sh_table.as<char>() + (size_t)num_rotations * kShRotStride * 4);
  CGS_CUDA(cudaMemsetAsync(bad, 0, 4, ctx->stream), "sh rotate status");
  CGS_CUDA(launch_sh_rotators(num_rotations, d_rotations, ctx->sh_basis.p, deg,
                              ctx->sh_table.as<float>(), ctx->stream), "sh rotators launch");
  CGS_CUDA(launch_sh_apply(n, d_sh, ctx->sh_table.as<float>(), num_rotations, d_index, deg, bad,
                           ctx->stream), "sh rotate launch");
  uint32_t h_bad = 0;
  CGS_CUDA(cudaMemcpyAsync(&h_bad, bad, 4, cudaMemcpyDeviceToHost, ctx->stream), "sh rotate status");
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "sh rotate");
  if (h_bad) return ctx->fail(CGS_E_ARG, "rotation index out of range (those blocks left unchanged)");
  return CGS_OK;
}

int cgs_export_deformed(cgs_ctx* ctx, uint32_t sh_degree, uint64_t capacity, float* pos, float* cov,
                        float* opa, float* sh, uint64_t* out_count) {
  if (!ctx || !out_count) return CGS_E_ARG;
  *out_count = 0;
  if (!ctx->scene_ready) return ctx->fail(CGS_E_STATE, "no scene uploaded");
  cudaSetDevice(ctx->device);
  CGS_TRY(drain(ctx, true));
  const bool deformed = ctx->deform_on();
  if (deformed && !ctx->deformed_valid)
    return ctx->fail(CGS_E_STATE, "the cage state has changed since the last frame; execute a frame first");
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "export");
  const uint32_t n = ctx->n;
  uint32_t splits = 0;
  if (deformed) CGS_CUDA(cudaMemcpy(&splits, ctx->persist.p, 4, cudaMemcpyDeviceToHost), "split count");
  const uint64_t total = (uint64_t)n + splits;
  *out_count = total;
  if (!pos && !cov && !opa && !sh) return CGS_OK;
  if (capacity < total) return ctx->fail(CGS_E_ARG, "capacity below the exported splat count");
  if (total == 0) return CGS_OK;
  const uint32_t deg = sh_degree > 3 ? 3u : sh_degree;
  cudaStream_t s = ctx->stream;

  ExportArgs a{};
  a.n_rest = n;
  if (deformed) {
    a.pos = ctx->def_pos.as<float4>();
    a.cova = ctx->def_cova.as<float4>();
    a.covb = ctx->def_covb.as<float2>();
  } else {
    a.pos = ctx->rest_pos.as<float4>();
    a.cova = ctx->rest_cova.as<float4>();
    a.covb = ctx->rest_covb.as<float2>();
  }
  a.sh = ctx->rest_sh.p;
  a.sh_f16 = ctx->sh_f16;
  a.sh_stride = n;
  a.degree = deg;
  if (deformed && sh && deg > 0) {
    // band matrices of every tet's and every MVC slot's rotation of the last
    // Stage 1, tets first
    const uint32_t T = ctx->has_cages ? ctx->num_tets : 0u, nb = ctx->mvc_nb;
    CGS_TRY(ensure_sh_basis(ctx));
    CGS_TRY(ctx->ensure(ctx->sh_table, ((size_t)T + nb) * kShRotStride * 4 + 64, "sh rotations"));
    float* table = ctx->sh_table.as<float>();
    CGS_CUDA(launch_sh_rotators(T, ctx->tet_R.as<float>(), ctx->sh_basis.p, deg, table, s),
             "sh rotators launch");
    if (nb)
      CGS_CUDA(launch_sh_rotators(nb, ctx->mvc_R.as<float>(), ctx->sh_basis.p, deg,
                                  table + (size_t)T * kShRotStride, s), "sh rotators launch");
    a.bind_tet = ctx->bind_tet.as<uint32_t>();
    a.bind_w = ctx->bind_w.as<float4>();
    a.split_meta = ctx->split_meta.as<uint2>();
    a.num_tets = T;
    a.mvc = nb > 0;
    a.table = table;
  } else if (deformed) {
    a.split_meta = ctx->split_meta.as<uint2>();
  }
  // Children read their parent's SH even when nothing rotates.
  if (!a.split_meta && splits) return ctx->fail(CGS_E_STATE, "split children without their meta");

  // Chunks of at most 2^20 splats through one device staging area (58 floats
  // a splat), copied into the caller's arrays.
  const uint32_t chunk = (uint32_t)std::min<uint64_t>(total, 1u << 20);
  CGS_TRY(ctx->ensure(ctx->sh_stage, (size_t)chunk * 58 * 4, "export staging"));
  float* st = ctx->sh_stage.as<float>();
  for (uint64_t first = 0; first < total; first += chunk) {
    const uint32_t cnt = (uint32_t)std::min<uint64_t>(chunk, total - first);
    a.first = (uint32_t)first;
    a.count = cnt;
    a.out_pos = pos ? st : nullptr;
    a.out_cov = cov ? st + (size_t)chunk * 3 : nullptr;
    a.out_opa = opa ? st + (size_t)chunk * 9 : nullptr;
    a.out_sh = sh ? st + (size_t)chunk * 10 : nullptr;
    CGS_CUDA(launch_export(a, s), "export launch");
    if (pos)
      CGS_CUDA(cudaMemcpyAsync(pos + 3 * first, a.out_pos, (size_t)cnt * 12, cudaMemcpyDeviceToHost, s),
               "export positions");
    if (cov)
      CGS_CUDA(cudaMemcpyAsync(cov + 6 * first, a.out_cov, (size_t)cnt * 24, cudaMemcpyDeviceToHost, s),
               "export covariances");
    if (opa)
      CGS_CUDA(cudaMemcpyAsync(opa + first, a.out_opa, (size_t)cnt * 4, cudaMemcpyDeviceToHost, s),
               "export opacities");
    if (sh)
      CGS_CUDA(cudaMemcpyAsync(sh + 48 * first, a.out_sh, (size_t)cnt * 192, cudaMemcpyDeviceToHost, s),
               "export sh");
  }
  CGS_CUDA(cudaStreamSynchronize(s), "export");
  return CGS_OK;
}

const char* cgs_kernel_name(int32_t id) {
  static const char* names[CGS_KERNEL_COUNT] = {"clear", "tet_transforms", "deform", "project",
                                                "bin", "entry_sort", "tile_ranges", "composite",
                                                "splat_sort", "mvc", "field"};
  return (id >= 0 && id < CGS_KERNEL_COUNT) ? names[id] : "unknown";
}

int cgs_kernel_profile_read(cgs_ctx* ctx, cgs_kernel_profile* out) {
  if (!ctx || !out) return CGS_E_ARG;
  cudaSetDevice(ctx->device);
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "profile read");
  CGS_TRY(drain(ctx, true));
  *out = ctx->kp_acc;
  return ctx->take_sticky();
}

int cgs_kernel_profile_reset(cgs_ctx* ctx) {
  if (!ctx) return CGS_E_ARG;
  cudaSetDevice(ctx->device);
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "profile reset");
  CGS_TRY(drain(ctx, true));
  ctx->kp_acc = cgs_kernel_profile{};
  return ctx->take_sticky();
}

int cgs_scan_u32(cgs_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint64_t n,
                 uint64_t* total) {
  if (!ctx) return CGS_E_ARG;
  if (n > 0 && (!d_in || !d_out)) return ctx->fail(CGS_E_ARG, "null device pointer");
  if (n >= 0xFFFFFFFFull) return ctx->fail(CGS_E_CAPACITY, "scan length must be < 2^32");
  cudaSetDevice(ctx->device);
  if (n == 0) {
    if (total) *total = 0;
    return CGS_OK;
  }
  const size_t tiles = scan_tiles((uint32_t)n);
  const size_t bytes = 256 + tiles * 8;
  CGS_TRY(ctx->ensure(ctx->prim[0], bytes, "scan scratch"));
  char* b = ctx->prim[0].as<char>();
  CGS_CUDA(cudaMemsetAsync(b, 0, bytes, ctx->stream), "clear scan scratch");
  uint32_t* words = (uint32_t*)b;  // [0] total, [1] tile counter, [2] status
  CGS_CUDA(launch_scan_u32(d_in, d_out, (uint32_t)n, words, (unsigned long long*)(b + 256),
                           words + 1, words + 2, ctx->stream),
           "scan launch");
  uint32_t h[3] = {0, 0, 0};
  CGS_CUDA(cudaMemcpyAsync(ctx->h_misc + 1, words, 12, cudaMemcpyDeviceToHost, ctx->stream), "scan total");
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "scan");
  std::memcpy(h, ctx->h_misc + 1, 12);
  if (h[2] & kStatusLookbackTimeout) return ctx->fail(CGS_E_TIMEOUT, "scan look-back wait gave up");
  if (total) *total = h[0];
  return CGS_OK;
}

static int sort_common(cgs_ctx* ctx, uint32_t* d_keys, uint32_t* d_vals, uint32_t* d_vals2,
                       uint64_t n, uint32_t key_bits, int32_t digit_bits, int* out_in_scratch,
                       uint32_t** alt) {
  const uint32_t rb = digit_bits == 0 ? 8u : (uint32_t)digit_bits;
  const uint32_t passes = sort_passes(key_bits, rb);
  const uint32_t stiles = sort_tiles((uint32_t)n);
  const size_t R = (size_t)1 << rb;
  const size_t hdr = 256 + 8 * 256 * 4;
  const size_t bytes = hdr + (size_t)passes * stiles * R * 4;
  CGS_TRY(ctx->ensure(ctx->prim[0], bytes, "sort scratch"));
  CGS_TRY(ctx->ensure(ctx->prim[1], (size_t)n * 4, "sort alt keys"));
  CGS_TRY(ctx->ensure(ctx->prim[2], (size_t)n * 4, "sort alt values"));
  if (d_vals2) CGS_TRY(ctx->ensure(ctx->prim[3], (size_t)n * 4, "sort alt values"));
  char* b = ctx->prim[0].as<char>();
  CGS_CUDA(cudaMemsetAsync(b, 0, bytes, ctx->stream), "clear sort scratch");
  uint32_t* words = (uint32_t*)b;  // [0] n, [1] status, [2..] tile counters
  const uint32_t n32 = (uint32_t)n;
  CGS_CUDA(cudaMemcpyAsync(words, &n32, 4, cudaMemcpyHostToDevice, ctx->stream), "sort n");
  uint32_t* hist = (uint32_t*)(b + 256);
  CGS_CUDA(launch_histogram(d_keys, words, n32, 0, key_bits, rb, hist, ctx->stream), "histogram");
  SortArgs sa{};
  sa.keys[0] = d_keys;
  sa.keys[1] = ctx->prim[1].as<uint32_t>();
  sa.vals[0] = d_vals;
  sa.vals[1] = ctx->prim[2].as<uint32_t>();
  if (d_vals2) {
    sa.vals2[0] = d_vals2;
    sa.vals2[1] = ctx->prim[3].as<uint32_t>();
  }
  sa.n_ptr = words;
  sa.capacity = n32;
  sa.first_bit = 0;
  sa.num_bits = key_bits;
  sa.radix_bits = rb;
  sa.hist = hist;
  sa.status = b + hdr;
  sa.tile_ctr = words + 2;
  sa.status_word = words + 1;
  sa.src = 0;
  int src = 0;
  CGS_CUDA(run_radix_sort(sa, &src, ctx->stream), "radix sort");
  *out_in_scratch = src;
  alt[0] = sa.keys[1];
  alt[1] = sa.vals[1];
  alt[2] = sa.vals2[1];
  return CGS_OK;
}

static int sort_status(cgs_ctx* ctx) {
  uint32_t* words = ctx->prim[0].as<uint32_t>();
  CGS_CUDA(cudaMemcpyAsync(ctx->h_misc + 1, words, 8, cudaMemcpyDeviceToHost, ctx->stream), "sort status");
  CGS_CUDA(cudaStreamSynchronize(ctx->stream), "sort");
  if (ctx->h_misc[2] & kStatusLookbackTimeout) return ctx->fail(CGS_E_TIMEOUT, "sort look-back wait gave up");
  return CGS_OK;
}

int cgs_sort_pairs_u32(cgs_ctx* ctx, uint32_t* d_keys, uint32_t* d_vals, uint64_t n,
                       uint32_t key_bits, int32_t digit_bits) {
  if (!ctx) return CGS_E_ARG;
  if (digit_bits != 0 && digit_bits != 4 && digit_bits != 8)
    return ctx->fail(CGS_E_ARG, "digit_bits must be 0, 4 or 8");
  if (key_bits == 0 || key_bits > 32) return ctx->fail(CGS_E_ARG, "key_bits must be in 1..32");
  if (n >= (1ull << 30)) return ctx->fail(CGS_E_CAPACITY, "sort length must be < 2^30");
  if (n > 0 && (!d_keys || !d_vals)) return ctx->fail(CGS_E_ARG, "null device pointer");
  if (n <= 1) return CGS_OK;
  cudaSetDevice(ctx->device);
  int src = 0;
  uint32_t* alt[3];
  CGS_TRY(sort_common(ctx, d_keys, d_vals, nullptr, n, key_bits, digit_bits, &src, alt));
  if (src == 1) {
    CGS_CUDA(cudaMemcpyAsync(d_keys, alt[0], n * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy keys");
    CGS_CUDA(cudaMemcpyAsync(d_vals, alt[1], n * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy values");
  }
  return sort_status(ctx);
}

int cgs_sort_pairs_u64(cgs_ctx* ctx, uint32_t* d_tiles, uint32_t* d_depths, uint32_t* d_ids,
                       uint64_t n, uint32_t tile_bits, int32_t digit_bits) {
  if (!ctx) return CGS_E_ARG;
  if (digit_bits != 0 && digit_bits != 4 && digit_bits != 8)
    return ctx->fail(CGS_E_ARG, "digit_bits must be 0, 4 or 8");
  if (tile_bits == 0 || tile_bits > 32) return ctx->fail(CGS_E_ARG, "tile_bits must be in 1..32");
  if (n >= (1ull << 30)) return ctx->fail(CGS_E_CAPACITY, "sort length must be < 2^30");
  if (n > 0 && (!d_tiles || !d_depths || !d_ids)) return ctx->fail(CGS_E_ARG, "null device pointer");
  if (n <= 1) return CGS_OK;
  cudaSetDevice(ctx->device);
  // Pass group 1: by depth, carrying (id, tile).
  int src = 0;
  uint32_t* alt[3];
  CGS_TRY(sort_common(ctx, d_depths, d_ids, d_tiles, n, 32, digit_bits, &src, alt));
  if (src == 1) {
    CGS_CUDA(cudaMemcpyAsync(d_depths, alt[0], n * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
    CGS_CUDA(cudaMemcpyAsync(d_ids, alt[1], n * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
    CGS_CUDA(cudaMemcpyAsync(d_tiles, alt[2], n * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
  }
  CGS_TRY(sort_status(ctx));
  // Pass group 2: by tile, carrying (id, depth).
  CGS_TRY(sort_common(ctx, d_tiles, d_ids, d_depths, n, tile_bits, digit_bits, &src, alt));
  if (src == 1) {
    CGS_CUDA(cudaMemcpyAsync(d_tiles, alt[0], n * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
    CGS_CUDA(cudaMemcpyAsync(d_ids, alt[1], n * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
    CGS_CUDA(cudaMemcpyAsync(d_depths, alt[2], n * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
  }
  return sort_status(ctx);
}

}  // extern "C"
#pragma GCC visibility pop
