// Host orchestration and the C ABI of include/gs_cuda.h.
//
// A gs_rasterizer owns every device buffer of the step, sized once at
// creation for a capacity of surfels, views, pixels and tile entries (the
// reference allocates once the same way and never reallocates,
// crates/gs-kernels/src/rasterizer.rs:108-316). Passes are stream-ordered and
// read element counts from device memory, so forward, loss, backward and the
// optimizer never synchronise with the host; the batched training step is
// captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "gs_cuda.h"
#include "gs_common.cuh"
#include "gs_kernels.h"

namespace gs {

static thread_local std::string g_last_error;

void set_error_message(const std::string& msg) { g_last_error = msg; }

int cuda_fail(cudaError_t e, const char* expr, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", expr, cudaGetErrorString(e), file, line);
  g_last_error = buf;
  return GS_ERR_CUDA;
}

}  // namespace gs

using namespace gs;

namespace {

constexpr int MAX_VIEWS_HARD = 64;

template <typename T>
cudaError_t dalloc(T*& p, size_t count) {
  p = nullptr;
  if (count == 0) count = 1;
  return cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
}

struct DynParams {
  float lr[5];
  float reg[5];
  float bc1, bc2;
};

}  // namespace

struct gs_rasterizer {
  gs_raster_config cfg{};
  int device = 0;
  int num_sms = 148;
  uint32_t cap = 0, max_views = 1;
  uint64_t max_pixels = 0, max_entries = 0, max_items = 0;
  uint32_t max_tiles = 0;
  float lambda_dist = 0.f;
  bool det = false, persistent = false, color_only = false, tight = false;
  // Raster launch shapes (autotuned): staging batch and pixels per thread.
  int fwd_batch = 128, fwd_ppt = 1, bwd_batch = 128, bwd_ppt = 2;
  int tile = 16;  // tile edge in pixels: 8, 16 (the reference's) or 32
  std::string err;

  // activated parameters (fp32) and the 16-bit SH copy
  float4* positions = nullptr;
  float2* scales = nullptr;
  float4* quats = nullptr;
  float* opacities = nullptr;
  float* sh = nullptr;
  void* sh_half = nullptr;
  uint32_t n_uploaded = 0;

  // per item (view*n + surfel)
  void* records = nullptr;
  uint4* rects = nullptr;
  uint32_t* item_keys[2] = {nullptr, nullptr};
  uint32_t* item_vals[2] = {nullptr, nullptr};
  uint32_t* counts = nullptr;
  uint32_t* offsets = nullptr;
  uint32_t* entry_offset = nullptr;

  // per entry: (tile, item) pairs, ping-pong buffers of the tile sort
  uint2* ent_pairs[2] = {nullptr, nullptr};
  uint32_t* exp_item = nullptr;
  float* partials = nullptr;
  uint2* ranges = nullptr;
  int ent_in1 = 0;
  double* normal_loss_sums = nullptr;  // per view: Σ α (1 − n̂·N_d) of the last gs_loss_normal
  // stored-state mode: contributor masks of the last colour-only forward
  uint32_t* mask = nullptr;
  uint32_t* mask_off = nullptr;
  uint32_t* mask_words = nullptr;
  bool stored_state = false, mask_valid = false;
  // colour-only forward on 16-pixel tiles: per tile entry, the 4-row pixel
  // groups it composited into (read by the matching backward)
  uint8_t* gmask = nullptr;
  bool gmask_valid = false;
  // persistent raster kernels: tiles in heaviest-first order (from the ranges
  // of the last persistent forward)
  uint32_t* tile_order = nullptr;
  bool order_valid = false;
  // per tile, the largest contributor count of the last persistent forward:
  // the backward's work, used to order its tiles
  uint32_t* tile_walk = nullptr;
  // Occlusion cut of the chosen-form step (off with GS_FLAG_FULL_LISTS and
  // in deterministic and stored-state modes): per tile the deepest depth key
  // the next step bins (all ones: the whole list), the tiles a truncated list
  // left unfinished, the items' depth keys and the completion pass's counts.
  bool cut_on = false;
  uint32_t* tile_cut = nullptr;
  uint32_t* inc_list = nullptr;
  uint32_t* inc_skip = nullptr;
  uint32_t* inc_src = nullptr;
  uint8_t* inc_flag = nullptr;
  uint32_t* item_key = nullptr;
  uint32_t* counts2 = nullptr;
  uint32_t* sorted_counts = nullptr;  // counts in depth order (written by the depth sort's final pass)
  uint32_t* cutw = nullptr;  // [0] unfinished tiles [1] completion items [2] completion entries (u32) [3] tile counter
  unsigned long long* entry_total2 = nullptr;
  std::vector<uint32_t> cut_sig;  // step shape and views the cuts were recorded for

  // device scalars: [0] entry total u64, then u32 words
  unsigned long long* entry_total = nullptr;
  uint32_t* words = nullptr;  // [0] entry count u32, [1] error word, [2] fwd tile counter, [3] bwd tile counter,
                              // [4..6] densify counts
  // per pixel
  float4 *out_color = nullptr, *out_aux = nullptr, *out_normal = nullptr, *dl_dcolor = nullptr,
         *dl_dnormal = nullptr, *target = nullptr;
  uint32_t* out_nc = nullptr;
  float* coef = nullptr;
  double* loss_sums = nullptr;

  // gradients
  float* grad_geom = nullptr;
  float4* grad_pos = nullptr;
  float2* grad_scales = nullptr;
  float4* grad_quat = nullptr;
  float* grad_opacity = nullptr;
  float* grad_sh = nullptr;
  float* grad_cam = nullptr;
  // deterministic mode: per (unit, view) camera partials of the projection
  // backward, summed in unit order
  float* cam_part = nullptr;

  // optimizer
  float* raw[5] = {};
  float* mom1[5] = {};
  float* mom2[5] = {};
  uint32_t t = 0;
  bool optim_ready = false;
  // limits (SM cycles) of the fused projection backward + Adam kernel's two
  // bounded waits on its optimizer-row copies (gs_rasterizer_set_wait_limits)
  long long wait_cycles[2] = {2000000000ll, 2000000000ll};
  float* accum_norm = nullptr;
  uint32_t accum_steps = 0;
  float* dyn_dev = nullptr;

  // densify scratch
  // MCMC relocation: scratch (allocated on first use) and device generator state
  uint32_t* mcmc_u32 = nullptr;           // 19 arrays of capacity u32
  unsigned long long* mcmc_u64 = nullptr;  // weight, cum (capacity each) + total
  uint64_t* mcmc_jump = nullptr;           // MCMC_JUMP_LEVELS x 64 rows
  uint64_t* mcmc_rng = nullptr;
  uint32_t* mcmc_counters = nullptr;
  uint32_t* dens_flags = nullptr;
  uint32_t* dens_slots = nullptr;
  float* dens_tmp = nullptr;

  // views: [0, max_views) batched layout, [max_views, 2*max_views) single-view layout
  ViewInfo* views_dev = nullptr;
  std::vector<ViewInfo> views_batched, views_single;
  uint32_t last_nv = 0, last_n = 0;
  int last_tiles = 0;
  bool last_batched = true;
  const ViewInfo* last_views_dev = nullptr;
  const ViewInfo* last_views_host = nullptr;
  bool have_forward = false;
  int last_prec = 0;  // storage precision of the last forward's records
  unsigned long long* work_counts = nullptr;  // gs_raster_work's device counters

  void* scan_scratch = nullptr;
  void* sort_scratch = nullptr;

  // graph of the chosen-form step
  cudaStream_t cap_stream = nullptr;
  // side stream of the chosen step: clears grad_geom and orders the
  // backward's tiles while the forward and the loss run
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_fwd = nullptr, ev_side = nullptr;
  cudaGraphExec_t graph = nullptr;
  std::vector<uint64_t> graph_key;
};

struct gs_binner {
  uint32_t max_items = 0, num_tiles = 0;
  uint64_t max_entries = 0;
  uint4* rects_tmp = nullptr;  // unused: rects come from the caller
  uint32_t* counts = nullptr;
  uint32_t* ref_offsets = nullptr;
  uint32_t* offsets = nullptr;
  uint32_t* item_keys[2] = {nullptr, nullptr};
  uint32_t* item_vals[2] = {nullptr, nullptr};
  uint2* ent_pairs[2] = {nullptr, nullptr};
  uint32_t* sorted_entries = nullptr;
  uint32_t* entry_items = nullptr;
  uint2* ranges = nullptr;
  unsigned long long* total = nullptr;
  uint32_t* words = nullptr;
  int ent_in1 = 0;
  void* scan_scratch = nullptr;
  void* sort_scratch = nullptr;
};

namespace {

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Stage timer of the profiled step: events recorded on the launch stream at
// stage boundaries; times of a stage are summed over the views of a step.
constexpr int N_STAGES = 9;
struct Prof {
  std::vector<cudaEvent_t> ev;
  std::vector<int> stage;  // stage index ending at ev[k]
  void mark(int stg, cudaStream_t st) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, st);
    ev.push_back(e);
    stage.push_back(stg);
  }
  ~Prof() { for (auto e : ev) cudaEventDestroy(e); }
};
inline void mark(Prof* p, int stg, cudaStream_t st) { if (p) p->mark(stg, st); }

gs_status fail(gs_rasterizer* r, gs_status st, const std::string& msg) {
  if (r) r->err = msg;
  g_last_error = msg;
  return st;
}

#define TRY_CUDA(r, expr)                                                                            \
  do {                                                                                               \
    cudaError_t _e = (expr);                                                                         \
    if (_e != cudaSuccess)                                                                           \
      return fail((r), GS_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e));             \
  } while (0)
#define TRY_LAUNCH(r, expr)                                                                          \
  do {                                                                                               \
    int _e = (expr);                                                                                 \
    if (_e != 0)                                                                                     \
      return fail((r), GS_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString((cudaError_t)_e)); \
  } while (0)

// glam Mat3::from_quat of the normalised quaternion (rasterizer.rs:410).
void rotation_of(const float q_in[4], float rot[9]) {
  const float inv = 1.0f / std::sqrt(q_in[0] * q_in[0] + q_in[1] * q_in[1] + q_in[2] * q_in[2] + q_in[3] * q_in[3]);
  const float x = q_in[0] * inv, y = q_in[1] * inv, z = q_in[2] * inv, w = q_in[3] * inv;
  const float x2 = x + x, y2 = y + y, z2 = z + z;
  const float xx = x * x2, xy = x * y2, xz = x * z2;
  const float yy = y * y2, yz = y * z2, zz = z * z2;
  const float wx = w * x2, wy = w * y2, wz = w * z2;
  rot[0] = 1.0f - (yy + zz); rot[1] = xy + wz; rot[2] = xz - wy;
  rot[3] = xy - wz; rot[4] = 1.0f - (xx + zz); rot[5] = yz + wx;
  rot[6] = xz + wy; rot[7] = yz - wx; rot[8] = 1.0f - (xx + yy);
}

// The same rotation in double (quaternion normalised in double, as the
// oracle's quat_to_mat does): the projection's accurate surfel centres.
void rotation64_of(const float q_in[4], double rot[9]) {
  const double q0 = q_in[0], q1 = q_in[1], q2 = q_in[2], q3 = q_in[3];
  const double n = std::sqrt(q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3);
  const double x = q0 / n, y = q1 / n, z = q2 / n, w = q3 / n;
  rot[0] = 1 - 2 * (y * y + z * z); rot[1] = 2 * (x * y + w * z); rot[2] = 2 * (x * z - w * y);
  rot[3] = 2 * (x * y - w * z); rot[4] = 1 - 2 * (x * x + z * z); rot[5] = 2 * (y * z + w * x);
  rot[6] = 2 * (x * z + w * y); rot[7] = 2 * (y * z - w * x); rot[8] = 1 - 2 * (x * x + y * y);
}

ViewInfo make_view(const gs_camera& c, int tile) {
  ViewInfo v{};
  rotation_of(c.quat, v.rot);
  rotation64_of(c.quat, v.rot64);
  for (int k = 0; k < 3; ++k) v.center[k] = c.center[k];
  v.focal = c.focal;
  v.width = (int)c.width;
  v.height = (int)c.height;
  v.cx = (float)c.width * 0.5f;
  v.cy = (float)c.height * 0.5f;
  v.tile = tile;
  v.tiles_x = (int)((c.width + tile - 1) / tile);
  v.tiles_y = (int)((c.height + tile - 1) / tile);
  v.sh_degree = (int)c.sh_degree;
  return v;
}

// Builds both view layouts for a set of cameras and checks capacities.
gs_status set_views(gs_rasterizer* r, const gs_camera* cams, uint32_t nv, uint32_t n) {
  if (!cams || nv == 0) return fail(r, GS_ERR_INVALID_ARG, "no cameras");
  if (nv > r->max_views) return fail(r, GS_ERR_CAPACITY, "more views than max_views");
  if (n > r->cap) return fail(r, GS_ERR_CAPACITY, "num_surfels exceeds capacity");
  if (n > r->n_uploaded && !r->optim_ready) return fail(r, GS_ERR_STATE, "num_surfels exceeds the uploaded scene");
  r->views_batched.assign(nv, ViewInfo{});
  r->views_single.assign(nv, ViewInfo{});
  long long pix = 0;
  int tiles = 0;
  for (uint32_t v = 0; v < nv; ++v) {
    const gs_camera& c = cams[v];
    if (c.width == 0 || c.height == 0 || !(c.focal > 0.f) || c.sh_degree > 3)
      return fail(r, GS_ERR_INVALID_ARG, "bad camera (size, focal or sh_degree)");
    if (r->cfg.precision != GS_PREC_F32 && (c.width > (uint32_t)REC_MAX_SIDE_H || c.height > (uint32_t)REC_MAX_SIDE_H))
      return fail(r, GS_ERR_INVALID_ARG, "16-bit storage supports images up to 32766 pixels per side");
    ViewInfo vi = make_view(c, r->tile);
    vi.pix_base = pix;
    vi.tile_base = tiles;
    r->views_batched[v] = vi;
    vi.tile_base = 0;
    r->views_single[v] = vi;
    pix += (long long)c.width * c.height;
    tiles += vi.tiles_x * vi.tiles_y;
  }
  if ((uint64_t)pix > r->max_pixels) return fail(r, GS_ERR_CAPACITY, "views exceed max_pixels");
  if ((uint32_t)tiles > r->max_tiles) return fail(r, GS_ERR_CAPACITY, "views exceed the tile budget");
  return GS_OK;
}

gs_status upload_views(gs_rasterizer* r, cudaStream_t st) {
  const uint32_t nv = (uint32_t)r->views_batched.size();
  TRY_CUDA(r, cudaMemcpyAsync(r->views_dev, r->views_batched.data(), sizeof(ViewInfo) * nv, cudaMemcpyHostToDevice, st));
  TRY_CUDA(r, cudaMemcpyAsync(r->views_dev + r->max_views, r->views_single.data(), sizeof(ViewInfo) * nv,
                              cudaMemcpyHostToDevice, st));
  return GS_OK;
}

// Whether (batch, pixels per thread) is a raster shape built for `tile`.
bool shape_listed(bool fwd, int tile, uint32_t batch, uint32_t ppt) {
  const RasterShape* tab = nullptr;
  const int n = fwd ? raster_fwd_shapes(tile, &tab) : raster_bwd_shapes(tile, &tab);
  for (int k = 0; k < n; ++k)
    if ((uint32_t)tab[k].batch == batch && (uint32_t)tab[k].ppt == ppt) return true;
  return false;
}

// Backward shape for the handle's tile size: (128, 2) where it is built,
// else the first shape built.
void default_bwd_shape(gs_rasterizer* r) {
  if (shape_listed(false, r->tile, 128, 2)) { r->bwd_batch = 128; r->bwd_ppt = 2; return; }
  const RasterShape* tab = nullptr;
  raster_bwd_shapes(r->tile, &tab);
  r->bwd_batch = tab[0].batch;
  r->bwd_ppt = tab[0].ppt;
}

const void* sh_for(gs_rasterizer* r, int prec) { return prec == 0 ? (const void*)r->sh : r->sh_half; }

// Projection + binning + forward raster for `nv` views starting at views_dev
// (already uploaded), `tiles` tiles in total, storage precision `prec`.
// cut: bin each tile only up to the depth recorded by the previous step's
// forward (tile_cut), then bin in full every tile whose truncated list ran
// out before all its pixels terminated and continue rendering it. A truncated list
// is a prefix of the full one (entries are ordered by depth), and a tile
// whose pixels all terminate inside it never reads past it, so images,
// contributor indices and gradients are those of the full lists.
gs_status run_forward(gs_rasterizer* r, const ViewInfo* vdev, const ViewInfo* vhost, uint32_t nv, int tiles, uint32_t n,
                      int prec, bool persistent, bool tight, cudaStream_t st, Prof* prof = nullptr,
                      bool color = false, bool cut = false) {
  const uint32_t items = nv * n;
  const bool cut_active = cut && r->cut_on && persistent;
  mark(prof, -1, st);
  if (cut_active) {
    TRY_CUDA(r, cudaMemsetAsync(r->cutw, 0, sizeof(uint32_t) * 4, st));
    TRY_CUDA(r, cudaMemsetAsync(r->inc_flag, 0, (size_t)tiles, st));
  }
  ProjectArgs pa{};
  pa.views = vdev; pa.n = n;
  pa.pos = r->positions; pa.scales = r->scales; pa.quats = r->quats; pa.opac = r->opacities;
  pa.sh = sh_for(r, prec);
  pa.records = r->records; pa.rects = r->rects;
  pa.keys = r->item_keys[0]; pa.vals = r->item_vals[0]; pa.counts = r->counts;
  pa.tight = tight ? 1 : 0;
  pa.cut = cut_active ? r->tile_cut : nullptr;
  pa.item_key = cut_active ? r->item_key : nullptr;
  TRY_LAUNCH(r, launch_project(pa, prec, nv, st));
  mark(prof, 0, st);
  int in1 = 0;
  // The final pass also lays the items' tile counts out in sorted order, so
  // the entry scan and the expansion read them sequentially.
  TRY_LAUNCH(r, launch_radix_sort(r->item_keys[0], r->item_vals[0], r->item_keys[1], r->item_vals[1], items, nullptr,
                                  32, r->sort_scratch, &in1, st, r->counts, r->sorted_counts));
  uint32_t* perm = r->item_vals[in1];
  uint32_t* n_entries = r->words;  // u32 saturated
  TRY_LAUNCH(r, launch_scan(r->sorted_counts, nullptr, r->offsets, items, nullptr, n_entries, r->entry_total,
                            r->scan_scratch, st));
  TRY_LAUNCH(r, launch_entry_guard(r->entry_total, n_entries, r->max_entries, r->words + 1, st));
  mark(prof, 1, st);
  ExpandArgs ea{};
  ea.perm = perm; ea.counts = r->counts; ea.sorted_counts = r->sorted_counts; ea.offsets = r->offsets;
  ea.rects = r->rects;
  ea.views = vdev; ea.items_per_view = n; ea.tiles_x = 0;
  ea.n_items_dev = nullptr; ea.n_items_host = items;
  ea.total = r->entry_total; ea.capacity = r->max_entries;
  ea.pairs = r->ent_pairs[0];
  ea.val_mode = r->det ? 1 : 0;
  ea.exp_item = r->exp_item;
  ea.entry_offset = r->det ? r->entry_offset : nullptr;
  ea.error_word = r->words + 1;
  ExpandFilterArgs fa{};
  fa.perm = perm; fa.counts = r->counts; fa.sorted_counts = r->sorted_counts; fa.offsets = r->offsets;
  fa.rects = r->rects;
  fa.views = vdev; fa.items_per_view = n; fa.n_items_host = items;
  fa.total = r->entry_total; fa.capacity = r->max_entries; fa.pairs = r->ent_pairs[0];
  fa.error_word = r->words + 1;
  if (cut_active) {
    fa.cut = r->tile_cut;
    fa.key_by_item = r->item_key;
    TRY_LAUNCH(r, launch_expand_filtered(fa, st));
  } else {
    TRY_LAUNCH(r, launch_expand(ea, st));
  }
  mark(prof, 2, st);
  const int bits = tile_key_bits((uint32_t)std::max(tiles, 1));
  // The tile sort's final pass also records each tile's range; the fix-up
  // turns it into [start, end).
  TRY_CUDA(r, cudaMemsetAsync(r->ranges, 0, sizeof(uint2) * (size_t)tiles, st));
  TRY_LAUNCH(r, launch_radix_sort_pairs(r->ent_pairs[0], r->ent_pairs[1], r->max_entries, n_entries, bits,
                                        r->sort_scratch, &r->ent_in1, st, r->ranges, (uint32_t)tiles));
  mark(prof, 3, st);
  TRY_LAUNCH(r, launch_ranges_fix(r->ranges, (uint32_t)tiles, st));
  r->order_valid = persistent;
  if (persistent) TRY_LAUNCH(r, launch_tile_order(r->ranges, nullptr, (uint32_t)tiles, r->tile_order, st));
  mark(prof, 4, st);
  RasterArgs ra{};
  ra.views = vdev; ra.n_views = (int)nv; ra.total_tiles = tiles;
  ra.ranges = r->ranges; ra.sorted_pairs = r->ent_pairs[r->ent_in1]; ra.exp_item = r->exp_item;
  ra.records = r->records;
  ra.out_color = r->out_color; ra.out_aux = r->out_aux; ra.out_normal = r->out_normal; ra.out_nc = r->out_nc;
  ra.tile_counter = r->words + 2;
  ra.tile_order = persistent ? r->tile_order : nullptr;
  ra.tile_walk = persistent ? r->tile_walk : nullptr;
  r->mask_valid = r->stored_state && color && persistent && r->tile == 16;
  r->gmask_valid = color && persistent && r->tile == 16 && !r->mask_valid && r->gmask != nullptr;
  if (r->gmask_valid) ra.gmask = r->gmask;
  if (r->mask_valid) {
    TRY_LAUNCH(r, launch_mask_offsets(r->ranges, (uint32_t)tiles, r->mask_words, r->mask_off, r->scan_scratch, st));
    ra.mask = r->mask;
    ra.mask_off = r->mask_off;
  }
  const int batch = r->fwd_batch, ppt = r->fwd_ppt;
  int grid = tiles;
  if (persistent) {
    TRY_CUDA(r, cudaMemsetAsync(r->words + 2, 0, sizeof(uint32_t), st));
    grid = std::min(tiles, r->num_sms * raster_fwd_occupancy(r->tile, prec, batch, ppt, r->det, color,
                                                              ra.mask != nullptr));
  }
  if (cut_active) {
    ra.tile_cut = r->tile_cut; ra.cut_pass = 1; ra.item_key = r->item_key;
    ra.inc_count = r->cutw; ra.inc_list = r->inc_list; ra.inc_flag = r->inc_flag;
    ra.inc_skip = r->inc_skip; ra.inc_src = r->inc_src;
  }
  TRY_LAUNCH(r, launch_raster_fwd(ra, r->tile, prec, batch, ppt, r->det, persistent, color && persistent, grid, st));
  mark(prof, 5, st);
  if (cut_active) {
    // Completion pass (every kernel finds zero work when no tile is listed):
    // the listed tiles' full lists are binned after the entries in use,
    // sorted there and their ranges replaced; each tile's rendering then
    // continues after the prefix pass 1 composited.
    TRY_LAUNCH(r, launch_cut_gate(r->cutw, items, r->cutw + 1, st));
    TRY_LAUNCH(r, launch_count_flagged(r->rects, vdev, nv, n, items, r->cutw, r->inc_list, r->inc_flag, r->counts2,
                                       st));
    TRY_LAUNCH(r, launch_scan(r->counts2, perm, r->offsets, items, r->cutw + 1, r->cutw + 2, r->entry_total2,
                              r->scan_scratch, st));
    TRY_LAUNCH(r, launch_entry_guard2(r->entry_total, r->entry_total2, r->cutw + 2, r->max_entries, r->words + 1, st));
    TRY_LAUNCH(r, launch_ranges_reset_list(r->inc_list, r->cutw, r->ranges, (uint32_t)tiles, st));
    mark(prof, 1, st);
    ExpandFilterArgs fb = fa;
    fb.counts = r->counts2; fb.sorted_counts = nullptr; fb.n_items_dev = r->cutw + 1;
    fb.total = r->entry_total2; fb.base = r->entry_total;
    fb.cut = nullptr; fb.key_by_item = nullptr; fb.flag = r->inc_flag;
    TRY_LAUNCH(r, launch_expand_filtered(fb, st));
    mark(prof, 2, st);
    int in1b = 0;
    TRY_LAUNCH(r, launch_radix_sort_pairs(r->ent_pairs[0], r->ent_pairs[1], r->max_entries, r->cutw + 2, bits,
                                          r->sort_scratch, &in1b, st, r->ranges, (uint32_t)tiles, r->entry_total));
    if (in1b != r->ent_in1) return fail(r, GS_ERR_STATE, "completion sort ended in the other buffer");
    mark(prof, 3, st);
    TRY_LAUNCH(r, launch_ranges_fix_list(r->inc_list, r->cutw, r->ranges, (uint32_t)tiles, r->entry_total,
                                         r->entry_total2, r->gmask_valid ? r->gmask : nullptr, r->inc_skip,
                                         r->inc_src, st));
    mark(prof, 4, st);
    RasterArgs rb = ra;
    rb.cut_pass = 2;
    rb.tile_order = r->inc_list;
    rb.tile_limit = r->cutw;
    rb.tile_counter = r->cutw + 3;
    TRY_LAUNCH(r, launch_raster_fwd(rb, r->tile, prec, batch, ppt, r->det, persistent, color && persistent, grid, st));
    mark(prof, 5, st);
  }
  r->last_nv = nv; r->last_n = n; r->last_tiles = tiles; r->last_views_dev = vdev; r->last_views_host = vhost;
  r->last_prec = prec;
  r->have_forward = true;
  return GS_OK;
}

RasterArgs bwd_args(gs_rasterizer* r, const ViewInfo* vdev, uint32_t nv, int tiles) {
  RasterArgs ra{};
  ra.views = vdev; ra.n_views = (int)nv; ra.total_tiles = tiles;
  ra.ranges = r->ranges; ra.sorted_pairs = r->ent_pairs[r->ent_in1]; ra.exp_item = r->exp_item;
  ra.records = r->records;
  ra.out_color = r->out_color; ra.out_aux = r->out_aux; ra.out_normal = r->out_normal; ra.out_nc = r->out_nc;
  ra.dl_dcolor = r->dl_dcolor; ra.dl_dnormal = r->dl_dnormal;
  ra.grad_geom = r->grad_geom; ra.partials = r->partials;
  ra.lambda_dist = r->lambda_dist;
  ra.tile_counter = r->words + 3;
  ra.tile_order = nullptr;
  return ra;
}

// prepared: grad_geom already cleared and the tile order already computed
// (the chosen step does both on its side stream).
gs_status run_backward_raster(gs_rasterizer* r, const ViewInfo* vdev, uint32_t nv, int tiles, uint32_t n, int prec,
                              bool aux, bool persistent, cudaStream_t st, bool prepared = false) {
  if (!r->det && !prepared)
    TRY_CUDA(r, cudaMemsetAsync(r->grad_geom, 0, sizeof(float) * GG_STRIDE * (size_t)nv * n, st));
  RasterArgs ra = bwd_args(r, vdev, nv, tiles);
  if (r->gmask_valid && !aux && r->tile == 16) ra.gmask = r->gmask;  // summary of the matching forward
  if (r->mask_valid && !aux) {  // masks of the matching colour-only forward
    ra.mask = r->mask;
    ra.mask_off = r->mask_off;
  }
  int grid = tiles;
  if (persistent) {
    TRY_CUDA(r, cudaMemsetAsync(r->words + 3, 0, sizeof(uint32_t), st));
    grid = std::min(tiles, r->num_sms * raster_bwd_occupancy(r->tile, prec, aux, r->bwd_ppt, r->bwd_batch, r->det,
                                                              ra.mask != nullptr));
    if (r->order_valid) {  // heaviest first by how far each tile's walk goes
      if (!prepared) TRY_LAUNCH(r, launch_tile_order(r->ranges, r->tile_walk, (uint32_t)tiles, r->tile_order, st));
      ra.tile_order = r->tile_order;
    }
  }
  TRY_LAUNCH(r, launch_raster_bwd(ra, r->tile, prec, aux, r->bwd_ppt, r->bwd_batch, r->det, persistent, grid, st));
  return GS_OK;
}

ProjectBwdArgs pbwd_args(gs_rasterizer* r, const ViewInfo* vdev, uint32_t nv, uint32_t n, int prec) {
  ProjectBwdArgs b{};
  b.views = vdev; b.n = n; b.n_views = (int)nv; b.view = 0;
  b.pos = r->positions; b.scales = r->scales; b.quats = r->quats; b.sh = sh_for(r, prec);
  b.grad_geom = r->grad_geom;
  b.partials = r->det ? r->partials : nullptr;
  b.entry_offset = r->entry_offset;
  b.entry_total = r->entry_total;
  b.counts = r->counts;
  b.grad_pos = r->grad_pos; b.grad_scales = r->grad_scales; b.grad_quat = r->grad_quat;
  b.grad_opacity = r->grad_opacity; b.grad_sh = r->grad_sh; b.grad_cam = r->grad_cam;
  b.cam_partials = r->det ? r->cam_part : nullptr;
  return b;
}

gs_status clear_param_grads(gs_rasterizer* r, uint32_t n, uint32_t nv, cudaStream_t st) {
  TRY_CUDA(r, cudaMemsetAsync(r->grad_pos, 0, sizeof(float4) * (size_t)n, st));
  TRY_CUDA(r, cudaMemsetAsync(r->grad_scales, 0, sizeof(float2) * (size_t)n, st));
  TRY_CUDA(r, cudaMemsetAsync(r->grad_quat, 0, sizeof(float4) * (size_t)n, st));
  TRY_CUDA(r, cudaMemsetAsync(r->grad_opacity, 0, sizeof(float) * (size_t)n, st));
  TRY_CUDA(r, cudaMemsetAsync(r->grad_sh, 0, sizeof(float) * SH_FLOATS * (size_t)n, st));
  TRY_CUDA(r, cudaMemsetAsync(r->grad_cam, 0, sizeof(float) * 16 * (size_t)nv, st));
  return GS_OK;
}

// Projection backward for each view of the last forward, adding into the
// parameter gradients (plain form).
gs_status run_project_bwd(gs_rasterizer* r, const ViewInfo* vdev, uint32_t nv, uint32_t n, int prec, bool aux,
                          float* grad_cam_base, cudaStream_t st) {
  for (uint32_t v = 0; v < nv; ++v) {
    ProjectBwdArgs b = pbwd_args(r, vdev, nv, n, prec);
    b.view = (int)v;
    b.grad_cam = grad_cam_base;
    TRY_LAUNCH(r, launch_project_bwd(b, prec, aux, st));
    if (b.cam_partials)  // deterministic mode: this view's camera gradient, summed in warp order
      TRY_LAUNCH(r, launch_cam_reduce(b.cam_partials, cam_partial_units(n, 0), 1, grad_cam_base + 16 * v, st));
  }
  return GS_OK;
}

gs_status run_loss(gs_rasterizer* r, const ViewInfo* vdev, const ViewInfo* vhost, uint32_t nv, float w_l1,
                   float w_ssim, double* sums, cudaStream_t st) {
  SsimArgs a{};
  a.views = vdev; a.n_views = (int)nv;
  int t16 = 0;
  for (uint32_t v = 0; v < nv; ++v) t16 += ((vhost[v].width + 15) / 16) * ((vhost[v].height + 15) / 16);
  a.total_tiles16 = t16;
  a.img = r->out_color; a.target = r->target; a.coef = r->coef; a.coef_stride = r->max_pixels;
  a.dl_dcolor = r->dl_dcolor;
  a.loss_sums = sums;
  a.w_l1 = w_l1; a.w_ssim = w_ssim;
  TRY_LAUNCH(r, launch_ssim(a, st));
  return GS_OK;
}

const int ACT[5] = {0, 1, 0, 2, 0};
const int WIDTH[5] = {4, 2, 4, 1, SH_FLOATS};

float* act_ptr(gs_rasterizer* r, int c) {
  switch (c) {
    case 0: return reinterpret_cast<float*>(r->positions);
    case 1: return reinterpret_cast<float*>(r->scales);
    case 2: return reinterpret_cast<float*>(r->quats);
    case 3: return r->opacities;
    default: return r->sh;
  }
}
float* grad_ptr(gs_rasterizer* r, int c) {
  switch (c) {
    case 0: return reinterpret_cast<float*>(r->grad_pos);
    case 1: return reinterpret_cast<float*>(r->grad_scales);
    case 2: return reinterpret_cast<float*>(r->grad_quat);
    case 3: return r->grad_opacity;
    default: return r->grad_sh;
  }
}

gs_status refresh_half(gs_rasterizer* r, uint32_t n, cudaStream_t st) {
  if (r->cfg.precision == GS_PREC_F32 || !r->sh_half) return GS_OK;
  TRY_LAUNCH(r, launch_to_half(r->sh, r->sh_half, (uint64_t)n * SH_FLOATS, r->cfg.precision == GS_PREC_BF16, st));
  return GS_OK;
}

// Bias corrections in f32 as the reference computes them (optim.rs:188-189).
void bias_corrections(float b1, float b2, uint32_t t, float& bc1, float& bc2) {
  float p1 = 1.f, p2 = 1.f;
  for (uint32_t k = 0; k < t; ++k) { p1 *= b1; p2 *= b2; }
  bc1 = 1.0f / (1.0f - p1);
  bc2 = 1.0f / (1.0f - p2);
}

gs_status adam_plain(gs_rasterizer* r, const gs_adam_config* c, uint32_t n, cudaStream_t st) {
  // Densify statistic: running sum of |dL/dpos| per surfel (the fused chosen
  // form adds it inside its kernel).
  TRY_LAUNCH(r, launch_accum_norm(r->grad_pos, r->accum_norm, n, st));
  r->accum_steps += 1;
  r->t += 1;
  float bc1, bc2;
  bias_corrections(c->beta1, c->beta2, r->t, bc1, bc2);
  for (int k = 0; k < 5; ++k) {
    AdamClass ac{r->raw[k], r->mom1[k], r->mom2[k], act_ptr(r, k), c->lr[k], c->reg[k]};
    TRY_LAUNCH(r, launch_adam_grad(ac, grad_ptr(r, k), (uint64_t)n * WIDTH[k], ACT[k], c->beta1, c->beta2, c->eps,
                                   bc1, bc2, st));
  }
  return refresh_half(r, n, st);
}

// The cuts hold for the step shape and views they were recorded with; any
// other step starts from full lists (results are exact either way; this only
// keeps stale cuts from sending most tiles through the completion pass).
gs_status cut_refresh(gs_rasterizer* r, uint32_t nv, uint32_t n, cudaStream_t st) {
  if (!r->cut_on) return GS_OK;
  std::vector<uint32_t> sig = {nv, n, (uint32_t)r->tile};
  for (const ViewInfo& v : r->views_batched) {
    const size_t w = sizeof(ViewInfo) / sizeof(uint32_t);
    const size_t at = sig.size();
    sig.resize(at + w);
    std::memcpy(sig.data() + at, &v, w * sizeof(uint32_t));
  }
  if (sig != r->cut_sig) {
    TRY_CUDA(r, cudaMemsetAsync(r->tile_cut, 0xff, sizeof(uint32_t) * (size_t)r->max_tiles, st));
    r->cut_sig = sig;
  }
  return GS_OK;
}

gs_status ensure_graph_stream(gs_rasterizer* r) {
  if (!r->cap_stream) TRY_CUDA(r, cudaStreamCreateWithFlags(&r->cap_stream, cudaStreamNonBlocking));
  return GS_OK;
}

gs_status ensure_side_stream(gs_rasterizer* r) {
  if (!r->side_stream) TRY_CUDA(r, cudaStreamCreateWithFlags(&r->side_stream, cudaStreamNonBlocking));
  for (cudaEvent_t* e : {&r->ev_fork, &r->ev_fwd, &r->ev_side})
    if (!*e) TRY_CUDA(r, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  return GS_OK;
}

// The chosen-form step body: batched forward, loss, backward raster, fused
// projection backward + Adam. Recorded into a graph by train_step.
gs_status chosen_body(gs_rasterizer* r, uint32_t nv, uint32_t n, const gs_step_config* cfg, cudaStream_t st,
                      Prof* prof = nullptr) {
  const int prec = (int)r->cfg.precision;
  const ViewInfo* vdev = r->views_dev;
  int tiles = 0;
  for (const ViewInfo& v : r->views_batched) tiles += v.tiles_x * v.tiles_y;
  // Side stream (forked from and joined into st, so it is part of a captured
  // graph): grad_geom is cleared during the forward; the backward's tile
  // order is computed during the loss.
  cudaStream_t side = r->side_stream;
  TRY_CUDA(r, cudaEventRecord(r->ev_fork, st));
  TRY_CUDA(r, cudaStreamWaitEvent(side, r->ev_fork, 0));
  if (!r->det) TRY_CUDA(r, cudaMemsetAsync(r->grad_geom, 0, sizeof(float) * GG_STRIDE * (size_t)nv * n, side));
  // With GS_FLAG_COLOR_ONLY the step's forward leaves depth and normal unwritten (nothing reads them).
  gs_status s = run_forward(r, vdev, r->views_batched.data(), nv, tiles, n, prec, true, true, st, prof, r->color_only,
                            true);
  if (s) return s;
  TRY_CUDA(r, cudaEventRecord(r->ev_fwd, st));
  TRY_CUDA(r, cudaStreamWaitEvent(side, r->ev_fwd, 0));
  if (r->order_valid)
    TRY_LAUNCH(r, launch_tile_order(r->ranges, r->tile_walk, (uint32_t)tiles, r->tile_order, side));
  TRY_CUDA(r, cudaEventRecord(r->ev_side, side));
  TRY_CUDA(r, cudaMemsetAsync(r->loss_sums, 0, sizeof(double) * 2 * nv, st));
  if (cfg->loss == GS_LOSS_L1_SSIM) {
    s = run_loss(r, vdev, r->views_batched.data(), nv, cfg->w_l1, cfg->w_ssim, r->loss_sums, st);
    if (s) return s;
  }
  mark(prof, 6, st);
  TRY_CUDA(r, cudaStreamWaitEvent(st, r->ev_side, 0));
  s = run_backward_raster(r, vdev, nv, tiles, n, prec, false, true, st, true);
  if (s) return s;
  mark(prof, 7, st);
  TRY_CUDA(r, cudaMemsetAsync(r->grad_cam, 0, sizeof(float) * 16 * nv, st));
  ProjectBwdArgs b = pbwd_args(r, vdev, nv, n, prec);
  AdamFusedArgs o{};
  for (int k = 0; k < 5; ++k) o.cls[k] = AdamClass{r->raw[k], r->mom1[k], r->mom2[k], act_ptr(r, k), 0.f, 0.f};
  o.beta1 = cfg->adam.beta1; o.beta2 = cfg->adam.beta2; o.eps = cfg->adam.eps;
  o.dyn = r->dyn_dev;
  o.sh_half = prec == 0 ? nullptr : r->sh_half;
  o.sh_half_is_bf16 = prec == 2;
  o.accum_grad_norm = r->accum_norm;
  o.error_word = r->words + 1;
  o.wait_cycles[0] = r->wait_cycles[0];
  o.wait_cycles[1] = r->wait_cycles[1];
  TRY_LAUNCH(r, launch_project_bwd_adam(b, o, prec, false, st));
  if (b.cam_partials)  // deterministic mode: camera gradients summed in block order
    TRY_LAUNCH(r, launch_cam_reduce(b.cam_partials, cam_partial_units(n, (int)nv), (int)nv, r->grad_cam, st));
  mark(prof, 8, st);
  return GS_OK;
}

// Plain-form step body (views one at a time, FP32, separate Adam).
gs_status plain_body(gs_rasterizer* r, uint32_t nv, uint32_t n, const gs_step_config* cfg, cudaStream_t st,
                     Prof* prof = nullptr) {
  gs_status s = clear_param_grads(r, n, nv, st);
  if (s) return s;
  TRY_CUDA(r, cudaMemsetAsync(r->loss_sums, 0, sizeof(double) * 2 * nv, st));
  for (uint32_t v = 0; v < nv; ++v) {
    const ViewInfo* vd = r->views_dev + r->max_views + v;
    const ViewInfo& vi = r->views_single[v];
    const int tiles = vi.tiles_x * vi.tiles_y;
    s = run_forward(r, vd, &r->views_single[v], 1, tiles, n, 0, false, false, st, prof);
    if (s) return s;
    if (cfg->loss == GS_LOSS_L1_SSIM) {
      s = run_loss(r, vd, &r->views_single[v], 1, cfg->w_l1, cfg->w_ssim, r->loss_sums + 2 * v, st);
      if (s) return s;
    }
    mark(prof, 6, st);
    s = run_backward_raster(r, vd, 1, tiles, n, 0, false, false, st);
    if (s) return s;
    mark(prof, 7, st);
    s = run_project_bwd(r, vd, 1, n, 0, false, r->grad_cam + 16 * v, st);
    if (s) return s;
    mark(prof, 8, st);
  }
  s = adam_plain(r, &cfg->adam, n, st);
  mark(prof, 8, st);
  return s;
}

}  // namespace

// ============================================================== C ABI
extern "C" {

const char* gs_version(void) { return "gs_cuda 0.1 sm_100a"; }

gs_status gs_last_error(gs_rasterizer* r, char* msg, size_t cap) {
  if (!msg || cap == 0) return GS_ERR_INVALID_ARG;
  const std::string& e = r ? r->err : g_last_error;
  snprintf(msg, cap, "%s", e.c_str());
  return GS_OK;
}

gs_status gs_camera_rotation(const gs_camera* cam, float rot9[9]) {
  if (!cam || !rot9) return GS_ERR_INVALID_ARG;
  rotation_of(cam->quat, rot9);
  return GS_OK;
}

gs_status gs_rasterizer_create(const gs_raster_config* cfg_in, gs_rasterizer** out) {
  if (!cfg_in || !out) return fail(nullptr, GS_ERR_INVALID_ARG, "null config or output");
  *out = nullptr;
  gs_raster_config c = *cfg_in;
  if (c.capacity == 0) return fail(nullptr, GS_ERR_INVALID_ARG, "capacity must be > 0");
  if (c.tile == 0) c.tile = 16;
  if (c.tile != 8 && c.tile != 16 && c.tile != 32) return fail(nullptr, GS_ERR_INVALID_ARG, "tile must be 8, 16 or 32");
  if (c.tile != 16 && (c.flags & GS_FLAG_STORED_STATE))
    return fail(nullptr, GS_ERR_INVALID_ARG, "the stored-state backward is built for 16-pixel tiles");
  if (c.max_views == 0) c.max_views = 1;
  if (c.max_views > MAX_VIEWS_HARD) return fail(nullptr, GS_ERR_INVALID_ARG, "max_views > 64");
  if (c.batch == 0) c.batch = 128;
  if (c.batch != 64 && c.batch != 128 && c.batch != 256) return fail(nullptr, GS_ERR_INVALID_ARG, "batch must be 64/128/256");
  if (c.pixels_per_thread == 0) c.pixels_per_thread = c.tile == 32 ? 4 : 1;
  if (!shape_listed(true, (int)c.tile, c.batch, c.pixels_per_thread))
    return fail(nullptr, GS_ERR_INVALID_ARG,
                "(batch, pixels_per_thread) not built for this tile: tile 8 -> ppt 1/2 with batch 64/128/256; tile 16 -> "
                "ppt 1 with batch 64/128/256, 2 with 64/128, 4 with 64; tile 32 -> ppt 2/4 with batch 64/128/256");
  if (c.precision > 2) return fail(nullptr, GS_ERR_INVALID_ARG, "bad precision");
  if (c.max_pixels == 0) c.max_pixels = (uint64_t)c.width * c.height * c.max_views;
  if (c.max_pixels == 0) return fail(nullptr, GS_ERR_INVALID_ARG, "width/height or max_pixels required");
  if (c.max_entries == 0) c.max_entries = 64ull * c.capacity * c.max_views;
  if (c.max_entries >= 0xffffffffull) return fail(nullptr, GS_ERR_INVALID_ARG, "max_entries must be < 2^32");
  if ((uint64_t)c.capacity * c.max_views >= 0xffffffffull) return fail(nullptr, GS_ERR_INVALID_ARG, "items must be < 2^32");

  gs_rasterizer* r = new (std::nothrow) gs_rasterizer();
  if (!r) return fail(nullptr, GS_ERR_CUDA, "host allocation failed");
  r->cfg = c;
  r->cap = c.capacity;
  r->max_views = c.max_views;
  r->max_pixels = c.max_pixels;
  r->max_entries = c.max_entries;
  r->max_items = (uint64_t)c.capacity * c.max_views;
  // Tile budget: every pixel in its own tile row/column worst case is
  // bounded by the pixel budget; views of at least 1 px add at most one
  // partial tile row and column each.
  r->max_tiles = (uint32_t)std::min<uint64_t>(0xffffffffull, c.max_pixels / 64 + 4096ull * c.max_views + 1024);
  r->det = (c.flags & GS_FLAG_DETERMINISTIC) != 0;
  r->persistent = (c.flags & GS_FLAG_PERSISTENT) != 0;
  r->color_only = (c.flags & GS_FLAG_COLOR_ONLY) != 0;
  r->tight = (c.flags & GS_FLAG_TIGHT_BINNING) != 0;
  r->stored_state = (c.flags & GS_FLAG_STORED_STATE) != 0;
  r->cut_on = (c.flags & GS_FLAG_FULL_LISTS) == 0 && !r->det && !r->stored_state;
  r->fwd_batch = (int)c.batch;
  r->fwd_ppt = (int)c.pixels_per_thread;
  r->tile = (int)c.tile;
  default_bwd_shape(r);
  auto bail = [&](cudaError_t e, const char* what) {
    std::string m = std::string("allocation of ") + what + " failed: " + cudaGetErrorString(e);
    gs_rasterizer_destroy(r);
    return fail(nullptr, GS_ERR_CUDA, m);
  };
#define ALLOC(ptr, n)                            \
  do {                                           \
    cudaError_t _e = dalloc(ptr, (n));           \
    if (_e != cudaSuccess) return bail(_e, #ptr); \
  } while (0)
  cudaGetDevice(&r->device);
  cudaDeviceGetAttribute(&r->num_sms, cudaDevAttrMultiProcessorCount, r->device);
  {
    const int pe = prepare_project_kernels();
    if (pe) return bail((cudaError_t)pe, "kernel shared-memory opt-in");
  }
  const size_t N = c.capacity, I = r->max_items, E = r->max_entries, P = r->max_pixels;
  ALLOC(r->positions, N); ALLOC(r->scales, N); ALLOC(r->quats, N); ALLOC(r->opacities, N);
  ALLOC(r->sh, N * SH_FLOATS);
  if (c.precision != GS_PREC_F32) {
    unsigned short* h = nullptr;
    ALLOC(h, N * SH_FLOATS);
    r->sh_half = h;
  }
  {
    float4* rec = nullptr;
    ALLOC(rec, I * REC_F4_F32);
    r->records = rec;
  }
  ALLOC(r->rects, I);
  for (int k = 0; k < 2; ++k) { ALLOC(r->item_keys[k], I); ALLOC(r->item_vals[k], I); }
  ALLOC(r->counts, I); ALLOC(r->offsets, I); ALLOC(r->sorted_counts, I);
  for (int k = 0; k < 2; ++k) ALLOC(r->ent_pairs[k], E);
  if (r->det) {
    ALLOC(r->exp_item, E);
    ALLOC(r->partials, E * GG_STRIDE);
    ALLOC(r->entry_offset, I);
    uint64_t units = cam_partial_units(c.capacity, 0);
    for (uint32_t v = 1; v <= c.max_views; ++v) units = std::max<uint64_t>(units, cam_partial_units(c.capacity, (int)v) * v);
    ALLOC(r->cam_part, units * 16);
  }
  ALLOC(r->ranges, r->max_tiles);
  ALLOC(r->tile_order, r->max_tiles);
  ALLOC(r->tile_walk, r->max_tiles);
  if (r->cut_on) {
    ALLOC(r->tile_cut, r->max_tiles);
    ALLOC(r->inc_list, r->max_tiles);
    ALLOC(r->inc_skip, r->max_tiles);
    ALLOC(r->inc_src, r->max_tiles);
    ALLOC(r->inc_flag, r->max_tiles);
    ALLOC(r->item_key, I);
    ALLOC(r->counts2, I);
    ALLOC(r->cutw, 4);
    ALLOC(r->entry_total2, 1);
  }
  if (r->stored_state) {
    // One bit per (pixel, tile entry): 32 bytes per entry, whole 32-entry words per tile.
    ALLOC(r->mask, ((size_t)E / 32 + r->max_tiles) * 256);
    ALLOC(r->mask_off, r->max_tiles);
    ALLOC(r->mask_words, r->max_tiles);
  }
  if (r->color_only && !r->stored_state) {
    // One byte per tile entry: the 4-row groups of a 16-pixel tile it composited into.
    ALLOC(r->gmask, E);
  }
  ALLOC(r->entry_total, 1);
  ALLOC(r->words, 8);
  ALLOC(r->work_counts, 4);
  ALLOC(r->out_color, P); ALLOC(r->out_aux, P); ALLOC(r->out_normal, P); ALLOC(r->dl_dcolor, P);
  ALLOC(r->dl_dnormal, P); ALLOC(r->target, P); ALLOC(r->out_nc, P);
  ALLOC(r->coef, P * 9);
  ALLOC(r->loss_sums, 2 * (size_t)c.max_views);
  ALLOC(r->normal_loss_sums, (size_t)c.max_views);
  ALLOC(r->grad_geom, I * GG_STRIDE);
  ALLOC(r->grad_pos, N); ALLOC(r->grad_scales, N); ALLOC(r->grad_quat, N); ALLOC(r->grad_opacity, N);
  ALLOC(r->grad_sh, N * SH_FLOATS);
  ALLOC(r->grad_cam, 16 * (size_t)c.max_views);
  for (int k = 0; k < 5; ++k) {
    // whole multiples of 64 surfels: the fused Adam kernel copies full 32-surfel rows
    const size_t NP = (N + 63) / 64 * 64;
    ALLOC(r->raw[k], NP * WIDTH[k]); ALLOC(r->mom1[k], NP * WIDTH[k]); ALLOC(r->mom2[k], NP * WIDTH[k]);
  }
  ALLOC(r->accum_norm, N);
  ALLOC(r->dyn_dev, sizeof(DynParams) / sizeof(float));
  ALLOC(r->views_dev, 2 * (size_t)c.max_views);
  {
    unsigned char* s1 = nullptr;
    ALLOC(s1, scan_scratch_bytes());
    r->scan_scratch = s1;
    unsigned char* s2 = nullptr;
    ALLOC(s2, sort_scratch_bytes());
    r->sort_scratch = s2;
  }
#undef ALLOC
  cudaError_t e = cudaMemset(r->words, 0, 8 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(r->entry_total, 0, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(r->grad_cam, 0, 16 * sizeof(float) * c.max_views);
  if (e == cudaSuccess) e = cudaMemset(r->accum_norm, 0, sizeof(float) * N);
  if (e == cudaSuccess && r->cut_on) e = cudaMemset(r->tile_cut, 0xff, sizeof(uint32_t) * (size_t)r->max_tiles);
  if (e == cudaSuccess && r->cut_on) e = cudaMemset(r->cutw, 0, sizeof(uint32_t) * 4);
  if (e != cudaSuccess) return bail(e, "initial memset");
  *out = r;
  return GS_OK;
}

gs_status gs_rasterizer_destroy(gs_rasterizer* r) {
  if (!r) return GS_OK;
  if (r->graph) cudaGraphExecDestroy(r->graph);
  if (r->cap_stream) cudaStreamDestroy(r->cap_stream);
  if (r->side_stream) cudaStreamDestroy(r->side_stream);
  for (cudaEvent_t e : {r->ev_fork, r->ev_fwd, r->ev_side})
    if (e) cudaEventDestroy(e);
  void* ptrs[] = {r->positions, r->scales, r->quats, r->opacities, r->sh, r->sh_half, r->records, r->rects,
                  r->item_keys[0], r->item_keys[1], r->item_vals[0], r->item_vals[1], r->counts, r->offsets,
                  r->entry_offset, r->ent_pairs[0], r->ent_pairs[1], r->exp_item,
                  r->partials, r->ranges, r->entry_total, r->words, r->out_color, r->out_aux, r->out_normal,
                  r->dl_dcolor, r->dl_dnormal, r->target, r->out_nc, r->coef, r->loss_sums, r->grad_geom,
                  r->grad_pos, r->grad_scales, r->grad_quat, r->grad_opacity, r->grad_sh, r->grad_cam, r->cam_part,
                  r->accum_norm, r->dyn_dev, r->dens_flags, r->dens_slots, r->dens_tmp, r->views_dev,
                  r->mcmc_u32, r->mcmc_u64, r->mcmc_jump, r->mcmc_rng, r->mcmc_counters, r->mask, r->mask_off, r->gmask, r->tile_order, r->tile_walk,
                  r->normal_loss_sums,
                  r->mask_words,
                  r->tile_cut, r->inc_list, r->inc_skip, r->inc_src, r->inc_flag, r->item_key, r->counts2, r->sorted_counts, r->cutw, r->entry_total2,
                  r->scan_scratch, r->sort_scratch, r->work_counts};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int k = 0; k < 5; ++k) {
    if (r->raw[k]) cudaFree(r->raw[k]);
    if (r->mom1[k]) cudaFree(r->mom1[k]);
    if (r->mom2[k]) cudaFree(r->mom2[k]);
  }
  delete r;
  return GS_OK;
}

gs_status gs_rasterizer_upload_scene(gs_rasterizer* r, const gs_scene_input* s, void* stream) {
  if (!r || !s) return GS_ERR_INVALID_ARG;
  if (s->n > r->cap) return fail(r, GS_ERR_CAPACITY, "scene larger than capacity");
  if (s->sh_coeffs == 0 || s->sh_coeffs > 16) return fail(r, GS_ERR_INVALID_ARG, "sh_coeffs must be 1..16");
  if (s->n && (!s->positions || !s->scales || !s->quats || !s->opacities || !s->sh))
    return fail(r, GS_ERR_INVALID_ARG, "null scene array");
  const size_t n = s->n;
  std::vector<float> pos(n * 4), sh(n * SH_FLOATS, 0.f);
  for (size_t i = 0; i < n; ++i) {
    pos[4 * i] = s->positions[3 * i]; pos[4 * i + 1] = s->positions[3 * i + 1];
    pos[4 * i + 2] = s->positions[3 * i + 2]; pos[4 * i + 3] = 1.0f;
    std::memcpy(&sh[i * SH_FLOATS], s->sh + i * s->sh_coeffs * 3, sizeof(float) * s->sh_coeffs * 3);
  }
  cudaStream_t st = S(stream);
  TRY_CUDA(r, cudaMemcpyAsync(r->positions, pos.data(), sizeof(float) * 4 * n, cudaMemcpyHostToDevice, st));
  TRY_CUDA(r, cudaMemcpyAsync(r->scales, s->scales, sizeof(float) * 2 * n, cudaMemcpyHostToDevice, st));
  TRY_CUDA(r, cudaMemcpyAsync(r->quats, s->quats, sizeof(float) * 4 * n, cudaMemcpyHostToDevice, st));
  TRY_CUDA(r, cudaMemcpyAsync(r->opacities, s->opacities, sizeof(float) * n, cudaMemcpyHostToDevice, st));
  TRY_CUDA(r, cudaMemcpyAsync(r->sh, sh.data(), sizeof(float) * SH_FLOATS * n, cudaMemcpyHostToDevice, st));
  gs_status x = refresh_half(r, (uint32_t)n, st);
  if (x) return x;
  TRY_CUDA(r, cudaStreamSynchronize(st));
  r->n_uploaded = s->n;
  r->optim_ready = false;
  r->cut_sig.clear();
  return GS_OK;
}

gs_status gs_rasterizer_set_lambda_dist(gs_rasterizer* r, float lambda_dist) {
  if (!r) return GS_ERR_INVALID_ARG;
  r->lambda_dist = lambda_dist;
  return GS_OK;
}

gs_status gs_rasterizer_set_wait_limits(gs_rasterizer* r, uint64_t copy_wait_cycles, uint64_t drain_wait_cycles) {
  if (!r) return GS_ERR_INVALID_ARG;
  // The drain wait keeps an expired block from exiting while its copies are
  // in flight; it must stay long enough for them to land.
  if (drain_wait_cycles < 100000000ull || drain_wait_cycles > (1ull << 62) || copy_wait_cycles > (1ull << 62))
    return fail(r, GS_ERR_INVALID_ARG, "drain wait below 1e8 cycles, or a limit beyond 2^62");
  r->wait_cycles[0] = (long long)copy_wait_cycles;
  r->wait_cycles[1] = (long long)drain_wait_cycles;
  return GS_OK;
}

gs_status gs_rasterizer_forward(gs_rasterizer* r, const gs_camera* cams, uint32_t nv, uint32_t n, void* stream) {
  if (!r) return GS_ERR_INVALID_ARG;
  gs_status s = set_views(r, cams, nv, n);
  if (s) return s;
  cudaStream_t st = S(stream);
  s = upload_views(r, st);
  if (s) return s;
  int tiles = 0;
  for (const ViewInfo& v : r->views_batched) tiles += v.tiles_x * v.tiles_y;
  r->last_batched = true;
  return run_forward(r, r->views_dev, r->views_batched.data(), nv, tiles, n, (int)r->cfg.precision, r->persistent,
                     r->tight, st);
}

gs_status gs_rasterizer_backward(gs_rasterizer* r, uint32_t n, void* stream) {
  if (!r) return GS_ERR_INVALID_ARG;
  if (!r->have_forward || n != r->last_n) return fail(r, GS_ERR_STATE, "backward needs a matching forward");
  cudaStream_t st = S(stream);
  const int prec = (int)r->cfg.precision;
  const bool aux = !r->color_only;
  gs_status s = clear_param_grads(r, n, r->last_nv, st);
  if (s) return s;
  s = run_backward_raster(r, r->last_views_dev, r->last_nv, r->last_tiles, n, prec, aux, r->persistent, st);
  if (s) return s;
  return run_project_bwd(r, r->last_views_dev, r->last_nv, n, prec, aux, r->grad_cam, st);
}

static gs_status buffer_info(gs_rasterizer* r, gs_buffer_id id, void** p, size_t* bytes) {
  const size_t N = r->cap, P = r->max_pixels, I = r->max_items, E = r->max_entries;
  switch (id) {
    case GS_BUF_POSITIONS: *p = r->positions; *bytes = 16 * N; break;
    case GS_BUF_SCALES: *p = r->scales; *bytes = 8 * N; break;
    case GS_BUF_QUATS: *p = r->quats; *bytes = 16 * N; break;
    case GS_BUF_OPACITIES: *p = r->opacities; *bytes = 4 * N; break;
    case GS_BUF_SH: *p = r->sh; *bytes = 4 * SH_FLOATS * N; break;
    case GS_BUF_OUT_COLOR: *p = r->out_color; *bytes = 16 * P; break;
    case GS_BUF_OUT_AUX: *p = r->out_aux; *bytes = 16 * P; break;
    case GS_BUF_OUT_NORMAL: *p = r->out_normal; *bytes = 16 * P; break;
    case GS_BUF_OUT_NCONTRIB: *p = r->out_nc; *bytes = 4 * P; break;
    case GS_BUF_DL_DCOLOR: *p = r->dl_dcolor; *bytes = 16 * P; break;
    case GS_BUF_DL_DNORMAL: *p = r->dl_dnormal; *bytes = 16 * P; break;
    case GS_BUF_GRAD_POS: *p = r->grad_pos; *bytes = 16 * N; break;
    case GS_BUF_GRAD_SCALES: *p = r->grad_scales; *bytes = 8 * N; break;
    case GS_BUF_GRAD_QUAT: *p = r->grad_quat; *bytes = 16 * N; break;
    case GS_BUF_GRAD_OPACITY: *p = r->grad_opacity; *bytes = 4 * N; break;
    case GS_BUF_GRAD_SH: *p = r->grad_sh; *bytes = 4 * SH_FLOATS * N; break;
    case GS_BUF_GRAD_CAM: *p = r->grad_cam; *bytes = 64 * (size_t)r->max_views; break;
    case GS_BUF_TARGET: *p = r->target; *bytes = 16 * P; break;
    case GS_BUF_RANGES: *p = r->ranges; *bytes = 8 * (size_t)r->max_tiles; break;
    case GS_BUF_SORTED_ITEMS: *p = r->ent_pairs[r->ent_in1]; *bytes = 8 * E; break;
    case GS_BUF_ENTRY_COUNT: *p = r->entry_total; *bytes = 8; break;
    case GS_BUF_LOSS: *p = r->loss_sums; *bytes = 16 * (size_t)r->max_views; break;
    case GS_BUF_RAW_POS: *p = r->raw[0]; *bytes = 16 * N; break;
    case GS_BUF_RAW_SCALES: *p = r->raw[1]; *bytes = 8 * N; break;
    case GS_BUF_RAW_QUAT: *p = r->raw[2]; *bytes = 16 * N; break;
    case GS_BUF_RAW_OPACITY: *p = r->raw[3]; *bytes = 4 * N; break;
    case GS_BUF_RAW_SH: *p = r->raw[4]; *bytes = 4 * SH_FLOATS * N; break;
    case GS_BUF_RECTS: *p = r->rects; *bytes = 16 * I; break;
    case GS_BUF_DEPTH_KEYS: *p = r->item_keys[0]; *bytes = 4 * I; break;
    case GS_BUF_DEPTH_ORDER: *p = r->item_vals[0]; *bytes = 4 * I; break;
    case GS_BUF_GRAD_NORM_SUM: *p = r->accum_norm; *bytes = 4 * N; break;
    case GS_BUF_NORMAL_LOSS: *p = r->normal_loss_sums; *bytes = 8 * (size_t)r->max_views; break;
    case GS_BUF_INCOMPLETE_TILES:
    case GS_BUF_TILE_CUT:
      if (!r->cut_on) return fail(r, GS_ERR_STATE, "the occlusion cut is off for this handle");
      if (id == GS_BUF_INCOMPLETE_TILES) { *p = r->cutw; *bytes = 4; }
      else { *p = r->tile_cut; *bytes = 4 * (size_t)r->max_tiles; }
      break;
    case GS_BUF_M_POS: case GS_BUF_M_SCALES: case GS_BUF_M_QUAT: case GS_BUF_M_OPACITY: case GS_BUF_M_SH: {
      const int k = (int)id - (int)GS_BUF_M_POS;
      *p = r->mom1[k]; *bytes = 4 * N * WIDTH[k];
      break;
    }
    case GS_BUF_V_POS: case GS_BUF_V_SCALES: case GS_BUF_V_QUAT: case GS_BUF_V_OPACITY: case GS_BUF_V_SH: {
      const int k = (int)id - (int)GS_BUF_V_POS;
      *p = r->mom2[k]; *bytes = 4 * N * WIDTH[k];
      break;
    }
    default: return fail(r, GS_ERR_INVALID_ARG, "unknown buffer id");
  }
  return GS_OK;
}

gs_status gs_rasterizer_buffer(gs_rasterizer* r, gs_buffer_id id, void** dptr, size_t* bytes) {
  if (!r || !dptr || !bytes) return GS_ERR_INVALID_ARG;
  return buffer_info(r, id, dptr, bytes);
}

gs_status gs_rasterizer_view_offset(gs_rasterizer* r, uint32_t view, uint64_t* pixel_offset, uint32_t* tile_offset) {
  if (!r) return GS_ERR_INVALID_ARG;
  if (view >= r->views_batched.size()) return fail(r, GS_ERR_INVALID_ARG, "view out of range");
  if (pixel_offset) *pixel_offset = (uint64_t)r->views_batched[view].pix_base;
  if (tile_offset) *tile_offset = (uint32_t)r->views_batched[view].tile_base;
  return GS_OK;
}

static gs_status copy_common(gs_rasterizer* r, gs_buffer_id id, uint64_t off, size_t bytes, void** dev) {
  void* p = nullptr;
  size_t total = 0;
  gs_status s = buffer_info(r, id, &p, &total);
  if (s) return s;
  if (off > total || bytes > total - off) return fail(r, GS_ERR_INVALID_ARG, "copy range outside the buffer");
  *dev = static_cast<char*>(p) + off;
  return GS_OK;
}

gs_status gs_rasterizer_read(gs_rasterizer* r, gs_buffer_id id, uint64_t off, void* host, size_t bytes, void* stream) {
  if (!r || (!host && bytes)) return GS_ERR_INVALID_ARG;
  void* d = nullptr;
  gs_status s = copy_common(r, id, off, bytes, &d);
  if (s) return s;
  TRY_CUDA(r, cudaMemcpyAsync(host, d, bytes, cudaMemcpyDeviceToHost, S(stream)));
  TRY_CUDA(r, cudaStreamSynchronize(S(stream)));
  return GS_OK;
}

gs_status gs_rasterizer_write(gs_rasterizer* r, gs_buffer_id id, uint64_t off, const void* host, size_t bytes,
                              void* stream) {
  if (!r || (!host && bytes)) return GS_ERR_INVALID_ARG;
  void* d = nullptr;
  gs_status s = copy_common(r, id, off, bytes, &d);
  if (s) return s;
  TRY_CUDA(r, cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, S(stream)));
  TRY_CUDA(r, cudaStreamSynchronize(S(stream)));
  return GS_OK;
}

gs_status gs_rasterizer_read_async(gs_rasterizer* r, gs_buffer_id id, uint64_t off, void* host, size_t bytes,
                                   void* stream) {
  if (!r || (!host && bytes)) return GS_ERR_INVALID_ARG;
  void* d = nullptr;
  gs_status s = copy_common(r, id, off, bytes, &d);
  if (s) return s;
  TRY_CUDA(r, cudaMemcpyAsync(host, d, bytes, cudaMemcpyDefault, S(stream)));  // host or device destination
  return GS_OK;
}

gs_status gs_rasterizer_write_async(gs_rasterizer* r, gs_buffer_id id, uint64_t off, const void* host, size_t bytes,
                                    void* stream) {
  if (!r || (!host && bytes)) return GS_ERR_INVALID_ARG;
  void* d = nullptr;
  gs_status s = copy_common(r, id, off, bytes, &d);
  if (s) return s;
  TRY_CUDA(r, cudaMemcpyAsync(d, host, bytes, cudaMemcpyDefault, S(stream)));  // host or device source
  return GS_OK;
}

gs_status gs_rasterizer_check(gs_rasterizer* r, void* stream) {
  if (!r) return GS_ERR_INVALID_ARG;
  TRY_CUDA(r, cudaStreamSynchronize(S(stream)));
  uint32_t w = 0;
  TRY_CUDA(r, cudaMemcpy(&w, r->words + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (w) {
    TRY_CUDA(r, cudaMemset(r->words + 1, 0, sizeof(uint32_t)));
    if (w & ERR_ENTRY_CAPACITY) return fail(r, GS_ERR_CAPACITY, "tile entries exceeded max_entries");
    if (w & ERR_TIMEOUT) return fail(r, GS_ERR_DEVICE_TIMEOUT, "a bounded device wait expired");
  }
  return GS_OK;
}

gs_status gs_loss_l1_ssim(gs_rasterizer* r, float w_l1, float w_ssim, void* stream) {
  if (!r) return GS_ERR_INVALID_ARG;
  if (!r->have_forward) return fail(r, GS_ERR_STATE, "loss needs a forward");
  cudaStream_t st = S(stream);
  TRY_CUDA(r, cudaMemsetAsync(r->loss_sums, 0, sizeof(double) * 2 * r->last_nv, st));
  return run_loss(r, r->last_views_dev, r->last_views_host, r->last_nv, w_l1, w_ssim, r->loss_sums, st);
}

gs_status gs_loss_normal(gs_rasterizer* r, float lambda, float alpha_min, void* stream) {
  if (!r) return GS_ERR_INVALID_ARG;
  if (!r->have_forward) return fail(r, GS_ERR_STATE, "normal loss needs a forward");
  cudaStream_t st = S(stream);
  uint64_t px = 0;
  for (uint32_t v = 0; v < r->last_nv; ++v) px += (uint64_t)r->last_views_host[v].width * r->last_views_host[v].height;
  TRY_CUDA(r, cudaMemsetAsync(r->normal_loss_sums, 0, sizeof(double) * r->last_nv, st));
  NormalArgs a{};
  a.views = r->last_views_dev; a.n_views = (int)r->last_nv; a.total_px = px;
  a.color = r->out_color; a.aux = r->out_aux; a.normal = r->out_normal;
  a.cp = r->coef; a.stride = r->max_pixels;  // the SSIM coefficient planes are free after the colour loss
  a.dl_dnormal = r->dl_dnormal; a.dl_dcolor = r->dl_dcolor; a.loss = r->normal_loss_sums;
  a.lambda = lambda; a.alpha_min = alpha_min;
  TRY_LAUNCH(r, launch_normal_loss(a, st));
  return GS_OK;
}

// ------------------------------------------------------ camera pose step
// crates/gs-track/src/lib.rs:289-337: the Riemannian rotation gradient, one
// Adam step over (rotation, centre) and the right-perturbation update.
gs_status gs_camera_step_grad(const float grad_cam[16], const float quat[4], float out6[6]) {
  if (!grad_cam || !quat || !out6) return GS_ERR_INVALID_ARG;
  for (int k = 0; k < 12; ++k)
    if (!std::isfinite(grad_cam[k])) return fail(nullptr, GS_ERR_NONFINITE, "non-finite camera gradient");
  float R[9];
  rotation_of(quat, R);  // column-major
  // B = Rᵀ·A with A = dL/dR (column-major): B[c][r] = Σ_k R[r][k]·A[c][k] ... as columns
  float B[9];
  for (int c = 0; c < 3; ++c)
    for (int rr = 0; rr < 3; ++rr) {
      float acc = 0.f;
      for (int k = 0; k < 3; ++k) acc += R[3 * rr + k] * grad_cam[3 * c + k];  // (Rᵀ)[rr][k] = R[k][rr] = col rr, row k
      B[3 * c + rr] = acc;
    }
  out6[0] = B[3 * 1 + 2] - B[3 * 2 + 1];
  out6[1] = B[3 * 2 + 0] - B[3 * 0 + 2];
  out6[2] = B[3 * 0 + 1] - B[3 * 1 + 0];
  out6[3] = grad_cam[9]; out6[4] = grad_cam[10]; out6[5] = grad_cam[11];
  return GS_OK;
}

gs_status gs_camera_adam6(float m[6], float v[6], uint32_t t, const float grad[6], float lr_rot, float lr_center,
                          float step[6]) {
  if (!m || !v || !grad || !step || t == 0) return GS_ERR_INVALID_ARG;
  float p1 = 1.f, p2 = 1.f;
  for (uint32_t k = 0; k < t; ++k) { p1 *= 0.9f; p2 *= 0.999f; }
  const float bc1 = 1.0f - p1, bc2 = 1.0f - p2;
  for (int k = 0; k < 6; ++k) {
    m[k] = 0.9f * m[k] + 0.1f * grad[k];
    v[k] = 0.999f * v[k] + 0.001f * grad[k] * grad[k];
    const float lr = k < 3 ? lr_rot : lr_center;
    step[k] = lr * (m[k] / bc1) / (std::sqrt(v[k] / bc2) + 1e-10f);
  }
  return GS_OK;
}

// ------------------------------------------------------- trainer schedule
// first_attempt/crates/gs-train/src/trainer.rs:740-746, 407-416, 1150.
gs_status gs_scene_extent(const float* positions, uint32_t n, uint32_t stride, float* extent) {
  if (!extent || (n && !positions) || stride < 3) return GS_ERR_INVALID_ARG;
  if (n == 0) { *extent = 1e-3f; return GS_OK; }
  float lo[3], hi[3];
  for (int c = 0; c < 3; ++c) lo[c] = hi[c] = positions[c];
  for (uint32_t i = 1; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      const float v = positions[(size_t)i * stride + c];
      lo[c] = std::min(lo[c], v);
      hi[c] = std::max(hi[c], v);
    }
  const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
  *extent = std::max(std::sqrt(dx * dx + dy * dy + dz * dz), 1e-3f) * 0.5f;
  return GS_OK;
}

gs_status gs_schedule_t(uint32_t iter, uint32_t iters, const gs_anneal* anneal, float* t) {
  if (!t) return GS_ERR_INVALID_ARG;
  if (!anneal) {
    *t = (float)iter / (float)std::max(iters, 1u);
    return GS_OK;
  }
  const uint32_t since = iter > anneal->start ? iter - anneal->start : 0u;
  const float done = std::min((float)since / (float)std::max(anneal->len, 1u), 1.0f);
  *t = anneal->t0 + (1.0f - anneal->t0) * done;
  return GS_OK;
}

gs_status gs_position_lr(float lr_pos, float extent, float final_factor, float t, float* lr) {
  if (!lr) return GS_ERR_INVALID_ARG;
  *lr = lr_pos * extent * std::pow(final_factor, t);
  return GS_OK;
}

gs_status gs_camera_apply_step(gs_camera* cam, const float step[6]) {
  if (!cam || !step) return GS_ERR_INVALID_ARG;
  // R' = R·exp([δ]×) with δ = −step[0..3]: q' = normalize(q · from_scaled_axis(δ)).
  const float dx = -step[0], dy = -step[1], dz = -step[2];
  const float ang = std::sqrt(dx * dx + dy * dy + dz * dz);
  float e[4] = {0.f, 0.f, 0.f, 1.f};
  if (ang != 0.f) {
    const float s = std::sin(0.5f * ang) / ang;
    e[0] = dx * s; e[1] = dy * s; e[2] = dz * s; e[3] = std::cos(0.5f * ang);
  }
  const float* q = cam->quat;
  float o[4];
  o[0] = q[3] * e[0] + q[0] * e[3] + q[1] * e[2] - q[2] * e[1];
  o[1] = q[3] * e[1] - q[0] * e[2] + q[1] * e[3] + q[2] * e[0];
  o[2] = q[3] * e[2] + q[0] * e[1] - q[1] * e[0] + q[2] * e[3];
  o[3] = q[3] * e[3] - q[0] * e[0] - q[1] * e[1] - q[2] * e[2];
  const float n = std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2] + o[3] * o[3]);
  for (int k = 0; k < 4; ++k) cam->quat[k] = o[k] / n;
  cam->center[0] -= step[3]; cam->center[1] -= step[4]; cam->center[2] -= step[5];
  return GS_OK;
}

gs_status gs_optimizer_init(gs_rasterizer* r, uint32_t n, void* stream) {
  if (!r) return GS_ERR_INVALID_ARG;
  if (n > r->cap) return fail(r, GS_ERR_CAPACITY, "num_surfels exceeds capacity");
  cudaStream_t st = S(stream);
  for (int k = 0; k < 5; ++k) {
    AdamClass ac{r->raw[k], r->mom1[k], r->mom2[k], act_ptr(r, k), 0.f, 0.f};
    TRY_LAUNCH(r, launch_activate_init(ac, (uint64_t)n * WIDTH[k], ACT[k], st));
  }
  gs_status s = refresh_half(r, n, st);
  if (s) return s;
  TRY_CUDA(r, cudaMemsetAsync(r->accum_norm, 0, sizeof(float) * r->cap, st));
  r->t = 0;
  r->accum_steps = 0;
  r->optim_ready = true;
  if (n > r->n_uploaded) r->n_uploaded = n;
  return GS_OK;
}

gs_status gs_optimizer_step(gs_rasterizer* r, const gs_adam_config* c, uint32_t n, void* stream) {
  if (!r || !c) return GS_ERR_INVALID_ARG;
  if (!r->optim_ready) return fail(r, GS_ERR_STATE, "gs_optimizer_init first");
  return adam_plain(r, c, n, S(stream));
}

gs_status gs_adam_flat(float* raw, const float* grad, float* m, float* v, float* act, uint64_t n, uint32_t activation,
                       float lr, float beta1, float beta2, float eps, float reg, uint32_t t, void* stream) {
  if (!raw || !grad || !m || !v || activation > 2 || t == 0) return fail(nullptr, GS_ERR_INVALID_ARG, "bad adam args");
  float bc1, bc2;
  bias_corrections(beta1, beta2, t, bc1, bc2);
  AdamClass ac{raw, m, v, act, lr, reg};
  int e = launch_adam_grad(ac, grad, n, (int)activation, beta1, beta2, eps, bc1, bc2, S(stream));
  if (e) return fail(nullptr, GS_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
  return GS_OK;
}

gs_status gs_train_step(gs_rasterizer* r, const gs_camera* cams, uint32_t nv, uint32_t n, const gs_step_config* cfg,
                        void* stream) {
  if (!r || !cfg || cfg->loss > GS_LOSS_GIVEN) return GS_ERR_INVALID_ARG;
  if (!r->optim_ready) return fail(r, GS_ERR_STATE, "gs_optimizer_init first");
  gs_status s = set_views(r, cams, nv, n);
  if (s) return s;
  cudaStream_t st = S(stream);
  s = upload_views(r, st);
  if (s) return s;
  if (cfg->form == 0) return plain_body(r, nv, n, cfg, st);
  // Chosen form: batched step replayed from a CUDA graph; per-step values
  // (cameras, learning rates, bias corrections) are uploaded before replay.
  s = cut_refresh(r, nv, n, st);
  if (s) return s;
  r->t += 1;
  DynParams dp{};
  for (int k = 0; k < 5; ++k) { dp.lr[k] = cfg->adam.lr[k]; dp.reg[k] = cfg->adam.reg[k]; }
  bias_corrections(cfg->adam.beta1, cfg->adam.beta2, r->t, dp.bc1, dp.bc2);
  TRY_CUDA(r, cudaMemcpyAsync(r->dyn_dev, &dp, sizeof(dp), cudaMemcpyHostToDevice, st));
  std::vector<uint64_t> key = {n, nv, (uint64_t)cfg->form, (uint64_t)r->cfg.precision};
  uint32_t bits[3];
  std::memcpy(&bits[0], &cfg->adam.beta1, 4);
  std::memcpy(&bits[1], &cfg->adam.beta2, 4);
  std::memcpy(&bits[2], &cfg->adam.eps, 4);
  for (uint32_t b : bits) key.push_back(b);
  uint32_t wb[2];
  std::memcpy(&wb[0], &cfg->w_l1, 4);
  std::memcpy(&wb[1], &cfg->w_ssim, 4);
  key.push_back(wb[0]); key.push_back(wb[1]);
  key.push_back(cfg->loss);
  key.push_back((uint64_t)r->wait_cycles[0]);
  key.push_back((uint64_t)r->wait_cycles[1]);
  for (const ViewInfo& v : r->views_batched) key.push_back(((uint64_t)v.width << 32) | (uint64_t)v.height);
  if (!r->graph || key != r->graph_key) {
    if (r->graph) { cudaGraphExecDestroy(r->graph); r->graph = nullptr; }
    s = ensure_graph_stream(r);
    if (!s) s = ensure_side_stream(r);
    if (s) return s;
    TRY_CUDA(r, cudaStreamSynchronize(st));
    TRY_CUDA(r, cudaStreamBeginCapture(r->cap_stream, cudaStreamCaptureModeThreadLocal));
    gs_status body = chosen_body(r, nv, n, cfg, r->cap_stream);
    cudaGraph_t g = nullptr;
    cudaError_t ec = cudaStreamEndCapture(r->cap_stream, &g);
    if (body) { if (g) cudaGraphDestroy(g); return body; }
    if (ec != cudaSuccess) return fail(r, GS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
    cudaError_t ei = cudaGraphInstantiate(&r->graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) { r->graph = nullptr; return fail(r, GS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei)); }
    r->graph_key = key;
  }
  TRY_CUDA(r, cudaGraphLaunch(r->graph, st));
  r->accum_steps += 1;
  return GS_OK;
}

gs_status gs_train_step_profiled(gs_rasterizer* r, const gs_camera* cams, uint32_t nv, uint32_t n,
                                 const gs_step_config* cfg, void* stream, float* stage_ms, uint32_t* n_stages) {
  if (!r || !cfg || !stage_ms || !n_stages || cfg->loss > GS_LOSS_GIVEN) return GS_ERR_INVALID_ARG;
  if (!r->optim_ready) return fail(r, GS_ERR_STATE, "gs_optimizer_init first");
  gs_status s = set_views(r, cams, nv, n);
  if (s) return s;
  cudaStream_t st = S(stream);
  s = upload_views(r, st);
  if (s) return s;
  Prof prof;
  if (cfg->form == 0) {
    s = plain_body(r, nv, n, cfg, st, &prof);
  } else {
    s = cut_refresh(r, nv, n, st);
    if (s) return s;
    r->t += 1;
    DynParams dp{};
    for (int k = 0; k < 5; ++k) { dp.lr[k] = cfg->adam.lr[k]; dp.reg[k] = cfg->adam.reg[k]; }
    bias_corrections(cfg->adam.beta1, cfg->adam.beta2, r->t, dp.bc1, dp.bc2);
    TRY_CUDA(r, cudaMemcpyAsync(r->dyn_dev, &dp, sizeof(dp), cudaMemcpyHostToDevice, st));
    s = ensure_side_stream(r);
    if (!s) s = chosen_body(r, nv, n, cfg, st, &prof);
    r->accum_steps += 1;
  }
  if (s) return s;
  TRY_CUDA(r, cudaStreamSynchronize(st));
  for (int k = 0; k < N_STAGES; ++k) stage_ms[k] = 0.f;
  for (size_t k = 1; k < prof.ev.size(); ++k) {
    float ms = 0.f;
    TRY_CUDA(r, cudaEventElapsedTime(&ms, prof.ev[k - 1], prof.ev[k]));
    const int stg = prof.stage[k];
    if (stg >= 0 && stg < N_STAGES) stage_ms[stg] += ms;
  }
  *n_stages = N_STAGES;
  return GS_OK;
}

gs_status gs_raster_work(gs_rasterizer* r, uint64_t out[4], void* stream) {
  if (!r || !out) return GS_ERR_INVALID_ARG;
  if (!r->have_forward) return fail(r, GS_ERR_STATE, "gs_raster_work needs a forward");
  cudaStream_t st = S(stream);
  RasterArgs ra{};
  ra.views = r->last_views_dev; ra.n_views = (int)r->last_nv; ra.total_tiles = r->last_tiles;
  ra.ranges = r->ranges; ra.sorted_pairs = r->ent_pairs[r->ent_in1];
  ra.exp_item = r->det ? r->exp_item : nullptr;
  ra.records = r->records;
  ra.out_nc = r->out_nc; ra.out_aux = r->out_aux;
  ra.gmask = r->gmask_valid ? r->gmask : nullptr;
  TRY_CUDA(r, cudaMemsetAsync(r->work_counts, 0, 4 * sizeof(unsigned long long), st));
  TRY_LAUNCH(r, launch_raster_work(ra, r->tile, r->last_prec, r->work_counts, st));
  unsigned long long h[4] = {0, 0, 0, 0};
  TRY_CUDA(r, cudaMemcpyAsync(h, r->work_counts, sizeof(h), cudaMemcpyDeviceToHost, st));
  TRY_CUDA(r, cudaStreamSynchronize(st));
  for (int k = 0; k < 4; ++k) out[k] = h[k];
  // The stored-state backward evaluates only the recorded contributors.
  if (r->mask_valid) out[2] = out[1];
  return GS_OK;
}

gs_status gs_set_launch_shapes(gs_rasterizer* r, const uint32_t shapes[4]) {
  if (!r || !shapes) return GS_ERR_INVALID_ARG;
  if (!shape_listed(true, r->tile, shapes[0], shapes[1]))
    return fail(r, GS_ERR_INVALID_ARG, "gs_set_launch_shapes: forward (batch, pixels per thread) not built for this tile");
  if (!shape_listed(false, r->tile, shapes[2], shapes[3]))
    return fail(r, GS_ERR_INVALID_ARG, "gs_set_launch_shapes: backward (batch, pixels per thread) not built for this tile");
  r->fwd_batch = (int)shapes[0];
  r->fwd_ppt = (int)shapes[1];
  r->bwd_batch = (int)shapes[2];
  r->bwd_ppt = (int)shapes[3];
  if (r->graph) { cudaGraphExecDestroy(r->graph); r->graph = nullptr; }
  return GS_OK;
}

gs_status gs_set_tile_size(gs_rasterizer* r, uint32_t tile) {
  if (!r) return GS_ERR_INVALID_ARG;
  if (tile != 8 && tile != 16 && tile != 32) return fail(r, GS_ERR_INVALID_ARG, "tile must be 8, 16 or 32");
  if (tile != 16 && r->stored_state)
    return fail(r, GS_ERR_INVALID_ARG, "the stored-state backward is built for 16-pixel tiles");
  if ((int)tile == r->tile) return GS_OK;
  r->tile = (int)tile;
  if (!shape_listed(true, r->tile, r->fwd_batch, r->fwd_ppt)) {
    const RasterShape* tab = nullptr;
    raster_fwd_shapes(r->tile, &tab);
    r->fwd_batch = tab[0].batch;
    r->fwd_ppt = tab[0].ppt;
  }
  if (!shape_listed(false, r->tile, r->bwd_batch, r->bwd_ppt)) default_bwd_shape(r);
  r->have_forward = false;  // tile lists of the last forward belong to the old tiling
  r->mask_valid = false;
  r->gmask_valid = false;
  if (r->graph) { cudaGraphExecDestroy(r->graph); r->graph = nullptr; }
  return GS_OK;
}

uint32_t gs_tile_size(const gs_rasterizer* r) { return r ? (uint32_t)r->tile : 0u; }

namespace {

// Times every forward and backward raster shape built for the handle's
// current tile size on these views (forward = projection + binning + raster,
// as the step runs it; backward = the colour-only backward raster) and
// keeps the fastest of each. *fwd_ms / *bwd_ms receive the winners' times
// (three launches each after one warm-up). *overflow is set, and nothing
// timed, when the tile entries exceed max_entries at this tile size.
gs_status tune_current_tile(gs_rasterizer* r, uint32_t nv, uint32_t n, cudaStream_t st, float* fwd_ms, float* bwd_ms,
                            bool* overflow) {
  *overflow = false;
  gs_status s = upload_views(r, st);
  if (s) return s;
  int tiles = 0;
  for (const ViewInfo& v : r->views_batched) tiles += v.tiles_x * v.tiles_y;
  const int prec = (int)r->cfg.precision;
  // Entry budget check at this tile size (the entry guard's sticky bit is
  // restored afterwards: an overflow here only rules the tile size out).
  uint32_t err_before = 0;
  TRY_CUDA(r, cudaMemcpyAsync(&err_before, r->words + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  s = run_forward(r, r->views_dev, r->views_batched.data(), nv, tiles, n, prec, true, true, st, nullptr,
                  r->color_only);
  if (s) return s;
  unsigned long long total = 0;
  TRY_CUDA(r, cudaMemcpyAsync(&total, r->entry_total, sizeof(total), cudaMemcpyDeviceToHost, st));
  TRY_CUDA(r, cudaStreamSynchronize(st));
  if (total > r->max_entries) {
    TRY_CUDA(r, cudaMemcpyAsync(r->words + 1, &err_before, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    TRY_CUDA(r, cudaStreamSynchronize(st));
    r->have_forward = false;
    *overflow = true;
    return GS_OK;
  }
  cudaEvent_t e0, e1;
  TRY_CUDA(r, cudaEventCreate(&e0));
  TRY_CUDA(r, cudaEventCreate(&e1));
  auto time_it = [&](auto&& fn) -> float {
    fn();  // warm-up
    cudaEventRecord(e0, st);
    for (int k = 0; k < 3; ++k) fn();
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms / 3.f;
  };
  const RasterShape* fshape = nullptr;
  const int nf = raster_fwd_shapes(r->tile, &fshape);
  float best = 1e30f;
  int bf = 0;
  for (int k = 0; k < nf; ++k) {
    r->fwd_batch = fshape[k].batch;
    r->fwd_ppt = fshape[k].ppt;
    gs_status fs = GS_OK;
    const float ms = time_it([&] { fs = run_forward(r, r->views_dev, r->views_batched.data(), nv, tiles, n, prec, true,
                                                    true, st, nullptr, r->color_only); });
    if (fs) { cudaEventDestroy(e0); cudaEventDestroy(e1); return fs; }
    if (ms < best) { best = ms; bf = k; }
  }
  *fwd_ms = best;
  r->fwd_batch = fshape[bf].batch;
  r->fwd_ppt = fshape[bf].ppt;
  // The forward the backward shapes are timed after is the step's own (the
  // colour-only forward also writes the row-group contributor summary).
  s = run_forward(r, r->views_dev, r->views_batched.data(), nv, tiles, n, prec, true, true, st, nullptr,
                  r->color_only);
  if (!s) {
    TRY_CUDA(r, cudaMemsetAsync(r->loss_sums, 0, sizeof(double) * 2 * nv, st));
    s = run_loss(r, r->views_dev, r->views_batched.data(), nv, 0.8f, 0.2f, r->loss_sums, st);
  }
  if (s) { cudaEventDestroy(e0); cudaEventDestroy(e1); return s; }
  const RasterShape* bshape = nullptr;
  const int nb = raster_bwd_shapes(r->tile, &bshape);
  best = 1e30f;
  int bb = 0;
  for (int k = 0; k < nb; ++k) {
    r->bwd_batch = bshape[k].batch;
    r->bwd_ppt = bshape[k].ppt;
    gs_status bs = GS_OK;
    const float ms = time_it([&] { bs = run_backward_raster(r, r->views_dev, nv, tiles, n, prec, false, true, st); });
    if (bs) { cudaEventDestroy(e0); cudaEventDestroy(e1); return bs; }
    if (ms < best) { best = ms; bb = k; }
  }
  *bwd_ms = best;
  r->bwd_batch = bshape[bb].batch;
  r->bwd_ppt = bshape[bb].ppt;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return GS_OK;
}

}  // namespace

gs_status gs_autotune(gs_rasterizer* r, const gs_camera* cams, uint32_t nv, uint32_t n, void* stream, uint32_t out[4]) {
  if (!r || !out) return GS_ERR_INVALID_ARG;
  gs_status s = set_views(r, cams, nv, n);
  if (s) return s;
  float fms = 0.f, bms = 0.f;
  bool overflow = false;
  s = tune_current_tile(r, nv, n, S(stream), &fms, &bms, &overflow);
  if (s) return s;
  if (overflow) return fail(r, GS_ERR_CAPACITY, "gs_autotune: tile entries exceed max_entries");
  if (r->graph) { cudaGraphExecDestroy(r->graph); r->graph = nullptr; }
  out[0] = (uint32_t)r->fwd_batch; out[1] = (uint32_t)r->fwd_ppt;
  out[2] = (uint32_t)r->bwd_batch; out[3] = (uint32_t)r->bwd_ppt;
  return GS_OK;
}

gs_status gs_autotune_tiles(gs_rasterizer* r, const gs_camera* cams, uint32_t nv, uint32_t n, void* stream,
                            uint32_t out[5], float times_ms[6]) {
  if (!r || !out) return GS_ERR_INVALID_ARG;
  cudaStream_t st = S(stream);
  const int tiles[3] = {8, 16, 32};
  float best = 1e30f;
  uint32_t best_cfg[5] = {0, 0, 0, 0, 0};
  for (int i = 0; i < 3; ++i) {
    if (times_ms) { times_ms[2 * i] = -1.f; times_ms[2 * i + 1] = -1.f; }
    if (tiles[i] != 16 && r->stored_state) continue;
    gs_status s = gs_set_tile_size(r, (uint32_t)tiles[i]);
    if (s) return s;
    s = set_views(r, cams, nv, n);
    if (s == GS_ERR_CAPACITY) continue;  // the tile budget of the handle is too small for this tiling
    if (s) return s;
    float fms = 0.f, bms = 0.f;
    bool overflow = false;
    s = tune_current_tile(r, nv, n, st, &fms, &bms, &overflow);
    if (s) return s;
    if (overflow) continue;
    if (times_ms) { times_ms[2 * i] = fms; times_ms[2 * i + 1] = bms; }
    if (fms + bms < best) {
      best = fms + bms;
      best_cfg[0] = (uint32_t)tiles[i];
      best_cfg[1] = (uint32_t)r->fwd_batch; best_cfg[2] = (uint32_t)r->fwd_ppt;
      best_cfg[3] = (uint32_t)r->bwd_batch; best_cfg[4] = (uint32_t)r->bwd_ppt;
    }
  }
  if (best_cfg[0] == 0) return fail(r, GS_ERR_CAPACITY, "gs_autotune_tiles: no tile size fits max_entries");
  gs_status s = gs_set_tile_size(r, best_cfg[0]);
  if (s) return s;
  s = gs_set_launch_shapes(r, best_cfg + 1);
  if (s) return s;
  s = set_views(r, cams, nv, n);
  if (s) return s;
  if (r->graph) { cudaGraphExecDestroy(r->graph); r->graph = nullptr; }
  for (int k = 0; k < 5; ++k) out[k] = best_cfg[k];
  return GS_OK;
}

gs_status gs_densify_prune(gs_rasterizer* r, const gs_densify_config* c, uint32_t n, uint32_t* n_out, void* stream) {
  if (!r || !c || !n_out) return GS_ERR_INVALID_ARG;
  if (!r->optim_ready) return fail(r, GS_ERR_STATE, "gs_optimizer_init first");
  if (n > r->cap) return fail(r, GS_ERR_CAPACITY, "num_surfels exceeds capacity");
  r->cut_sig.clear();  // the surfel set changes: the next step starts from full lists
  cudaStream_t st = S(stream);
  const size_t N = r->cap;
  if (!r->dens_flags) {
    TRY_CUDA(r, dalloc(r->dens_flags, 2 * N));
    TRY_CUDA(r, dalloc(r->dens_slots, 2 * N));
    TRY_CUDA(r, dalloc(r->dens_tmp, N * SH_FLOATS));
  }
  DensifyArgs a{};
  a.n = n; a.capacity = r->cap;
  a.grad_threshold = c->grad_threshold; a.opacity_threshold = c->opacity_threshold;
  a.inv_steps = r->accum_steps ? 1.0f / (float)r->accum_steps : 0.f;
  a.accum = r->accum_norm; a.opacity_act = r->opacities;
  a.flags = r->dens_flags; a.slots = r->dens_slots; a.tmp = r->dens_tmp; a.n_out_dev = r->words + 4;
  int k = 0;
  for (int c5 = 0; c5 < 5; ++c5) {
    a.arrays[k] = r->raw[c5]; a.widths[k++] = WIDTH[c5];
    a.arrays[k] = act_ptr(r, c5); a.widths[k++] = WIDTH[c5];
    a.arrays[k] = r->mom1[c5]; a.widths[k++] = -WIDTH[c5];
    a.arrays[k] = r->mom2[c5]; a.widths[k++] = -WIDTH[c5];
  }
  a.n_arrays = k;
  TRY_LAUNCH(r, launch_densify(a, r->scan_scratch, st));
  uint32_t out = 0;
  TRY_CUDA(r, cudaMemcpyAsync(&out, r->words + 4, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  TRY_CUDA(r, cudaStreamSynchronize(st));
  TRY_CUDA(r, cudaMemsetAsync(r->accum_norm, 0, sizeof(float) * N, st));
  r->accum_steps = 0;
  gs_status s = refresh_half(r, out, st);
  if (s) return s;
  TRY_CUDA(r, cudaStreamSynchronize(st));
  if (r->graph) { cudaGraphExecDestroy(r->graph); r->graph = nullptr; }
  r->n_uploaded = out;
  *n_out = out;
  return GS_OK;
}

// ------------------------------------------------------------------ MCMC
static gs_status mcmc_ready(gs_rasterizer* r, cudaStream_t st) {
  if (r->mcmc_u32) return GS_OK;
  const size_t N = r->cap;
  TRY_CUDA(r, dalloc(r->mcmc_u32, 19 * N));
  TRY_CUDA(r, dalloc(r->mcmc_u64, 2 * N + 1));
  TRY_CUDA(r, dalloc(r->mcmc_jump, 64 * (size_t)MCMC_JUMP_LEVELS));
  TRY_CUDA(r, dalloc(r->mcmc_rng, 1));
  TRY_CUDA(r, dalloc(r->mcmc_counters, 8));
  std::vector<uint64_t> jump(64 * (size_t)MCMC_JUMP_LEVELS);
  mcmc_jump_tables(jump.data());
  TRY_CUDA(r, cudaMemcpyAsync(r->mcmc_jump, jump.data(), jump.size() * 8, cudaMemcpyHostToDevice, st));
  const uint64_t seed = 0x853c49e6748fea9bull;
  TRY_CUDA(r, cudaMemcpyAsync(r->mcmc_rng, &seed, 8, cudaMemcpyHostToDevice, st));
  TRY_CUDA(r, cudaStreamSynchronize(st));  // the host sources above are stack/heap temporaries
  return GS_OK;
}

gs_status gs_mcmc_seed(gs_rasterizer* r, uint64_t state, void* stream) {
  if (!r || state == 0) return fail(r, GS_ERR_INVALID_ARG, "xorshift64 state must be nonzero");
  cudaStream_t st = S(stream);
  gs_status s = mcmc_ready(r, st);
  if (s) return s;
  TRY_CUDA(r, cudaMemcpyAsync(r->mcmc_rng, &state, 8, cudaMemcpyHostToDevice, st));
  TRY_CUDA(r, cudaStreamSynchronize(st));
  return GS_OK;
}

gs_status gs_mcmc_relocate(gs_rasterizer* r, const gs_mcmc_config* c, uint32_t n, void* stream) {
  if (!r || !c) return GS_ERR_INVALID_ARG;
  if (!r->optim_ready) return fail(r, GS_ERR_STATE, "gs_optimizer_init first");
  if (n > r->cap) return fail(r, GS_ERR_CAPACITY, "num_surfels exceeds capacity");
  if (n == 0) return GS_OK;
  r->cut_sig.clear();  // relocated surfels: the next step starts from full lists
  cudaStream_t st = S(stream);
  gs_status s = mcmc_ready(r, st);
  if (s) return s;
  const size_t N = r->cap;
  McmcArgs a{};
  a.n = n; a.dead_threshold = c->dead_threshold; a.split_ratio = c->split_ratio;
  a.jump = r->mcmc_jump; a.rng_state = r->mcmc_rng; a.counters = r->mcmc_counters;
  uint32_t* u = r->mcmc_u32;
  uint32_t** fields[] = {&a.dead, &a.dead_rank, &a.dead_idx, &a.owner, &a.used, &a.pick, &a.leftover_flag,
                         &a.left_rank, &a.left_idx, &a.size_key, &a.size_val, &a.key2, &a.val2, &a.over_flag,
                         &a.over_rank, &a.over_key, &a.over_val};
  for (size_t k = 0; k < sizeof(fields) / sizeof(fields[0]); ++k) *fields[k] = u + k * N;
  a.weight = r->mcmc_u64; a.cum = r->mcmc_u64 + N; a.total_weight = r->mcmc_u64 + 2 * N;
  a.opac_act = r->opacities; a.scales_act = r->scales;
  a.pos_raw = reinterpret_cast<float4*>(r->raw[0]); a.scales_raw = reinterpret_cast<float2*>(r->raw[1]);
  a.quat_raw = reinterpret_cast<float4*>(r->raw[2]); a.opac_raw = r->raw[3]; a.sh_raw = r->raw[4];
  a.pos_act = r->positions; a.scales_act_w = r->scales; a.quat_act = r->quats; a.opac_act_w = r->opacities;
  a.sh_act = r->sh;
  a.sh_half = r->cfg.precision == GS_PREC_F32 ? nullptr : r->sh_half;
  for (int k = 0; k < 5; ++k) { a.m[k] = r->mom1[k]; a.v[k] = r->mom2[k]; }
  TRY_LAUNCH(r, launch_mcmc_relocate(a, (int)r->cfg.precision, r->scan_scratch, r->sort_scratch, st));
  return GS_OK;
}

gs_status gs_mcmc_stats(gs_rasterizer* r, uint32_t out[4], uint64_t* rng_state, void* stream) {
  if (!r || !out) return GS_ERR_INVALID_ARG;
  cudaStream_t st = S(stream);
  gs_status s = mcmc_ready(r, st);
  if (s) return s;
  uint32_t c[8];
  uint64_t x = 0;
  TRY_CUDA(r, cudaMemcpyAsync(c, r->mcmc_counters, sizeof(c), cudaMemcpyDeviceToHost, st));
  TRY_CUDA(r, cudaMemcpyAsync(&x, r->mcmc_rng, 8, cudaMemcpyDeviceToHost, st));
  TRY_CUDA(r, cudaStreamSynchronize(st));
  out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = c[3];
  if (rng_state) *rng_state = x;
  return GS_OK;
}

gs_status gs_mcmc_noise(gs_rasterizer* r, uint32_t n, uint32_t seed, float sigma, float opacity_k, void* stream) {
  if (!r) return GS_ERR_INVALID_ARG;
  if (!r->optim_ready) return fail(r, GS_ERR_STATE, "gs_optimizer_init first");
  if (n > r->cap) return fail(r, GS_ERR_CAPACITY, "num_surfels exceeds capacity");
  TRY_LAUNCH(r, launch_mcmc_noise(reinterpret_cast<float4*>(r->raw[0]), r->positions, r->scales, r->opacities, n,
                                  seed, sigma, opacity_k, S(stream)));
  return GS_OK;
}

// ------------------------------------------------------------------- PLY
gs_status gs_rasterizer_save_ply(gs_rasterizer* r, const char* path, uint32_t n, void* stream) {
  if (!r || !path) return GS_ERR_INVALID_ARG;
  if (n > r->cap) return fail(r, GS_ERR_CAPACITY, "num_surfels exceeds capacity");
  cudaStream_t st = S(stream);
  std::vector<float> pos(4 * (size_t)n), sc(2 * (size_t)n), q(4 * (size_t)n), op(n), sh(SH_FLOATS * (size_t)n);
  TRY_CUDA(r, cudaMemcpyAsync(pos.data(), r->positions, pos.size() * 4, cudaMemcpyDeviceToHost, st));
  TRY_CUDA(r, cudaMemcpyAsync(sc.data(), r->scales, sc.size() * 4, cudaMemcpyDeviceToHost, st));
  TRY_CUDA(r, cudaMemcpyAsync(q.data(), r->quats, q.size() * 4, cudaMemcpyDeviceToHost, st));
  TRY_CUDA(r, cudaMemcpyAsync(op.data(), r->opacities, op.size() * 4, cudaMemcpyDeviceToHost, st));
  TRY_CUDA(r, cudaMemcpyAsync(sh.data(), r->sh, sh.size() * 4, cudaMemcpyDeviceToHost, st));
  TRY_CUDA(r, cudaStreamSynchronize(st));
  const gs_status s = gs_ply_write(path, n, pos.data(), sc.data(), q.data(), op.data(), sh.data());
  if (s) r->err = g_last_error;
  return s;
}

gs_status gs_rasterizer_load_ply(gs_rasterizer* r, const char* path, uint32_t* n_out, void* stream) {
  if (!r || !path || !n_out) return GS_ERR_INVALID_ARG;
  uint32_t n = 0, nc = 0;
  gs_status s = gs_ply_info(path, &n, &nc);
  if (!s && n > r->cap) s = fail(nullptr, GS_ERR_CAPACITY, "ply holds more surfels than the capacity");
  std::vector<float> pos3(3 * (size_t)n), sc3(3 * (size_t)n), q(4 * (size_t)n), op(n), sh(3 * (size_t)nc * n);
  if (!s) s = gs_ply_read(path, r->cap, pos3.data(), sc3.data(), q.data(), op.data(), sh.data(), &n);
  if (s) {
    r->err = g_last_error;
    return s;
  }
  std::vector<float> sc2(2 * (size_t)n);
  for (size_t i = 0; i < n; ++i) { sc2[2 * i] = sc3[3 * i]; sc2[2 * i + 1] = sc3[3 * i + 1]; }
  gs_scene_input in{pos3.data(), sc2.data(), q.data(), op.data(), sh.data(), nc, n};
  s = gs_rasterizer_upload_scene(r, &in, stream);
  if (!s) *n_out = n;
  return s;
}

// ---------------------------------------------------------------- binner
gs_status gs_binner_create(uint32_t max_items, uint64_t max_entries, uint32_t num_tiles, gs_binner** out) {
  if (!out || max_items == 0 || num_tiles == 0 || max_entries >= 0xffffffffull)
    return fail(nullptr, GS_ERR_INVALID_ARG, "bad binner sizes");
  gs_binner* b = new (std::nothrow) gs_binner();
  if (!b) return fail(nullptr, GS_ERR_CUDA, "host allocation failed");
  b->max_items = max_items; b->max_entries = std::max<uint64_t>(max_entries, 1); b->num_tiles = num_tiles;
  const size_t I = max_items, E = b->max_entries;
  cudaError_t e = cudaSuccess;
  auto A = [&](auto*& p, size_t n) { if (e == cudaSuccess) e = dalloc(p, n); };
  A(b->counts, I); A(b->ref_offsets, I); A(b->offsets, I);
  for (int k = 0; k < 2; ++k) { A(b->item_keys[k], I); A(b->item_vals[k], I); A(b->ent_pairs[k], E); }
  A(b->sorted_entries, E); A(b->entry_items, E); A(b->ranges, num_tiles); A(b->total, 1); A(b->words, 8);
  unsigned char *s1 = nullptr, *s2 = nullptr;
  A(s1, scan_scratch_bytes()); A(s2, sort_scratch_bytes());
  b->scan_scratch = s1; b->sort_scratch = s2;
  if (e == cudaSuccess) e = cudaMemset(b->words, 0, 32);
  if (e == cudaSuccess) e = cudaMemset(b->total, 0, 8);
  if (e != cudaSuccess) {
    gs_binner_destroy(b);
    return fail(nullptr, GS_ERR_CUDA, std::string("binner allocation: ") + cudaGetErrorString(e));
  }
  *out = b;
  return GS_OK;
}

gs_status gs_binner_destroy(gs_binner* b) {
  if (!b) return GS_OK;
  void* ptrs[] = {b->counts, b->ref_offsets, b->offsets, b->item_keys[0], b->item_keys[1], b->item_vals[0],
                  b->item_vals[1], b->ent_pairs[0], b->ent_pairs[1], b->sorted_entries,
                  b->entry_items, b->ranges, b->total, b->words, b->scan_scratch, b->sort_scratch};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete b;
  return GS_OK;
}

}  // extern "C"

namespace gs {
int launch_rect_counts(const uint4* rects, const uint32_t* depths, uint32_t n, uint32_t* counts, uint32_t* keys,
                       uint32_t* vals, cudaStream_t st);
}

extern "C" gs_status gs_binner_encode(gs_binner* b, const uint32_t* rects_dev, const uint32_t* depths_dev, uint32_t n,
                                      uint32_t tiles_x, void* stream) {
  if (!b || (n && (!rects_dev || !depths_dev)) || tiles_x == 0 || b->num_tiles % tiles_x != 0)
    return fail(nullptr, GS_ERR_INVALID_ARG, "bad binner encode args");
  if (n > b->max_items) return fail(nullptr, GS_ERR_CAPACITY, "more items than max_items");
  cudaStream_t st = S(stream);
  const uint4* rects = reinterpret_cast<const uint4*>(rects_dev);
  int e = launch_rect_counts(rects, depths_dev, n, b->counts, b->item_keys[0], b->item_vals[0], st);
  if (!e) e = launch_scan(b->counts, nullptr, b->ref_offsets, n, nullptr, nullptr, nullptr, b->scan_scratch, st);
  int in1 = 0;
  if (!e) e = launch_radix_sort(b->item_keys[0], b->item_vals[0], b->item_keys[1], b->item_vals[1], n, nullptr, 32,
                                b->sort_scratch, &in1, st);
  uint32_t* perm = b->item_vals[in1];
  if (!e) e = launch_scan(b->counts, perm, b->offsets, n, nullptr, b->words, b->total, b->scan_scratch, st);
  if (!e) e = launch_entry_guard(b->total, b->words, b->max_entries, b->words + 1, st);
  if (!e) {
    ExpandArgs ea{};
    ea.perm = perm; ea.counts = b->counts; ea.offsets = b->offsets; ea.rects = rects;
    ea.views = nullptr; ea.items_per_view = n ? n : 1; ea.tiles_x = tiles_x;
    ea.n_items_dev = nullptr; ea.n_items_host = n;
    ea.total = b->total; ea.capacity = b->max_entries;
    ea.pairs = b->ent_pairs[0];
    ea.val_mode = 2; ea.ref_offsets = b->ref_offsets; ea.entry_items = b->entry_items;
    ea.error_word = b->words + 1;
    e = launch_expand(ea, st);
  }
  if (!e) e = launch_radix_sort_pairs(b->ent_pairs[0], b->ent_pairs[1], b->max_entries, b->words,
                                      tile_key_bits(b->num_tiles), b->sort_scratch, &b->ent_in1, st);
  if (!e) e = launch_ranges(b->ent_pairs[b->ent_in1], b->total, b->max_entries, b->ranges, b->num_tiles, st);
  if (!e) e = launch_pair_values(b->ent_pairs[b->ent_in1], b->sorted_entries, b->total, b->max_entries, st);
  if (e) return fail(nullptr, GS_ERR_CUDA, std::string("binner encode: ") + cudaGetErrorString((cudaError_t)e));
  // The reference asserts on overflow; report it here (blocking).
  uint32_t w = 0;
  cudaError_t ce = cudaMemcpyAsync(&w, b->words + 1, 4, cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess) return fail(nullptr, GS_ERR_CUDA, cudaGetErrorString(ce));
  if (w & ERR_ENTRY_CAPACITY) {
    cudaMemset(b->words + 1, 0, 4);
    return fail(nullptr, GS_ERR_CAPACITY, "tile entries exceeded max_entries");
  }
  return GS_OK;
}

extern "C" gs_status gs_binner_buffer(gs_binner* b, uint32_t which, void** dptr, size_t* bytes) {
  if (!b || !dptr || !bytes) return GS_ERR_INVALID_ARG;
  switch (which) {
    case 0: *dptr = b->sorted_entries; *bytes = 4 * b->max_entries; break;
    case 1: *dptr = b->entry_items; *bytes = 4 * b->max_entries; break;
    case 2: *dptr = b->ranges; *bytes = 8ull * b->num_tiles; break;
    case 3: *dptr = b->total; *bytes = 8; break;
    default: return fail(nullptr, GS_ERR_INVALID_ARG, "unknown binner buffer");
  }
  return GS_OK;
}

// ------------------------------------------------------- sort / scan API
namespace {
struct GlobalScratch {
  std::mutex mu;
  int device = -1;
  void* scan = nullptr;
  void* sort = nullptr;
  uint32_t* words = nullptr;
};
GlobalScratch g_scratch;

gs_status global_scratch(void** scan, void** sort, uint32_t** words) {
  std::lock_guard<std::mutex> lk(g_scratch.mu);
  int dev = 0;
  cudaGetDevice(&dev);
  if (g_scratch.device != dev) {
    if (g_scratch.scan) { cudaFree(g_scratch.scan); cudaFree(g_scratch.sort); cudaFree(g_scratch.words); }
    g_scratch.scan = g_scratch.sort = nullptr;
    g_scratch.words = nullptr;
    cudaError_t e = cudaMalloc(&g_scratch.scan, scan_scratch_bytes());
    if (e == cudaSuccess) e = cudaMalloc(&g_scratch.sort, sort_scratch_bytes());
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g_scratch.words), 64);
    if (e != cudaSuccess) return fail(nullptr, GS_ERR_CUDA, std::string("scratch: ") + cudaGetErrorString(e));
    g_scratch.device = dev;
  }
  *scan = g_scratch.scan;
  *sort = g_scratch.sort;
  *words = g_scratch.words;
  return GS_OK;
}
}  // namespace

extern "C" gs_status gs_radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint64_t n, uint32_t key_bits, void* stream) {
  if (n == 0) return GS_OK;
  if (!keys || !vals || key_bits == 0 || key_bits > 32 || n >= 0xffffffffull)
    return fail(nullptr, GS_ERR_INVALID_ARG, "bad sort args");
  void *scan = nullptr, *sort = nullptr;
  uint32_t* words = nullptr;
  gs_status s = global_scratch(&scan, &sort, &words);
  if (s) return s;
  cudaStream_t st = S(stream);
  uint32_t *k1 = nullptr, *v1 = nullptr;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&k1), n * 4, st);
  if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void**>(&v1), n * 4, st);
  if (e != cudaSuccess) return fail(nullptr, GS_ERR_CUDA, std::string("sort buffers: ") + cudaGetErrorString(e));
  int in1 = 0;
  int le = launch_radix_sort(keys, vals, k1, v1, n, nullptr, (int)key_bits, sort, &in1, st);
  if (!le && in1) {  // an odd number of passes ends in the ping-pong buffers
    le = (int)cudaMemcpyAsync(keys, k1, n * 4, cudaMemcpyDeviceToDevice, st);
    if (!le) le = (int)cudaMemcpyAsync(vals, v1, n * 4, cudaMemcpyDeviceToDevice, st);
  }
  cudaFreeAsync(k1, st);
  cudaFreeAsync(v1, st);
  if (le) return fail(nullptr, GS_ERR_CUDA, cudaGetErrorString((cudaError_t)le));
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(nullptr, GS_ERR_CUDA, cudaGetErrorString(e));
  return GS_OK;
}

extern "C" gs_status gs_exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* total_dev,
                                           void* stream) {
  if ((!in || !out) && n) return fail(nullptr, GS_ERR_INVALID_ARG, "bad scan args");
  if (n >= 0xffffffffull) return fail(nullptr, GS_ERR_INVALID_ARG, "scan length must be < 2^32");
  void *scan = nullptr, *sort = nullptr;
  uint32_t* words = nullptr;
  gs_status s = global_scratch(&scan, &sort, &words);
  if (s) return s;
  int e = launch_scan(in, nullptr, out, n, nullptr, total_dev, nullptr, scan, S(stream));
  if (e) return fail(nullptr, GS_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
  return GS_OK;
}

extern "C" gs_status gs_shutdown(void) {
  std::lock_guard<std::mutex> lk(g_scratch.mu);
  if (g_scratch.scan) { cudaFree(g_scratch.scan); cudaFree(g_scratch.sort); cudaFree(g_scratch.words); }
  g_scratch.scan = g_scratch.sort = nullptr;
  g_scratch.words = nullptr;
  g_scratch.device = -1;
  return GS_OK;
}
