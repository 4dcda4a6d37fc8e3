// Internal launch interface between the host orchestration (gs_api.cu) and
// the kernel translation units. Launchers return a cudaError_t value (0 = ok).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "gs_common.cuh"

namespace gs {

// Sets the text gs_last_error(NULL) reports.
void set_error_message(const std::string& msg);

struct ProjectArgs {
  const ViewInfo* views;
  uint32_t n;             // surfels of this step; item = view*n + surfel
  const float4* pos;
  const float2* scales;
  const float4* quats;
  const float* opac;
  const void* sh;         // 48 per surfel, f32 or 16-bit by precision
  void* records;
  uint4* rects;
  uint32_t* keys;
  uint32_t* vals;
  uint32_t* counts;
  int tight;              // bin only tiles the α-box overlaps (contributor indices then refer to that list)
  // Occlusion cut (null: off): per global tile id, the largest depth key
  // binned into the tile; counts[item] then covers only the rect's tiles with
  // key <= cut[tile]. item_key receives every item's depth key by item index.
  const uint32_t* cut;
  uint32_t* item_key;
};

struct ProjectBwdArgs {
  const ViewInfo* views;
  uint32_t n;
  int n_views;
  int view;               // plain form: the view of this launch
  const float4* pos;
  const float2* scales;
  const float4* quats;
  const void* sh;
  const float* grad_geom;     // atomic mode: [item][GG_STRIDE]
  const float* partials;      // deterministic mode: [entry][GG_STRIDE], or null
  const uint32_t* entry_offset;  // deterministic mode: first entry of each item
  const unsigned long long* entry_total;  // deterministic mode: entries of the last forward
  const uint32_t* counts;
  float4* grad_pos;
  float2* grad_scales;
  float4* grad_quat;
  float* grad_opacity;
  float* grad_sh;
  float* grad_cam;        // 16 per view, or null
  // Deterministic mode: per (unit, view) camera partial sums, 16 floats each
  // (units: warps of the plain kernel, blocks of the fused one), summed in
  // unit order by launch_cam_reduce; null: added into grad_cam by atomics.
  float* cam_partials;
};

struct AdamClass {
  float* raw;
  float* m;
  float* v;
  float* act;
  float lr;
  float reg;
};

struct AdamFusedArgs {
  AdamClass cls[5];
  float beta1, beta2, eps, bc1_inv, bc2_inv;
  const float* dyn;       // optional device copy of {lr[5], reg[5], bc1_inv, bc2_inv} (graph replay)
  void* sh_half;          // 16-bit activated SH copy for mixed precision, or null
  int sh_half_is_bf16;
  float* accum_grad_norm; // per-surfel running sum of |dL/dpos| (densify), or null
  uint32_t* error_word;   // sticky device error word (bounded-wait expiry)
  // Limits in SM cycles of the two bounded waits on the optimizer-row copies:
  // [0] before the Adam update (expiry sets ERR_TIMEOUT and skips the block's
  // update; 0 gives up at once), [1] the drain wait that lets the copies land
  // before an expired block exits.
  long long wait_cycles[2];
};

struct RasterArgs {
  const ViewInfo* views;
  int n_views;
  int total_tiles;
  const uint2* ranges;
  const uint2* sorted_pairs;    // (tile, item id) (atomic mode) or (tile, expansion index) (deterministic mode)
  const uint32_t* exp_item;     // expansion index -> item (deterministic mode)
  const void* records;
  float4* out_color;
  float4* out_aux;
  float4* out_normal;
  uint32_t* out_nc;
  const float4* dl_dcolor;
  const float4* dl_dnormal;
  float* grad_geom;
  float* partials;
  float lambda_dist;
  uint32_t* tile_counter;       // persistent kernels: zeroed before each launch
  const uint32_t* tile_order;   // persistent kernels: the tile taken at each counter value (null: identity)
  uint32_t* tile_walk;          // forward (optional): per tile, the largest contributor count of its pixels
  // Stored-state mode (16-pixel tiles): per-pixel contributor bitmasks. Word w of
  // pixel i (0..255, row-major in the tile) of tile t is mask[(mask_off[t] + w)·256 + i];
  // bit b of word w is set when list position 32w + b composited into the pixel.
  // Colour-only forward on 16-pixel tiles: per tile entry (index into
  // sorted_pairs), bit g set when a pixel of rows 4g..4g+3 composited it.
  // Written by the forward and read by the backward when non-null.
  uint8_t* gmask;
  uint32_t* mask;               // null: the backward re-evaluates every entry
  const uint32_t* mask_off;     // per tile, in 256-word groups
  // Persistent kernels: number of tile_order entries to take (device count);
  // null: total_tiles.
  const uint32_t* tile_limit;
  // Occlusion cut bookkeeping (persistent forward with tile_walk): null: off.
  // cut_pass 1 renders lists truncated at tile_cut and records every tile
  // that ran out of its truncated list with pixels still alive (inc_flag[t]
  // = 1; slot i of inc_count holds the tile in inc_list, its truncated
  // length in inc_skip and start in inc_src). cut_pass 2 takes the listed
  // tiles (tile_order = inc_list) and resumes each after its first inc_skip
  // entries from the pixel state pass 1 left in the outputs (their gmask
  // bytes are moved by launch_ranges_fix_list). Both write each
  // finished tile's next cut: the depth key (item_key) at list position
  // walk + walk/4 + 32, or past the list's end when it is shorter.
  uint32_t* tile_cut;
  int cut_pass;
  const uint32_t* item_key;
  uint32_t* inc_count;
  uint32_t* inc_list;
  uint32_t* inc_skip;
  uint32_t* inc_src;
  uint8_t* inc_flag;
};
// Raster launch shapes built for a tile size (8, 16, 32): (staging batch,
// pixels per thread). Returns the count and points *out at the table.
struct RasterShape { int batch, ppt; };
int raster_fwd_shapes(int tile, const RasterShape** out);
int raster_bwd_shapes(int tile, const RasterShape** out);
// Blocks per SM the raster kernels sustain (for persistent grids).
int raster_fwd_occupancy(int tile, int prec, int batch, int ppt, bool det, bool color, bool mask);
int raster_bwd_occupancy(int tile, int prec, bool aux, int ppt, int batch, bool det, bool mask);
// Per tile size (defined by the unit that instantiates it).
template <int TS> int raster_fwd_occupancy_t(int prec, int batch, int ppt, bool det, bool color, bool mask);
template <int TS> int raster_bwd_occupancy_t(int prec, bool aux, int ppt, int batch, bool det, bool mask);
template <int TS> int launch_raster_fwd_t(const RasterArgs& a, int prec, int batch, int ppt, bool det,
                                          bool persistent, bool color, int grid, cudaStream_t st);
template <int TS> int launch_raster_bwd_t(const RasterArgs& a, int prec, bool aux, int ppt, int batch, bool det,
                                          bool persistent, int grid, cudaStream_t st);

int launch_project(const ProjectArgs& a, int prec, uint32_t n_views, cudaStream_t st);
int launch_project_bwd(const ProjectBwdArgs& a, int prec, bool aux, cudaStream_t st);
int prepare_project_kernels();
int launch_project_bwd_adam(const ProjectBwdArgs& a, const AdamFusedArgs& opt, int prec, bool aux, cudaStream_t st);
// Units of camera partials a projection-backward launch writes per view
// (deterministic mode): warps of the plain kernel (n_views 0) or blocks of the
// fused kernel over n_views views.
uint64_t cam_partial_units(uint32_t n, int n_views);
// grad_cam[16 v + c] = sum over units u, in unit order, of
// partials[(u * n_views + v) * 16 + c], c < 13 (one block per view).
int launch_cam_reduce(const float* partials, uint64_t units, int n_views, float* grad_cam, cudaStream_t st);
int launch_raster_fwd(const RasterArgs& a, int tile, int prec, int batch, int ppt, bool det, bool persistent,
                      bool color, int grid, cudaStream_t st);
// Counts the raster kernels' work on the last forward (k_raster_work): adds
// {forward hit evaluations, contributing pairs, backward hit evaluations,
// pixels} into out4 (zeroed by the caller).
int launch_raster_work(const RasterArgs& a, int tile, int prec, unsigned long long* out4, cudaStream_t st);
int launch_raster_bwd(const RasterArgs& a, int tile, int prec, bool aux, int ppt, int batch, bool det,
                      bool persistent, int grid, cudaStream_t st);

// ---- sort / scan / binning (gs_sort.cu) ----
// Scratch for the scan and the radix sort; sized by the caller through
// scan_scratch_bytes / sort_scratch_bytes.
constexpr int SCAN_GRID = 512;    // blocks of the chunked scan
constexpr int SORT_GRID = 444;    // blocks of the chunked radix passes (3 per SM, one wave)
size_t scan_scratch_bytes();
size_t sort_scratch_bytes();

// Exclusive scan of n u32 values read as in[perm ? perm[i] : i] (n from
// n_dev when non-null, else n_host). Writes out[i], and the total to
// total_u32 (saturated) / total_u64 when non-null.
int launch_scan(const uint32_t* in, const uint32_t* perm, uint32_t* out, uint64_t n_host, const uint32_t* n_dev,
                uint32_t* total_u32, unsigned long long* total_u64, void* scratch, cudaStream_t st);
// Stable LSD radix sort of (key, val) over bits [0, key_bits). Ping-pongs
// between (k0,v0) and (k1,v1); returns in *result_in_1 where the output is.
// With gather_dst, the final pass also writes gather_dst[i] = gather_src[val]
// for every sorted position i.
int launch_radix_sort(uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1, uint64_t n_host, const uint32_t* n_dev,
                      int key_bits, void* scratch, int* result_in_1, cudaStream_t st,
                      const uint32_t* gather_src = nullptr, uint32_t* gather_dst = nullptr);
// The same sort on interleaved (key, val) pairs, ping-ponging between p0 and p1.
int launch_radix_sort_pairs(uint2* p0, uint2* p1, uint64_t n_host, const uint32_t* n_dev, int key_bits, void* scratch,
                            int* result_in_1, cudaStream_t st, uint2* ranges = nullptr, uint32_t num_ranges = 0,
                            const unsigned long long* base = nullptr);
// With `ranges` (zero-filled, num_ranges entries) the sort's final pass also
// records each key's output range; launch_ranges_fix then converts it to
// [start, end) per key ((0, 0) for absent keys) — the tile ranges without a
// separate pass over the sorted entries. With `base` (device), the sort
// covers elements [*base, *base + n) of both buffers and the recorded ranges
// are positions in the whole buffer.
int launch_ranges_fix(uint2* ranges, uint32_t num_tiles, cudaStream_t st);
// Tile order for the persistent raster kernels: tiles bucketed by the
// logarithm of their work (four buckets per octave; the work is lengths[t]
// when given, else the tile's entry count), heaviest bucket first. Order
// within a bucket is arbitrary; results do not depend on it.
int launch_tile_order(const uint2* ranges, const uint32_t* lengths, uint32_t num_tiles, uint32_t* order,
                      cudaStream_t st);
// dst[i] = src[i].y for i < min(*n, capacity).
int launch_pair_values(const uint2* src, uint32_t* dst, const unsigned long long* n, uint64_t capacity,
                       cudaStream_t st);

struct ExpandArgs {
  const uint32_t* perm;        // depth-sorted item order
  const uint32_t* counts;      // per item
  const uint32_t* sorted_counts;  // counts in sorted order (counts[perm[k]]), or null
  const uint32_t* offsets;     // exclusive scan of counts in sorted order
  const uint4* rects;          // per item
  const ViewInfo* views;       // null for the standalone binner
  uint32_t items_per_view;     // item / items_per_view = view (when views != null)
  uint32_t tiles_x;            // standalone binner grid width
  const uint32_t* n_items_dev; // null: n_items_host
  uint32_t n_items_host;
  const unsigned long long* total;  // entries
  uint64_t capacity;
  uint2* pairs;                // per entry: (tile id relative to the launch's first view, value per val_mode:
                               // 0 item, 1 expansion index, 2 reference entry index)
  int val_mode;
  uint32_t* exp_item;          // val_mode 1: expansion index -> item
  uint32_t* entry_offset;      // item -> first expansion index, or null
  const uint32_t* ref_offsets; // val_mode 2: exclusive scan of counts in item order
  uint32_t* entry_items;       // val_mode 2: reference entry index -> item
  uint32_t* error_word;
};
int launch_expand(const ExpandArgs& a, cudaStream_t st);

// Expansion restricted to some tiles of each item's rect, in the same order
// as launch_expand (items in depth order, a rect's tiles row-major): a tile
// is taken when key_by_item[item] <= cut[tile] (cut != null) or when
// flag[tile] != 0 (flag != null). counts/offsets hold the restricted counts.
// Entries go to pairs[*base + offset] (base null: 0) as (tile, item).
struct ExpandFilterArgs {
  const uint32_t* perm;
  const uint32_t* counts;
  const uint32_t* sorted_counts;  // counts in sorted order, or null
  const uint32_t* offsets;
  const uint4* rects;
  const ViewInfo* views;
  uint32_t items_per_view;
  const uint32_t* n_items_dev;       // null: n_items_host
  uint32_t n_items_host;
  const unsigned long long* total;   // entries of this expansion
  const unsigned long long* base;    // entries already in pairs, or null
  uint64_t capacity;
  uint2* pairs;
  const uint32_t* cut;
  const uint32_t* key_by_item;
  const uint8_t* flag;
  uint32_t* error_word;
};
int launch_expand_filtered(const ExpandFilterArgs& a, cudaStream_t st);
// Completion pass of the occlusion cut. gate_n = *inc_count ? n_items : 0.
int launch_cut_gate(const uint32_t* inc_count, uint32_t n_items, uint32_t* gate_n, cudaStream_t st);
// counts[item] = tiles of rects[item] that are listed (inc_list, *inc_count
// of them; flag[t] set for each). The kernel returns at once when the list
// is empty (the counts are then not read).
int launch_count_flagged(const uint4* rects, const ViewInfo* views, uint32_t n_views, uint32_t items_per_view,
                         uint32_t n_items, const uint32_t* inc_count, const uint32_t* inc_list, const uint8_t* flag,
                         uint32_t* counts, cudaStream_t st);
// When base + total2 exceeds the capacity: flag the entry-capacity error and
// zero total2 and count2.
int launch_entry_guard2(const unsigned long long* base, unsigned long long* total2, uint32_t* count2,
                        uint64_t capacity, uint32_t* error_word, cudaStream_t st);
// ranges[list[i]] = (0, 0) for i < *count.
int launch_ranges_reset_list(const uint32_t* list, const uint32_t* count, uint2* ranges, uint32_t max_list,
                             cudaStream_t st);
// launch_ranges_fix for the listed tiles only, then *entry_total += *total2.
// With gmask, the first skip[i] bytes of listed tile i's summary move from
// gmask[src[i]] to the tile's new start.
int launch_ranges_fix_list(const uint32_t* list, const uint32_t* count, uint2* ranges, uint32_t max_list,
                           unsigned long long* entry_total, const unsigned long long* total2, uint8_t* gmask,
                           const uint32_t* skip, const uint32_t* src, cudaStream_t st);
// ranges[t] = [start, end) of tile t in the sorted pairs (ranges zeroed by the callee).
// mask_off[t] = Σ_{t' < t} ⌈len(t')/32⌉ over the tiles' entry ranges.
int launch_mask_offsets(const uint2* ranges, uint32_t num_tiles, uint32_t* words, uint32_t* mask_off, void* scratch,
                        cudaStream_t st);
int launch_ranges(const uint2* sorted_pairs, const unsigned long long* total, uint64_t capacity, uint2* ranges,
                  uint32_t num_tiles, cudaStream_t st);
// After the entry scan: on overflow flag the error and zero the entry counts.
int launch_entry_guard(unsigned long long* total, uint32_t* count, uint64_t capacity, uint32_t* error_word,
                       cudaStream_t st);
// Number of key bits needed for num_tiles tile ids.
int tile_key_bits(uint32_t num_tiles);
// dst[i] = src[idx[i]] for i < n (device n).
int launch_gather_u32(const uint32_t* src, const uint32_t* idx, uint32_t* dst, const unsigned long long* n,
                      uint64_t capacity, cudaStream_t st);

// ---- loss, optimizer, densify ----
struct SsimArgs {
  const ViewInfo* views;
  int n_views;
  int total_tiles16;          // 16x16 tiles over all views
  const float4* img;
  const float4* target;
  float* coef;                // 9 planes of coef_stride floats (scratch)
  uint64_t coef_stride;       // pixels per plane (the pixel budget)
  float4* dl_dcolor;
  double* loss_sums;          // 2 per view
  float w_l1, w_ssim;
  float w[6];                 // Gaussian window taps 0..5 (set by the launcher)
};
int launch_ssim(const SsimArgs& a, cudaStream_t st);

struct NormalArgs {
  const ViewInfo* views;
  int n_views;
  uint64_t total_px;
  const float4* color;     // alpha in .w
  const float4* aux;       // depth_acc in .y
  const float4* normal;
  float* cp;               // 6 planes of `stride` floats (stencil coefficients)
  uint64_t stride;
  float4* dl_dnormal;
  float4* dl_dcolor;       // .w written
  double* loss;            // per view: Σ α (1 − n̂·N_d)
  float lambda, alpha_min;
};
int launch_normal_loss(const NormalArgs& a, cudaStream_t st);

int launch_adam_grad(const AdamClass& c, const float* grad, uint64_t n, int activation, float beta1, float beta2,
                     float eps, float bc1_inv, float bc2_inv, cudaStream_t st);
int launch_accum_norm(const float4* grad_pos, float* accum, uint32_t n, cudaStream_t st);
int launch_activate_init(const AdamClass& c, uint64_t n, int activation, cudaStream_t st);
int launch_to_half(const float* src, void* dst, uint64_t n, bool bf16, cudaStream_t st);

struct DensifyArgs {
  uint32_t n, capacity;
  float grad_threshold, opacity_threshold;
  float inv_steps;                 // 1 / steps accumulated
  const float* accum;              // per-surfel Σ|dL/dpos|
  const float* opacity_act;
  uint32_t* flags;                 // per surfel: keep (bit0), clone (bit1)
  uint32_t* slots;                 // scan scratch
  // parameter classes to compact: raw, m, v, act, floats per surfel
  float* arrays[20];
  int widths[20];
  int n_arrays;
  float* tmp;                      // capacity * max width staging
  uint32_t* n_out_dev;
};
int launch_densify(DensifyArgs& a, void* scan_scratch, cudaStream_t st);

// ---- MCMC relocation and noise (gs_mcmc.cu) ----
constexpr int MCMC_JUMP_LEVELS = 33;  // powers M^(2^j) of the xorshift64 step, j < 33
struct McmcArgs {
  uint32_t n;
  float dead_threshold, split_ratio;
  const uint64_t* jump;          // MCMC_JUMP_LEVELS × 64 rows
  uint64_t* rng_state;           // device xorshift64 state, advanced by one step per dead surfel
  uint32_t* counters;            // [0] dead [1] relocated [2] split [3] deferred [5] oversized [6] leftover
  unsigned long long* total_weight;
  // per-surfel scratch (capacity entries each)
  uint32_t *dead, *dead_rank, *dead_idx, *owner, *used, *pick, *leftover_flag, *left_rank, *left_idx;
  unsigned long long *weight, *cum;
  uint32_t *size_key, *size_val, *key2, *val2, *over_flag, *over_rank, *over_key, *over_val;
  const uint32_t* sorted_size_key;
  const uint32_t* over_sorted_val;
  // parameters
  const float* opac_act;         // read for sampling
  const float2* scales_act;
  float4* pos_raw; float2* scales_raw; float4* quat_raw; float* opac_raw; float* sh_raw;
  float4* pos_act; float2* scales_act_w; float4* quat_act; float* opac_act_w; float* sh_act;
  void* sh_half;
  float* m[5];
  float* v[5];
};
void mcmc_jump_tables(uint64_t* out);
int launch_mcmc_relocate(McmcArgs& a, int prec, void* scan_scratch, void* sort_scratch, cudaStream_t st);
int launch_mcmc_noise(float4* pos_raw, float4* pos_act, const float2* scales_act, const float* opac_act, uint32_t n,
                      uint32_t seed, float sigma, float opacity_k, cudaStream_t st);

}  // namespace gs
