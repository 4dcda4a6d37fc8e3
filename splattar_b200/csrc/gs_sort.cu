// Prefix scan, stable LSD radix sort and tile binning.
//
// The reference bins with count → scan → expand (item-major) → stable 32-bit
// sort by depth → gather tile keys → stable 32-bit sort by tile → ranges
// (crates/gs-kernels/src/binning.rs:171-238, tile_binning.wgsl:30-103,
// crates/gs-wgpu/src/shaders/radix_sort.wgsl): sixteen 4-bit passes over the
// entries, equivalent to one sort by (tile, depth, entry index).
//
// Here the depth order is established on the ITEMS (one per surfel and view,
// 4 passes of 8 bits over N·V keys), items are expanded in that order, and
// the entries are stably sorted by tile id alone (⌈log2 tiles / 8⌉ passes,
// usually 2). Within one tile each item owns at most one entry and entry
// indices grow with item index, so the result is exactly the reference's
// (tile, depth, entry) order.
//
// All passes read element counts from device memory, so a step needs no host
// synchronisation and can be captured in a CUDA graph. Every block of a
// chunked pass handles a fixed contiguous share of the input; nothing waits
// on another block.
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include "gs_common.cuh"
#include "gs_kernels.h"

namespace gs {
namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ uint64_t read_n(uint64_t n_host, const uint32_t* n_dev) {
  if (n_dev == nullptr) return n_host;
  uint64_t d = *n_dev;
  return d < n_host ? d : n_host;
}

// ------------------------------------------------------------------ scan
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ uint32_t scan_in(const uint32_t* in, const uint32_t* perm, uint64_t i) {
  return perm ? in[perm[i]] : in[i];
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const uint32_t* in, const uint32_t* perm, uint64_t n_host,
                                                              const uint32_t* n_dev, unsigned long long* bsum) {
  const uint64_t n = read_n(n_host, n_dev);
  const uint64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const uint64_t beg = blockIdx.x * chunk, end = min(n, beg + chunk);
  unsigned long long s = 0;
  for (uint64_t i = beg + threadIdx.x; i < end; i += SCAN_THREADS) s += scan_in(in, perm, i);
  using BR = cub::BlockReduce<unsigned long long, SCAN_THREADS>;
  __shared__ typename BR::TempStorage tmp;
  s = BR(tmp).Sum(s);
  if (threadIdx.x == 0) bsum[blockIdx.x] = s;
}

__global__ void __launch_bounds__(SCAN_GRID) k_scan_blocks(unsigned long long* bsum, uint32_t* total_u32,
                                                           unsigned long long* total_u64) {
  using BS = cub::BlockScan<unsigned long long, SCAN_GRID>;
  __shared__ typename BS::TempStorage tmp;
  unsigned long long v = bsum[threadIdx.x], excl, agg;
  BS(tmp).ExclusiveSum(v, excl, agg);
  bsum[threadIdx.x] = excl;
  if (threadIdx.x == 0) {
    if (total_u32) *total_u32 = agg > 0xffffffffull ? 0xffffffffu : (uint32_t)agg;
    if (total_u64) *total_u64 = agg;
  }
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_down(const uint32_t* in, const uint32_t* perm, uint32_t* out,
                                                            uint64_t n_host, const uint32_t* n_dev,
                                                            const unsigned long long* boff) {
  const uint64_t n = read_n(n_host, n_dev);
  const uint64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const uint64_t beg = blockIdx.x * chunk, end = min(n, beg + chunk);
  using BS = cub::BlockScan<uint32_t, SCAN_THREADS>;
  __shared__ typename BS::TempStorage tmp;
  uint32_t running = (uint32_t)boff[blockIdx.x];
  for (uint64_t t0 = beg; t0 < end; t0 += SCAN_TILE) {
    uint32_t v[SCAN_ITEMS];
    uint32_t loc = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
      const uint64_t i = t0 + (uint64_t)threadIdx.x * SCAN_ITEMS + k;
      v[k] = i < end ? scan_in(in, perm, i) : 0u;
      loc += v[k];
    }
    uint32_t excl, agg;
    BS(tmp).ExclusiveSum(loc, excl, agg);
    uint32_t r = running + excl;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
      const uint64_t i = t0 + (uint64_t)threadIdx.x * SCAN_ITEMS + k;
      if (i < end) out[i] = r;
      r += v[k];
    }
    running += agg;
    __syncthreads();
  }
}

// ------------------------------------------------------------ radix sort
// Reduce-then-scan LSD passes of 8-bit digits. Every block owns a contiguous
// chunk of the input and walks it in tiles of RS_TILE elements.
//   upsweep: per-warp digit histograms in shared memory by shared atomics
//     (four independent loads in flight per thread), summed per block;
//   downsweep: warp w holds elements [256w, 256w+256) of the tile in 8 rounds
//     of 32, ranks them stably by ballot multi-split, the block combines the
//     warps' digit counts in warp order, the tile is reordered through shared
//     memory and written out in digit runs. The next tile's elements are
//     loaded while the current one is ranked and written.
// The per-(digit, block) counts are scanned between the two. Elements are
// (key, value) pairs, either in two arrays or interleaved as uint2.
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ROUNDS = 8;                        // elements per thread per tile
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;     // 2048
constexpr int RS_BINS = 256;
static_assert(SORT_GRID % 148 == 0, "whole waves of the downsweep (3 blocks per SM)");

// Lanes of the warp whose digit equals this lane's (multi-split by ballots).
__device__ __forceinline__ uint32_t match_digit(uint32_t d, int nbits, uint32_t active) {
  uint32_t peers = active;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    if (b < nbits) {
      const uint32_t bit = (d >> b) & 1u;
      const uint32_t bal = __ballot_sync(FULL, bit);
      peers &= bit ? bal : ~bal;
    }
  }
  return peers;
}

// Element access: two arrays, or one interleaved uint2 array.
// SplitIO's optional gather (final pass only): gdst[position] = gsrc[value],
// e.g. each item's tile count in sorted order for the entry scan, which then
// reads it sequentially instead of through the permutation.
struct SplitIO {
  const uint32_t* kin; const uint32_t* vin; uint32_t* kout; uint32_t* vout;
  const uint32_t* gsrc = nullptr; uint32_t* gdst = nullptr;
  SplitIO plain() const { SplitIO y = *this; y.gdst = nullptr; return y; }
  __device__ __forceinline__ void skip(uint64_t b) { kin += b; vin += b; kout += b; vout += b; }
  __device__ __forceinline__ uint32_t key(uint64_t i) const { return __ldg(kin + i); }
  __device__ __forceinline__ uint2 load(uint64_t i) const { return make_uint2(__ldg(kin + i), __ldg(vin + i)); }
  __device__ __forceinline__ void store(size_t g, uint2 e) const {
    kout[g] = e.x;
    vout[g] = e.y;
    if (gdst != nullptr) gdst[g] = __ldg(gsrc + e.y);
  }
};
struct PairIO {
  const uint2* in; uint2* out;
  PairIO plain() const { return *this; }
  __device__ __forceinline__ void skip(uint64_t b) { in += b; out += b; }
  __device__ __forceinline__ uint32_t key(uint64_t i) const {
    return __ldg(reinterpret_cast<const uint32_t*>(in + i));
  }
  __device__ __forceinline__ uint2 load(uint64_t i) const { return __ldg(in + i); }
  __device__ __forceinline__ void store(size_t g, uint2 e) const { out[g] = e; }
};

template <class IO>
__global__ void __launch_bounds__(RS_THREADS) k_rs_upsweep(IO io, uint64_t n_host, const uint32_t* n_dev, int shift,
                                                           int nbits, uint32_t* __restrict__ hist,
                                                           const unsigned long long* base) {
  __shared__ uint32_t s_hist[RS_WARPS][RS_BINS];
  if (base != nullptr) io.skip(*base);
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int k = tid; k < RS_WARPS * RS_BINS; k += RS_THREADS) (&s_hist[0][0])[k] = 0;
  __syncthreads();
  const uint64_t n = read_n(n_host, n_dev);
  const uint64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const uint64_t beg = blockIdx.x * chunk, end = min(n, beg + chunk);
  const uint32_t mask = (1u << nbits) - 1u;
  uint32_t* h = s_hist[warp];
  uint64_t i = beg + tid;
  for (; i + 3 * RS_THREADS < end; i += 4 * RS_THREADS) {
    const uint32_t k0 = io.key(i), k1 = io.key(i + RS_THREADS), k2 = io.key(i + 2 * RS_THREADS),
                   k3 = io.key(i + 3 * RS_THREADS);
    atomicAdd(h + ((k0 >> shift) & mask), 1u);
    atomicAdd(h + ((k1 >> shift) & mask), 1u);
    atomicAdd(h + ((k2 >> shift) & mask), 1u);
    atomicAdd(h + ((k3 >> shift) & mask), 1u);
  }
  for (; i < end; i += RS_THREADS) atomicAdd(h + ((io.key(i) >> shift) & mask), 1u);
  __syncthreads();
  for (int dd = tid; dd < RS_BINS; dd += RS_THREADS) {
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) s += s_hist[w][dd];
    hist[(size_t)dd * gridDim.x + blockIdx.x] = s;
  }
}

// ranges (final pass of a key sort only, else null): every run of one key
// inside a staged tile is folded into that key's output range, stored as
// (~first position, one past the last position) with atomicMax on both, so
// the zero-filled buffer needs no other initialisation (launch_ranges_fix
// turns it into [start, end) afterwards). Staged tiles are ordered by the
// full key in the final pass: by this pass's digit, and within a digit by
// the lower digits the earlier passes sorted.
template <class IO>
__global__ void __launch_bounds__(RS_THREADS, 3) k_rs_downsweep(IO io, uint64_t n_host, const uint32_t* n_dev,
                                                                int shift, int nbits,
                                                                const uint32_t* __restrict__ hist,
                                                                uint2* ranges, uint32_t num_ranges,
                                                                const unsigned long long* base) {
  __shared__ uint2 s_e[RS_TILE];
  __shared__ uint32_t s_wh[RS_WARPS][RS_BINS];
  __shared__ uint32_t s_start[RS_BINS], s_gofs[RS_BINS], s_run[RS_BINS];
  using BS = cub::BlockScan<uint32_t, RS_THREADS>;
  __shared__ typename BS::TempStorage tmp;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t n = read_n(n_host, n_dev);
  const uint64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const uint64_t beg = blockIdx.x * chunk, end = min(n, beg + chunk);
  if (beg >= end) return;
  const uint32_t b0 = base != nullptr ? (uint32_t)*base : 0u;  // range positions are whole-buffer positions
  if (b0) io.skip(b0);
  const uint32_t mask = (1u << nbits) - 1u;
  s_run[tid] = hist[(size_t)tid * gridDim.x + blockIdx.x];  // RS_THREADS == RS_BINS
  uint2 e[RS_ROUNDS];
  {
    const int tn = (int)min((uint64_t)RS_TILE, end - beg);
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
      const int idx = warp * (RS_ROUNDS * 32) + r * 32 + lane;
      e[r] = idx < tn ? io.load(beg + idx) : make_uint2(0u, 0u);
    }
  }
  for (uint64_t t0 = beg; t0 < end; t0 += RS_TILE) {
    const int tn = (int)min((uint64_t)RS_TILE, end - t0);
#pragma unroll
    for (int k = tid; k < RS_WARPS * RS_BINS; k += RS_THREADS) (&s_wh[0][0])[k] = 0;
    __syncthreads();
    uint32_t pre[RS_ROUNDS];
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
      const int idx = warp * (RS_ROUNDS * 32) + r * 32 + lane;
      const bool valid = idx < tn;
      const uint32_t d = (e[r].x >> shift) & mask;
      const uint32_t act = __ballot_sync(FULL, valid);
      const uint32_t peers = match_digit(d, nbits, act);
      uint32_t basev = 0;
      if (valid) basev = s_wh[warp][d];
      __syncwarp();
      if (valid && (peers & lanemask_lt()) == 0) s_wh[warp][d] = basev + __popc(peers);
      __syncwarp();
      pre[r] = basev + __popc(peers & lanemask_lt());
    }
    __syncthreads();
    {
      const int d = tid;
      uint32_t s = 0;
#pragma unroll
      for (int w = 0; w < RS_WARPS; ++w) {
        const uint32_t c = s_wh[w][d];
        s_wh[w][d] = s;
        s += c;
      }
      uint32_t excl;
      BS(tmp).ExclusiveSum(s, excl);
      s_start[d] = excl;
      s_gofs[d] = s_run[d] - excl;  // global position = s_gofs[d] + position in the tile
      s_run[d] += s;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
      const int idx = warp * (RS_ROUNDS * 32) + r * 32 + lane;
      if (idx < tn) {
        const uint32_t d = (e[r].x >> shift) & mask;
        s_e[s_start[d] + s_wh[warp][d] + pre[r]] = e[r];
      }
    }
    {  // the next tile's elements are in flight during the write-out
      const uint64_t t1 = t0 + RS_TILE;
      const int tn1 = t1 < end ? (int)min((uint64_t)RS_TILE, end - t1) : 0;
#pragma unroll
      for (int r = 0; r < RS_ROUNDS; ++r) {
        const int idx = warp * (RS_ROUNDS * 32) + r * 32 + lane;
        e[r] = idx < tn1 ? io.load(t1 + idx) : make_uint2(0u, 0u);
      }
    }
    __syncthreads();
#pragma unroll 4
    for (int i = tid; i < tn; i += RS_THREADS) {
      const uint2 v = s_e[i];
      const uint32_t pos = s_gofs[(v.x >> shift) & mask] + (uint32_t)i;
      io.store((size_t)pos, v);
      if (ranges != nullptr && v.x < num_ranges) {
        if (i == 0 || s_e[i - 1].x != v.x) atomicMax(&ranges[v.x].x, ~(b0 + pos));
        if (i == tn - 1 || s_e[i + 1].x != v.x) atomicMax(&ranges[v.x].y, b0 + pos + 1u);
      }
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------- binning
__global__ void __launch_bounds__(256) k_expand(ExpandArgs a) {
  const uint64_t n = read_n(a.n_items_host, a.n_items_dev);
  const uint64_t tot = *a.total;  // zeroed by the entry guard on overflow
  if (tot == 0 || tot > a.capacity) return;
  const int lane = threadIdx.x & 31;
  const uint64_t warps_total = (uint64_t)gridDim.x * (blockDim.x / 32);
  for (uint64_t w = (uint64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); w * 32 < n; w += warps_total) {
    const uint64_t k0 = w * 32, k = k0 + lane;
    const bool valid = k < n;
    uint32_t item = 0, cnt = 0, x0 = 0, y0 = 0, wd = 1, tb = 0, tx = a.tiles_x;
    if (valid) {
      item = a.perm[k];
      cnt = a.sorted_counts != nullptr ? a.sorted_counts[k] : a.counts[item];
      if (cnt) {
        const uint4 r = a.rects[item];
        x0 = r.x; y0 = r.y; wd = r.z - r.x + 1u;
      }
      if (a.views) {
        const ViewInfo* V = a.views + item / a.items_per_view;
        tb = (uint32_t)__ldg(&V->tile_base);
        tx = (uint32_t)__ldg(&V->tiles_x);
      }
    }
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += t;
    }
    const uint32_t excl = incl - cnt;
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    const uint32_t off0 = a.offsets[k0];
    if ((uint64_t)off0 + total > a.capacity) {
      if (lane == 0 && total) atomicOr(a.error_word, ERR_ENTRY_CAPACITY);
      continue;
    }
    if (valid && a.entry_offset) a.entry_offset[item] = off0 + excl;
    for (uint32_t base = 0; base < total; base += 32) {
      const uint32_t j = base + lane;
      int owner = 0;
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) {
        const int c = owner + s;
        const uint32_t ec = __shfl_sync(FULL, excl, c < 32 ? c : 31);
        if (c < 32 && ec <= j) owner = c;
      }
      const uint32_t o_excl = __shfl_sync(FULL, excl, owner);
      const uint32_t o_wd = __shfl_sync(FULL, wd, owner);
      const uint32_t o_x0 = __shfl_sync(FULL, x0, owner);
      const uint32_t o_y0 = __shfl_sync(FULL, y0, owner);
      const uint32_t o_item = __shfl_sync(FULL, item, owner);
      const uint32_t o_tb = __shfl_sync(FULL, tb, owner);
      const uint32_t o_tx = __shfl_sync(FULL, tx, owner);
      if (j < total) {
        const uint32_t local = j - o_excl;
        const uint32_t ly = local / o_wd, lx = local - ly * o_wd;
        const uint32_t pos = off0 + j;
        const uint32_t key = o_tb + (o_y0 + ly) * o_tx + (o_x0 + lx);
        uint32_t val = o_item;
        if (a.val_mode == 1) {
          val = pos;
          a.exp_item[pos] = o_item;
        } else if (a.val_mode == 2) {
          val = a.ref_offsets[o_item] + local;
          if (val < tot) a.entry_items[val] = o_item;
        }
        a.pairs[pos] = make_uint2(key, val);
      }
    }
  }
}

// Filtered expansion (occlusion cut and its completion pass): the warp walks
// the candidate tiles of its 32 items' rects in launch_expand's order and
// keeps those the filter accepts, compacted by ballot, so each item's kept
// tiles land at its restricted offset in rect order.
__global__ void __launch_bounds__(256) k_expand_filtered(ExpandFilterArgs a) {
  const uint64_t n = read_n(a.n_items_host, a.n_items_dev);
  const uint64_t tot = *a.total;
  const uint64_t b = a.base != nullptr ? *a.base : 0ull;
  if (tot == 0 || b + tot > a.capacity) return;
  const int lane = threadIdx.x & 31;
  const uint64_t warps_total = (uint64_t)gridDim.x * (blockDim.x / 32);
  for (uint64_t w = (uint64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); w * 32 < n; w += warps_total) {
    const uint64_t k0 = w * 32, k = k0 + lane;
    uint32_t item = 0, cnt = 0, full = 0, x0 = 0, y0 = 0, wd = 1, tb = 0, tx = 0, key = 0;
    if (k < n) {
      item = a.perm[k];
      cnt = a.sorted_counts != nullptr ? a.sorted_counts[k] : a.counts[item];
      if (cnt) {
        const uint4 r = a.rects[item];
        x0 = r.x; y0 = r.y; wd = r.z - r.x + 1u;
        full = wd * (r.w - r.y + 1u);
        const ViewInfo* V = a.views + item / a.items_per_view;
        tb = (uint32_t)__ldg(&V->tile_base);
        tx = (uint32_t)__ldg(&V->tiles_x);
        if (a.cut != nullptr) key = a.key_by_item[item];
      }
    }
    uint32_t incl = full, incl_c = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(FULL, incl, o), tc = __shfl_up_sync(FULL, incl_c, o);
      if (lane >= o) { incl += t; incl_c += tc; }
    }
    const uint32_t excl = incl - full;
    const uint32_t total_full = __shfl_sync(FULL, incl, 31), total_cnt = __shfl_sync(FULL, incl_c, 31);
    if (total_cnt == 0) continue;
    const uint32_t off0 = a.offsets[k0];
    if ((uint64_t)off0 + total_cnt > tot) {
      if (lane == 0) atomicOr(a.error_word, ERR_ENTRY_CAPACITY);
      continue;
    }
    uint32_t run = 0;
    for (uint32_t basej = 0; basej < total_full; basej += 32) {
      const uint32_t j = basej + lane;
      int owner = 0;
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) {
        const int c = owner + s;
        const uint32_t ec = __shfl_sync(FULL, excl, c < 32 ? c : 31);
        if (c < 32 && ec <= j) owner = c;
      }
      const uint32_t o_excl = __shfl_sync(FULL, excl, owner);
      const uint32_t o_wd = __shfl_sync(FULL, wd, owner);
      const uint32_t o_x0 = __shfl_sync(FULL, x0, owner);
      const uint32_t o_y0 = __shfl_sync(FULL, y0, owner);
      const uint32_t o_item = __shfl_sync(FULL, item, owner);
      const uint32_t o_tb = __shfl_sync(FULL, tb, owner);
      const uint32_t o_tx = __shfl_sync(FULL, tx, owner);
      const uint32_t o_key = __shfl_sync(FULL, key, owner);
      bool take = false;
      uint32_t tile = 0;
      if (j < total_full) {
        const uint32_t local = j - o_excl;
        const uint32_t ly = local / o_wd, lx = local - ly * o_wd;
        tile = o_tb + (o_y0 + ly) * o_tx + (o_x0 + lx);
        take = a.cut != nullptr ? o_key <= __ldg(a.cut + tile) : __ldg(a.flag + tile) != 0;
      }
      const uint32_t bal = __ballot_sync(FULL, take);
      if (take) {
        const uint32_t slot = run + __popc(bal & lanemask_lt());
        if (slot < total_cnt) a.pairs[b + off0 + slot] = make_uint2(tile, o_item);
        else atomicOr(a.error_word, ERR_ENTRY_CAPACITY);  // counts disagree with the filter: never written past them
      }
      run += __popc(bal);
    }
  }
}

__global__ void k_cut_gate(const uint32_t* inc_count, uint32_t n_items, uint32_t* gate_n) {
  *gate_n = *inc_count ? n_items : 0u;
}

// Listed tiles are held in shared memory as (view, x, y) when there are few
// of them; each item then checks its rect against the list instead of
// reading the flags of every tile in the rect.
constexpr int FLAG_LIST_SMEM = 512;
__global__ void __launch_bounds__(256) k_count_flagged(const uint4* rects, const ViewInfo* views, uint32_t nv,
                                                       uint32_t ipv, uint32_t n, const uint32_t* inc_count,
                                                       const uint32_t* inc_list, const uint8_t* flag,
                                                       uint32_t* counts) {
  const uint32_t m = *inc_count;
  if (m == 0) return;
  __shared__ uint32_t s_v[FLAG_LIST_SMEM], s_x[FLAG_LIST_SMEM], s_y[FLAG_LIST_SMEM];
  const bool listed = m <= (uint32_t)FLAG_LIST_SMEM;
  if (listed) {
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
      const uint32_t t = inc_list[i];
      uint32_t v = 0;
      while (v + 1 < nv && t >= (uint32_t)__ldg(&views[v + 1].tile_base)) ++v;
      const uint32_t lt = t - (uint32_t)__ldg(&views[v].tile_base), tx = (uint32_t)__ldg(&views[v].tiles_x);
      s_v[i] = v; s_y[i] = lt / tx; s_x[i] = lt - (lt / tx) * tx;
    }
    __syncthreads();
  }
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint4 r = rects[i];
    uint32_t c = 0;
    if (r.z >= r.x && r.w >= r.y) {
      const uint32_t v = i / ipv;
      if (listed) {
        for (uint32_t k = 0; k < m; ++k)
          c += (s_v[k] == v && s_x[k] >= r.x && s_x[k] <= r.z && s_y[k] >= r.y && s_y[k] <= r.w) ? 1u : 0u;
      } else {
        const ViewInfo* V = views + v;
        const uint32_t tb = (uint32_t)__ldg(&V->tile_base), tx = (uint32_t)__ldg(&V->tiles_x);
        for (uint32_t y = r.y; y <= r.w; ++y)
          for (uint32_t x = r.x; x <= r.z; ++x) c += __ldg(flag + tb + y * tx + x) != 0 ? 1u : 0u;
      }
    }
    counts[i] = c;
  }
}

__global__ void k_entry_guard2(const unsigned long long* base, unsigned long long* total2, uint32_t* count2,
                               uint64_t capacity, uint32_t* error_word) {
  if (*base + *total2 > capacity) {
    atomicOr(error_word, ERR_ENTRY_CAPACITY);
    *total2 = 0;
    *count2 = 0;
  }
}

__global__ void __launch_bounds__(256) k_ranges_reset_list(const uint32_t* list, const uint32_t* count, uint2* ranges,
                                                           uint32_t max_list) {
  const uint32_t m = min(*count, max_list);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    ranges[list[i]] = make_uint2(0u, 0u);
}

// One block per listed tile: the range recorded by the completion sort
// becomes [start, end), and the row-group summary of the first skip[i]
// entries (those pass 1 composited) moves from src[i] to the new start.
__global__ void __launch_bounds__(256) k_ranges_fix_list(const uint32_t* list, const uint32_t* count, uint2* ranges,
                                                         uint32_t max_list, unsigned long long* entry_total,
                                                         const unsigned long long* total2, uint8_t* gmask,
                                                         const uint32_t* skip, const uint32_t* src) {
  const uint32_t m = min(*count, max_list);
  for (uint32_t i = blockIdx.x; i < m; i += gridDim.x) {
    const uint32_t t = list[i];
    const uint2 r = ranges[t];
    __syncthreads();  // every thread holds the recorded range before it is replaced
    const uint2 f = r.y ? make_uint2(~r.x, r.y) : make_uint2(0u, 0u);
    if (threadIdx.x == 0) ranges[t] = f;
    if (gmask != nullptr) {
      const uint32_t sk = skip[i], from = src[i];
      if (f.y - f.x >= sk)
        for (uint32_t j = threadIdx.x; j < sk; j += blockDim.x) gmask[f.x + j] = gmask[from + j];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *entry_total += *total2;
}

__global__ void __launch_bounds__(256) k_ranges(const uint2* pairs, const unsigned long long* total,
                                                uint64_t capacity, uint2* ranges, uint32_t num_tiles) {
  const uint64_t n = min((uint64_t)*total, capacity);
  const uint32_t* keys = reinterpret_cast<const uint32_t*>(pairs);  // key of pair p at 2p
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t t = __ldg(keys + 2 * p);
    if (t >= num_tiles) continue;
    if (p == 0 || __ldg(keys + 2 * (p - 1)) != t) ranges[t].x = (uint32_t)p;
    if (p == n - 1 || __ldg(keys + 2 * (p + 1)) != t) ranges[t].y = (uint32_t)(p + 1);
  }
}

__global__ void __launch_bounds__(256) k_pair_values(const uint2* src, uint32_t* dst, const unsigned long long* total,
                                                     uint64_t capacity) {
  const uint64_t n = min((uint64_t)*total, capacity);
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x)
    dst[p] = src[p].y;
}

// Entry-capacity guard, run right after the entry scan: when the scene needs
// more entries than were allocated, flag GS_ERR_CAPACITY and set the entry
// count to zero so no later pass reads an entry that was never written.
__global__ void k_entry_guard(unsigned long long* total, uint32_t* count, uint64_t capacity, uint32_t* error_word) {
  if (*total > capacity) {
    atomicOr(error_word, ERR_ENTRY_CAPACITY);
    *total = 0;
    *count = 0;
  }
}

__global__ void __launch_bounds__(256) k_gather(const uint32_t* src, const uint32_t* idx, uint32_t* dst,
                                                const unsigned long long* total, uint64_t capacity) {
  const uint64_t n = min((uint64_t)*total, capacity);
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x)
    dst[p] = src[idx[p]];
}

// Standalone binner: tiles per rect (tile_binning.wgsl:30-43), depth keys and
// the identity permutation for the item sort.
__global__ void __launch_bounds__(256) k_rect_counts(const uint4* rects, const uint32_t* depths, uint32_t n,
                                                     uint32_t* counts, uint32_t* keys, uint32_t* vals) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint4 r = rects[i];
    counts[i] = (r.z >= r.x && r.w >= r.y) ? (r.z - r.x + 1u) * (r.w - r.y + 1u) : 0u;
    keys[i] = depths[i];
    vals[i] = i;
  }
}

int grid_for(uint64_t n_max, int per_block, int cap_blocks) {
  uint64_t g = (n_max + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > (uint64_t)cap_blocks) g = cap_blocks;
  return (int)g;
}

}  // namespace

size_t scan_scratch_bytes() { return sizeof(unsigned long long) * SCAN_GRID; }
size_t sort_scratch_bytes() { return sizeof(uint32_t) * RS_BINS * SORT_GRID + scan_scratch_bytes(); }

int launch_scan(const uint32_t* in, const uint32_t* perm, uint32_t* out, uint64_t n_host, const uint32_t* n_dev,
                uint32_t* total_u32, unsigned long long* total_u64, void* scratch, cudaStream_t st) {
  auto* bsum = reinterpret_cast<unsigned long long*>(scratch);
  k_scan_reduce<<<SCAN_GRID, SCAN_THREADS, 0, st>>>(in, perm, n_host, n_dev, bsum);
  k_scan_blocks<<<1, SCAN_GRID, 0, st>>>(bsum, total_u32, total_u64);
  k_scan_down<<<SCAN_GRID, SCAN_THREADS, 0, st>>>(in, perm, out, n_host, n_dev, bsum);
  return (int)cudaGetLastError();
}

template <class IO, class SWAP>
int radix_passes(IO io, uint64_t n_host, const uint32_t* n_dev, int key_bits, void* scratch, int* result_in_1,
                 cudaStream_t st, SWAP swap, uint2* ranges = nullptr, uint32_t num_ranges = 0,
                 const unsigned long long* base = nullptr) {
  auto* hist = reinterpret_cast<uint32_t*>(scratch);
  int in1 = 0;
  for (int shift = 0; shift < key_bits; shift += 8) {
    const int nbits = key_bits - shift < 8 ? key_bits - shift : 8;
    k_rs_upsweep<IO><<<SORT_GRID, RS_THREADS, 0, st>>>(io, n_host, n_dev, shift, nbits, hist, base);
    const int e = launch_scan(hist, nullptr, hist, (uint64_t)RS_BINS * SORT_GRID, nullptr, nullptr, nullptr,
                              hist + RS_BINS * SORT_GRID, st);
    if (e) return e;
    const bool last = shift + 8 >= key_bits;
    k_rs_downsweep<IO><<<SORT_GRID, RS_THREADS, 0, st>>>(last ? io : io.plain(), n_host, n_dev, shift, nbits, hist,
                                                         last ? ranges : nullptr, num_ranges, base);
    swap(io);
    in1 ^= 1;
  }
  *result_in_1 = in1;
  return (int)cudaGetLastError();
}

int launch_radix_sort(uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1, uint64_t n_host, const uint32_t* n_dev,
                      int key_bits, void* scratch, int* result_in_1, cudaStream_t st, const uint32_t* gather_src,
                      uint32_t* gather_dst) {
  SplitIO io{k0, v0, k1, v1, gather_src, gather_dst};
  return radix_passes(io, n_host, n_dev, key_bits, scratch, result_in_1, st, [](SplitIO& x) {
    SplitIO y{x.kout, x.vout, const_cast<uint32_t*>(x.kin), const_cast<uint32_t*>(x.vin), x.gsrc, x.gdst};
    x = y;
  });
}

int launch_radix_sort_pairs(uint2* p0, uint2* p1, uint64_t n_host, const uint32_t* n_dev, int key_bits, void* scratch,
                            int* result_in_1, cudaStream_t st, uint2* ranges, uint32_t num_ranges,
                            const unsigned long long* base) {
  PairIO io{p0, p1};
  return radix_passes(
      io, n_host, n_dev, key_bits, scratch, result_in_1, st,
      [](PairIO& x) {
        PairIO y{x.out, const_cast<uint2*>(x.in)};
        x = y;
      },
      ranges, num_ranges, base);
}

int launch_expand(const ExpandArgs& a, cudaStream_t st) {
  const int grid = grid_for((uint64_t)a.n_items_host, 256, 148 * 16);
  k_expand<<<grid, 256, 0, st>>>(a);
  return (int)cudaGetLastError();
}

int launch_expand_filtered(const ExpandFilterArgs& a, cudaStream_t st) {
  const int grid = grid_for((uint64_t)a.n_items_host, 256, 148 * 16);
  k_expand_filtered<<<grid, 256, 0, st>>>(a);
  return (int)cudaGetLastError();
}

int launch_cut_gate(const uint32_t* inc_count, uint32_t n_items, uint32_t* gate_n, cudaStream_t st) {
  k_cut_gate<<<1, 1, 0, st>>>(inc_count, n_items, gate_n);
  return (int)cudaGetLastError();
}

int launch_count_flagged(const uint4* rects, const ViewInfo* views, uint32_t n_views, uint32_t items_per_view,
                         uint32_t n_items, const uint32_t* inc_count, const uint32_t* inc_list, const uint8_t* flag,
                         uint32_t* counts, cudaStream_t st) {
  if (n_items == 0) return 0;
  k_count_flagged<<<grid_for(n_items, 256, 148 * 4), 256, 0, st>>>(rects, views, n_views, items_per_view, n_items,
                                                                    inc_count, inc_list, flag, counts);
  return (int)cudaGetLastError();
}

int launch_entry_guard2(const unsigned long long* base, unsigned long long* total2, uint32_t* count2,
                        uint64_t capacity, uint32_t* error_word, cudaStream_t st) {
  k_entry_guard2<<<1, 1, 0, st>>>(base, total2, count2, capacity, error_word);
  return (int)cudaGetLastError();
}

int launch_ranges_reset_list(const uint32_t* list, const uint32_t* count, uint2* ranges, uint32_t max_list,
                             cudaStream_t st) {
  if (max_list == 0) return 0;
  k_ranges_reset_list<<<grid_for(max_list, 256, 148), 256, 0, st>>>(list, count, ranges, max_list);
  return (int)cudaGetLastError();
}

int launch_ranges_fix_list(const uint32_t* list, const uint32_t* count, uint2* ranges, uint32_t max_list,
                           unsigned long long* entry_total, const unsigned long long* total2, uint8_t* gmask,
                           const uint32_t* skip, const uint32_t* src, cudaStream_t st) {
  k_ranges_fix_list<<<148, 256, 0, st>>>(list, count, ranges, max_list, entry_total, total2, gmask, skip, src);
  return (int)cudaGetLastError();
}

int launch_ranges(const uint2* sorted_pairs, const unsigned long long* total, uint64_t capacity, uint2* ranges,
                  uint32_t num_tiles, cudaStream_t st) {
  cudaMemsetAsync(ranges, 0, sizeof(uint2) * (size_t)num_tiles, st);
  k_ranges<<<148 * 8, 256, 0, st>>>(sorted_pairs, total, capacity, ranges, num_tiles);
  return (int)cudaGetLastError();
}

namespace {
// (~first, end) from the final sort pass → [first, end); (0, 0) for a key no
// element carried.
__global__ void __launch_bounds__(256) k_ranges_fix(uint2* ranges, uint32_t num_tiles) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < num_tiles; t += gridDim.x * blockDim.x) {
    const uint2 r = ranges[t];
    ranges[t] = r.y ? make_uint2(~r.x, r.y) : make_uint2(0u, 0u);
  }
}

__global__ void __launch_bounds__(256) k_tile_words(const uint2* ranges, uint32_t num_tiles, uint32_t* words) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < num_tiles; t += gridDim.x * blockDim.x) {
    const uint2 r = ranges[t];
    words[t] = r.y > r.x ? (r.y - r.x + 31u) / 32u : 0u;
  }
}
}  // namespace

int launch_ranges_fix(uint2* ranges, uint32_t num_tiles, cudaStream_t st) {
  if (num_tiles == 0) return 0;
  k_ranges_fix<<<grid_for(num_tiles, 256, 148 * 8), 256, 0, st>>>(ranges, num_tiles);
  return (int)cudaGetLastError();
}

namespace {
// Bucket of a work amount w: 4·⌊log2(w + 1)⌋ plus the two bits below the
// leading one, so four buckets per octave (0..127).
__device__ __forceinline__ uint32_t work_bucket(uint32_t w) {
  const uint32_t x = w + 1u > w ? w + 1u : w;
  const int e = 31 - __clz(x);
  const uint32_t frac = e >= 2 ? (x >> (e - 2)) & 3u : (x << (2 - e)) & 3u;
  return 4u * (uint32_t)e + frac;
}

__global__ void __launch_bounds__(1024) k_tile_order(const uint2* ranges, const uint32_t* lengths, uint32_t num_tiles,
                                                     uint32_t* order) {
  constexpr int NB = 128;
  __shared__ uint32_t s_cnt[NB];
  const int tid = threadIdx.x;
  if (tid < NB) s_cnt[tid] = 0u;
  __syncthreads();
  auto work = [&](uint32_t t) {
    if (lengths) return lengths[t];
    const uint2 r = ranges[t];
    return r.y - r.x;
  };
  for (uint32_t t = tid; t < num_tiles; t += blockDim.x) atomicAdd(&s_cnt[work_bucket(work(t))], 1u);
  __syncthreads();
  if (tid == 0) {  // exclusive offsets, heaviest bucket first
    uint32_t run = 0;
    for (int b = NB - 1; b >= 0; --b) {
      const uint32_t c = s_cnt[b];
      s_cnt[b] = run;
      run += c;
    }
  }
  __syncthreads();
  for (uint32_t t = tid; t < num_tiles; t += blockDim.x) order[atomicAdd(&s_cnt[work_bucket(work(t))], 1u)] = t;
}
}  // namespace

int launch_tile_order(const uint2* ranges, const uint32_t* lengths, uint32_t num_tiles, uint32_t* order,
                      cudaStream_t st) {
  if (num_tiles == 0) return 0;
  k_tile_order<<<1, 1024, 0, st>>>(ranges, lengths, num_tiles, order);
  return (int)cudaGetLastError();
}

int launch_mask_offsets(const uint2* ranges, uint32_t num_tiles, uint32_t* words, uint32_t* mask_off, void* scratch,
                        cudaStream_t st) {
  if (num_tiles == 0) return 0;
  k_tile_words<<<grid_for(num_tiles, 256, 148 * 8), 256, 0, st>>>(ranges, num_tiles, words);
  return launch_scan(words, nullptr, mask_off, num_tiles, nullptr, nullptr, nullptr, scratch, st);
}

int launch_pair_values(const uint2* src, uint32_t* dst, const unsigned long long* n, uint64_t capacity,
                       cudaStream_t st) {
  k_pair_values<<<148 * 8, 256, 0, st>>>(src, dst, n, capacity);
  return (int)cudaGetLastError();
}

int launch_entry_guard(unsigned long long* total, uint32_t* count, uint64_t capacity, uint32_t* error_word,
                       cudaStream_t st) {
  k_entry_guard<<<1, 1, 0, st>>>(total, count, capacity, error_word);
  return (int)cudaGetLastError();
}

int launch_gather_u32(const uint32_t* src, const uint32_t* idx, uint32_t* dst, const unsigned long long* n,
                      uint64_t capacity, cudaStream_t st) {
  k_gather<<<148 * 8, 256, 0, st>>>(src, idx, dst, n, capacity);
  return (int)cudaGetLastError();
}

int launch_rect_counts(const uint4* rects, const uint32_t* depths, uint32_t n, uint32_t* counts, uint32_t* keys,
                       uint32_t* vals, cudaStream_t st) {
  if (n == 0) return 0;
  k_rect_counts<<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(rects, depths, n, counts, keys, vals);
  return (int)cudaGetLastError();
}

int tile_key_bits(uint32_t num_tiles) {
  int b = 1;
  while (b < 32 && (1ull << b) < (unsigned long long)num_tiles) ++b;
  return b;
}

}  // namespace gs
