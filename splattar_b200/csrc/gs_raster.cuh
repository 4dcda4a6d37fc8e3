// Tile rasterizers: forward front-to-back compositing and its adjoint,
// templated on the tile edge TS (8, 16 or 32 pixels; the reference uses 16,
// crates/gs-kernels/src/rasterizer.rs:13). Each tile size is instantiated in
// its own translation unit (gs_raster.cu, gs_raster_t8.cu, gs_raster_t32.cu).
//
// Forward: crates/gs-kernels/src/shaders/rasterize_fwd.wgsl:20-85 with the hit
// test of raster_common.wgsl:69-95. One CTA per TS×TS tile, PPT pixels per
// thread; the tile's depth-sorted entries are staged in shared
// memory in batches and composited front to back in FP32. Beyond the
// reference:
//   * the whole CTA stops as soon as every pixel has terminated
//     (__syncthreads_count);
//   * while a batch is staged, entries whose α-box (the projection's
//     conservative pixel box of α ≥ 1/255) misses the tile are dropped and
//     the rest compacted, each keeping its original list position, and a
//     pixel outside an entry's box skips it — exact, because such entries
//     cannot reach the 1/255 threshold there;
//   * the ray–splat intersection is evaluated from the precomputed record
//     (three 3-term dot products, one reciprocal, one exp):
//     ĝ = max(G_ray, G_screen) = exp(−min(q_ray, q_screen)).
//
// Backward: rasterize_bwd.wgsl:113-312. Each pixel walks its contributors in
// reverse from the stored final transmittance and last-contributor index,
// recovering T_before = T/(1−α), with suffix sums for colour (and depth,
// normal and depth distortion when aux losses are on). Per-entry gradients
// are taken with respect to the record fields (M, Bu, Bv, tn, px, py, colour,
// opacity, …) and reduced across the warp by a 16-lane transpose reduction,
// then (CTAs of several warps) across the warps in a fixed order, then either
// added to the per-surfel accumulator with one vector reduction per 4
// components (default) or stored per entry for an ordered reduction
// (deterministic mode).
#pragma once

#include <type_traits>

#include "gs_common.cuh"
#include "gs_kernels.h"

namespace gs {
namespace {

constexpr unsigned FULL = 0xffffffffu;

struct Hit {
  float ghat, u, v, t, inv_det, q2, dy;
  bool ray;
};

// Approximate reciprocal (MUFU, ≤ 1 ulp): the only reciprocal either kernel
// uses, so forward and backward stay bit-consistent.
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// A staged record's centre as offsets from the tile's first pixel centre
// (bx0, by0): r1.w = (bx0 − px_hi) − px_lo, r2.w = (by0 − py_hi) − py_lo, done
// once per staged entry. A pixel k columns and l rows into the tile then has
// dx = r1.w + k and dy = r2.w + l: one add each, computed the same way by
// every kernel, so forward and backward evaluate bit-identical hits.
__device__ __forceinline__ void stage_offsets(float4& r1, float4& r2, float bx0, float by0) {
  r1.w = __fsub_rn(__fsub_rn(bx0, r1.w), r1.z);
  r2.w = __fsub_rn(__fsub_rn(by0, r2.w), r2.z);
}

// The part of the hit test that depends on the pixel column only: a thread's
// pixels share sx and dx, so det, u·det and v·det are one FMA per pixel from
// these partial sums, and the screen-space distance needs dy alone. kx is the
// pixel's column within the tile (records staged with stage_offsets).
struct ColPart {
  float det0, un0, vn0, dx, dx2;
};
__device__ __forceinline__ ColPart col_part(const float4& r0, const float4& r1, const float4& r2, float sx,
                                            float kx) {
  ColPart c;
  c.det0 = fmaf(r0.x, sx, r0.z);
  c.dx = __fadd_rn(r1.w, kx);
  c.un0 = __fmul_rn(r1.x, c.dx);
  c.vn0 = __fmul_rn(r2.x, c.dx);
  c.dx2 = __fmul_rn(c.dx, c.dx);
  return c;
}

// raster_common.wgsl:69-95 on the record parameterisation, branch-free.
// Written with explicit rounding intrinsics so the forward and backward
// kernels compute bit-identical alphas. When the ray branch is unavailable
// (|det| ≤ 1e-12 or t ≤ near) q_ray is +inf and u, v, t are unused.
// q2 = u² + v² (= 2·q_ray) is kept for the backward.
// Fast forms, decided per staged entry and tile, with the same α, skip
// decision and branch for every pixel that takes the entry as the full test:
//   RAY_OK (1): the entry's ray branch is available at every pixel of the
//     tile (ray_available), so the per-pixel ray test is left out;
//   RAY_FAR (2): besides, its screen-space low-pass disc stays away from the
//     tile (screen_far), so q_screen is left out too: where q_screen < q_ray,
//     q_screen > ln(255·o) + 0.05 already puts α below 1/255.
constexpr int HIT_FULL = 0, HIT_RAY_OK = 1, HIT_RAY_FAR = 2;
template <int FAST = HIT_FULL>
__device__ __forceinline__ Hit eval_hit(const ColPart& c, const float4& r0, const float4& r1, const float4& r2,
                                        float depth, float sy, float ky) {
  Hit h;
  const float det = fmaf(r0.y, sy, c.det0);
  const float inv = rcp_approx(det);
  h.dy = __fadd_rn(r2.w, ky);
  // (u·det, v·det) and (u, v) as packed pairs, rounding per component as fmaf / __fmul_rn.
  const float2 uvn = __ffma2_rn(make_float2(r1.y, r2.y), make_float2(h.dy, h.dy), make_float2(c.un0, c.vn0));
  const float2 uv = __fmul2_rn(uvn, make_float2(inv, inv));
  const float u = uv.x, v = uv.y;
  const float t = __fmul_rn(r0.w, inv);
  if constexpr (FAST == HIT_RAY_FAR) {
    h.q2 = fmaf(u, u, __fmul_rn(v, v));
    h.ray = true;
    h.u = u; h.v = v; h.inv_det = inv;
    h.t = t;
    h.ghat = __expf(-__fmul_rn(0.5f, h.q2));
    return h;
  }
  const bool ray_ok = FAST == HIT_RAY_OK || (fabsf(det) > 1e-12f && t > NEAR_DEPTH);
  h.q2 = fmaf(u, u, __fmul_rn(v, v));
  const float qr = ray_ok ? __fmul_rn(0.5f, h.q2) : __int_as_float(0x7f800000);
  const float qs = fmaf(h.dy, h.dy, c.dx2);  // (dx²+dy²)/(2σ²) with σ² = 0.5
  h.ray = qr <= qs;
  const float q = fminf(qr, qs);  // = ray ? qr : qs (neither is NaN; equal values are the same value)
  h.u = u; h.v = v; h.inv_det = inv;
  h.t = h.ray ? t : depth;
  h.ghat = __expf(-q);
  return h;
}

// eval_hit for two pixels of one column (rows with sy.x, sy.y) with the
// packed two-wide FP32 instructions of sm_100 (FFMA2/FMUL2/FADD2): every
// product and sum of the hit test takes one instruction for both pixels.
// Each component rounds exactly as the scalar operation of eval_hit, so
// either form gives bit-identical results for a pixel.
template <int FAST = HIT_FULL>
__device__ __forceinline__ void eval_hit2(const ColPart& c, const float4& r0, const float4& r1, const float4& r2,
                                          float depth, float2 sy, float2 ky, Hit& ha, Hit& hb) {
  const float2 det = __ffma2_rn(make_float2(r0.y, r0.y), sy, make_float2(c.det0, c.det0));
  const float2 inv = make_float2(rcp_approx(det.x), rcp_approx(det.y));
  const float2 dy = __fadd2_rn(make_float2(r2.w, r2.w), ky);  // as eval_hit's __fadd_rn, per component
  const float2 un = __ffma2_rn(make_float2(r1.y, r1.y), dy, make_float2(c.un0, c.un0));
  const float2 vn = __ffma2_rn(make_float2(r2.y, r2.y), dy, make_float2(c.vn0, c.vn0));
  const float2 u = __fmul2_rn(un, inv), v = __fmul2_rn(vn, inv);
  const float2 t = __fmul2_rn(make_float2(r0.w, r0.w), inv);
  const float2 q2 = __ffma2_rn(u, u, __fmul2_rn(v, v));
  const float2 qr0 = __fmul2_rn(make_float2(0.5f, 0.5f), q2);
  if constexpr (FAST == HIT_RAY_FAR) {  // as eval_hit
    ha.ray = hb.ray = true;
    ha.u = u.x; ha.v = v.x; ha.inv_det = inv.x; ha.q2 = q2.x; ha.dy = dy.x; ha.t = t.x;
    hb.u = u.y; hb.v = v.y; hb.inv_det = inv.y; hb.q2 = q2.y; hb.dy = dy.y; hb.t = t.y;
    ha.ghat = __expf(-qr0.x);
    hb.ghat = __expf(-qr0.y);
    return;
  }
  const float2 qs = __ffma2_rn(dy, dy, make_float2(c.dx2, c.dx2));
  const float inf = __int_as_float(0x7f800000);
  const float qra = FAST == HIT_RAY_OK || (fabsf(det.x) > 1e-12f && t.x > NEAR_DEPTH) ? qr0.x : inf;
  const float qrb = FAST == HIT_RAY_OK || (fabsf(det.y) > 1e-12f && t.y > NEAR_DEPTH) ? qr0.y : inf;
  ha.ray = qra <= qs.x;
  hb.ray = qrb <= qs.y;
  ha.u = u.x; ha.v = v.x; ha.inv_det = inv.x; ha.q2 = q2.x; ha.dy = dy.x;
  hb.u = u.y; hb.v = v.y; hb.inv_det = inv.y; hb.q2 = q2.y; hb.dy = dy.y;
  ha.t = ha.ray ? t.x : depth;
  hb.t = hb.ray ? t.y : depth;
  ha.ghat = __expf(-fminf(qra, qs.x));  // = ray ? q_ray : q_screen, as in eval_hit
  hb.ghat = __expf(-fminf(qrb, qs.y));
}

// Thread → pixel layout of a TS×TS tile with PPT pixels of one column per
// thread. Threads form TS/PPT thread rows; warps own blocks of WC columns × WR
// thread rows (16 × 2 for tiles of 16 and 32, 8 × 4 for tiles of 8), laid
// row-major over the tile. Blocked (IL false): thread row t holds the PPT
// adjacent pixel rows t·PPT .. t·PPT+PPT−1. Interleaved (IL true): thread row
// t holds rows t, t+RS, t+2·RS, … with RS = TS/PPT, so a warp whose thread
// rows span the tile covers a box of h rows with about h/RS + 1 distinct
// pixel slots instead of min(h, PPT).
template <int TS, int PPT, bool IL = false>
struct Layout {
  static constexpr int NT = TS * TS / PPT;       // threads per CTA
  static constexpr int WC = TS < 16 ? TS : 16;   // pixel columns of a warp's block
  static constexpr int WR = 32 / WC;             // thread rows of a warp's block
  static constexpr int BPR = TS / WC;            // warp blocks across the tile
  static constexpr int RS = IL ? TS / PPT : 1;   // row step between a thread's pixels
  static_assert(NT % 32 == 0 && NT <= 1024, "whole warps, at most 1024 threads");
  static __device__ __forceinline__ int col(int tid) { return ((tid >> 5) % BPR) * WC + (tid & 31) % WC; }
  static __device__ __forceinline__ int trow(int tid) { return ((tid >> 5) / BPR) * WR + (tid & 31) / WC; }
  // row of the thread's pixel 0 (pixel p: row(tid) + p·RS)
  static __device__ __forceinline__ int row(int tid) { return IL ? trow(tid) : trow(tid) * PPT; }
  // the thread's PPT bits in a staged row mask (box_masks)
  static __device__ __forceinline__ int mshift(int tid) { return trow(tid) * PPT; }
};

template <int PPT>
struct TileGeo {
  int W, H;
  long long row0;               // pix_base + y(p=0)·W + x
  long long pstride;            // buffer offset between a thread's pixels (RS·W)
  float pxc, sx, kx;                 // kx: column within the tile
  float pyc[PPT], sy[PPT], ky[PPT];   // ky: rows within the tile
  bool inside[PPT];
  float bx0, bx1, by0, by1;     // pixel-centre extent of the tile's in-image pixels
  float sxa, sxb, sya, syb;     // ray components of the tile's first and last pixel column and row
};

template <int TS, int PPT, bool IL = false>
__device__ __forceinline__ TileGeo<PPT> tile_geo(const RasterArgs& a, int tile) {
  using L = Layout<TS, PPT, IL>;
  TileGeo<PPT> g;
  int v = 0;
  while (v + 1 < a.n_views && tile >= __ldg(&a.views[v + 1].tile_base)) ++v;
  const ViewInfo* V = a.views + v;
  const int tiles_x = __ldg(&V->tiles_x);
  g.W = __ldg(&V->width);
  g.H = __ldg(&V->height);
  const int lt = tile - __ldg(&V->tile_base);
  const int x0 = (lt % tiles_x) * TS, y0 = (lt / tiles_x) * TS;
  const int x = x0 + L::col(threadIdx.x), yb = y0 + L::row(threadIdx.x);
  const float f = __ldg(&V->focal), cx = __ldg(&V->cx), cy = __ldg(&V->cy);
  g.pxc = (float)x + 0.5f;
  g.sx = -((g.pxc - cx) / f);  // s = −d
  g.kx = (float)(x - x0);
#pragma unroll
  for (int p = 0; p < PPT; ++p) {
    const int y = yb + p * L::RS;
    g.pyc[p] = (float)y + 0.5f;
    g.sy[p] = (g.pyc[p] - cy) / f;
    g.ky[p] = (float)(y - y0);
    g.inside[p] = x < g.W && y < g.H;
  }
  g.row0 = __ldg(&V->pix_base) + (long long)yb * g.W + x;
  g.pstride = (long long)L::RS * g.W;
  g.bx0 = (float)x0 + 0.5f;
  g.bx1 = (float)(min(x0 + TS, g.W) - 1) + 0.5f;
  g.by0 = (float)y0 + 0.5f;
  g.by1 = (float)(min(y0 + TS, g.H) - 1) + 0.5f;
  g.sxa = -(((float)x0 + 0.5f - cx) / f);
  g.sxb = -(((float)(x0 + TS - 1) + 0.5f - cx) / f);
  g.sya = ((float)y0 + 0.5f - cy) / f;
  g.syb = ((float)(y0 + TS - 1) + 0.5f - cy) / f;
  return g;
}

// True when an entry's ray branch is available at every pixel of the tile:
// |det| > 1e-12 and t = tn/det > NEAR_DEPTH. det = M·(sx, sy, 1) is affine
// in the pixel's ray components, which are monotone in the pixel column and
// row, so over the tile it lies between its values at the four corner
// pixels; the margins (1e-5 of the terms' magnitude, 1e-5 of NEAR_DEPTH)
// cover the rounding of the corner and per-pixel evaluations and of the
// approximate reciprocal. A false answer only keeps the per-pixel test.
template <int PPT>
__device__ __forceinline__ bool ray_available(const float4& r0, const TileGeo<PPT>& g) {
  const float e0 = fmaf(r0.x, g.sxa, r0.z), e1 = fmaf(r0.x, g.sxb, r0.z);
  const float d00 = fmaf(r0.y, g.sya, e0), d01 = fmaf(r0.y, g.syb, e0);
  const float d10 = fmaf(r0.y, g.sya, e1), d11 = fmaf(r0.y, g.syb, e1);
  const float err = 1e-5f * (fabsf(r0.x) * fmaxf(fabsf(g.sxa), fabsf(g.sxb)) +
                             fabsf(r0.y) * fmaxf(fabsf(g.sya), fabsf(g.syb)) + fabsf(r0.z));
  const float lo = fminf(fminf(d00, d01), fminf(d10, d11)) - err;
  const float hi = fmaxf(fmaxf(d00, d01), fmaxf(d10, d11)) + err;
  const float near = NEAR_DEPTH * (1.0f + 1e-5f);
  if (lo > 1e-12f) return r0.w > near * hi;     // det > 0 everywhere: t ≥ tn / hi
  if (hi < -1e-12f) return -r0.w > near * -lo;  // det < 0 everywhere: t ≥ tn / lo
  return false;
}

// True when q_screen = dx² + dy² exceeds ln(255·max(o, 1)) + 0.05 at every
// pixel of the tile, for a record staged with stage_offsets (dx = r1.w +
// column, dy = r2.w + row) and opacity o: there o·exp(−q_screen) < 1/255, so
// the screen branch never decides a pixel that takes the entry.
template <int TS>
__device__ __forceinline__ bool screen_far(const float4& r1, const float4& r2, float o) {
  const float ex = r1.w > 0.f ? r1.w : fmaxf(-(r1.w + (float)(TS - 1)), 0.f);
  const float ey = r2.w > 0.f ? r2.w : fmaxf(-(r2.w + (float)(TS - 1)), 0.f);
  const float lim = 5.5913f + fmaxf(__logf(o), 0.f) * 1.001f;  // ln 255 = 5.5413
  return fmaf(ex, ex, ey * ey) > lim;
}

template <int PPT>
__device__ __forceinline__ bool box_hits_tile(const float4& b, const TileGeo<PPT>& g) {
  return b.x <= g.bx1 && b.y >= g.bx0 && b.z <= g.by1 && b.w >= g.by0;
}

// Bits r (0 <= r < TS) with c0 + r in [z0, z1], for pixel centres c0 + r.
// The candidate ends come from the float differences (off by at most one
// for |z - c0| < 2^23; larger values are clamped) and are corrected with the
// same comparisons the per-pixel test makes, so the result is exact.
template <int TS>
__device__ __forceinline__ void span_range(float c0, float z0, float z1, int& lo, int& hi) {
  lo = (int)ceilf(fminf(fmaxf(z0 - c0, -1.0f), (float)TS));
  if (lo < TS && !(c0 + (float)lo >= z0)) ++lo;
  if (lo > 0 && c0 + (float)(lo - 1) >= z0) --lo;
  hi = (int)floorf(fminf(fmaxf(z1 - c0, -1.0f), (float)TS));
  if (hi >= 0 && !(c0 + (float)hi <= z1)) --hi;
  if (hi < TS - 1 && c0 + (float)(hi + 1) <= z1) ++hi;
  lo = max(lo, 0);
  hi = min(hi, TS - 1);
}
template <int TS>
__device__ __forceinline__ uint32_t span_bits(float c0, float z0, float z1) {
  int lo, hi;
  span_range<TS>(c0, z0, z1, lo, hi);
  if (hi < lo) return 0u;
  return ((2u << hi) - 1u) & ~((1u << lo) - 1u);
}

// Pixel masks of an entry's α-box over the tile, the per-pixel box test
// decided once per staged entry; a lane then tests bits instead of comparing
// per pixel. .y: bit c when column c (centre bx0 + c) lies in [b.x, b.y].
// .x: the rows (centres by0 + r) in [b.z, b.w] in the layout's order: PPT bits
// per thread row t, bit t·PPT + p for the thread's pixel p (row t·PPT + p when
// blocked, which is bit r for row r; row t + p·RS when interleaved).
template <int TS, int PPT, bool IL = false>
__device__ __forceinline__ uint2 box_masks(const float4& b, const TileGeo<PPT>& g) {
  if constexpr (!IL) {
    return make_uint2(span_bits<TS>(g.by0, b.z, b.w), span_bits<TS>(g.bx0, b.x, b.y));
  } else {
    constexpr int RS = TS / PPT;
    int lo, hi;
    span_range<TS>(g.by0, b.z, b.w, lo, hi);
    uint32_t m = 0u;
    if (hi >= lo) {
#pragma unroll
      for (int t = 0; t < RS; ++t) {
        // pixels p with lo <= t + p·RS <= hi
        const int plo = lo <= t ? 0 : (lo - t + RS - 1) / RS;
        const int phi = hi < t ? -1 : min((hi - t) / RS, PPT - 1);
        if (phi >= plo) m |= (((2u << phi) - 1u) & ~((1u << plo) - 1u)) << (t * PPT);
      }
    }
    return make_uint2(m, span_bits<TS>(g.bx0, b.x, b.y));
  }
}

// Compaction of one staging round: returns this thread's slot among the kept
// entries of the round (valid when keep) and the number kept. Order is
// preserved. Rounds alternate between two s_wcount rows, so the next round's
// writes never meet a slower warp still reading this one.
template <int NW>
__device__ __forceinline__ int compact_slot(bool keep, int* s_wcount, int& kept) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned bal = __ballot_sync(FULL, keep);
  if (lane == 0) s_wcount[warp] = __popc(bal);
  __syncthreads();
  int off = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < NW; ++w) {
    const int c = s_wcount[w];
    if (w < warp) off += c;
    tot += c;
  }
  kept = tot;
  return off + __popc(bal & lanemask_lt());
}

// Row-group word flush of the colour-only forward: ORs a 32-entry word of
// contributor bits over the lanes that share a row group (the 16 lanes of a
// thread row, and both thread rows of a warp when a thread covers fewer than
// 4 rows) and adds it into s_gw[group][word]; clears the lane's words.
template <int PPT, int GPL, int GW>
__device__ __forceinline__ void flush_row_groups(uint32_t (&gcur)[GPL], uint32_t (*s_gw)[GW], int g0, int word) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i < GPL; ++i) {
    uint32_t v = gcur[i];
    v |= __shfl_xor_sync(FULL, v, 1);
    v |= __shfl_xor_sync(FULL, v, 2);
    v |= __shfl_xor_sync(FULL, v, 4);
    v |= __shfl_xor_sync(FULL, v, 8);
    if (PPT < 4) v |= __shfl_xor_sync(FULL, v, 16);
    if (v && (lane & (PPT < 4 ? 31 : 15)) == 0) atomicOr(&s_gw[g0 + i][word], v);
    gcur[i] = 0u;
  }
}

// Occlusion-cut bookkeeping of a tile at the end of a persistent colour-only
// forward pass (one thread): `complete` when every pixel terminated, `walk`
// the tile's largest contributor count. A truncated list that ran out first
// is listed for the completion pass; otherwise the tile's next cut is
// recorded.
__device__ __forceinline__ void cut_tile_end(const RasterArgs& a, int tile, uint2 range, bool complete,
                                             uint32_t walk) {
  const uint32_t used = a.cut_pass == 1 ? a.tile_cut[tile] : 0xffffffffu;
  const uint32_t len = range.y - range.x;
  if (!complete && used != 0xffffffffu) {
    // the truncated list ran out first: the completion pass continues the tile
    a.inc_flag[tile] = 1u;
    const uint32_t slot = atomicAdd(a.inc_count, 1u);
    a.inc_list[slot] = (uint32_t)tile;
    a.inc_skip[slot] = len;
    a.inc_src[slot] = range.x;
  } else {
    // next cut: the depth key at list position walk + walk/4 + 32 (the last
    // contributor plus a margin for the next step's changes). A truncated list
    // shorter than that extends its cut past its last key by the key span from
    // the last contributor to the list's end (at least 2^14 units in the last
    // place, about 0.2 % of depth).
    uint32_t next = 0xffffffffu;
    if (complete) {
      const uint32_t keep = walk + walk / 4u + 32u;
      if (keep < len) {
        next = __ldg(a.item_key + a.sorted_pairs[range.x + keep - 1u].y);
      } else if (used == 0xffffffffu || walk == 0u || len == 0u) {
        next = used;
      } else {
        const uint32_t kl = __ldg(a.item_key + a.sorted_pairs[range.y - 1u].y);
        const uint32_t kw = __ldg(a.item_key + a.sorted_pairs[range.x + walk - 1u].y);
        const uint32_t span = max(kl - kw, 1u << 14);
        next = kl < 0x7f7fffffu - span ? kl + span : 0x7f7fffffu;
      }
    }
    a.tile_cut[tile] = next;
  }
}

// COLOR: colour, alpha and final transmittance only (the training step's
// loss reads nothing else); depth and normal are neither accumulated nor
// written.
// Resident two-warp colour-only forward CTAs per SM that the register
// allocation must allow (1: the compiler's choice). 16 caps the registers at
// 64 (8 warps per SM sub-partition, 40 B of spills): on 1M surfels × 8 ×
// 1080p the colour-only (64, 4) forward ran 2.74 ms against 2.82 ms at 14
// CTAs (72 registers) and 3.32 → 4.21 ms earlier between 72 registers and
// the compiler's 99. With the per-entry hit forms the walk needs fewer live
// values; before them 64 registers ran slower than 72.
#ifndef GS_FWD_2WARP_CTAS
#define GS_FWD_2WARP_CTAS 16
#endif
template <int TS, int BATCH, int PREC, bool DET, bool PERSIST, int PPT, bool COLOR = false, bool MASK = false>
__global__ void __launch_bounds__(TS * TS / PPT, ((TS * TS / PPT) == 64 && COLOR && !MASK) ? GS_FWD_2WARP_CTAS : 1)
    k_raster_fwd(RasterArgs a) {
  static_assert(!MASK || COLOR, "contributor masks belong to the colour-only variant");
  using L = Layout<TS, PPT>;
  constexpr int NT = L::NT, NW = NT / 32, TP = TS * TS;
  constexpr int ROUNDS = (BATCH + NT - 1) / NT;  // staging rounds per batch
  // Row-group contributor summary (colour-only forward, 16-pixel tiles): for
  // every staged entry, bit g is set when some pixel of rows 4g..4g+3 of the
  // tile composited it; written to gmask[entry] for the backward. Each lane
  // collects the entries its pixels composited as bits of a 32-entry word per
  // row group it covers (GPL = 1, or 2 at 8 pixels per thread); every 32
  // entries the lanes of a row group OR their words together and one lane
  // adds the result into s_gw[group][word].
  constexpr bool GM = COLOR && !MASK && TS == 16;
  constexpr int GPL = PPT >= 8 ? 2 : 1;              // row groups per lane
  constexpr int GW = (BATCH + 31) / 32;              // 32-entry words per batch
  __shared__ float4 s_r0[BATCH], s_r1[BATCH], s_r2[BATCH], s_r3[BATCH];
  __shared__ uint2 s_msk[BATCH];  // box_masks of the staged entry
  __shared__ float4 s_r4[COLOR ? 1 : BATCH];
  __shared__ int s_j[BATCH];
  __shared__ uint32_t s_gw[GM ? 4 : 1][GM ? GW : 1];
  __shared__ int s_wcount[2][NW];
  __shared__ int s_tile;
  __shared__ uint32_t s_walk;  // tile_walk: the tile's largest contributor count
  __shared__ uint32_t s_slot;  // counter value the tile was taken at
  // Bits 31 and 30 of a staged column mask (free on tiles of up to 16
  // pixels): RAYBIT when the entry's ray branch is available at every pixel
  // of the tile (ray_available) and its opacity is below the α clamp (α =
  // o·ĝ with ĝ ≤ 1 is never clamped): the HIT_RAY_OK form; with FARBIT its
  // screen-space disc also stays away from the tile (screen_far): the
  // HIT_RAY_FAR form.
  constexpr bool RAYFLAG = TS <= 16;
  constexpr uint32_t RAYBIT = 0x80000000u, FARBIT = 0x40000000u;
  const int tid = threadIdx.x, lane = tid & 31;
  const bool gm_on = GM && a.gmask != nullptr;
  const int g0 = L::row(tid) >> 2;  // first row group of this lane's pixels
  constexpr uint32_t PMASK = (1u << PPT) - 1u;  // a lane's pixels p as bits
  uint32_t gcur[GPL];
  int tile = blockIdx.x;
  for (;;) {
    if (PERSIST) {
      if (tid == 0) {
        const uint32_t slot = atomicAdd(a.tile_counter, 1u);
        const uint32_t lim = a.tile_limit != nullptr ? *a.tile_limit : (uint32_t)a.total_tiles;
        // heaviest tiles first when an order is given (a shorter tail)
        s_tile = slot >= lim ? a.total_tiles : (int)(a.tile_order != nullptr ? __ldg(a.tile_order + slot) : slot);
        s_slot = slot;
      }
      __syncthreads();
      tile = s_tile;
      if (tile >= a.total_tiles) return;
    }
    const TileGeo<PPT> g = tile_geo<TS, PPT>(a, tile);
    const uint2 range = __ldg(&a.ranges[tile]);
    // Completion pass of the occlusion cut: the tile's full list begins with
    // the skip entries pass 1 composited (their row-group summary was moved
    // along with the range); continue after them from the pixel state pass 1
    // wrote.
    const bool resume = PERSIST && a.cut_pass == 2;
    uint32_t skip = 0;
    if (resume) {
      skip = a.inc_skip[s_slot];
      if (range.y - range.x < skip) skip = 0;  // list not rebuilt (entry capacity error already flagged)
    }
    float T[PPT], cr[PPT], cg[PPT], cb[PPT], aa[PPT], ad[PPT], nx[PPT], ny[PPT], nz[PPT];
    uint32_t nc[PPT];
    uint32_t dm = 0u;  // bit p: pixel p terminated (or lies outside the image)
    // Stored-state contributor masks (colour-only variant): the word being
    // filled and its index, per pixel.
    uint32_t mw[PPT];
    int mi[PPT];
    constexpr bool masks = MASK;
    const size_t mbase = masks ? (size_t)__ldg(&a.mask_off[tile]) * TP : 0;
    const int mpix = L::row(tid) * TS + L::col(tid);  // pixel p is mpix + p·TS
#pragma unroll
    for (int p = 0; p < PPT; ++p) {
      T[p] = 1.f; cr[p] = cg[p] = cb[p] = aa[p] = ad[p] = nx[p] = ny[p] = nz[p] = 0.f;
      nc[p] = 0;
      if (!g.inside[p]) dm |= 1u << p;
      if (resume && g.inside[p]) {
        const long long pix = g.row0 + (long long)p * g.W;
        const float4 c = a.out_color[pix], x = a.out_aux[pix];
        cr[p] = c.x; cg[p] = c.y; cb[p] = c.z; aa[p] = c.w;
        T[p] = x.x;
        if (!COLOR) {
          ad[p] = x.y;
          const float4 nn = a.out_normal[pix];
          nx[p] = nn.x; ny[p] = nn.y; nz[p] = nn.z;
        }
        nc[p] = a.out_nc[pix];
        if (T[p] < T_TERMINATE) dm |= 1u << p;
      }
      mw[p] = 0u;
      mi[p] = 0;
    }
    bool tdone = dm == PMASK;
    for (uint32_t base = range.x + skip; base < range.y; base += BATCH) {
      if (__syncthreads_count(tdone) == NT) break;
      const int count = (int)min((uint32_t)BATCH, range.y - base);
      int kept = 0;
#pragma unroll
      for (int rd = 0; rd < ROUNDS; ++rd) {
        const int j = rd * NT + tid;
        bool keep = false;
        uint32_t item = 0;
        float4 bb = make_float4(0.f, 0.f, 0.f, 0.f);
        if (j < count) {
          item = __ldg(&a.sorted_pairs[base + j].y);
          if (DET) item = __ldg(&a.exp_item[item]);
          bb = load_record_box<PREC>(a.records, item);
          keep = box_hits_tile(bb, g);
        }
        int kr;
        const int slot = kept + compact_slot<NW>(keep, s_wcount[rd & 1], kr);
        if (keep) {
          float4 r0, r1, r2, r3, r4;
          if (COLOR) load_record4<PREC>(a.records, item, r0, r1, r2, r3);
          else load_record<PREC>(a.records, item, r0, r1, r2, r3, r4);
          stage_offsets(r1, r2, g.bx0, g.by0);
          s_r0[slot] = r0; s_r1[slot] = r1; s_r2[slot] = r2; s_r3[slot] = r3;
          if (!COLOR) s_r4[slot] = r4;
          uint2 mk = box_masks<TS, PPT>(bb, g);
          if (RAYFLAG && r3.w < ALPHA_CLAMP && ray_available(r0, g)) {
            mk.y |= RAYBIT;
            if (screen_far<TS>(r1, r2, r3.w)) mk.y |= FARBIT;
          }
          s_msk[slot] = mk;
          s_j[slot] = j;
        }
        kept += kr;
      }
      if (GM && tid < 4 * GW) (&s_gw[0][0])[tid] = 0u;
#pragma unroll
      for (int i = 0; i < GPL; ++i) gcur[i] = 0u;
      __syncthreads();
      // Warp-synchronous walk: every lane runs every iteration (lanes whose
      // pixels are done idle), so the per-entry warp reduction is legal.
      if (__any_sync(FULL, !tdone)) {
        int k = 0;
        for (; k < kept; ++k) {
          const uint32_t kbit = 1u << (k & 31);
          const uint2 mk = s_msk[k];
          // need: bit p when pixel p is live and inside the entry's α-box
          const uint32_t need = ((mk.y >> L::col(tid)) & 1u) ? (mk.x >> L::row(tid)) & ~dm & PMASK : 0u;
          if (need) {
            const float4 r0 = s_r0[k], r1 = s_r1[k], r2 = s_r2[k];
            const float4 r3 = s_r3[k];
            const float4 r4 = COLOR ? make_float4(0.f, 0.f, 0.f, 0.f) : s_r4[k];
            const uint32_t idx1 = base - range.x + (uint32_t)s_j[k] + 1u;
            const ColPart cp = col_part(r0, r1, r2, g.sx, g.kx);
            constexpr int PS = PPT >= 2 ? 2 : 1;  // pixels per hit evaluation
            // the pixel walk, with or without the per-pixel ray test
            auto walk = [&](auto ray_tag) {
            constexpr int FAST = decltype(ray_tag)::value;
#pragma unroll
            for (int pp = 0; pp < PPT; pp += PS) {
            bool need_q[PS];
            Hit hh[PS];
#pragma unroll
            for (int q = 0; q < PS; ++q) need_q[q] = (need >> (pp + q)) & 1u;
            if constexpr (PS == 2) {
              if (!((need >> pp) & 3u)) continue;
              eval_hit2<FAST>(cp, r0, r1, r2, r4.w, make_float2(g.sy[pp], g.sy[pp + 1]),
                                make_float2(g.ky[pp], g.ky[pp + 1]), hh[0], hh[PS - 1]);
            } else {
              if (!need_q[0]) continue;
              hh[0] = eval_hit<FAST>(cp, r0, r1, r2, r4.w, g.sy[pp], g.ky[pp]);
            }
            if constexpr (PS == 2 && COLOR && !MASK && PPT <= 4) {  // (8 pixels per thread would spill)
              // Both pixels of the pair composited at once in packed FP32: a
              // pixel that does not take the entry gets α = 0, so its weight is
              // 0 and its T is multiplied by 1 (both exact); each component
              // rounds as the scalar code below would.
              // (fast form: opacity < ALPHA_CLAMP and ĝ ≤ 1, so the clamp never acts)
              const float a0 = FAST ? __fmul_rn(r3.w, hh[0].ghat) : fminf(__fmul_rn(r3.w, hh[0].ghat), ALPHA_CLAMP);
              const float a1 = FAST ? __fmul_rn(r3.w, hh[PS - 1].ghat)
                                    : fminf(__fmul_rn(r3.w, hh[PS - 1].ghat), ALPHA_CLAMP);
              const bool c0 = need_q[0] && !(a0 < ALPHA_SKIP), c1 = need_q[PS - 1] && !(a1 < ALPHA_SKIP);
              if (c0 || c1) {
                const float2 al = make_float2(c0 ? a0 : 0.f, c1 ? a1 : 0.f);
                const float2 Tp = make_float2(T[pp], T[pp + 1]);
                const float2 w = __fmul2_rn(Tp, al);
                float2 vr = __ffma2_rn(make_float2(r3.x, r3.x), w, make_float2(cr[pp], cr[pp + 1]));
                float2 vg = __ffma2_rn(make_float2(r3.y, r3.y), w, make_float2(cg[pp], cg[pp + 1]));
                float2 vb = __ffma2_rn(make_float2(r3.z, r3.z), w, make_float2(cb[pp], cb[pp + 1]));
                float2 va = __fadd2_rn(make_float2(aa[pp], aa[pp + 1]), w);
                const float2 Tn = __fmul2_rn(Tp, __fadd2_rn(make_float2(1.0f, 1.0f), make_float2(-al.x, -al.y)));
                cr[pp] = vr.x; cr[pp + 1] = vr.y; cg[pp] = vg.x; cg[pp + 1] = vg.y;
                cb[pp] = vb.x; cb[pp + 1] = vb.y; aa[pp] = va.x; aa[pp + 1] = va.y;
                T[pp] = Tn.x; T[pp + 1] = Tn.y;
                // both pixels of a pair lie in one 4-row group (a thread's first row is even)
                if (GM) gcur[(((L::row(tid) & 3) + pp) >> 2) & (GPL - 1)] |= kbit;
                if (c0) {
                  nc[pp] = idx1;
                  if (Tn.x < T_TERMINATE) dm |= 1u << pp;
                }
                if (c1) {
                  nc[pp + 1] = idx1;
                  if (Tn.y < T_TERMINATE) dm |= 2u << pp;
                }
              }
              continue;
            }
#pragma unroll
            for (int q = 0; q < PS; ++q) {
              const int p = pp + q;
              if (!need_q[q]) continue;
              const Hit& h = hh[q];
              const float alpha = FAST ? __fmul_rn(r3.w, h.ghat) : fminf(__fmul_rn(r3.w, h.ghat), ALPHA_CLAMP);
              if (alpha < ALPHA_SKIP) continue;
              const float w = T[p] * alpha;
              cr[p] += r3.x * w; cg[p] += r3.y * w; cb[p] += r3.z * w;
              aa[p] += w;
              if (!COLOR) {
                ad[p] += h.t * w;
                nx[p] += r4.x * w; ny[p] += r4.y * w; nz[p] += r4.z * w;
              }
              T[p] = __fmul_rn(T[p], 1.0f - alpha);
              nc[p] = idx1;
              if (GM) gcur[(((L::row(tid) & 3) + p) >> 2) & (GPL - 1)] |= kbit;
              if (masks) {
                const uint32_t cidx = idx1 - 1u;
                const int w = (int)(cidx >> 5);
                if (w != mi[p]) {  // close the current word, zero the words skipped
                  uint32_t* m = a.mask + mbase + mpix + p * TS;
                  m[(size_t)mi[p] * TP] = mw[p];
                  for (int z = mi[p] + 1; z < w; ++z) m[(size_t)z * TP] = 0u;
                  mi[p] = w;
                  mw[p] = 0u;
                }
                mw[p] |= 1u << (cidx & 31u);
              }
              if (T[p] < T_TERMINATE) dm |= 1u << p;
            }
            }
            };
            if (RAYFLAG && (mk.y & FARBIT)) walk(std::integral_constant<int, HIT_RAY_FAR>{});
            else if (RAYFLAG && (mk.y & RAYBIT)) walk(std::integral_constant<int, HIT_RAY_OK>{});
            else walk(std::integral_constant<int, HIT_FULL>{});
            tdone = dm == PMASK;
          }
          if (GM && gm_on && (k & 31) == 31) flush_row_groups<PPT, GPL, GM ? GW : 1>(gcur, s_gw, g0, k >> 5);
          if (__all_sync(FULL, tdone)) break;
        }
        const int last = k < kept ? k : kept - 1;  // last entry walked (the walk breaks after it)
        if (GM && gm_on && last >= 0 && (last & 31) != 31) flush_row_groups<PPT, GPL, GM ? GW : 1>(gcur, s_gw, g0, last >> 5);
      }
      if (GM && gm_on) {
        __syncthreads();
        for (int k = tid; k < kept; k += NT) {
          const int w = k >> 5, b = k & 31;
          const uint32_t m = ((s_gw[0][w] >> b) & 1u) | (((s_gw[1][w] >> b) & 1u) << 1) |
                             (((s_gw[2][w] >> b) & 1u) << 2) | (((s_gw[3][w] >> b) & 1u) << 3);
          a.gmask[base + (uint32_t)s_j[k]] = (uint8_t)m;
        }
      }
    }
#pragma unroll
    for (int p = 0; p < PPT; ++p) {
      if (!g.inside[p]) continue;
      const long long pix = g.row0 + (long long)p * g.W;
      a.out_color[pix] = make_float4(cr[p], cg[p], cb[p], aa[p]);
      if (masks && nc[p] > 0) a.mask[mbase + mpix + p * TS + (size_t)mi[p] * TP] = mw[p];
      if (COLOR) {
        a.out_aux[pix].x = T[p];
      } else {
        a.out_aux[pix] = make_float4(T[p], ad[p], 0.f, 0.f);
        a.out_normal[pix] = make_float4(nx[p], ny[p], nz[p], 0.f);
      }
      a.out_nc[pix] = nc[p];
    }
    if (a.tile_walk != nullptr) {  // how far the backward will walk this tile's list
      uint32_t m = 0;
#pragma unroll
      for (int p = 0; p < PPT; ++p) m = max(m, nc[p]);
      m = __reduce_max_sync(FULL, m);
      if (tid == 0) s_walk = 0u;
      __syncthreads();
      if (lane == 0) atomicMax(&s_walk, m);
      __syncthreads();
      if (tid == 0) a.tile_walk[tile] = s_walk;
    }
    if (a.tile_cut != nullptr) {  // occlusion cut bookkeeping (set together with tile_walk)
      const bool complete = __syncthreads_count(tdone) == NT;  // every pixel terminated
      if (tid == 0) cut_tile_end(a, tile, range, complete, s_walk);
    }
    if (!PERSIST) return;
    __syncthreads();
  }
}

// Resident single-warp backward CTAs per SM (without stored-state masks, which
// would spill) that the register allocation must allow (1: the compiler's
// choice). 24 caps the registers at 80 (6 warps per
// SM sub-partition instead of 4 at the compiler's 115): on 1M surfels × 8 ×
// 1080p the (32, 8) backward ran 3.31 ms against 3.70 ms (24 B of spills;
// at 72 registers the spills grew to 68 B and it ran 3.63 ms).
#ifndef GS_BWD_WARP_CTAS
#define GS_BWD_WARP_CTAS 24
#endif
template <int TS, int BATCH, int PREC, bool AUX, bool DET, bool PERSIST, int PPT, bool MASK = false>
__global__ void __launch_bounds__(TS * TS / PPT, ((TS * TS / PPT) == 32 && !MASK) ? GS_BWD_WARP_CTAS : 1)
    k_raster_bwd(RasterArgs a) {
  static_assert(!MASK || !AUX, "contributor masks cover the colour-only backward");
  // Interleaved pixel rows (Layout) for single-warp CTAs with two or more
  // pixels per thread: on 16-pixel tiles with 8 pixels per thread, a box of
  // h ≤ 8 rows takes about h/2 + 1 pixel slots of the warp instead of h. With
  // several warps, interleaving would spread every box over all of them (one
  // more warp reduction per warp an entry reaches), so they stay blocked.
#ifndef GS_BWD_INTERLEAVE
#define GS_BWD_INTERLEAVE 1
#endif
  constexpr bool IL = GS_BWD_INTERLEAVE && PPT >= 2 && TS * TS / PPT == 32;
  using L = Layout<TS, PPT, IL>;
  constexpr int NT = L::NT, NW = NT / 32, TP = TS * TS;
  constexpr int ROUNDS = (BATCH + NT - 1) / NT;  // staging rounds per batch
  constexpr int NG = AUX ? 32 : 16;  // reduced components per entry (AUX: 20 used)
  constexpr int NQ = AUX ? 5 : 4;    // float4 groups per entry written out
  // Row-group contributor summary of the matching colour-only forward
  // (16-pixel tiles): entries no pixel of a group composited are skipped for
  // that group's pixels without evaluating them.
  constexpr bool GM = !AUX && !MASK && TS == 16;
  // Interleaved single-warp tiles fold the summary into the staged row mask
  // (a pixel's group depends on its slot alone there, not on its thread row).
  constexpr bool GM_FOLD = GM && IL && L::RS == 2;
  // A single-warp CTA (8 pixels per thread on 16-pixel tiles) has nothing to
  // sum across warps: the lanes holding each group of four reduced components
  // gather them by shuffles and emit the vector reduction (or ordered store)
  // at once, without staging them in shared memory.
  constexpr bool DIRECT = !AUX && NW == 1;
  __shared__ float4 s_r0[BATCH], s_r1[BATCH], s_r2[BATCH], s_r3[BATCH];
  __shared__ uint2 s_msk[BATCH];  // box_masks of the staged entry
  __shared__ float4 s_r4[AUX ? BATCH : 1];
  __shared__ uint32_t s_item[BATCH];
  __shared__ uint32_t s_q[DET ? BATCH : 1];
  __shared__ int s_j[BATCH];
  __shared__ uint8_t s_gm[GM ? BATCH : 1];
  __shared__ float s_part[DIRECT ? 1 : NW][DIRECT ? 1 : BATCH][NG];
  __shared__ int s_wcount[2][NW];
  __shared__ int s_tile, s_maxnc;
  // Colour-only: the tile's dL/dcolour per pixel (each thread reads back only
  // its own pixels), read where a pair contributes instead of held in three
  // registers per pixel.
#ifndef GS_BWD_DLC_SMEM
#define GS_BWD_DLC_SMEM 1
#endif
  constexpr bool DLC_SMEM = GS_BWD_DLC_SMEM && !AUX && TS <= 16;  // (tiles of 32: 16 KB more than the static limit allows)
  __shared__ float4 s_dlc[DLC_SMEM ? TP : 1];
  // Optionally each pixel's walked-back transmittance and colour suffix too
  // (again read and written only by the thread that owns the pixel).
#ifndef GS_BWD_STATE_SMEM
#define GS_BWD_STATE_SMEM 0
#endif
  constexpr bool ST_SMEM = GS_BWD_STATE_SMEM && DLC_SMEM && DIRECT;  // single-warp CTAs
  __shared__ float2 s_ts[ST_SMEM ? TP : 1];
  // Single-warp interleaved colour-only CTAs keep the pixels' contributor
  // counts in shared memory (read only when the walk mask is rebuilt), and
  // optionally the rows' ray components (read once per evaluated pixel
  // pair), instead of registers; a pixel's tile-local row offset is then
  // formed from its first.
#ifndef GS_BWD_SY_SMEM
#define GS_BWD_SY_SMEM 0
#endif
  constexpr bool LEAN = DIRECT && IL && DLC_SMEM && !MASK;
  constexpr bool SYS = LEAN && GS_BWD_SY_SMEM;
  __shared__ uint32_t s_nc[LEAN ? TP : 1];
  __shared__ float s_sy[SYS ? TS : 1];
  // Bits 31 and 30 of a staged column mask, as in the forward: RAYBIT for
  // the HIT_RAY_OK form, with FARBIT for the HIT_RAY_FAR form.
  constexpr bool RAYFLAG = TS <= 16;
  constexpr uint32_t RAYBIT = 0x80000000u;
  constexpr uint32_t FARBIT = 0x40000000u;  // with RAYBIT: the HIT_RAY_FAR form (screen_far)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool gm_on = GM && a.gmask != nullptr;
  // A lane's pixels p (rows row(tid) + p·RS) as bits of a PPT-bit mask. Row
  // group g covers rows 4g..4g+3. Blocked, a lane's first row is a multiple of
  // min(PPT, 4), so its pixels fall in GPT whole groups of GSZ pixels.
  constexpr uint32_t PMASK = (1u << PPT) - 1u;
  constexpr int GSZ = PPT < 4 ? PPT : 4, GPT = PPT / GSZ;
  const int g0 = L::row(tid) >> 2;  // the lane's first row group
  uint32_t thread_gbits = 0u;
#pragma unroll
  for (int p = 0; p < PPT; ++p) thread_gbits |= 1u << ((L::row(tid) + p * L::RS) >> 2);
  const uint32_t warp_gbits = __reduce_or_sync(FULL, thread_gbits);
  const int lpix = L::row(tid) * TS + L::col(tid);  // tile-local index of pixel 0 (pixel p: + p·RS·TS)
  constexpr int PSTEP = L::RS * TS;
  // Results of staged entry k: group q4 of four reduced components, or zeros
  // for an entry this warp's pixels did not composite.
  auto emit4 = [&](int k, int q4, float s0, float s1, float s2, float s3) {
    if (DET) {
      reinterpret_cast<float4*>(a.partials + (size_t)s_q[k] * GG_STRIDE)[q4] = make_float4(s0, s1, s2, s3);
    } else if (s0 != 0.f || s1 != 0.f || s2 != 0.f || s3 != 0.f) {
      red_add_v4(a.grad_geom + (size_t)s_item[k] * GG_STRIDE + 4 * q4, s0, s1, s2, s3);
    }
  };
  auto emit_zero = [&](int k) {
    if constexpr (DIRECT) {
      if (DET && lane < NQ) emit4(k, lane, 0.f, 0.f, 0.f, 0.f);
    } else {
      if (lane < 16) s_part[warp][k][lane] = 0.f;
      if (AUX && lane >= 16) s_part[warp][k][lane] = 0.f;
    }
  };
  int tile = blockIdx.x;
  for (;;) {
    if (PERSIST) {
      if (tid == 0) {
        const uint32_t slot = atomicAdd(a.tile_counter, 1u);
        const uint32_t lim = a.tile_limit != nullptr ? *a.tile_limit : (uint32_t)a.total_tiles;
        // heaviest tiles first when an order is given (a shorter tail)
        s_tile = slot >= lim ? a.total_tiles : (int)(a.tile_order != nullptr ? __ldg(a.tile_order + slot) : slot);
      }
      __syncthreads();
      tile = s_tile;
      if (tile >= a.total_tiles) return;
    }
    const uint2 range = __ldg(&a.ranges[tile]);
    if (range.y <= range.x) {
      if (!PERSIST) return;
      __syncthreads();
      continue;
    }
    const TileGeo<PPT> g = tile_geo<TS, PPT, IL>(a, tile);
    // Suffix sums of what lies behind the current entry: colour and normal
    // enter only through their dot products with dL/dcolour and dL/dnormal,
    // so those scalars are carried instead of the vectors.
    float3 dlc[PPT], dln[PPT];
    float suf_c[PPT], suf_n[PPT];
    float dld[PPT], wtot[PPT], wttot[PPT], T[PPT], suf_d[PPT], suf_w[PPT], suf_cw[PPT];
    uint32_t nc[PPT];
    uint32_t my_max = 0;
#pragma unroll
    for (int p = 0; p < PPT; ++p) {
      dlc[p] = dln[p] = make_float3(0.f, 0.f, 0.f);
      suf_c[p] = suf_n[p] = 0.f;
      dld[p] = wtot[p] = wttot[p] = suf_d[p] = suf_w[p] = suf_cw[p] = 0.f;
      T[p] = 1.f;
      nc[p] = 0;
      if (g.inside[p]) {
        const long long pix = g.row0 + (long long)p * g.pstride;
        const float4 gc = a.dl_dcolor[pix];
        dlc[p] = make_float3(gc.x, gc.y, gc.z);
        if (DLC_SMEM) s_dlc[lpix + p * PSTEP] = gc;
        const float4 aux = a.out_aux[pix];
        T[p] = aux.x;
        if (ST_SMEM) s_ts[lpix + p * PSTEP] = make_float2(aux.x, 0.f);
        nc[p] = a.out_nc[pix];
        if (AUX) {
          dld[p] = gc.w;
          const float4 gn = a.dl_dnormal[pix];
          dln[p] = make_float3(gn.x, gn.y, gn.z);
          wtot[p] = a.out_color[pix].w;
          wttot[p] = aux.y;
        }
      }
      bool has_loss = g.inside[p] && (dlc[p].x != 0.f || dlc[p].y != 0.f || dlc[p].z != 0.f);
      if (AUX) has_loss = g.inside[p] && (has_loss || dld[p] != 0.f || dln[p].x != 0.f || dln[p].y != 0.f ||
                                          dln[p].z != 0.f || a.lambda_dist != 0.f);
      if (!has_loss) nc[p] = 0;  // nc = 0 disables the pixel's walk
      my_max = max(my_max, nc[p]);
      if (LEAN) s_nc[lpix + p * PSTEP] = nc[p];
    }
    if (SYS && (lane % L::WC) == 0) {  // one lane per thread row writes its rows' sy
#pragma unroll
      for (int p = 0; p < PPT; ++p) s_sy[L::row(tid) + p * L::RS] = g.sy[p];
    }
    // the ray component and tile-local row of pixel p (as tile_geo computes them)
    auto sy_of = [&](int p) { return SYS ? s_sy[L::row(tid) + p * L::RS] : g.sy[p]; };
    auto ky_of = [&](int p) { return LEAN ? __fadd_rn(g.ky[0], (float)(p * L::RS)) : g.ky[p]; };
    // Entries at or past this warp's last contributor are skipped warp-wide.
    const uint32_t warp_maxnc = __reduce_max_sync(FULL, my_max);
    if (tid == 0) s_maxnc = 0;
    __syncthreads();
    if (my_max) atomicMax(&s_maxnc, (int)my_max);
    __syncthreads();
    const uint32_t maxnc = min((uint32_t)s_maxnc, range.y - range.x);
    // Pixels whose walk has reached the current entry (cidx < nc[p]) as a
    // mask. cidx only decreases, so the mask is rebuilt only when cidx drops
    // below `thr`, the largest nc among the pixels not yet walking.
    uint32_t alive = 0u, thr = 0u;
#pragma unroll
    for (int p = 0; p < PPT; ++p) thr = max(thr, nc[p]);
    // Stored-state mode: contributor masks written by the forward; the word
    // cached per pixel and its index (list positions are walked downwards).
    constexpr bool masks = MASK;
    const size_t mbase = masks ? (size_t)__ldg(&a.mask_off[tile]) * TP : 0;
    const int mpix = lpix;
    uint32_t cm[PPT];
    int cw[PPT];
#pragma unroll
    for (int p = 0; p < PPT; ++p) { cm[p] = 0u; cw[p] = -1; }

    if (DET) {
      // Entries past the tile's last contributor get zero partials.
      for (uint32_t e = range.x + maxnc + tid; e < range.y; e += NT) {
        const uint32_t q = __ldg(&a.sorted_pairs[e].y);
        float4* pp = reinterpret_cast<float4*>(a.partials + (size_t)q * GG_STRIDE);
#pragma unroll
        for (int k = 0; k < NQ; ++k) pp[k] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }

    uint32_t hi = range.x + maxnc;
    while (hi > range.x) {
      const uint32_t lo = (hi - range.x > (uint32_t)BATCH) ? hi - BATCH : range.x;
      const int count = (int)(hi - lo);
      int kept = 0;
#pragma unroll
      for (int rd = 0; rd < ROUNDS; ++rd) {
        const int j = rd * NT + tid;
        bool keep = false;
        uint32_t item = 0, q = 0;
        float4 bb = make_float4(0.f, 0.f, 0.f, 0.f);
        if (j < count) {
          item = __ldg(&a.sorted_pairs[lo + j].y);
          q = item;
          if (DET) item = __ldg(&a.exp_item[q]);
          bb = load_record_box<PREC>(a.records, item);
          keep = box_hits_tile(bb, g);
          if (DET && !keep) {
            float4* pp = reinterpret_cast<float4*>(a.partials + (size_t)q * GG_STRIDE);
#pragma unroll
            for (int k = 0; k < NQ; ++k) pp[k] = make_float4(0.f, 0.f, 0.f, 0.f);
          }
        }
        int kr;
        const int slot = kept + compact_slot<NW>(keep, s_wcount[rd & 1], kr);
        if (keep) {
          float4 r0, r1, r2, r3, r4;
          if (AUX) load_record<PREC>(a.records, item, r0, r1, r2, r3, r4);
          else load_record4<PREC>(a.records, item, r0, r1, r2, r3);
          stage_offsets(r1, r2, g.bx0, g.by0);
          s_r0[slot] = r0; s_r1[slot] = r1; s_r2[slot] = r2; s_r3[slot] = r3;
          if (AUX) s_r4[slot] = r4;
          {
            uint2 mk = box_masks<TS, PPT, IL>(bb, g);
            if (RAYFLAG && r3.w < ALPHA_CLAMP && ray_available(r0, g)) {
              mk.y |= RAYBIT;
              if (screen_far<TS>(r1, r2, r3.w)) mk.y |= FARBIT;
            }
            s_msk[slot] = mk;
          }
          s_item[slot] = item;
          if (DET) s_q[slot] = q;
          s_j[slot] = j;
          if (GM) {
            const uint8_t gm = gm_on ? __ldg(a.gmask + lo + j) : (uint8_t)0xffu;
            if constexpr (GM_FOLD) {
              // every thread row's pixel p lies in group p / 2: AND the doubled
              // group bits into both thread rows' halves of the row mask
              uint32_t x = gm & 0xfu;
              x = (x | (x << 2)) & 0x33u;
              x = (x | (x << 1)) & 0x55u;
              x |= x << 1;
              s_msk[slot].x &= x | (x << PPT);
            } else {
              s_gm[slot] = gm;
            }
          }
        }
        kept += kr;
      }
      __syncthreads();
      for (int k = kept - 1; k >= 0; --k) {
        const uint32_t cidx = lo - range.x + (uint32_t)s_j[k];
        if (cidx >= warp_maxnc) {
          emit_zero(k);
          continue;
        }
        // need: bit p when pixel p evaluates the entry
        uint32_t need = 0u;
        if (masks) {
#pragma unroll
          for (int p = 0; p < PPT; ++p) {
            if (cidx < nc[p]) {
              const int w = (int)(cidx >> 5);
              if (w != cw[p]) {
                cw[p] = w;
                cm[p] = __ldg(a.mask + mbase + mpix + p * PSTEP + (size_t)w * TP);
              }
              need |= ((cm[p] >> (cidx & 31u)) & 1u) << p;
            }
          }
          if (!__any_sync(FULL, need != 0u)) {  // no pixel of this warp composited the entry
            emit_zero(k);
            continue;
          }
        } else {
          const uint2 mk = s_msk[k];  // bit p of mk.x >> mshift: pixel p's row is inside the box
          uint32_t gmp = PMASK;  // pixels in row groups that composited the entry
          if constexpr (GM_FOLD) {
            if (!mk.x) {  // no row of the box holds a contributor
              emit_zero(k);
              continue;
            }
          } else if (GM) {
            const uint32_t gm = s_gm[k];
            if (!(gm & warp_gbits)) {  // no pixel of this warp's row groups composited the entry
              emit_zero(k);
              continue;
            }
            if constexpr (!IL) {
              gmp = 0u;
#pragma unroll
              for (int i = 0; i < GPT; ++i) gmp |= ((gm >> (g0 + i)) & 1u) ? ((1u << GSZ) - 1u) << (GSZ * i) : 0u;
            } else if constexpr (L::RS == 2) {  // pixel p in group p / 2: each bit of gm doubled
              uint32_t x = gm & 0xfu;
              x = (x | (x << 2)) & 0x33u;
              x = (x | (x << 1)) & 0x55u;
              gmp = x | (x << 1);
            } else if constexpr (L::RS == 4) {  // pixel p in group p
              gmp = gm & PMASK;
            } else {
              gmp = 0u;
#pragma unroll
              for (int p = 0; p < PPT; ++p) gmp |= ((gm >> ((L::row(tid) + p * L::RS) >> 2)) & 1u) << p;
            }
          }
          if (cidx < thr) {  // a pixel's walk starts here
            alive = 0u;
            thr = 0u;
#pragma unroll
            for (int p = 0; p < PPT; ++p) {
              const uint32_t ncp = LEAN ? s_nc[lpix + p * PSTEP] : nc[p];
              if (cidx < ncp) alive |= 1u << p;
              else thr = max(thr, ncp);
            }
          }
          need = ((mk.y >> L::col(tid)) & 1u) ? (mk.x >> L::mshift(tid)) & alive & gmp : 0u;
        }
        float gg[NG];
#pragma unroll
        for (int c = 0; c < NG; ++c) gg[c] = 0.f;
        bool contrib = false;
        if (need) {
          const float4 r0 = s_r0[k], r1 = s_r1[k], r2 = s_r2[k], r3 = s_r3[k];
          float4 r4 = make_float4(0.f, 0.f, 0.f, 0.f);
          float depth = 0.f;  // feeds t in the screen branch, used by aux terms alone
          if (AUX) { r4 = s_r4[k]; depth = r4.w; }
          const ColPart cp = col_part(r0, r1, r2, g.sx, g.kx);
          // Pixel slots tested in pairs: with interleaved rows a box's slots
          // are consecutive, so both pixels of a pair are mostly needed (one
          // slot at a time ran 3.31 against 3.25 ms on 1M surfels × 8 × 1080p).
          constexpr int PS = PPT >= 2 ? 2 : 1;
          // the pixel walk, with or without the per-pixel ray test
          auto walk = [&](auto ray_tag) {
          constexpr int FAST = decltype(ray_tag)::value;
#pragma unroll
          for (int pp = 0; pp < PPT; pp += PS) {
          bool need_q[PS];
          Hit hh[PS];
#pragma unroll
          for (int q = 0; q < PS; ++q) need_q[q] = (need >> (pp + q)) & 1u;
          if constexpr (PS == 2) {
            if (!((need >> pp) & 3u)) continue;
            // both hits, evaluated one at a time: in this register-capped
            // kernel the packed form's operand pairs cost more moves than
            // its paired arithmetic saves
            hh[0] = eval_hit<FAST>(cp, r0, r1, r2, depth, sy_of(pp), ky_of(pp));
            hh[PS - 1] = eval_hit<FAST>(cp, r0, r1, r2, depth, sy_of(pp + 1), ky_of(pp + 1));
          } else {
            if (!need_q[0]) continue;
            hh[0] = eval_hit<FAST>(cp, r0, r1, r2, depth, sy_of(pp), ky_of(pp));
          }
#pragma unroll
          for (int q = 0; q < PS; ++q) {
            const int p = pp + q;
            if (!need_q[q]) continue;
            const Hit& h = hh[q];
            const float raw_alpha = __fmul_rn(r3.w, h.ghat);
            // (fast form: opacity < ALPHA_CLAMP and ĝ ≤ 1, so the clamp never acts)
            const float alpha = FAST ? raw_alpha : fminf(raw_alpha, ALPHA_CLAMP);
            if (alpha < ALPHA_SKIP) continue;
            contrib = true;
            const float inv_oma = rcp_approx(1.0f - alpha);
            float2 ts = make_float2(T[p], suf_c[p]);
            if (ST_SMEM) ts = s_ts[lpix + p * PSTEP];
            const float t_before = ts.x * inv_oma;
            const float w = t_before * alpha;
            float3 gcol = dlc[p];
            if (DLC_SMEM) {
              const float4 g4 = s_dlc[lpix + p * PSTEP];
              gcol = make_float3(g4.x, g4.y, g4.z);
            }
            const float dc = gcol.x * r3.x + gcol.y * r3.y + gcol.z * r3.z;
            float dl_dalpha = dc * t_before - ts.y * inv_oma;
            float dl_dt = 0.f;
            if (AUX) {
              const float t_hit = h.t;
              float dt_dist = 0.f, coef = 0.f;
              if (a.lambda_dist != 0.f) {
                const float a_pre = wtot[p] - suf_w[p] - w;
                const float b_pre = wttot[p] - suf_d[p] - w * t_hit;
                dt_dist = a.lambda_dist * 2.0f * w * (a_pre - suf_w[p]);
                coef = a.lambda_dist * (2.0f * (t_hit * a_pre - b_pre) + 2.0f * (suf_d[p] - t_hit * suf_w[p]));
              }
              dl_dt = dld[p] * w + dt_dist;
              const float dn = dln[p].x * r4.x + dln[p].y * r4.y + dln[p].z * r4.z;
              dl_dalpha += dld[p] * (t_hit * t_before - suf_d[p] * inv_oma) + dn * t_before -
                           suf_n[p] * inv_oma + coef * t_before - suf_cw[p] * inv_oma;
              suf_d[p] += t_hit * w;
              suf_n[p] += dn * w;
              suf_w[p] += w;
              suf_cw[p] += coef * w;
              gg[17] += dln[p].x * w; gg[18] += dln[p].y * w; gg[19] += dln[p].z * w;
            }
            if (ST_SMEM) {
              s_ts[lpix + p * PSTEP] = make_float2(t_before, ts.y + dc * w);
            } else {
              suf_c[p] += dc * w;
              T[p] = t_before;
            }
            {  // packed pairs round per component as the scalar FFMAs (x·1 is exact)
              const float2 c2 = __ffma2_rn(make_float2(gcol.x, gcol.y), make_float2(w, w), make_float2(gg[11], gg[12]));
              gg[11] = c2.x; gg[12] = c2.y;
              gg[13] += gcol.z * w;
            }
            if (FAST || raw_alpha <= ALPHA_CLAMP) {
              // dL/dĝ·ĝ = dL/dα·o·ĝ; ray branch: ĝ = exp(−(u²+v²)/2) with
              // u = (s·Bu)/det, v = (s·Bv)/det, det = s·M, so dL/d(s·Bu) = −u·K/det,
              // dL/d(s·Bv) = −v·K/det and dL/ddet = (u²+v²)·K/det (− t·dL/dt/det
              // through t = tn/det).
              const float dg = dl_dalpha * h.ghat;
              gg[14] += dg;
              const float K = dl_dalpha * raw_alpha;  // = dg·o, without waiting for dg
              if (h.ray) {
                const float Ki = K * h.inv_det;
                const float2 guv = __fmul2_rn(make_float2(-h.u, -h.v), make_float2(Ki, Ki));
                float gdet = h.q2 * Ki;
                if (AUX) gdet -= h.t * dl_dt * h.inv_det;
                const float2 sy1 = make_float2(sy_of(p), 1.0f);
                const float2 m0 = __ffma2_rn(make_float2(gdet, gdet), sy1, make_float2(gg[1], gg[2]));
                const float2 m1 = __ffma2_rn(make_float2(guv.x, guv.x), sy1, make_float2(gg[4], gg[5]));
                const float2 m2 = __ffma2_rn(make_float2(guv.y, guv.y), sy1, make_float2(gg[7], gg[8]));
                gg[1] = m0.x; gg[2] = m0.y; gg[4] = m1.x; gg[5] = m1.y; gg[7] = m2.x; gg[8] = m2.y;
                if (AUX) gg[15] += dl_dt * h.inv_det;
              } else {
                const float kk = K * (1.0f / LOWPASS_SIGMA2);
                const float2 sd = __ffma2_rn(make_float2(cp.dx, h.dy), make_float2(kk, kk), make_float2(gg[9], gg[10]));
                gg[9] = sd.x;
                gg[10] = sd.y;
                if (AUX) gg[16] += dl_dt;
              }
            }
          }
          }
          };
          const uint32_t fm = RAYFLAG ? s_msk[k].y : 0u;
          if (fm & FARBIT) walk(std::integral_constant<int, HIT_RAY_FAR>{});
          else if (fm & RAYBIT) walk(std::integral_constant<int, HIT_RAY_OK>{});
          else walk(std::integral_constant<int, HIT_FULL>{});
          // A thread's pixels share sx: the sx moments are sx times the plain sums.
          gg[0] = gg[2] * g.sx; gg[3] = gg[5] * g.sx; gg[6] = gg[8] * g.sx;
        }
        if (__any_sync(FULL, contrib)) {
          float lo16[16];
#pragma unroll
          for (int c = 0; c < 16; ++c) lo16[c] = gg[c];
          const float r = warp_reduce16(lo16);
          if constexpr (DIRECT) {
            // component c sits in lanes 2c and 2c+1: lane 8q gathers 4q..4q+3
            const float r1 = __shfl_down_sync(FULL, r, 2), r2 = __shfl_down_sync(FULL, r, 4);
            const float r3 = __shfl_down_sync(FULL, r, 6);
            if ((lane & 7) == 0) emit4(k, lane >> 3, r, r1, r2, r3);
          } else {
            if (!(lane & 1)) s_part[warp][k][lane >> 1] = r;
          }
          if (AUX) {
            float hi16[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) hi16[c] = gg[16 + c];
            const float r2 = warp_reduce16(hi16);
            if (!(lane & 1)) s_part[warp][k][16 + (lane >> 1)] = r2;
          }
        } else {
          emit_zero(k);
        }
      }
      __syncthreads();
      // Cross-warp sum in fixed warp order, then one vector reduction (or
      // one ordered store) per 4 components.
      for (int w4 = tid; !DIRECT && w4 < kept * NQ; w4 += NT) {
        const int k = w4 / NQ, q4 = w4 % NQ;
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
        for (int ww = 0; ww < NW; ++ww) {
          s0 += s_part[ww][k][4 * q4]; s1 += s_part[ww][k][4 * q4 + 1];
          s2 += s_part[ww][k][4 * q4 + 2]; s3 += s_part[ww][k][4 * q4 + 3];
        }
        emit4(k, q4, s0, s1, s2, s3);
      }
      __syncthreads();
      hi = lo;
    }
    if (!PERSIST) return;
    __syncthreads();
  }
}

// Work of the raster kernels on the last forward, counted by replaying each
// pixel's walk (outside any timed region): one thread per pixel, TS·TS/NPT
// threads per tile. Per pixel, the forward evaluates the hit of every list
// entry whose α-box holds the pixel until the pixel terminates (its last
// contributor when T < 1e-4 at the end, else the whole list); a pair
// contributes when α ≥ 1/255 (the same eval_hit, so the same decisions as
// the forward); the backward evaluates the entries before the pixel's last
// contributor whose box holds it and, with the row-group summary, whose
// summary byte has the pixel's group. out: {forward evaluations,
// contributing pairs, backward evaluations, pixels}.
template <int TS, int PREC>
__global__ void __launch_bounds__(256) k_raster_work(RasterArgs a, unsigned long long* out) {
  constexpr int NP = TS * TS, NT = NP < 256 ? NP : 256;
  __shared__ unsigned long long s_cnt[4];
  if (threadIdx.x < 4) s_cnt[threadIdx.x] = 0ull;
  __syncthreads();
  const int tile = blockIdx.x;
  int v = 0;
  while (v + 1 < a.n_views && tile >= __ldg(&a.views[v + 1].tile_base)) ++v;
  const ViewInfo* V = a.views + v;
  const int tiles_x = __ldg(&V->tiles_x), W = __ldg(&V->width), H = __ldg(&V->height);
  const int lt = tile - __ldg(&V->tile_base);
  const int x0 = (lt % tiles_x) * TS, y0 = (lt / tiles_x) * TS;
  const float f = __ldg(&V->focal), cx = __ldg(&V->cx), cy = __ldg(&V->cy);
  const uint2 range = __ldg(&a.ranges[tile]);
  const uint32_t len = range.y > range.x ? range.y - range.x : 0u;
  unsigned long long fe = 0, co = 0, be = 0, px = 0;
  for (int q = threadIdx.x; q < NP; q += NT) {
    const int x = x0 + q % TS, y = y0 + q / TS;
    if (x >= W || y >= H) continue;
    ++px;
    const long long pix = __ldg(&V->pix_base) + (long long)y * W + x;
    const uint32_t nc = a.out_nc[pix];
    const float Tf = a.out_aux[pix].x;
    const uint32_t stop = Tf < T_TERMINATE ? min(nc, len) : len;
    const float pxc = (float)x + 0.5f, pyc = (float)y + 0.5f;
    const float sx = -((pxc - cx) / f), sy = (pyc - cy) / f;
    const uint32_t gbit = 1u << ((q / TS) >> 2);
    for (uint32_t j = 0; j < stop; ++j) {
      uint32_t item = __ldg(&a.sorted_pairs[range.x + j].y);
      if (a.exp_item != nullptr) item = __ldg(&a.exp_item[item]);
      const float4 bb = load_record_box<PREC>(a.records, item);
      if (!(pxc >= bb.x && pxc <= bb.y && pyc >= bb.z && pyc <= bb.w)) continue;
      ++fe;
      float4 r0, r1, r2, r3;
      load_record4<PREC>(a.records, item, r0, r1, r2, r3);
      stage_offsets(r1, r2, (float)x0 + 0.5f, (float)y0 + 0.5f);
      const ColPart cp = col_part(r0, r1, r2, sx, (float)(x - x0));
      const Hit h = eval_hit(cp, r0, r1, r2, 0.0f, sy, (float)(y - y0));
      const float alpha = fminf(__fmul_rn(r3.w, h.ghat), ALPHA_CLAMP);
      if (!(alpha < ALPHA_SKIP)) ++co;
      if (j < nc && (TS != 16 || a.gmask == nullptr || (__ldg(a.gmask + range.x + j) & gbit))) ++be;
    }
  }
  atomicAdd(&s_cnt[0], fe);
  atomicAdd(&s_cnt[1], co);
  atomicAdd(&s_cnt[2], be);
  atomicAdd(&s_cnt[3], px);
  __syncthreads();
  if (threadIdx.x < 4) atomicAdd(out + threadIdx.x, s_cnt[threadIdx.x]);
}

// ---------------------------------------------------------------------------
// Pixel-compacted raster kernels: 16-pixel tiles, colour-only, persistent (the
// chosen training step). One warp owns a tile and keeps its per-pixel state in
// shared memory; for each staged entry it spreads the pixels of the entry's
// α-box ∩ tile (the only pixels whose α can reach 1/255) over its 32 lanes,
// so lanes do not idle on pixels the entry cannot touch. Entries are
// processed one after another, so each pixel still composites (or is walked
// back) in list order. The hit test and compositing are the same operations
// as in k_raster_fwd / k_raster_bwd: images, final T and contributor indices
// are bit-identical, and gradients equal up to the order of float sums.
constexpr int PX_TP = 256;  // pixels per tile
constexpr int PX_NB = 32;   // staged entries per round: one per lane

// Tile-local pixel rectangle of an α-box ∩ the tile's in-image pixels
// (columns < tw, rows < th), packed x0 | x1 << 8 | y0 << 16 | y1 << 24;
// 0xffffffff when empty. Same pixel decisions as the per-pixel box test.
__device__ __forceinline__ uint32_t px_rect(const float4& b, float bx0, float by0, int tw, int th) {
  const uint32_t cm = span_bits<16>(bx0, b.x, b.y) & ((1u << tw) - 1u);
  const uint32_t rm = span_bits<16>(by0, b.z, b.w) & ((1u << th) - 1u);
  if (!cm || !rm) return 0xffffffffu;
  const uint32_t x0 = (uint32_t)(__ffs(cm) - 1), x1 = 31u - (uint32_t)__clz(cm);
  const uint32_t y0 = (uint32_t)(__ffs(rm) - 1), y1 = 31u - (uint32_t)__clz(rm);
  return x0 | (x1 << 8) | (y0 << 16) | (y1 << 24);
}

struct PxTile {
  int tile;
  uint32_t slot;
  int W, tw, th;
  float bx0, by0;
  long long pbase;  // pixel (x0, y0) of the tile in per-pixel buffers
};

// Takes the next tile from the persistent queue (all lanes); false when done.
// Writes the tile's column and row ray components into s_sx / s_sy exactly
// as tile_geo computes them.
__device__ __forceinline__ bool px_next_tile(const RasterArgs& a, PxTile& t, float* s_sx, float* s_sy) {
  const int lane = threadIdx.x;
  uint32_t slot = 0;
  int tile = 0;
  if (lane == 0) {
    slot = atomicAdd(a.tile_counter, 1u);
    const uint32_t lim = a.tile_limit != nullptr ? *a.tile_limit : (uint32_t)a.total_tiles;
    tile = slot >= lim ? a.total_tiles : (int)(a.tile_order != nullptr ? __ldg(a.tile_order + slot) : slot);
  }
  t.tile = __shfl_sync(FULL, tile, 0);
  t.slot = __shfl_sync(FULL, slot, 0);
  if (t.tile >= a.total_tiles) return false;
  int v = 0;
  while (v + 1 < a.n_views && t.tile >= __ldg(&a.views[v + 1].tile_base)) ++v;
  const ViewInfo* V = a.views + v;
  const int tiles_x = __ldg(&V->tiles_x), H = __ldg(&V->height);
  t.W = __ldg(&V->width);
  const int lt = t.tile - __ldg(&V->tile_base);
  const int x0 = (lt % tiles_x) * 16, y0 = (lt / tiles_x) * 16;
  t.tw = min(16, t.W - x0);
  t.th = min(16, H - y0);
  const float f = __ldg(&V->focal), cx = __ldg(&V->cx), cy = __ldg(&V->cy);
  if (lane < 16) {
    const float pxc = (float)(x0 + lane) + 0.5f;
    s_sx[lane] = -((pxc - cx) / f);
  } else {
    const float pyc = (float)(y0 + lane - 16) + 0.5f;
    s_sy[lane - 16] = (pyc - cy) / f;
  }
  t.bx0 = (float)x0 + 0.5f;
  t.by0 = (float)y0 + 0.5f;
  t.pbase = __ldg(&V->pix_base) + (long long)y0 * t.W + x0;
  return true;
}

// Stages up to 32 entries of [j0, j1): each lane takes one, culls it by its
// α-box (and by an empty row-group summary when gm_mask), and the kept ones are
// compacted in list order into the shared arrays. Returns the number kept.
// In the deterministic backward (s_q given) every entry not kept gets its
// ordered zero partial here.
template <int PREC, bool DET>
__device__ __forceinline__ int px_stage(const RasterArgs& a, const PxTile& t, uint32_t j0, uint32_t j1,
                                        uint32_t rstart, bool use_gm, float4* s_r0, float4* s_r1, float4* s_r2,
                                        float4* s_r3, uint32_t* s_rect, uint32_t* s_j, uint32_t* s_item,
                                        uint32_t* s_q, uint8_t* s_gm) {
  const int lane = threadIdx.x;
  const uint32_t j = j0 + (uint32_t)lane;
  uint32_t item = 0, q = 0, rect = 0xffffffffu;
  uint32_t gm = 0xffu;
  if (j < j1) {
    q = __ldg(&a.sorted_pairs[j].y);
    item = DET ? __ldg(&a.exp_item[q]) : q;
    if (use_gm) gm = __ldg(a.gmask + j);
    if (gm) {
      rect = px_rect(load_record_box<PREC>(a.records, item), t.bx0, t.by0, t.tw, t.th);
      if (use_gm && rect != 0xffffffffu) {  // rows of the 4-row groups with a contributor
        const uint32_t g0 = (uint32_t)(__ffs(gm) - 1), g1 = 31u - (uint32_t)__clz(gm);
        const uint32_t y0 = max((rect >> 16) & 255u, 4u * g0), y1 = min(rect >> 24, 4u * g1 + 3u);
        rect = y0 <= y1 ? (rect & 0xffffu) | (y0 << 16) | (y1 << 24) : 0xffffffffu;
      }
    }
    if (DET && s_q != nullptr && rect == 0xffffffffu) {  // no contribution: an ordered zero partial
      float4* pp = reinterpret_cast<float4*>(a.partials + (size_t)q * GG_STRIDE);
#pragma unroll
      for (int k = 0; k < 4; ++k) pp[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  const bool keep = rect != 0xffffffffu;
  const unsigned bal = __ballot_sync(FULL, keep);
  if (keep) {
    const int sl = __popc(bal & lanemask_lt());
    float4 r0, r1, r2, r3;
    load_record4<PREC>(a.records, item, r0, r1, r2, r3);
    stage_offsets(r1, r2, t.bx0, t.by0);
    s_r0[sl] = r0; s_r1[sl] = r1; s_r2[sl] = r2; s_r3[sl] = r3;
    s_rect[sl] = rect;
    s_j[sl] = j - rstart;
    if (s_item) s_item[sl] = item;
    if (DET && s_q) s_q[sl] = q;
    if (s_gm) s_gm[sl] = (uint8_t)gm;
  }
  __syncwarp();
  return __popc(bal);
}

template <int PREC, bool DET>
__global__ void __launch_bounds__(32) k_raster_fwd_px(RasterArgs a) {
  __shared__ float s_T[PX_TP];
  __shared__ float4 s_c[PX_TP];
  __shared__ uint32_t s_nc[PX_TP];
  __shared__ float s_sx[16], s_sy[16];
  __shared__ float4 s_r0[PX_NB], s_r1[PX_NB], s_r2[PX_NB], s_r3[PX_NB];
  __shared__ uint32_t s_rect[PX_NB], s_j[PX_NB];
  const int lane = threadIdx.x;
  const bool gm_on = a.gmask != nullptr;
  PxTile t;
  while (px_next_tile(a, t, s_sx, s_sy)) {
    const uint2 range = __ldg(&a.ranges[t.tile]);
    // Completion pass of the occlusion cut: continue after the entries pass 1
    // composited, from the pixel state it wrote.
    const bool resume = a.cut_pass == 2;
    uint32_t skip = 0;
    if (resume) {
      skip = a.inc_skip[t.slot];
      if (range.y - range.x < skip) skip = 0;  // list not rebuilt (entry capacity error already flagged)
    }
    int alive = 0;
    uint32_t walk = 0;
    for (int p = lane; p < PX_TP; p += 32) {
      const int ly = p >> 4, lx = p & 15;
      float T = 0.f;  // pixels outside the image count as terminated
      float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
      uint32_t nc = 0;
      if (lx < t.tw && ly < t.th) {
        T = 1.f;
        if (resume) {
          const long long pix = t.pbase + (long long)ly * t.W + lx;
          c = a.out_color[pix];
          T = a.out_aux[pix].x;
          nc = a.out_nc[pix];
        }
        if (!(T < T_TERMINATE)) ++alive;
      }
      s_T[p] = T;
      s_c[p] = c;
      s_nc[p] = nc;
      walk = max(walk, nc);
    }
    alive = __reduce_add_sync(FULL, alive);
    walk = __reduce_max_sync(FULL, walk);
    __syncwarp();
    for (uint32_t base = range.x + skip; base < range.y && alive > 0; base += PX_NB) {
      const int kept = px_stage<PREC, DET>(a, t, base, min(base + (uint32_t)PX_NB, range.y), range.x, false, s_r0,
                                           s_r1, s_r2, s_r3, s_rect, s_j, nullptr, nullptr, nullptr);
      for (int k = 0; k < kept; ++k) {
        const uint32_t rc = s_rect[k];
        const int rx0 = (int)(rc & 255u), rx1 = (int)((rc >> 8) & 255u), ry0 = (int)((rc >> 16) & 255u);
        const int w = rx1 - rx0 + 1, cnt = w * ((int)(rc >> 24) - ry0 + 1);
        const int rw = (4096 + w - 1) / w;  // q / w = (q·rw) >> 12 exactly for q < 256, w <= 16
        const float4 r0 = s_r0[k], r1 = s_r1[k], r2 = s_r2[k], r3 = s_r3[k];
        const uint32_t idx1 = s_j[k] + 1u;
        uint32_t gbits = 0;
        int nd = 0;
        for (int q = lane; q < cnt; q += 32) {
          const int dy = (q * rw) >> 12, ly = ry0 + dy, lx = rx0 + q - dy * w;
          const int p = ly * 16 + lx;
          const float T = s_T[p];
          if (T < T_TERMINATE) continue;
          const ColPart cp = col_part(r0, r1, r2, s_sx[lx], (float)lx);
          const Hit h = eval_hit(cp, r0, r1, r2, 0.0f, s_sy[ly], (float)ly);
          const float alpha = fminf(__fmul_rn(r3.w, h.ghat), ALPHA_CLAMP);
          if (alpha < ALPHA_SKIP) continue;
          const float wt = T * alpha;
          float4 c = s_c[p];
          c.x += r3.x * wt; c.y += r3.y * wt; c.z += r3.z * wt;
          c.w += wt;
          const float Tn = __fmul_rn(T, 1.0f - alpha);
          s_c[p] = c;
          s_T[p] = Tn;
          s_nc[p] = idx1;
          gbits |= 1u << (ly >> 2);
          if (Tn < T_TERMINATE) ++nd;
        }
        const uint32_t gm = __reduce_or_sync(FULL, gbits);
        alive -= __reduce_add_sync(FULL, nd);
        if (gm) walk = idx1;  // entries come in list order: the latest contributor is the deepest
        if (gm_on && lane == 0) a.gmask[range.x + idx1 - 1u] = (uint8_t)gm;
        __syncwarp();
        if (alive <= 0) break;
      }
    }
    for (int p = lane; p < PX_TP; p += 32) {
      const int ly = p >> 4, lx = p & 15;
      if (lx < t.tw && ly < t.th) {
        const long long pix = t.pbase + (long long)ly * t.W + lx;
        a.out_color[pix] = s_c[p];
        a.out_aux[pix].x = s_T[p];
        a.out_nc[pix] = s_nc[p];
      }
    }
    if (lane == 0) {
      if (a.tile_walk != nullptr) a.tile_walk[t.tile] = walk;
      if (a.tile_cut != nullptr) cut_tile_end(a, t.tile, range, alive <= 0, walk);
    }
    __syncwarp();
  }
}

template <int PREC, bool DET>
__global__ void __launch_bounds__(32) k_raster_bwd_px(RasterArgs a) {
  __shared__ float s_T[PX_TP], s_suf[PX_TP];
  __shared__ uint32_t s_nc[PX_TP];
  __shared__ float4 s_dlc[PX_TP];
  __shared__ float s_sx[16], s_sy[16];
  __shared__ float4 s_r0[PX_NB], s_r1[PX_NB], s_r2[PX_NB], s_r3[PX_NB];
  __shared__ uint32_t s_rect[PX_NB], s_j[PX_NB], s_item[PX_NB];
  __shared__ uint32_t s_q[DET ? PX_NB : 1];
  __shared__ uint8_t s_gm[PX_NB];
  const int lane = threadIdx.x;
  const bool use_gm = a.gmask != nullptr;
  PxTile t;
  while (px_next_tile(a, t, s_sx, s_sy)) {
    const uint2 range = __ldg(&a.ranges[t.tile]);
    if (range.y <= range.x) continue;
    uint32_t mx = 0;
    for (int p = lane; p < PX_TP; p += 32) {
      const int ly = p >> 4, lx = p & 15;
      float T = 1.f;
      uint32_t nc = 0;
      float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
      if (lx < t.tw && ly < t.th) {
        const long long pix = t.pbase + (long long)ly * t.W + lx;
        g = a.dl_dcolor[pix];
        T = a.out_aux[pix].x;
        nc = a.out_nc[pix];
        if (g.x == 0.f && g.y == 0.f && g.z == 0.f) nc = 0;  // no loss at the pixel: nothing to walk
      }
      s_T[p] = T;
      s_suf[p] = 0.f;
      s_nc[p] = nc;
      s_dlc[p] = g;
      mx = max(mx, nc);
    }
    const uint32_t maxnc = min(__reduce_max_sync(FULL, mx), range.y - range.x);
    if (DET) {  // entries past the tile's last contributor get zero partials
      for (uint32_t e = range.x + maxnc + (uint32_t)lane; e < range.y; e += 32) {
        float4* pp = reinterpret_cast<float4*>(a.partials + (size_t)__ldg(&a.sorted_pairs[e].y) * GG_STRIDE);
#pragma unroll
        for (int k = 0; k < 4; ++k) pp[k] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    __syncwarp();
    uint32_t hi = range.x + maxnc;
    while (hi > range.x) {
      const uint32_t lo = hi - range.x > (uint32_t)PX_NB ? hi - PX_NB : range.x;
      const int kept = px_stage<PREC, DET>(a, t, lo, hi, range.x, use_gm, s_r0, s_r1, s_r2, s_r3, s_rect, s_j, s_item,
                                           DET ? s_q : nullptr, s_gm);
      for (int k = kept - 1; k >= 0; --k) {
        const uint32_t rc = s_rect[k];
        const int rx0 = (int)(rc & 255u), rx1 = (int)((rc >> 8) & 255u), ry0 = (int)((rc >> 16) & 255u);
        const int w = rx1 - rx0 + 1, cnt = w * ((int)(rc >> 24) - ry0 + 1);
        const int rw = (4096 + w - 1) / w;
        const float4 r0 = s_r0[k], r1 = s_r1[k], r2 = s_r2[k], r3 = s_r3[k];
        const uint32_t cidx = s_j[k];
        const uint32_t gm = s_gm[k];
        float gg[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) gg[c] = 0.f;
        bool contrib = false;
        for (int q = lane; q < cnt; q += 32) {
          const int dy = (q * rw) >> 12, ly = ry0 + dy, lx = rx0 + q - dy * w;
          if (!((gm >> (ly >> 2)) & 1u)) continue;
          const int p = ly * 16 + lx;
          if (cidx >= s_nc[p]) continue;
          const float sx = s_sx[lx], sy = s_sy[ly];
          const ColPart cp = col_part(r0, r1, r2, sx, (float)lx);
          const Hit h = eval_hit(cp, r0, r1, r2, 0.0f, sy, (float)ly);
          const float raw_alpha = __fmul_rn(r3.w, h.ghat);
          const float alpha = fminf(raw_alpha, ALPHA_CLAMP);
          if (alpha < ALPHA_SKIP) continue;
          contrib = true;
          const float inv_oma = rcp_approx(1.0f - alpha);
          const float t_before = s_T[p] * inv_oma;
          const float wt = t_before * alpha;
          const float4 g4 = s_dlc[p];
          const float dc = g4.x * r3.x + g4.y * r3.y + g4.z * r3.z;
          const float suf = s_suf[p];
          const float dl_dalpha = dc * t_before - suf * inv_oma;
          s_suf[p] = suf + dc * wt;
          s_T[p] = t_before;
          gg[11] += g4.x * wt; gg[12] += g4.y * wt; gg[13] += g4.z * wt;
          if (raw_alpha <= ALPHA_CLAMP) {
            const float dg = dl_dalpha * h.ghat;
            gg[14] += dg;
            const float K = dl_dalpha * raw_alpha;  // = dg·o
            if (h.ray) {
              // record moments sum over the pixel ray s = (sx, sy, 1) of the
              // ray-branch adjoints (see k_raster_bwd)
              const float Ki = K * h.inv_det;
              const float gu = -h.u * Ki, gv = -h.v * Ki, gdet = h.q2 * Ki;
              const float2 s2 = make_float2(sx, sy);
              const float2 m0 = __ffma2_rn(make_float2(gdet, gdet), s2, make_float2(gg[0], gg[1]));
              const float2 m1 = __ffma2_rn(make_float2(gu, gu), s2, make_float2(gg[3], gg[4]));
              const float2 m2 = __ffma2_rn(make_float2(gv, gv), s2, make_float2(gg[6], gg[7]));
              gg[0] = m0.x; gg[1] = m0.y; gg[3] = m1.x; gg[4] = m1.y; gg[6] = m2.x; gg[7] = m2.y;
              gg[2] += gdet; gg[5] += gu; gg[8] += gv;
            } else {
              const float kk = K * (1.0f / LOWPASS_SIGMA2);
              const float2 sd = __ffma2_rn(make_float2(cp.dx, h.dy), make_float2(kk, kk), make_float2(gg[9], gg[10]));
              gg[9] = sd.x;
              gg[10] = sd.y;
            }
          }
        }
        __syncwarp();
        if (__any_sync(FULL, contrib)) {
          const float r = warp_reduce16(gg);
          // component c sits in lanes 2c and 2c+1: lane 8q gathers 4q..4q+3
          const float u1 = __shfl_down_sync(FULL, r, 2), u2 = __shfl_down_sync(FULL, r, 4);
          const float u3 = __shfl_down_sync(FULL, r, 6);
          if ((lane & 7) == 0) {
            const int q4 = lane >> 3;
            if (DET) {
              reinterpret_cast<float4*>(a.partials + (size_t)s_q[k] * GG_STRIDE)[q4] = make_float4(r, u1, u2, u3);
            } else if (r != 0.f || u1 != 0.f || u2 != 0.f || u3 != 0.f) {
              red_add_v4(a.grad_geom + (size_t)s_item[k] * GG_STRIDE + 4 * q4, r, u1, u2, u3);
            }
          }
        } else if (DET && lane < 4) {
          reinterpret_cast<float4*>(a.partials + (size_t)s_q[k] * GG_STRIDE)[lane] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
      hi = lo;
    }
    __syncwarp();
  }
}

}  // namespace

// ------------------------------------------------------------- dispatch
// Launch shapes (staging batch, pixels per thread) built per tile size.
// Forward: TS 8 → ppt 1/2 × batch 64/128/256; TS 16 → (64,1) (128,1) (256,1)
// (64,2) (128,2) (64,4) (64,8) (128,8); TS 32 → ppt 2/4 × batch 64/128/256
// and (128,8). Backward without aux losses: TS 8 → (64,1) (64,2) (128,2);
// TS 16 → (64,1) (64,2) (128,2) (64,4) (32,8) (64,8) (128,8); TS 32 → (64,4) (64,8). With aux losses: batch 32 at ppt 1 (TS 8,
// 16) or 4 (TS 32). The backward's per-warp partial buffer NW·BATCH·NG floats
// is static shared memory, which bounds the backward shapes.
template <int TS, int PREC, bool DET, bool PERSIST, bool COLOR, bool MASK, typename F>
bool fwd_shape(int batch, int ppt, F&& f) {
#define GS_FWD(B, P)                                                                   \
  if (batch == B && ppt == P) {                                                        \
    f(k_raster_fwd<TS, B, PREC, DET, PERSIST, P, COLOR, MASK>, TS * TS / P);           \
    return true;                                                                       \
  }
  if constexpr (TS == 8) {
    GS_FWD(64, 1) GS_FWD(128, 1) GS_FWD(256, 1) GS_FWD(64, 2) GS_FWD(128, 2) GS_FWD(256, 2)
  } else if constexpr (TS == 16) {
    GS_FWD(64, 1) GS_FWD(128, 1) GS_FWD(256, 1) GS_FWD(64, 2) GS_FWD(128, 2) GS_FWD(64, 4) GS_FWD(64, 8)
    GS_FWD(128, 8)
  } else {
    GS_FWD(64, 2) GS_FWD(128, 2) GS_FWD(256, 2) GS_FWD(64, 4) GS_FWD(128, 4) GS_FWD(256, 4) GS_FWD(128, 8)
  }
#undef GS_FWD
  return false;
}

template <int TS, int PREC, bool AUX, bool DET, bool PERSIST, bool MASK, typename F>
bool bwd_shape(int batch, int ppt, F&& f) {
#define GS_BWD(B, P)                                                                   \
  if (batch == B && ppt == P) {                                                        \
    f(k_raster_bwd<TS, B, PREC, AUX, DET, PERSIST, P, MASK>, TS * TS / P);             \
    return true;                                                                       \
  }
  if constexpr (AUX) {
    if constexpr (TS == 32) {
      GS_BWD(32, 4)
    } else {
      GS_BWD(32, 1)
    }
  } else if constexpr (TS == 8) {
    GS_BWD(64, 1) GS_BWD(64, 2) GS_BWD(128, 2)
  } else if constexpr (TS == 16) {
    GS_BWD(64, 1) GS_BWD(64, 2) GS_BWD(128, 2) GS_BWD(64, 4) GS_BWD(32, 8) GS_BWD(64, 8) GS_BWD(128, 8)
  } else {
    GS_BWD(64, 4) GS_BWD(64, 8)
  }
#undef GS_BWD
  return false;
}

template <int V>
using IC = std::integral_constant<int, V>;

template <typename G>
bool by_prec(int prec, G&& g) {
  return prec == 0 ? g(IC<0>{}) : prec == 1 ? g(IC<1>{}) : g(IC<2>{});
}

// Calls f(kernel, threads) with the forward kernel of these options, or
// returns false when the combination is not built. Contributor masks exist
// for TS 16 only; the colour-only variant is persistent.
// Launch shape (32, 0) on 16-pixel tiles selects the pixel-compacted kernels,
// which exist for the colour-only persistent passes without contributor
// masks; elsewhere that shape stands for (64, 4) forward and (64, 8) backward.
template <int TS, typename F>
bool fwd_kernel(int prec, int batch, int ppt, bool det, bool persistent, bool color, bool mask, F&& f) {
  if constexpr (TS == 16) {
    if (ppt == 0 && batch == PX_NB) {
      if (color && persistent && !mask) {
        return by_prec(prec, [&](auto pc) -> bool {
          constexpr int P = decltype(pc)::value;
          if (det) f(k_raster_fwd_px<P, true>, 32);
          else f(k_raster_fwd_px<P, false>, 32);
          return true;
        });
      }
      batch = 64;
      ppt = 4;
    }
  }
  return by_prec(prec, [&](auto pc) -> bool {
    constexpr int P = decltype(pc)::value;
    if (color) {
      if (!persistent) return false;
      if (mask) {
        if constexpr (TS == 16) {
          return det ? fwd_shape<TS, P, true, true, true, true>(batch, ppt, f)
                     : fwd_shape<TS, P, false, true, true, true>(batch, ppt, f);
        } else {
          return false;
        }
      }
      return det ? fwd_shape<TS, P, true, true, true, false>(batch, ppt, f)
                 : fwd_shape<TS, P, false, true, true, false>(batch, ppt, f);
    }
    if (det) return persistent ? fwd_shape<TS, P, true, true, false, false>(batch, ppt, f)
                               : fwd_shape<TS, P, true, false, false, false>(batch, ppt, f);
    return persistent ? fwd_shape<TS, P, false, true, false, false>(batch, ppt, f)
                      : fwd_shape<TS, P, false, false, false, false>(batch, ppt, f);
  });
}

template <int TS, typename F>
bool bwd_kernel(int prec, bool aux, int batch, int ppt, bool det, bool persistent, bool mask, F&& f) {
  if constexpr (TS == 16) {
    if (ppt == 0 && batch == PX_NB) {
      if (!aux && persistent && !mask) {
        return by_prec(prec, [&](auto pc) -> bool {
          constexpr int P = decltype(pc)::value;
          if (det) f(k_raster_bwd_px<P, true>, 32);
          else f(k_raster_bwd_px<P, false>, 32);
          return true;
        });
      }
      batch = 64;
      ppt = 8;
    }
  }
  if (aux) {  // one shape per tile size with aux losses
    batch = 32;
    ppt = TS == 32 ? 4 : 1;
  }
  return by_prec(prec, [&](auto pc) -> bool {
    constexpr int P = decltype(pc)::value;
    if (aux) {
      if (mask) return false;
      if (det) return persistent ? bwd_shape<TS, P, true, true, true, false>(batch, ppt, f)
                                 : bwd_shape<TS, P, true, true, false, false>(batch, ppt, f);
      return persistent ? bwd_shape<TS, P, true, false, true, false>(batch, ppt, f)
                        : bwd_shape<TS, P, true, false, false, false>(batch, ppt, f);
    }
    if (mask) {
      if constexpr (TS == 16) {
        if (!persistent) return false;
        return det ? bwd_shape<TS, P, false, true, true, true>(batch, ppt, f)
                   : bwd_shape<TS, P, false, false, true, true>(batch, ppt, f);
      } else {
        return false;
      }
    }
    if (det) return persistent ? bwd_shape<TS, P, false, true, true, false>(batch, ppt, f)
                               : bwd_shape<TS, P, false, true, false, false>(batch, ppt, f);
    return persistent ? bwd_shape<TS, P, false, false, true, false>(batch, ppt, f)
                      : bwd_shape<TS, P, false, false, false, false>(batch, ppt, f);
  });
}

template <typename K>
int occupancy_of(K kernel, int threads) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, 0) != cudaSuccess) return 1;
  return n < 1 ? 1 : n;
}

template <int TS>
int raster_fwd_occupancy_t(int prec, int batch, int ppt, bool det, bool color, bool mask) {
  int n = 1;
  fwd_kernel<TS>(prec, batch, ppt, det, true, color, mask, [&](auto k, int threads) { n = occupancy_of(k, threads); });
  return n;
}

template <int TS>
int raster_bwd_occupancy_t(int prec, bool aux, int ppt, int batch, bool det, bool mask) {
  int n = 1;
  bwd_kernel<TS>(prec, aux, batch, ppt, det, true, mask, [&](auto k, int threads) { n = occupancy_of(k, threads); });
  return n;
}

template <int TS>
int launch_raster_fwd_t(const RasterArgs& a, int prec, int batch, int ppt, bool det, bool persistent, bool color,
                        int grid, cudaStream_t st) {
  if (a.total_tiles == 0) return 0;
  const bool mask = color && a.mask != nullptr;
  const bool ok = fwd_kernel<TS>(prec, batch, ppt, det, persistent, color, mask,
                                 [&](auto k, int threads) { k<<<grid, threads, 0, st>>>(a); });
  if (!ok) return (int)cudaErrorInvalidValue;
  return (int)cudaGetLastError();
}

template <int TS>
int launch_raster_bwd_t(const RasterArgs& a, int prec, bool aux, int ppt, int batch, bool det, bool persistent,
                        int grid, cudaStream_t st) {
  if (a.total_tiles == 0) return 0;
  const bool mask = !aux && a.mask != nullptr;
  const bool ok = bwd_kernel<TS>(prec, aux, batch, ppt, det, persistent, mask,
                                 [&](auto k, int threads) { k<<<grid, threads, 0, st>>>(a); });
  if (!ok) return (int)cudaErrorInvalidValue;
  return (int)cudaGetLastError();
}

// Explicit instantiation of one tile size's launchers (one translation unit each).
#define GS_RASTER_INSTANTIATE(TS)                                                                             \
  template int raster_fwd_occupancy_t<TS>(int, int, int, bool, bool, bool);                                  \
  template int raster_bwd_occupancy_t<TS>(int, bool, int, int, bool, bool);                                  \
  template int launch_raster_fwd_t<TS>(const RasterArgs&, int, int, int, bool, bool, bool, int, cudaStream_t); \
  template int launch_raster_bwd_t<TS>(const RasterArgs&, int, bool, int, int, bool, bool, int, cudaStream_t);

}  // namespace gs
