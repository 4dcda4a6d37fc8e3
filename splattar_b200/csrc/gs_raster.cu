// Tile rasterizers: forward front-to-back compositing and its adjoint.
//
// Forward: crates/gs-kernels/src/shaders/rasterize_fwd.wgsl:20-85 with the hit
// test of raster_common.wgsl:69-95. One CTA of 256 threads per 16×16 tile,
// one pixel per thread; the tile's depth-sorted entries are staged in shared
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
// then across the CTA's 8 warps in a fixed order, then either added to the
// per-surfel accumulator with one vector reduction per 4 components (default)
// or stored per entry for an ordered reduction (deterministic mode).
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

// The part of the hit test that depends on the pixel column only: a thread's
// pixels share sx, so det, u·det and v·det are one FMA per pixel from these
// partial sums, and the screen-space distance needs dy alone.
struct ColPart {
  float det0, un0, vn0, dx, dx2;
};
__device__ __forceinline__ ColPart col_part(const float4& r0, const float4& r1, const float4& r2, float sx,
                                            float pxc) {
  ColPart c;
  c.det0 = fmaf(r0.x, sx, r0.z);
  c.un0 = fmaf(r1.x, sx, r1.z);
  c.vn0 = fmaf(r2.x, sx, r2.z);
  c.dx = __fsub_rn(pxc, r1.w);
  c.dx2 = __fmul_rn(c.dx, c.dx);
  return c;
}

// raster_common.wgsl:69-95 on the record parameterisation, branch-free.
// Written with explicit rounding intrinsics so the forward and backward
// kernels compute bit-identical alphas. When the ray branch is unavailable
// (|det| ≤ 1e-12 or t ≤ near) q_ray is +inf and u, v, t are unused.
// q2 = u² + v² (= 2·q_ray) is kept for the backward.
__device__ __forceinline__ Hit eval_hit(const ColPart& c, const float4& r0, const float4& r1, const float4& r2,
                                        float depth, float sy, float pyc) {
  Hit h;
  const float det = fmaf(r0.y, sy, c.det0);
  const float inv = rcp_approx(det);
  const float u = __fmul_rn(fmaf(r1.y, sy, c.un0), inv);
  const float v = __fmul_rn(fmaf(r2.y, sy, c.vn0), inv);
  const float t = __fmul_rn(r0.w, inv);
  const bool ray_ok = fabsf(det) > 1e-12f && t > NEAR_DEPTH;
  h.q2 = fmaf(u, u, __fmul_rn(v, v));
  const float qr = ray_ok ? __fmul_rn(0.5f, h.q2) : __int_as_float(0x7f800000);
  h.dy = __fsub_rn(pyc, r2.w);
  const float qs = fmaf(h.dy, h.dy, c.dx2);  // (dx²+dy²)/(2σ²) with σ² = 0.5
  h.ray = qr <= qs;
  const float q = h.ray ? qr : qs;
  h.u = u; h.v = v; h.inv_det = inv;
  h.t = h.ray ? t : depth;
  h.ghat = __expf(-q);
  return h;
}

// Tile geometry for a CTA working on `tile` with PPT vertically adjacent
// pixels per thread: thread t owns column t & 15 and rows (t >> 4)·PPT + p,
// so each warp covers a compact 16 × (2·PPT) block.
template <int PPT>
struct TileGeo {
  int W, H;
  long long row0;               // pix_base + y(p=0)·W + x
  float pxc, sx;
  float pyc[PPT], sy[PPT];
  bool inside[PPT];
  float bx0, bx1, by0, by1;     // pixel-centre extent of the tile's in-image pixels
};

template <int PPT>
__device__ __forceinline__ TileGeo<PPT> tile_geo(const RasterArgs& a, int tile) {
  TileGeo<PPT> g;
  int v = 0;
  while (v + 1 < a.n_views && tile >= __ldg(&a.views[v + 1].tile_base)) ++v;
  const ViewInfo* V = a.views + v;
  const int tiles_x = __ldg(&V->tiles_x);
  g.W = __ldg(&V->width);
  g.H = __ldg(&V->height);
  const int lt = tile - __ldg(&V->tile_base);
  const int x0 = (lt % tiles_x) * TILE, y0 = (lt / tiles_x) * TILE;
  const int x = x0 + (threadIdx.x & 15), yb = y0 + (threadIdx.x >> 4) * PPT;
  const float f = __ldg(&V->focal), cx = __ldg(&V->cx), cy = __ldg(&V->cy);
  g.pxc = (float)x + 0.5f;
  g.sx = -((g.pxc - cx) / f);  // s = −d
#pragma unroll
  for (int p = 0; p < PPT; ++p) {
    g.pyc[p] = (float)(yb + p) + 0.5f;
    g.sy[p] = (g.pyc[p] - cy) / f;
    g.inside[p] = x < g.W && yb + p < g.H;
  }
  g.row0 = __ldg(&V->pix_base) + (long long)yb * g.W + x;
  g.bx0 = (float)x0 + 0.5f;
  g.bx1 = (float)(min(x0 + TILE, g.W) - 1) + 0.5f;
  g.by0 = (float)y0 + 0.5f;
  g.by1 = (float)(min(y0 + TILE, g.H) - 1) + 0.5f;
  return g;
}

template <int PPT>
__device__ __forceinline__ bool box_hits_tile(const float4& b, const TileGeo<PPT>& g) {
  return b.x <= g.bx1 && b.y >= g.bx0 && b.z <= g.by1 && b.w >= g.by0;
}
__device__ __forceinline__ bool box_has_pixel(const float4& b, float pxc, float pyc) {
  return pxc >= b.x && pxc <= b.y && pyc >= b.z && pyc <= b.w;
}

// Compaction of the staged batch: returns this thread's slot among the kept
// entries (valid when keep) and the number kept. Order is preserved.
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

// COLOR: colour, alpha and final transmittance only (the training step's
// loss reads nothing else); depth and normal are neither accumulated nor
// written.
template <int BATCH, int PREC, bool DET, bool PERSIST, int PPT, bool COLOR = false, bool MASK = false>
__global__ void __launch_bounds__(256 / PPT) k_raster_fwd(RasterArgs a) {
  static_assert(!MASK || COLOR, "contributor masks belong to the colour-only variant");
  constexpr int NT = 256 / PPT, NW = NT / 32;
  static_assert(BATCH <= NT, "one staging pass per batch");
  __shared__ float4 s_r0[BATCH], s_r1[BATCH], s_r2[BATCH], s_r3[BATCH], s_bb[BATCH];
  __shared__ float4 s_r4[COLOR ? 1 : BATCH];
  __shared__ int s_j[BATCH];
  __shared__ int s_wcount[NW];
  __shared__ int s_tile;
  const int tid = threadIdx.x;
  int tile = blockIdx.x;
  for (;;) {
    if (PERSIST) {
      if (tid == 0) s_tile = (int)atomicAdd(a.tile_counter, 1u);
      __syncthreads();
      tile = s_tile;
      if (tile >= a.total_tiles) return;
    }
    const TileGeo<PPT> g = tile_geo<PPT>(a, tile);
    const uint2 range = __ldg(&a.ranges[tile]);
    float T[PPT], cr[PPT], cg[PPT], cb[PPT], aa[PPT], ad[PPT], nx[PPT], ny[PPT], nz[PPT];
    uint32_t nc[PPT];
    bool done[PPT];
    bool tdone = true;
    // Stored-state contributor masks (colour-only variant): the word being
    // filled and its index, per pixel.
    uint32_t mw[PPT];
    int mi[PPT];
    constexpr bool masks = MASK;
    const size_t mbase = masks ? (size_t)__ldg(&a.mask_off[tile]) * 256 : 0;
    const int mpix = ((tid >> 4) * PPT) * TILE + (tid & 15);  // pixel p is mpix + p·TILE
#pragma unroll
    for (int p = 0; p < PPT; ++p) {
      T[p] = 1.f; cr[p] = cg[p] = cb[p] = aa[p] = ad[p] = nx[p] = ny[p] = nz[p] = 0.f;
      nc[p] = 0;
      done[p] = !g.inside[p];
      tdone &= done[p];
      mw[p] = 0u;
      mi[p] = 0;
    }
    for (uint32_t base = range.x; base < range.y; base += BATCH) {
      if (__syncthreads_count(tdone) == NT) break;
      const int count = (int)min((uint32_t)BATCH, range.y - base);
      bool keep = false;
      uint32_t item = 0;
      float4 bb = make_float4(0.f, 0.f, 0.f, 0.f);
      if (tid < count) {
        item = __ldg(&a.sorted_pairs[base + tid].y);
        if (DET) item = __ldg(&a.exp_item[item]);
        bb = load_record_box<PREC>(a.records, item);
        keep = box_hits_tile(bb, g);
      }
      int kept;
      const int slot = compact_slot<NW>(keep, s_wcount, kept);
      if (keep) {
        float4 r0, r1, r2, r3, r4;
        load_record<PREC>(a.records, item, r0, r1, r2, r3, r4);
        s_r0[slot] = r0; s_r1[slot] = r1; s_r2[slot] = r2; s_r3[slot] = r3;
        if (!COLOR) s_r4[slot] = r4;
        s_bb[slot] = bb;
        s_j[slot] = tid;
      }
      __syncthreads();
      if (!tdone) {
        for (int k = 0; k < kept; ++k) {
          const float4 bbk = s_bb[k];
          if (g.pxc < bbk.x || g.pxc > bbk.y) continue;
          const float4 r0 = s_r0[k], r1 = s_r1[k], r2 = s_r2[k];
          const float4 r3 = s_r3[k];
          const float4 r4 = COLOR ? make_float4(0.f, 0.f, 0.f, 0.f) : s_r4[k];
          const uint32_t idx1 = base - range.x + (uint32_t)s_j[k] + 1u;
          const ColPart cp = col_part(r0, r1, r2, g.sx, g.pxc);
#pragma unroll
          for (int p = 0; p < PPT; ++p) {
            if (done[p] || g.pyc[p] < bbk.z || g.pyc[p] > bbk.w) continue;
            const Hit h = eval_hit(cp, r0, r1, r2, r4.w, g.sy[p], g.pyc[p]);
            const float alpha = fminf(__fmul_rn(r3.w, h.ghat), ALPHA_CLAMP);
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
            if (masks) {
              const uint32_t cidx = idx1 - 1u;
              const int w = (int)(cidx >> 5);
              if (w != mi[p]) {  // close the current word, zero the words skipped
                uint32_t* m = a.mask + mbase + mpix + p * TILE;
                m[(size_t)mi[p] * 256] = mw[p];
                for (int z = mi[p] + 1; z < w; ++z) m[(size_t)z * 256] = 0u;
                mi[p] = w;
                mw[p] = 0u;
              }
              mw[p] |= 1u << (cidx & 31u);
            }
            if (T[p] < T_TERMINATE) done[p] = true;
          }
          bool all = true;
#pragma unroll
          for (int p = 0; p < PPT; ++p) all &= done[p];
          if (all) { tdone = true; break; }
        }
      }
    }
#pragma unroll
    for (int p = 0; p < PPT; ++p) {
      if (!g.inside[p]) continue;
      const long long pix = g.row0 + (long long)p * g.W;
      a.out_color[pix] = make_float4(cr[p], cg[p], cb[p], aa[p]);
      if (masks && nc[p] > 0) a.mask[mbase + mpix + p * TILE + (size_t)mi[p] * 256] = mw[p];
      if (COLOR) {
        a.out_aux[pix].x = T[p];
      } else {
        a.out_aux[pix] = make_float4(T[p], ad[p], 0.f, 0.f);
        a.out_normal[pix] = make_float4(nx[p], ny[p], nz[p], 0.f);
      }
      a.out_nc[pix] = nc[p];
    }
    if (!PERSIST) return;
    __syncthreads();
  }
}

template <int BATCH, int PREC, bool AUX, bool DET, bool PERSIST, int PPT, bool MASK = false>
__global__ void __launch_bounds__(256 / PPT) k_raster_bwd(RasterArgs a) {
  static_assert(!MASK || !AUX, "contributor masks cover the colour-only backward");
  constexpr int NT = 256 / PPT, NW = NT / 32;
  constexpr int NG = AUX ? 32 : 16;  // reduced components per entry (AUX: 20 used)
  constexpr int NQ = AUX ? 5 : 4;    // float4 groups per entry written out
  static_assert(BATCH <= NT, "one staging pass per batch");
  __shared__ float4 s_r0[BATCH], s_r1[BATCH], s_r2[BATCH], s_r3[BATCH], s_bb[BATCH];
  __shared__ float4 s_r4[AUX ? BATCH : 1];
  __shared__ uint32_t s_item[BATCH];
  __shared__ uint32_t s_q[DET ? BATCH : 1];
  __shared__ int s_j[BATCH];
  __shared__ float s_part[NW][BATCH][NG];
  __shared__ int s_wcount[NW];
  __shared__ int s_tile, s_maxnc;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int tile = blockIdx.x;
  for (;;) {
    if (PERSIST) {
      if (tid == 0) s_tile = (int)atomicAdd(a.tile_counter, 1u);
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
    const TileGeo<PPT> g = tile_geo<PPT>(a, tile);
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
        const long long pix = g.row0 + (long long)p * g.W;
        const float4 gc = a.dl_dcolor[pix];
        dlc[p] = make_float3(gc.x, gc.y, gc.z);
        const float4 aux = a.out_aux[pix];
        T[p] = aux.x;
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
    }
    // Entries at or past this warp's last contributor are skipped warp-wide.
    const uint32_t warp_maxnc = __reduce_max_sync(FULL, my_max);
    if (tid == 0) s_maxnc = 0;
    __syncthreads();
    if (my_max) atomicMax(&s_maxnc, (int)my_max);
    __syncthreads();
    const uint32_t maxnc = min((uint32_t)s_maxnc, range.y - range.x);
    // Stored-state mode: contributor masks written by the forward; the word
    // cached per pixel and its index (list positions are walked downwards).
    constexpr bool masks = MASK;
    const size_t mbase = masks ? (size_t)__ldg(&a.mask_off[tile]) * 256 : 0;
    const int mpix = ((tid >> 4) * PPT) * TILE + (tid & 15);
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
      bool keep = false;
      uint32_t item = 0, q = 0;
      float4 bb = make_float4(0.f, 0.f, 0.f, 0.f);
      if (tid < count) {
        item = __ldg(&a.sorted_pairs[lo + tid].y);
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
      int kept;
      const int slot = compact_slot<NW>(keep, s_wcount, kept);
      if (keep) {
        float4 r0, r1, r2, r3, r4;
        load_record<PREC>(a.records, item, r0, r1, r2, r3, r4);
        s_r0[slot] = r0; s_r1[slot] = r1; s_r2[slot] = r2; s_r3[slot] = r3;
        if (AUX) s_r4[slot] = r4;
        s_bb[slot] = bb;
        s_item[slot] = item;
        if (DET) s_q[slot] = q;
        s_j[slot] = tid;
      }
      __syncthreads();
      for (int k = kept - 1; k >= 0; --k) {
        const uint32_t cidx = lo - range.x + (uint32_t)s_j[k];
        if (cidx >= warp_maxnc) {
          if (lane < 16) s_part[warp][k][lane] = 0.f;
          if (AUX && lane >= 16) s_part[warp][k][lane] = 0.f;
          continue;
        }
        bool bit[PPT];
        bool anybit = false;
        if (masks) {
#pragma unroll
          for (int p = 0; p < PPT; ++p) {
            bit[p] = false;
            if (cidx < nc[p]) {
              const int w = (int)(cidx >> 5);
              if (w != cw[p]) {
                cw[p] = w;
                cm[p] = __ldg(a.mask + mbase + mpix + p * TILE + (size_t)w * 256);
              }
              bit[p] = (cm[p] >> (cidx & 31u)) & 1u;
              anybit |= bit[p];
            }
          }
          if (!__any_sync(FULL, anybit)) {  // no pixel of this warp composited the entry
            if (lane < 16) s_part[warp][k][lane] = 0.f;
            continue;
          }
        }
        const float4 bbk = s_bb[k];
        float gg[NG];
#pragma unroll
        for (int c = 0; c < NG; ++c) gg[c] = 0.f;
        bool contrib = false;
        if (masks ? anybit : (g.pxc >= bbk.x && g.pxc <= bbk.y)) {
          const float4 r0 = s_r0[k], r1 = s_r1[k], r2 = s_r2[k], r3 = s_r3[k];
          float4 r4 = make_float4(0.f, 0.f, 0.f, 0.f);
          float depth = 0.f;  // feeds t in the screen branch, used by aux terms alone
          if (AUX) { r4 = s_r4[k]; depth = r4.w; }
          const ColPart cp = col_part(r0, r1, r2, g.sx, g.pxc);
#pragma unroll
          for (int p = 0; p < PPT; ++p) {
            if (masks ? !bit[p] : (!(cidx < nc[p]) || g.pyc[p] < bbk.z || g.pyc[p] > bbk.w)) continue;
            const Hit h = eval_hit(cp, r0, r1, r2, depth, g.sy[p], g.pyc[p]);
            const float raw_alpha = __fmul_rn(r3.w, h.ghat);
            const float alpha = fminf(raw_alpha, ALPHA_CLAMP);
            if (alpha < ALPHA_SKIP) continue;
            contrib = true;
            const float inv_oma = rcp_approx(1.0f - alpha);
            const float t_before = T[p] * inv_oma;
            const float w = t_before * alpha;
            const float dc = dlc[p].x * r3.x + dlc[p].y * r3.y + dlc[p].z * r3.z;
            float dl_dalpha = dc * t_before - suf_c[p] * inv_oma;
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
            suf_c[p] += dc * w;
            T[p] = t_before;
            gg[11] += dlc[p].x * w; gg[12] += dlc[p].y * w; gg[13] += dlc[p].z * w;
            if (raw_alpha <= ALPHA_CLAMP) {
              // dL/dĝ·ĝ = dL/dα·o·ĝ; ray branch: ĝ = exp(−(u²+v²)/2) with
              // u = (s·Bu)/det, v = (s·Bv)/det, det = s·M, so dL/d(s·Bu) = −u·K/det,
              // dL/d(s·Bv) = −v·K/det and dL/ddet = (u²+v²)·K/det (− t·dL/dt/det
              // through t = tn/det).
              const float dg = dl_dalpha * h.ghat;
              gg[14] += dg;
              const float K = dg * r3.w;
              if (h.ray) {
                const float Ki = K * h.inv_det;
                const float gun = -h.u * Ki, gvn = -h.v * Ki;
                float gdet = h.q2 * Ki;
                if (AUX) gdet -= h.t * dl_dt * h.inv_det;
                gg[1] += gdet * g.sy[p]; gg[2] += gdet;
                gg[4] += gun * g.sy[p]; gg[5] += gun;
                gg[7] += gvn * g.sy[p]; gg[8] += gvn;
                if (AUX) gg[15] += dl_dt * h.inv_det;
              } else {
                const float kk = K * (1.0f / LOWPASS_SIGMA2);
                gg[9] += cp.dx * kk;
                gg[10] += h.dy * kk;
                if (AUX) gg[16] += dl_dt;
              }
            }
          }
          // A thread's pixels share sx: the sx moments are sx times the plain sums.
          gg[0] = gg[2] * g.sx; gg[3] = gg[5] * g.sx; gg[6] = gg[8] * g.sx;
        }
        if (__any_sync(FULL, contrib)) {
          float lo16[16];
#pragma unroll
          for (int c = 0; c < 16; ++c) lo16[c] = gg[c];
          const float r = warp_reduce16(lo16);
          if (!(lane & 1)) s_part[warp][k][lane >> 1] = r;
          if (AUX) {
            float hi16[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) hi16[c] = gg[16 + c];
            const float r2 = warp_reduce16(hi16);
            if (!(lane & 1)) s_part[warp][k][16 + (lane >> 1)] = r2;
          }
        } else {
          if (lane < 16) s_part[warp][k][lane] = 0.f;
          if (AUX && lane >= 16) s_part[warp][k][lane] = 0.f;
        }
      }
      __syncthreads();
      // Cross-warp sum in fixed warp order, then one vector reduction (or
      // one ordered store) per 4 components.
      for (int w4 = tid; w4 < kept * NQ; w4 += NT) {
        const int k = w4 / NQ, q4 = w4 % NQ;
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
        for (int ww = 0; ww < NW; ++ww) {
          s0 += s_part[ww][k][4 * q4]; s1 += s_part[ww][k][4 * q4 + 1];
          s2 += s_part[ww][k][4 * q4 + 2]; s3 += s_part[ww][k][4 * q4 + 3];
        }
        if (DET) {
          reinterpret_cast<float4*>(a.partials + (size_t)s_q[k] * GG_STRIDE)[q4] = make_float4(s0, s1, s2, s3);
        } else if (s0 != 0.f || s1 != 0.f || s2 != 0.f || s3 != 0.f) {
          red_add_v4(a.grad_geom + (size_t)s_item[k] * GG_STRIDE + 4 * q4, s0, s1, s2, s3);
        }
      }
      __syncthreads();
      hi = lo;
    }
    if (!PERSIST) return;
    __syncthreads();
  }
}

// ------------------------------------------------------------- launchers
// Forward variants: (pixels per thread, staging batch) ∈ {(1, 64), (1, 128),
// (1, 256), (2, 64), (2, 128)}; `batch` selects one, `ppt` the pixel split.
// Backward: two pixels per thread and 128-entry batches without aux
// losses; one pixel per thread and 32-entry batches with aux losses (the
// per-warp partial buffer is NW·BATCH·NG floats of static shared memory).
template <int PREC, bool DET, bool PERSIST, bool COLOR = false, bool MASK = false>
void fwd_dispatch(const RasterArgs& a, int batch, int ppt, int grid, cudaStream_t st) {
  if (ppt == 4) {
    k_raster_fwd<64, PREC, DET, PERSIST, 4, COLOR, MASK><<<grid, 64, 0, st>>>(a);
  } else if (ppt == 2) {
    if (batch == 64) k_raster_fwd<64, PREC, DET, PERSIST, 2, COLOR, MASK><<<grid, 128, 0, st>>>(a);
    else k_raster_fwd<128, PREC, DET, PERSIST, 2, COLOR, MASK><<<grid, 128, 0, st>>>(a);
  } else {
    if (batch == 64) k_raster_fwd<64, PREC, DET, PERSIST, 1, COLOR, MASK><<<grid, 256, 0, st>>>(a);
    else if (batch == 256) k_raster_fwd<256, PREC, DET, PERSIST, 1, COLOR, MASK><<<grid, 256, 0, st>>>(a);
    else k_raster_fwd<128, PREC, DET, PERSIST, 1, COLOR, MASK><<<grid, 256, 0, st>>>(a);
  }
}

// Backward variants without aux losses: (pixels per thread, batch) ∈
// {(1, 64), (2, 64), (2, 128)}; with aux losses (1, 32).
template <int PREC, bool AUX, bool DET, bool PERSIST, bool MASK = false>
void bwd_dispatch(const RasterArgs& a, int ppt, int batch, int grid, cudaStream_t st) {
  if constexpr (AUX) {
    k_raster_bwd<32, PREC, true, DET, PERSIST, 1><<<grid, 256, 0, st>>>(a);
  } else {
    if (ppt == 4) k_raster_bwd<64, PREC, false, DET, PERSIST, 4, MASK><<<grid, 64, 0, st>>>(a);
    else if (ppt == 1) k_raster_bwd<64, PREC, false, DET, PERSIST, 1, MASK><<<grid, 256, 0, st>>>(a);
    else if (batch == 64) k_raster_bwd<64, PREC, false, DET, PERSIST, 2, MASK><<<grid, 128, 0, st>>>(a);
    else k_raster_bwd<128, PREC, false, DET, PERSIST, 2, MASK><<<grid, 128, 0, st>>>(a);
  }
}

template <typename K>
int occ(K kernel, int threads) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, 0) != cudaSuccess) return 1;
  return n < 1 ? 1 : n;
}

}  // namespace

int raster_fwd_occupancy(int prec, int batch, int ppt, bool det, bool color, bool mask) {
#define GS_OC(B, P, D, PPT, NT) (mask ? occ(k_raster_fwd<B, P, D, true, PPT, true, true>, NT)  \
                                 : color ? occ(k_raster_fwd<B, P, D, true, PPT, true>, NT) \
                                         : occ(k_raster_fwd<B, P, D, true, PPT, false>, NT))
#define GS_O1(B, P) (det ? GS_OC(B, P, true, 1, 256) : GS_OC(B, P, false, 1, 256))
#define GS_O2(B, P) (det ? GS_OC(B, P, true, 2, 128) : GS_OC(B, P, false, 2, 128))
#define GS_O4(P) (det ? GS_OC(64, P, true, 4, 64) : GS_OC(64, P, false, 4, 64))
#define GS_OB(P) (ppt == 4 ? GS_O4(P) : ppt == 2 ? (batch == 64 ? GS_O2(64, P) : GS_O2(128, P)) \
                           : (batch == 64 ? GS_O1(64, P) : (batch == 256 ? GS_O1(256, P) : GS_O1(128, P))))
  return prec == 0 ? GS_OB(0) : (prec == 1 ? GS_OB(1) : GS_OB(2));
#undef GS_OB
#undef GS_O4
#undef GS_O2
#undef GS_O1
#undef GS_OC
}

int raster_bwd_occupancy(int prec, bool aux, int ppt, int batch, bool det, bool mask) {
#define GS_OM(P, D, M) (ppt == 4 ? occ(k_raster_bwd<64, P, false, D, true, 4, M>, 64)                \
                         : ppt == 1 ? occ(k_raster_bwd<64, P, false, D, true, 1, M>, 256)               \
                                     : (batch == 64 ? occ(k_raster_bwd<64, P, false, D, true, 2, M>, 128) \
                                                    : occ(k_raster_bwd<128, P, false, D, true, 2, M>, 128)))
#define GS_OV(P, D) (aux ? occ(k_raster_bwd<32, P, true, D, true, 1>, 256) \
                         : (mask ? GS_OM(P, D, true) : GS_OM(P, D, false)))
#define GS_O2(P) (det ? GS_OV(P, true) : GS_OV(P, false))
  return prec == 0 ? GS_O2(0) : (prec == 1 ? GS_O2(1) : GS_O2(2));
#undef GS_O2
#undef GS_OV
#undef GS_OM
}

int launch_raster_fwd(const RasterArgs& a, int prec, int batch, int ppt, bool det, bool persistent, bool color,
                      int grid, cudaStream_t st) {
  if (a.total_tiles == 0) return 0;
  if (color && !persistent) return (int)cudaErrorInvalidValue;  // the colour-only variant is persistent
  const bool mask = color && a.mask != nullptr;
#define GS_F(P, D, S) fwd_dispatch<P, D, S>(a, batch, ppt, grid, st)
#define GS_FC(P, D) \
  if (mask) fwd_dispatch<P, D, true, true, true>(a, batch, ppt, grid, st); \
  else fwd_dispatch<P, D, true, true>(a, batch, ppt, grid, st);
#define GS_F2(P)                                   \
  if (det) { if (color) { GS_FC(P, true) } else if (persistent) GS_F(P, true, true); else GS_F(P, true, false); } \
  else { if (color) { GS_FC(P, false) } else if (persistent) GS_F(P, false, true); else GS_F(P, false, false); }
  if (prec == 0) { GS_F2(0) } else if (prec == 1) { GS_F2(1) } else { GS_F2(2) }
#undef GS_F2
#undef GS_FC
#undef GS_F
  return (int)cudaGetLastError();
}

int launch_raster_bwd(const RasterArgs& a, int prec, bool aux, int ppt, int batch, bool det, bool persistent, int grid,
                      cudaStream_t st) {
  if (a.total_tiles == 0) return 0;
  const bool mask = !aux && a.mask != nullptr;
#define GS_B(P, X, D, S)                                                                  \
  do {                                                                                    \
    if (mask) bwd_dispatch<P, X, D, S, (!X && S)>(a, ppt, batch, grid, st);               \
    else bwd_dispatch<P, X, D, S>(a, ppt, batch, grid, st);                               \
  } while (0)
#define GS_B3(P, X)                                \
  if (det) { if (persistent) GS_B(P, X, true, true); else GS_B(P, X, true, false); } \
  else { if (persistent) GS_B(P, X, false, true); else GS_B(P, X, false, false); }
#define GS_B2(P) if (aux) { GS_B3(P, true) } else { GS_B3(P, false) }
  if (prec == 0) { GS_B2(0) } else if (prec == 1) { GS_B2(1) } else { GS_B2(2) }
#undef GS_B2
#undef GS_B3
#undef GS_B
  return (int)cudaGetLastError();
}

}  // namespace gs
