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
  float ghat, u, v, t, inv_det;
  bool ray;
};

// raster_common.wgsl:69-95 on the record parameterisation. Written with
// explicit rounding intrinsics so the forward and backward kernels compute
// bit-identical alphas.
__device__ __forceinline__ Hit eval_hit(const float4& r0, const float4& r1, const float4& r2, float depth, float sx,
                                        float sy, float pxc, float pyc) {
  Hit h;
  const float det = fmaf(r0.x, sx, fmaf(r0.y, sy, r0.z));
  float qr = __int_as_float(0x7f800000);  // +inf: ray branch unavailable
  h.u = 0.0f; h.v = 0.0f; h.t = 0.0f; h.inv_det = 0.0f;
  if (fabsf(det) > 1e-12f) {
    const float inv = __frcp_rn(det);
    const float u = __fmul_rn(fmaf(r1.x, sx, fmaf(r1.y, sy, r1.z)), inv);
    const float v = __fmul_rn(fmaf(r2.x, sx, fmaf(r2.y, sy, r2.z)), inv);
    const float t = __fmul_rn(r0.w, inv);
    h.u = u; h.v = v; h.t = t; h.inv_det = inv;
    if (t > NEAR_DEPTH) qr = __fmul_rn(0.5f, fmaf(u, u, __fmul_rn(v, v)));
  }
  const float dx = pxc - r1.w, dy = pyc - r2.w;
  const float qs = fmaf(dx, dx, __fmul_rn(dy, dy));  // (dx²+dy²)/(2σ²) with σ² = 0.5
  h.ray = qr <= qs;
  const float q = h.ray ? qr : qs;
  if (!h.ray) h.t = depth;
  h.ghat = __expf(-q);
  return h;
}

struct TileGeo {
  int v, x, y, W, H;
  bool inside;
  float pxc, pyc, sx, sy;
  float bx0, bx1, by0, by1;  // pixel-centre extent of the tile's in-image pixels
  long long pix;
};

__device__ __forceinline__ TileGeo tile_geo(const RasterArgs& a, int tile) {
  TileGeo g;
  int v = 0;
  while (v + 1 < a.n_views && tile >= __ldg(&a.views[v + 1].tile_base)) ++v;
  const ViewInfo* V = a.views + v;
  const int tiles_x = __ldg(&V->tiles_x);
  g.v = v;
  g.W = __ldg(&V->width);
  g.H = __ldg(&V->height);
  const int lt = tile - __ldg(&V->tile_base);
  const int x0 = (lt % tiles_x) * TILE, y0 = (lt / tiles_x) * TILE;
  g.x = x0 + (threadIdx.x & 15);
  g.y = y0 + (threadIdx.x >> 4);
  g.inside = g.x < g.W && g.y < g.H;
  const float f = __ldg(&V->focal), cx = __ldg(&V->cx), cy = __ldg(&V->cy);
  g.pxc = (float)g.x + 0.5f;
  g.pyc = (float)g.y + 0.5f;
  g.sx = -((g.pxc - cx) / f);  // s = −d
  g.sy = (g.pyc - cy) / f;
  g.bx0 = (float)x0 + 0.5f;
  g.bx1 = (float)(min(x0 + TILE, g.W) - 1) + 0.5f;
  g.by0 = (float)y0 + 0.5f;
  g.by1 = (float)(min(y0 + TILE, g.H) - 1) + 0.5f;
  g.pix = __ldg(&V->pix_base) + (long long)g.y * g.W + g.x;
  return g;
}

__device__ __forceinline__ bool box_hits_tile(const float4& b, const TileGeo& g) {
  return b.x <= g.bx1 && b.y >= g.bx0 && b.z <= g.by1 && b.w >= g.by0;
}
__device__ __forceinline__ bool box_has_pixel(const float4& b, float pxc, float pyc) {
  return pxc >= b.x && pxc <= b.y && pyc >= b.z && pyc <= b.w;
}

// Compaction of the staged batch: returns this thread's slot among the kept
// entries (valid when keep) and the number kept. Order is preserved.
__device__ __forceinline__ int compact_slot(bool keep, int* s_wcount, int& kept) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned bal = __ballot_sync(FULL, keep);
  if (lane == 0) s_wcount[warp] = __popc(bal);
  __syncthreads();
  int off = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < 8; ++w) {
    const int c = s_wcount[w];
    if (w < warp) off += c;
    tot += c;
  }
  kept = tot;
  return off + __popc(bal & lanemask_lt());
}

template <int BATCH, int PREC, bool DET, bool PERSIST>
__global__ void __launch_bounds__(256) k_raster_fwd(RasterArgs a) {
  static_assert(BATCH <= 256, "one staging pass per batch");
  __shared__ float4 s_r0[BATCH], s_r1[BATCH], s_r2[BATCH], s_r3[BATCH], s_r4[BATCH], s_bb[BATCH];
  __shared__ int s_j[BATCH];
  __shared__ int s_wcount[8];
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
    const TileGeo g = tile_geo(a, tile);
    const uint2 range = __ldg(&a.ranges[tile]);
    float T = 1.0f, cr = 0.f, cg = 0.f, cb = 0.f, aa = 0.f, ad = 0.f, nx = 0.f, ny = 0.f, nz = 0.f;
    uint32_t nc = 0;
    bool done = !g.inside;
    for (uint32_t base = range.x; base < range.y; base += BATCH) {
      if (__syncthreads_count(done) == 256) break;
      const int count = (int)min((uint32_t)BATCH, range.y - base);
      bool keep = false;
      uint32_t item = 0;
      float4 bb = make_float4(0.f, 0.f, 0.f, 0.f);
      if (tid < count) {
        item = __ldg(&a.sorted_vals[base + tid]);
        if (DET) item = __ldg(&a.exp_item[item]);
        bb = load_record_box<PREC>(a.records, item);
        keep = box_hits_tile(bb, g);
      }
      int kept;
      const int slot = compact_slot(keep, s_wcount, kept);
      if (keep) {
        float4 r0, r1, r2, r3, r4;
        load_record<PREC>(a.records, item, r0, r1, r2, r3, r4);
        s_r0[slot] = r0; s_r1[slot] = r1; s_r2[slot] = r2; s_r3[slot] = r3; s_r4[slot] = r4;
        s_bb[slot] = bb;
        s_j[slot] = tid;
      }
      __syncthreads();
      if (!done) {
        for (int k = 0; k < kept; ++k) {
          if (!box_has_pixel(s_bb[k], g.pxc, g.pyc)) continue;
          const float4 r0 = s_r0[k], r1 = s_r1[k], r2 = s_r2[k];
          const float4 r4 = s_r4[k];
          const Hit h = eval_hit(r0, r1, r2, r4.w, g.sx, g.sy, g.pxc, g.pyc);
          const float4 r3 = s_r3[k];
          const float alpha = fminf(__fmul_rn(r3.w, h.ghat), ALPHA_CLAMP);
          if (alpha < ALPHA_SKIP) continue;
          const float w = T * alpha;
          cr += r3.x * w; cg += r3.y * w; cb += r3.z * w;
          aa += w;
          ad += h.t * w;
          nx += r4.x * w; ny += r4.y * w; nz += r4.z * w;
          T = __fmul_rn(T, 1.0f - alpha);
          nc = base - range.x + (uint32_t)s_j[k] + 1u;
          if (T < T_TERMINATE) { done = true; break; }
        }
      }
    }
    if (g.inside) {
      a.out_color[g.pix] = make_float4(cr, cg, cb, aa);
      a.out_aux[g.pix] = make_float4(T, ad, 0.f, 0.f);
      a.out_normal[g.pix] = make_float4(nx, ny, nz, 0.f);
      a.out_nc[g.pix] = nc;
    }
    if (!PERSIST) return;
    __syncthreads();
  }
}

template <int BATCH, int PREC, bool AUX, bool DET, bool PERSIST>
__global__ void __launch_bounds__(256) k_raster_bwd(RasterArgs a) {
  constexpr int NW = 8;
  constexpr int NG = AUX ? 32 : 16;  // reduced components per entry (AUX: 20 used)
  constexpr int NQ = AUX ? 5 : 4;    // float4 groups per entry written out
  __shared__ float4 s_r0[BATCH], s_r1[BATCH], s_r2[BATCH], s_r3[BATCH], s_bb[BATCH];
  __shared__ float4 s_r4[AUX ? BATCH : 1];
  __shared__ uint32_t s_item[BATCH];
  __shared__ uint32_t s_q[DET ? BATCH : 1];
  __shared__ int s_j[BATCH];
  __shared__ float s_part[NW][BATCH][NG];
  __shared__ int s_wcount[8];
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
    const TileGeo g = tile_geo(a, tile);
    float3 dlc = make_float3(0.f, 0.f, 0.f);
    float dld = 0.f, wtot = 0.f, wttot = 0.f;
    float3 dln = make_float3(0.f, 0.f, 0.f);
    float T = 1.0f;
    uint32_t nc = 0;
    if (g.inside) {
      const float4 gc = a.dl_dcolor[g.pix];
      dlc = make_float3(gc.x, gc.y, gc.z);
      const float4 aux = a.out_aux[g.pix];
      T = aux.x;
      nc = a.out_nc[g.pix];
      if (AUX) {
        dld = gc.w;
        const float4 gn = a.dl_dnormal[g.pix];
        dln = make_float3(gn.x, gn.y, gn.z);
        wtot = a.out_color[g.pix].w;
        wttot = aux.y;
      }
    }
    bool has_loss = g.inside && (dlc.x != 0.f || dlc.y != 0.f || dlc.z != 0.f);
    if (AUX) has_loss = g.inside && (has_loss || dld != 0.f || dln.x != 0.f || dln.y != 0.f || dln.z != 0.f ||
                                     a.lambda_dist != 0.f);
    if (!has_loss) nc = 0;
    if (tid == 0) s_maxnc = 0;
    __syncthreads();
    if (nc) atomicMax(&s_maxnc, (int)nc);
    __syncthreads();
    const uint32_t maxnc = min((uint32_t)s_maxnc, range.y - range.x);

    if (DET) {
      // Entries past the tile's last contributor get zero partials.
      for (uint32_t e = range.x + maxnc + tid; e < range.y; e += 256) {
        const uint32_t q = __ldg(&a.sorted_vals[e]);
        float4* pp = reinterpret_cast<float4*>(a.partials + (size_t)q * GG_STRIDE);
#pragma unroll
        for (int k = 0; k < NQ; ++k) pp[k] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }

    float3 suf_c = make_float3(0.f, 0.f, 0.f), suf_n = make_float3(0.f, 0.f, 0.f);
    float suf_d = 0.f, suf_w = 0.f, suf_cw = 0.f;

    uint32_t hi = range.x + maxnc;
    while (hi > range.x) {
      const uint32_t lo = (hi - range.x > (uint32_t)BATCH) ? hi - BATCH : range.x;
      const int count = (int)(hi - lo);
      bool keep = false;
      uint32_t item = 0, q = 0;
      float4 bb = make_float4(0.f, 0.f, 0.f, 0.f);
      if (tid < count) {
        item = __ldg(&a.sorted_vals[lo + tid]);
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
      const int slot = compact_slot(keep, s_wcount, kept);
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
        float gg[NG];
#pragma unroll
        for (int c = 0; c < NG; ++c) gg[c] = 0.f;
        bool contrib = false;
        if (has_loss && cidx < nc && box_has_pixel(s_bb[k], g.pxc, g.pyc)) {
          const float4 r0 = s_r0[k], r1 = s_r1[k], r2 = s_r2[k], r3 = s_r3[k];
          float4 r4 = make_float4(0.f, 0.f, 0.f, 0.f);
          float depth = 0.f;  // feeds t in the screen branch, used by aux terms alone
          if (AUX) { r4 = s_r4[k]; depth = r4.w; }
          const Hit h = eval_hit(r0, r1, r2, depth, g.sx, g.sy, g.pxc, g.pyc);
          const float raw_alpha = __fmul_rn(r3.w, h.ghat);
          const float alpha = fminf(raw_alpha, ALPHA_CLAMP);
          if (alpha >= ALPHA_SKIP) {
            contrib = true;
            const float oma = 1.0f - alpha;
            const float inv_oma = 1.0f / oma;
            const float t_before = T / oma;
            const float w = t_before * alpha;
            float dl_dalpha = (dlc.x * r3.x + dlc.y * r3.y + dlc.z * r3.z) * t_before -
                              (dlc.x * suf_c.x + dlc.y * suf_c.y + dlc.z * suf_c.z) * inv_oma;
            float dl_dt = 0.f;
            if (AUX) {
              const float t_hit = h.t;
              float dt_dist = 0.f, coef = 0.f;
              if (a.lambda_dist != 0.f) {
                const float a_pre = wtot - suf_w - w;
                const float b_pre = wttot - suf_d - w * t_hit;
                dt_dist = a.lambda_dist * 2.0f * w * (a_pre - suf_w);
                coef = a.lambda_dist * (2.0f * (t_hit * a_pre - b_pre) + 2.0f * (suf_d - t_hit * suf_w));
              }
              dl_dt = dld * w + dt_dist;
              dl_dalpha += dld * (t_hit * t_before - suf_d * inv_oma) +
                           (dln.x * r4.x + dln.y * r4.y + dln.z * r4.z) * t_before -
                           (dln.x * suf_n.x + dln.y * suf_n.y + dln.z * suf_n.z) * inv_oma + coef * t_before -
                           suf_cw * inv_oma;
              suf_d += t_hit * w;
              suf_n.x += r4.x * w; suf_n.y += r4.y * w; suf_n.z += r4.z * w;
              suf_w += w;
              suf_cw += coef * w;
              gg[17] = dln.x * w; gg[18] = dln.y * w; gg[19] = dln.z * w;
            }
            suf_c.x += r3.x * w; suf_c.y += r3.y * w; suf_c.z += r3.z * w;
            T = t_before;
            gg[11] = dlc.x * w; gg[12] = dlc.y * w; gg[13] = dlc.z * w;
            if (raw_alpha <= ALPHA_CLAMP) {
              gg[14] = dl_dalpha * h.ghat;
              const float dl_dghat = dl_dalpha * r3.w;
              if (h.ray) {
                const float gu = -h.u * h.ghat * dl_dghat;
                const float gv = -h.v * h.ghat * dl_dghat;
                const float gun = gu * h.inv_det, gvn = gv * h.inv_det;
                const float gdet = -(h.u * gu + h.v * gv + (AUX ? h.t * dl_dt : 0.f)) * h.inv_det;
                gg[0] = gdet * g.sx; gg[1] = gdet * g.sy; gg[2] = gdet;
                gg[3] = gun * g.sx; gg[4] = gun * g.sy; gg[5] = gun;
                gg[6] = gvn * g.sx; gg[7] = gvn * g.sy; gg[8] = gvn;
                if (AUX) gg[15] = dl_dt * h.inv_det;
              } else {
                const float kk = h.ghat * dl_dghat / LOWPASS_SIGMA2;
                gg[9] = (g.pxc - r1.w) * kk;
                gg[10] = (g.pyc - r2.w) * kk;
                if (AUX) gg[16] = dl_dt;
              }
            }
          }
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
      for (int w4 = tid; w4 < kept * NQ; w4 += 256) {
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

template <int BATCH, int PREC, bool DET, bool PERSIST>
void fwd_launch(const RasterArgs& a, int grid, cudaStream_t st) {
  k_raster_fwd<BATCH, PREC, DET, PERSIST><<<grid, 256, 0, st>>>(a);
}

template <int PREC, bool DET, bool PERSIST>
void fwd_batch(const RasterArgs& a, int batch, int grid, cudaStream_t st) {
  if (batch == 64) fwd_launch<64, PREC, DET, PERSIST>(a, grid, st);
  else if (batch == 256) fwd_launch<256, PREC, DET, PERSIST>(a, grid, st);
  else fwd_launch<128, PREC, DET, PERSIST>(a, grid, st);
}

// The per-warp partial buffer is NW*BATCH*NG floats of static shared memory,
// so the backward stages 32 entries at a time with aux losses and 64 without.
template <bool AUX>
constexpr int bwd_batch() { return AUX ? 32 : 64; }

template <int PREC, bool AUX, bool DET, bool PERSIST>
void bwd_launch(const RasterArgs& a, int grid, cudaStream_t st) {
  k_raster_bwd<bwd_batch<AUX>(), PREC, AUX, DET, PERSIST><<<grid, 256, 0, st>>>(a);
}

template <typename K>
int occ(K kernel) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, 256, 0) != cudaSuccess) return 1;
  return n < 1 ? 1 : n;
}

}  // namespace

int raster_fwd_occupancy(int prec, int batch, bool det) {
#define GS_O(B, P) (det ? occ(k_raster_fwd<B, P, true, true>) : occ(k_raster_fwd<B, P, false, true>))
#define GS_OB(P) (batch == 64 ? GS_O(64, P) : (batch == 256 ? GS_O(256, P) : GS_O(128, P)))
  return prec == 0 ? GS_OB(0) : (prec == 1 ? GS_OB(1) : GS_OB(2));
#undef GS_OB
#undef GS_O
}

int raster_bwd_occupancy(int prec, bool aux, bool det) {
#define GS_O(P, X, D) occ(k_raster_bwd<bwd_batch<X>(), P, X, D, true>)
#define GS_O2(P) (aux ? (det ? GS_O(P, true, true) : GS_O(P, true, false)) : (det ? GS_O(P, false, true) : GS_O(P, false, false)))
  return prec == 0 ? GS_O2(0) : (prec == 1 ? GS_O2(1) : GS_O2(2));
#undef GS_O2
#undef GS_O
}

int launch_raster_fwd(const RasterArgs& a, int prec, int batch, bool det, bool persistent, int grid, cudaStream_t st) {
  if (a.total_tiles == 0) return 0;
#define GS_F(P, D, S) fwd_batch<P, D, S>(a, batch, grid, st)
#define GS_F2(P)                                   \
  if (det) { if (persistent) GS_F(P, true, true); else GS_F(P, true, false); } \
  else { if (persistent) GS_F(P, false, true); else GS_F(P, false, false); }
  if (prec == 0) { GS_F2(0) } else if (prec == 1) { GS_F2(1) } else { GS_F2(2) }
#undef GS_F2
#undef GS_F
  return (int)cudaGetLastError();
}

int launch_raster_bwd(const RasterArgs& a, int prec, bool aux, bool det, bool persistent, int grid, cudaStream_t st) {
  if (a.total_tiles == 0) return 0;
#define GS_B(P, X, D, S) bwd_launch<P, X, D, S>(a, grid, st)
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
