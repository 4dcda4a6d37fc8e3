// Surfel projection (forward): crates/gs-kernels/src/shaders/surfel_prep_fwd.wgsl:64-132 — world
// parameters to camera space, SH colour with clamp mask, camera-facing
// normal, projected centre, conservative 3σ pixel radius capped at 64 px, tile
// rect by truncation, depth key = f32 bits of the centre depth. One thread
// per (surfel, view); the tile count of the rect is written for the binner
// (the reference's separate count_tiles pass, tile_binning.wgsl:30-43),
// restricted under the occlusion cut to the tiles whose cut the key reaches.
//
// This translation unit is compiled with --fmad=false: the rect and key
// arithmetic is evaluated in the reference's operation order without
// contraction so an f32 restatement on the host reproduces it bit for bit.
// The adjoint lives in gs_project_bwd.cu.
#include "gs_geom.cuh"

namespace gs {
namespace {

// Range of N(θ)/D(θ) over θ for N = a0 + a1 cosθ + a2 sinθ and
// D = b0 + b1 cosθ + b2 sinθ > 0: the extremes solve
// P sinθ + Q cosθ + R = 0 with P = a0 b1 − a1 b0, Q = a2 b0 − a0 b2,
// R = a2 b1 − a1 b2. On the unit circle (s, c) = (sinθ, cosθ) that line meets
// it at (s, c) = (−R·(P, Q) ± (Q, −P)·√(h² − R²)) / h², h² = P² + Q². The
// result only bounds a box that gets a pixel of margin, so divisions are the
// fast ones.
__device__ __forceinline__ void ratio_range(float a0, float a1, float a2, float b0, float b1, float b2, float& lo,
                                            float& hi) {
  const float P = a0 * b1 - a1 * b0, Q = a2 * b0 - a0 * b2, R = a2 * b1 - a1 * b2;
  const float h2 = P * P + Q * Q;
  // Interval bound, always valid: |N| ≤ |a0| + |(a1,a2)|, D ≥ b0 − |(b1,b2)|.
  const float na = sqrtf(a1 * a1 + a2 * a2), nb = sqrtf(b1 * b1 + b2 * b2), dmin = b0 - nb;
  float blo = __fdividef(a0 - na, a0 - na < 0.f ? dmin : b0 + nb);
  float bhi = __fdividef(a0 + na, a0 + na > 0.f ? dmin : b0 + nb);
  if (h2 > 1e-24f && R * R <= h2) {
    const float w = sqrtf(h2 - R * R), ih2 = __fdividef(1.0f, h2);
    const float s0 = (-R * P + Q * w) * ih2, c0 = (-R * Q - P * w) * ih2;
    const float s1 = (-R * P - Q * w) * ih2, c1 = (-R * Q + P * w) * ih2;
    const float v0 = __fdividef(a0 + a1 * c0 + a2 * s0, b0 + b1 * c0 + b2 * s0);
    const float v1 = __fdividef(a0 + a1 * c1 + a2 * s1, b0 + b1 * c1 + b2 * s1);
    lo = fmaxf(fminf(v0, v1), blo);
    hi = fminf(fmaxf(v0, v1), bhi);
    if (!(lo <= hi)) { lo = blo; hi = bhi; }
  } else {
    lo = blo;
    hi = bhi;
  }
}

// Pixel-space bounding box of the region where the surfel can reach
// α = o·ĝ ≥ 1/255 (the kernels' skip threshold): ĝ ≥ τ = 1/(255 o) holds
// inside the screen low-pass disc (dx²+dy² ≤ ln(1/τ)) or where the ray hits
// the surfel plane inside the disc u²+v² ≤ 2 ln(1/τ) in front of the near
// plane — the perspective image of a 3D ellipse whose x and y extremes have a
// closed form. The box is widened by a safety margin; it is used only to skip
// evaluations that are guaranteed to fall below the threshold, so colours and
// contributor counts are unchanged. Returns (x0, x1, y0, y1) in pixel
// coordinates of pixel centres; an unbounded region gives ±1e30.
__device__ __forceinline__ float4 alpha_bbox(const Cam& k, float3 c, float3 tu, float3 tv, float px, float py, float o) {
  const float L = logf(255.0f * o) + 1e-3f;
  if (!(L > 0.f)) return make_float4(1e30f, -1e30f, 1e30f, -1e30f);  // never reaches the threshold
  const float rs = sqrtf(L);
  float x0 = px - rs, x1 = px + rs, y0 = py - rs, y1 = py + rs;
  const float r = sqrtf(2.0f * L);
  // Ellipse c + r cosθ τu + r sinθ τv, depth D = −Z.
  const float b0 = -c.z, b1 = -r * tu.z, b2 = -r * tv.z;
  if (b0 - sqrtf(b1 * b1 + b2 * b2) <= NEAR_DEPTH * 1.01f + 1e-6f) return make_float4(-1e30f, 1e30f, -1e30f, 1e30f);
  float lo, hi;
  ratio_range(c.x, r * tu.x, r * tv.x, b0, b1, b2, lo, hi);
  x0 = fminf(x0, k.cx + k.f * lo);
  x1 = fmaxf(x1, k.cx + k.f * hi);
  ratio_range(c.y, r * tu.y, r * tv.y, b0, b1, b2, lo, hi);
  y0 = fminf(y0, k.cy - k.f * hi);
  y1 = fmaxf(y1, k.cy - k.f * lo);
  const float m = 1.0f;  // pixels of margin for rounding in the box and in the per-pixel evaluation
  return make_float4(x0 - m - 1e-4f * fabsf(x0), x1 + m + 1e-4f * fabsf(x1), y0 - m - 1e-4f * fabsf(y0),
                     y1 + m + 1e-4f * fabsf(y1));
}

template <int PREC>
__global__ void __launch_bounds__(256) k_project(ProjectArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = blockIdx.y;
  if (i >= a.n) return;
  const uint32_t item = (uint32_t)v * a.n + i;
  const Cam k = load_cam(a.views, v);
  const float4 p = __ldg(a.pos + i);
  const float2 s = __ldg(a.scales + i);
  const float4 q = __ldg(a.quats + i);
  uint4 rect = make_uint4(1u, 1u, 0u, 0u);
  Geom g;
  g.x = f3(p.x, p.y, p.z) - k.C;
  g.c = rt_mul(k, g.x);
  g.depth = -g.c.z;
  a.vals[item] = item;
  if (g.depth < NEAR_DEPTH) {
    a.rects[item] = rect;
    a.keys[item] = 0u;
    if (a.item_key != nullptr) a.item_key[item] = 0u;
    a.counts[item] = 0u;
    return;
  }
  geom(k, p, s, q, g);
  const float3 c = g.c, tu = g.tu, tv = g.tv;
  const float depth = g.depth;

  // Colour (surfel_prep_fwd.wgsl:183-186).
  const float lx = sqrtf(dot3(g.x, g.x));
  const float3 dir = f3(g.x.x / lx, g.x.y / lx, g.x.z / lx);
  float b[16];
  int nb;
  ShRow<PREC> row;
  row.load(a.sh, i);
  float3 raw = sh_raw_color_with([&](int kk) { return row.coeff(kk); }, k.deg, dir, b, nb);
  float3 color = f3(fmaxf(raw.x, 0.0f), fmaxf(raw.y, 0.0f), fmaxf(raw.z, 0.0f));

  // Normal facing the camera (surfel_prep_fwd.wgsl:188-194).
  float3 M = cross3(tu, tv);
  float3 nrm = M;
  float m2 = dot3(M, M);
  if (m2 > 0.0f) {
    const float il = rsqrtf(m2);  // the normal feeds only the aux outputs: no exact division needed
    nrm = f3(M.x * il, M.y * il, M.z * il);
    if (dot3(nrm, c) > 0.0f) nrm = f3(-nrm.x, -nrm.y, -nrm.z);
  }

  // Projected centre, conservative radius and tile rect (surfel_prep_fwd.wgsl:196-226),
  // same operation order as the shader.
  const float w = depth;
  const float px = k.cx + k.f * c.x / w;
  const float py = k.cy - k.f * c.y / w;
  const float lu = sqrtf(dot3(tu, tu)), lv = sqrtf(dot3(tv, tv));
  const float r = fminf(3.0f * k.f * (lu + lv) / depth + 3.0f, 64.0f);
  const float tf = (float)k.tile;
  // The tile edge is a power of two (8, 16 or 32), so x·(1/tf) rounds exactly
  // as x/tf: the rect stays bit-identical to the reference's division.
  const float itf = 1.0f / tf;
  const float mx = (float)(k.tiles_x - 1), my = (float)(k.tiles_y - 1);
  const uint32_t x0 = (uint32_t)fminf(fmaxf((px - r) * itf, 0.0f), mx);
  const uint32_t y0 = (uint32_t)fminf(fmaxf((py - r) * itf, 0.0f), my);
  const uint32_t x1 = (uint32_t)fminf(fmaxf((px + r) * itf, 0.0f), mx);
  const uint32_t y1 = (uint32_t)fminf(fmaxf((py + r) * itf, 0.0f), my);
  uint32_t count = 0;
  if (px + r >= 0.0f && px - r < (float)k.W && py + r >= 0.0f && py - r < (float)k.H) {
    rect = make_uint4(x0, y0, x1, y1);
    count = (x1 - x0 + 1u) * (y1 - y0 + 1u);
  }
  const float o = __ldg(a.opac + i);
  const float4 box = count ? alpha_bbox(k, c, tu, tv, px, py, o) : make_float4(1e30f, -1e30f, 1e30f, -1e30f);
  if (a.tight && count) {
    // Tight binning: only the tiles of the reference rect that the α-box
    // overlaps. Tile t holds pixel centres [T·t + 0.5, T·t + T − 0.5].
    const float lim = 1e8f, hi = tf - 0.5f;
    const float fx0 = ceilf((fminf(fmaxf(box.x, -lim), lim) - hi) * itf);
    const float fx1 = floorf((fminf(fmaxf(box.y, -lim), lim) - 0.5f) * itf);
    const float fy0 = ceilf((fminf(fmaxf(box.z, -lim), lim) - hi) * itf);
    const float fy1 = floorf((fminf(fmaxf(box.w, -lim), lim) - 0.5f) * itf);
    const int tx0 = max((int)x0, (int)fmaxf(fx0, -1.f)), tx1 = min((int)x1, (int)fminf(fx1, 1e7f));
    const int ty0 = max((int)y0, (int)fmaxf(fy0, -1.f)), ty1 = min((int)y1, (int)fminf(fy1, 1e7f));
    if (tx0 <= tx1 && ty0 <= ty1) {
      rect = make_uint4(tx0, ty0, tx1, ty1);
      count = (uint32_t)(tx1 - tx0 + 1) * (uint32_t)(ty1 - ty0 + 1);
    } else {
      rect = make_uint4(1u, 1u, 0u, 0u);
      count = 0;
    }
  }
  a.rects[item] = rect;
  const uint32_t key = __float_as_uint(depth);
  a.keys[item] = key;
  if (a.item_key != nullptr) a.item_key[item] = key;
  if (a.cut != nullptr && count) {
    // Occlusion cut: only the rect's tiles whose binned depth reaches this key.
    // Four independent loads per round, walking the rect row-major.
    const uint32_t tb = (uint32_t)__ldg(&a.views[v].tile_base), txs = (uint32_t)k.tiles_x;
    uint32_t kept = 0, x = rect.x, y = rect.y;
    for (uint32_t j = 0; j < count; j += 4) {
      uint32_t idx[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        idx[u] = tb + y * txs + x;
        if (++x > rect.z) { x = rect.x; ++y; }
      }
      uint32_t c[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) c[u] = j + u < count ? __ldg(a.cut + idx[u]) : 0u;
#pragma unroll
      for (int u = 0; u < 4; ++u) kept += (j + u < count && key <= c[u]) ? 1u : 0u;
    }
    count = kept;
  }
  a.counts[item] = count;

  const float3 Bu = cross3(tv, c);
  const float3 Bv = cross3(c, tu);
  const float tn = -dot3(c, M);
  // The projected centre for the hit test, accurate to double: the camera
  // transform and the perspective division in double (the float px, py above
  // keep the reference's rect arithmetic), stored as hi + lo.
  const ViewInfo* V = a.views + v;
  const double xd = (double)p.x - (double)k.C.x, yd = (double)p.y - (double)k.C.y, zd = (double)p.z - (double)k.C.z;
  const double cxd = __ldg(&V->rot64[0]) * xd + __ldg(&V->rot64[1]) * yd + __ldg(&V->rot64[2]) * zd;
  const double cyd = __ldg(&V->rot64[3]) * xd + __ldg(&V->rot64[4]) * yd + __ldg(&V->rot64[5]) * zd;
  const double czd = __ldg(&V->rot64[6]) * xd + __ldg(&V->rot64[7]) * yd + __ldg(&V->rot64[8]) * zd;
  const double pxd = (double)k.cx + (double)k.f * cxd / -czd;
  const double pyd = (double)k.cy - (double)k.f * cyd / -czd;
  const float pxh = (float)pxd, pyh = (float)pyd;
  const float pxl = (float)(pxd - (double)pxh), pyl = (float)(pyd - (double)pyh);
  const float inv_f = 1.0f / k.f;
  store_record<PREC>(a.records, item, make_float4(M.x, M.y, M.z, tn),
                     make_float4(-Bu.x * inv_f, Bu.y * inv_f, pxl, pxh),
                     make_float4(-Bv.x * inv_f, Bv.y * inv_f, pyl, pyh), make_float4(color.x, color.y, color.z, o),
                     make_float4(nrm.x, nrm.y, nrm.z, depth), box);
}

}  // namespace

int launch_project(const ProjectArgs& a, int prec, uint32_t n_views, cudaStream_t st) {
  if (a.n == 0 || n_views == 0) return 0;
  dim3 grid((a.n + 255) / 256, n_views);
  if (prec == 0) k_project<0><<<grid, 256, 0, st>>>(a);
  else if (prec == 1) k_project<1><<<grid, 256, 0, st>>>(a);
  else k_project<2><<<grid, 256, 0, st>>>(a);
  return (int)cudaGetLastError();
}

}  // namespace gs
