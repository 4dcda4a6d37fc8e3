// Surfel projection (forward) and its adjoint.
//
// Forward: crates/gs-kernels/src/shaders/surfel_prep_fwd.wgsl:64-132 — world
// parameters to camera space, SH colour with clamp mask, camera-facing
// normal, projected centre, conservative 3σ pixel radius capped at 64 px, tile
// rect by truncation, depth key = f32 bits of the centre depth. One thread
// per (surfel, view); the tile count of the rect is written for the binner
// (the reference's separate count_tiles pass, tile_binning.wgsl:30-43).
//
// This translation unit is compiled with --fmad=false: the rect and key
// arithmetic is evaluated in the reference's operation order without
// contraction so an f32 restatement on the host reproduces it bit for bit.
//
// Backward: crates/gs-kernels/src/shaders/surfel_prep_bwd.wgsl:129-284 —
// chains the per-surfel record gradients (see GG_STRIDE in gs_common.cuh)
// into position, scales, quaternion (through normalisation), opacity, SH
// (clamp-masked, with the view-direction path) and the camera accumulators
// dL/dR, dL/dC, dL/dfocal.
#include "gs_common.cuh"
#include "gs_kernels.h"

namespace gs {
namespace {

// SH constants as the reference shader writes them (surfel_prep_fwd.wgsl:17-18, 129-142).
constexpr float C0 = 0.28209479f;
constexpr float C1 = 0.48860252f;
constexpr float C2a = 1.0925484f, C2b = 0.31539157f, C2c = 0.5462742f;
constexpr float C3a = 0.5900436f, C3b = 2.8906114f, C3c = 0.4570458f, C3d = 0.37317634f, C3e = 1.4453057f;

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
__device__ __forceinline__ float3& operator-=(float3& a, float3 b) { a = a - b; return a; }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

struct Cam {
  float3 r0, r1, r2;  // columns of R
  float3 C;
  float f, cx, cy;
  int W, H, tiles_x, tiles_y, deg;
};

__device__ __forceinline__ Cam load_cam(const ViewInfo* views, int v) {
  const ViewInfo* V = views + v;
  Cam c;
  c.r0 = f3(__ldg(&V->rot[0]), __ldg(&V->rot[1]), __ldg(&V->rot[2]));
  c.r1 = f3(__ldg(&V->rot[3]), __ldg(&V->rot[4]), __ldg(&V->rot[5]));
  c.r2 = f3(__ldg(&V->rot[6]), __ldg(&V->rot[7]), __ldg(&V->rot[8]));
  c.C = f3(__ldg(&V->center[0]), __ldg(&V->center[1]), __ldg(&V->center[2]));
  c.f = __ldg(&V->focal);
  c.cx = __ldg(&V->cx);
  c.cy = __ldg(&V->cy);
  c.W = __ldg(&V->width);
  c.H = __ldg(&V->height);
  c.tiles_x = __ldg(&V->tiles_x);
  c.tiles_y = __ldg(&V->tiles_y);
  c.deg = __ldg(&V->sh_degree);
  return c;
}

// Rᵀ v with R's columns r0..r2 (raster_common.wgsl:41-48).
__device__ __forceinline__ float3 rt_mul(const Cam& k, float3 v) { return f3(dot3(k.r0, v), dot3(k.r1, v), dot3(k.r2, v)); }
// R v.
__device__ __forceinline__ float3 r_mul(const Cam& k, float3 v) { return k.r0 * v.x + k.r1 * v.y + k.r2 * v.z; }

struct Geom {
  float3 x, c, tu, tv, col0, col1;
  float4 qh;
  float qn;
  float depth;
};

// Camera-space geometry of one surfel (surfel_prep_fwd.wgsl:82-95, 54-62).
__device__ __forceinline__ void geom(const Cam& k, float4 p, float2 s, float4 q, Geom& g) {
  g.x = f3(p.x, p.y, p.z) - k.C;
  g.c = rt_mul(k, g.x);
  g.depth = -g.c.z;
  g.qn = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  float x = q.x / g.qn, y = q.y / g.qn, z = q.z / g.qn, w = q.w / g.qn;
  g.qh = make_float4(x, y, z, w);
  g.col0 = f3(1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + w * z), 2.0f * (x * z - w * y));
  g.col1 = f3(2.0f * (x * y - w * z), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + w * x));
  g.tu = rt_mul(k, g.col0 * s.x);
  g.tv = rt_mul(k, g.col1 * s.y);
}

// Real SH basis up to degree 3 for a unit direction (crates/gs-cpu-ref/src/math.rs:127-152).
__device__ __forceinline__ int sh_basis(int deg, float3 d, float b[16]) {
  float x = d.x, y = d.y, z = d.z;
  b[0] = C0;
  if (deg < 1) return 1;
  b[1] = -C1 * y; b[2] = C1 * z; b[3] = -C1 * x;
  if (deg < 2) return 4;
  float xx = x * x, yy = y * y, zz = z * z;
  b[4] = C2a * x * y; b[5] = -C2a * y * z; b[6] = C2b * (2.0f * zz - xx - yy);
  b[7] = -C2a * x * z; b[8] = C2c * (xx - yy);
  if (deg < 3) return 9;
  b[9] = -C3a * y * (3.0f * xx - yy); b[10] = C3b * x * y * z; b[11] = -C3c * y * (4.0f * zz - xx - yy);
  b[12] = C3d * z * (2.0f * zz - 3.0f * xx - 3.0f * yy); b[13] = -C3c * x * (4.0f * zz - xx - yy);
  b[14] = C3e * z * (xx - yy); b[15] = -C3a * x * (xx - 3.0f * yy);
  return 16;
}

// d(basis)/d(direction) before the normalisation Jacobian (math.rs:155-191).
__device__ __forceinline__ void sh_basis_grad(int deg, float3 d, float3 g[16]) {
  float x = d.x, y = d.y, z = d.z;
  g[0] = f3(0, 0, 0);
  if (deg < 1) return;
  g[1] = f3(0, -C1, 0); g[2] = f3(0, 0, C1); g[3] = f3(-C1, 0, 0);
  if (deg < 2) return;
  g[4] = f3(y, x, 0) * C2a; g[5] = f3(0, z, y) * (-C2a); g[6] = f3(-2.0f * x, -2.0f * y, 4.0f * z) * C2b;
  g[7] = f3(z, 0, x) * (-C2a); g[8] = f3(2.0f * x, -2.0f * y, 0) * C2c;
  if (deg < 3) return;
  float xx = x * x, yy = y * y, zz = z * z;
  g[9] = f3(6.0f * x * y, 3.0f * xx - 3.0f * yy, 0) * (-C3a);
  g[10] = f3(y * z, x * z, x * y) * C3b;
  g[11] = f3(-2.0f * x * y, 4.0f * zz - xx - 3.0f * yy, 8.0f * y * z) * (-C3c);
  g[12] = f3(-6.0f * x * z, -6.0f * y * z, 6.0f * zz - 3.0f * xx - 3.0f * yy) * C3d;
  g[13] = f3(4.0f * zz - 3.0f * xx - yy, -2.0f * x * y, 8.0f * x * z) * (-C3c);
  g[14] = f3(2.0f * x * z, -2.0f * y * z, xx - yy) * C3e;
  g[15] = f3(3.0f * xx - 3.0f * yy, -6.0f * x * y, 0) * (-C3a);
}

template <int PREC>
__device__ __forceinline__ float3 sh_coeff(const void* sh, size_t i, int k) {
  if constexpr (PREC == 0) {
    const float* p = reinterpret_cast<const float*>(sh) + i * SH_FLOATS + 3 * k;
    return f3(__ldg(p), __ldg(p + 1), __ldg(p + 2));
  } else {
    using H = typename std::conditional<PREC == 1, __half, __nv_bfloat16>::type;
    const H* p = reinterpret_cast<const H*>(sh) + i * SH_FLOATS + 3 * k;
    return f3(h2f<H>(p[0]), h2f<H>(p[1]), h2f<H>(p[2]));
  }
}

// Raw SH colour 0.5 + Σ b_k sh_k (surfel_prep_fwd.wgsl:121-147).
template <int PREC>
__device__ __forceinline__ float3 sh_raw_color(const void* sh, size_t i, int deg, float3 dir, float b[16], int& nb) {
  nb = sh_basis(deg, dir, b);
  float3 acc = f3(0, 0, 0);
  for (int k = 0; k < nb; ++k) acc += sh_coeff<PREC>(sh, i, k) * b[k];
  return acc + f3(0.5f, 0.5f, 0.5f);
}

// Range of f·N(θ)/D(θ) over θ for N = a0 + a1 cosθ + a2 sinθ and
// D = b0 + b1 cosθ + b2 sinθ > 0: the extremes solve
// (a0 b1 − a1 b0) sinθ + (a2 b0 − a0 b2) cosθ + (a2 b1 − a1 b2) = 0.
__device__ __forceinline__ void ratio_range(float a0, float a1, float a2, float b0, float b1, float b2, float& lo,
                                            float& hi) {
  const float P = a0 * b1 - a1 * b0, Q = a2 * b0 - a0 * b2, R = a2 * b1 - a1 * b2;
  const float h = sqrtf(P * P + Q * Q);
  // Interval bound, always valid: |N| ≤ |a0| + |(a1,a2)|, D ≥ b0 − |(b1,b2)|.
  const float na = sqrtf(a1 * a1 + a2 * a2), dmin = b0 - sqrtf(b1 * b1 + b2 * b2);
  float blo = (a0 - na) / (a0 - na < 0.f ? dmin : b0 + sqrtf(b1 * b1 + b2 * b2));
  float bhi = (a0 + na) / (a0 + na > 0.f ? dmin : b0 + sqrtf(b1 * b1 + b2 * b2));
  if (h > 1e-12f && fabsf(R) <= h) {
    const float phi = atan2f(P, Q), dth = acosf(fminf(fmaxf(-R / h, -1.f), 1.f));
    float s0, c0, s1, c1;
    sincosf(phi + dth, &s0, &c0);
    sincosf(phi - dth, &s1, &c1);
    const float v0 = (a0 + a1 * c0 + a2 * s0) / (b0 + b1 * c0 + b2 * s0);
    const float v1 = (a0 + a1 * c1 + a2 * s1) / (b0 + b1 * c1 + b2 * s1);
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
  float3 raw = sh_raw_color<PREC>(a.sh, i, k.deg, dir, b, nb);
  float3 color = f3(fmaxf(raw.x, 0.0f), fmaxf(raw.y, 0.0f), fmaxf(raw.z, 0.0f));

  // Normal facing the camera (surfel_prep_fwd.wgsl:188-194).
  float3 M = cross3(tu, tv);
  float3 nrm = M;
  float m2 = dot3(M, M);
  if (m2 > 0.0f) {
    float ml = sqrtf(m2);
    nrm = f3(M.x / ml, M.y / ml, M.z / ml);
    if (dot3(nrm, c) > 0.0f) nrm = f3(-nrm.x, -nrm.y, -nrm.z);
  }

  // Projected centre, conservative radius and tile rect (surfel_prep_fwd.wgsl:196-226),
  // same operation order as the shader.
  const float w = depth;
  const float px = k.cx + k.f * c.x / w;
  const float py = k.cy - k.f * c.y / w;
  const float lu = sqrtf(dot3(tu, tu)), lv = sqrtf(dot3(tv, tv));
  const float r = fminf(3.0f * k.f * (lu + lv) / depth + 3.0f, 64.0f);
  const float tf = (float)TILE;
  const float mx = (float)(k.tiles_x - 1), my = (float)(k.tiles_y - 1);
  const uint32_t x0 = (uint32_t)fminf(fmaxf((px - r) / tf, 0.0f), mx);
  const uint32_t y0 = (uint32_t)fminf(fmaxf((py - r) / tf, 0.0f), my);
  const uint32_t x1 = (uint32_t)fminf(fmaxf((px + r) / tf, 0.0f), mx);
  const uint32_t y1 = (uint32_t)fminf(fmaxf((py + r) / tf, 0.0f), my);
  uint32_t count = 0;
  if (px + r >= 0.0f && px - r < (float)k.W && py + r >= 0.0f && py - r < (float)k.H) {
    rect = make_uint4(x0, y0, x1, y1);
    count = (x1 - x0 + 1u) * (y1 - y0 + 1u);
  }
  const float o = __ldg(a.opac + i);
  const float4 box = count ? alpha_bbox(k, c, tu, tv, px, py, o) : make_float4(1e30f, -1e30f, 1e30f, -1e30f);
  if (a.tight && count) {
    // Tight binning: only the tiles of the reference rect that the α-box
    // overlaps. Tile t holds pixel centres [16t + 0.5, 16t + 15.5].
    const float lim = 1e8f;
    const float fx0 = ceilf((fminf(fmaxf(box.x, -lim), lim) - 15.5f) / tf);
    const float fx1 = floorf((fminf(fmaxf(box.y, -lim), lim) - 0.5f) / tf);
    const float fy0 = ceilf((fminf(fmaxf(box.z, -lim), lim) - 15.5f) / tf);
    const float fy1 = floorf((fminf(fmaxf(box.w, -lim), lim) - 0.5f) / tf);
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
  a.keys[item] = __float_as_uint(depth);
  a.counts[item] = count;

  const float3 Bu = cross3(tv, c);
  const float3 Bv = cross3(c, tu);
  const float tn = -dot3(c, M);
  store_record<PREC>(a.records, item, make_float4(M.x, M.y, M.z, tn), make_float4(Bu.x, Bu.y, Bu.z, px),
                     make_float4(Bv.x, Bv.y, Bv.z, py), make_float4(color.x, color.y, color.z, o),
                     make_float4(nrm.x, nrm.y, nrm.z, depth), box);
}

// dL/dq for the unnormalised quaternion from the first two columns of dL/dR_q
// (the third is zero for surfels): crates/gs-cpu-ref/src/math.rs:38-88.
__device__ __forceinline__ float4 quat_grad2(const Geom& g, float3 d0, float3 d1) {
  const float x = g.qh.x, y = g.qh.y, z = g.qh.z, w = g.qh.w;
  float gx = dot3(d0, f3(0.0f, 2.0f * y, 2.0f * z)) + dot3(d1, f3(2.0f * y, -4.0f * x, 2.0f * w));
  float gy = dot3(d0, f3(-4.0f * y, 2.0f * x, -2.0f * w)) + dot3(d1, f3(2.0f * x, 0.0f, 2.0f * z));
  float gz = dot3(d0, f3(-4.0f * z, 2.0f * w, 2.0f * x)) + dot3(d1, f3(-2.0f * w, -4.0f * z, 2.0f * y));
  float gw = dot3(d0, f3(0.0f, 2.0f * z, -2.0f * y)) + dot3(d1, f3(-2.0f * z, 0.0f, 2.0f * x));
  float dt = gx * x + gy * y + gz * z + gw * w;
  return make_float4((gx - x * dt) / g.qn, (gy - y * dt) / g.qn, (gz - z * dt) / g.qn, (gw - w * dt) / g.qn);
}

struct ParamGrads {
  float3 pos;
  float2 scales;
  float4 quat;
  float opacity;
  float sh[48];
  float cam[13];  // dL/dR (column-major 9), dL/dC 3, dL/dfocal
};

// Chains one (surfel, view) record gradient into parameter and camera
// gradients, ADDING into `o` (the reference's backward.rs:176-248 /
// surfel_prep_bwd.wgsl:135-283, restated on the record parameterisation).
template <int PREC, bool AUX>
__device__ __forceinline__ void chain_one(const Cam& k, const float4 p, const float2 s, const float4 q, const void* sh,
                                          size_t i, const float* G, ParamGrads& o) {
  Geom g;
  geom(k, p, s, q, g);
  const float3 c = g.c, tu = g.tu, tv = g.tv;
  const float3 M = cross3(tu, tv), Bu = cross3(tv, c), Bv = cross3(c, tu);
  const float3 GM = f3(G[0], G[1], G[2]), GBu = f3(G[3], G[4], G[5]), GBv = f3(G[6], G[7], G[8]);
  const float Gpx = G[9], Gpy = G[10];
  float3 dc = f3(0, 0, 0), dtu = f3(0, 0, 0), dtv = f3(0, 0, 0);
  float3 GMt = GM;
  if (AUX) {
    const float Gtn = G[15];
    GMt -= c * Gtn;   // tn = −c·M
    dc -= M * Gtn;
  }
  dtu += cross3(tv, GMt);  // M = τu × τv
  dtv += cross3(GMt, tu);
  dtv += cross3(c, GBu);   // Bu = τv × c
  dc += cross3(GBu, tv);
  dc += cross3(tu, GBv);   // Bv = c × τu
  dtu += cross3(GBv, c);
  // Screen branch: px = cx + f c.x/w, py = cy − f c.y/w, w = −c.z (backward.rs:329-336).
  const float w = g.depth, f = k.f;
  dc.x += Gpx * f / w;
  dc.z += Gpx * f * c.x / (w * w);
  dc.y += Gpy * (-f / w);
  dc.z += Gpy * (-f * c.y / (w * w));
  float dfocal = Gpx * c.x / w + Gpy * (-c.y / w);
  // Ray branch focal path: s depends on f as ∂s/∂f = (−s.x/f, −s.y/f, 0), so
  // dL/df = −(1/f) Σ_K (K.x G_K.x + K.y G_K.y) over K ∈ {M, Bu, Bv}.
  dfocal -= (M.x * GM.x + M.y * GM.y + Bu.x * GBu.x + Bu.y * GBu.y + Bv.x * GBv.x + Bv.y * GBv.y) / f;
  if (AUX) {
    dc.z -= G[16];  // screen-branch t = centre depth = −c.z
    const float3 Gn = f3(G[17], G[18], G[19]);
    if (Gn.x != 0.0f || Gn.y != 0.0f || Gn.z != 0.0f) {
      const float len2 = dot3(M, M);
      if (len2 > 1e-24f) {
        const float len = sqrtf(len2);
        const float3 mh = M * (1.0f / len);
        const float sign = dot3(mh, c) > 0.0f ? -1.0f : 1.0f;
        const float3 dlm = (Gn - mh * dot3(mh, Gn)) * (sign / len);
        dtu += cross3(tv, dlm);
        dtv += cross3(dlm, tu);
      }
    }
  }
  // c = Rᵀ(p − C)
  const float3 dx = r_mul(k, dc);
  o.pos += dx;
  float3 dcenter = f3(-dx.x, -dx.y, -dx.z);
  float dR[9];
#pragma unroll
  for (int kk = 0; kk < 3; ++kk) {
    const float a = kk == 0 ? dc.x : (kk == 1 ? dc.y : dc.z);
    dR[3 * kk] = g.x.x * a; dR[3 * kk + 1] = g.x.y * a; dR[3 * kk + 2] = g.x.z * a;
  }
  // τ = Rᵀ(s R_q e_axis)
  const float3 dyu = r_mul(k, dtu), dyv = r_mul(k, dtv);
  o.scales.x += dot3(dyu, g.col0);
  o.scales.y += dot3(dyv, g.col1);
  const float4 dq = quat_grad2(g, dyu * s.x, dyv * s.y);
  o.quat.x += dq.x; o.quat.y += dq.y; o.quat.z += dq.z; o.quat.w += dq.w;
  const float3 yu = g.col0 * s.x, yv = g.col1 * s.y;
#pragma unroll
  for (int kk = 0; kk < 3; ++kk) {
    const float au = kk == 0 ? dtu.x : (kk == 1 ? dtu.y : dtu.z);
    const float av = kk == 0 ? dtv.x : (kk == 1 ? dtv.y : dtv.z);
    dR[3 * kk] += yu.x * au + yv.x * av;
    dR[3 * kk + 1] += yu.y * au + yv.y * av;
    dR[3 * kk + 2] += yu.z * au + yv.z * av;
  }
  // Colour → SH and the view-direction path, masked where the forward clamped.
  float3 dcol = f3(G[11], G[12], G[13]);
  const float lx = sqrtf(dot3(g.x, g.x));
  const float3 dir = f3(g.x.x / lx, g.x.y / lx, g.x.z / lx);
  float b[16];
  int nb;
  const float3 raw = sh_raw_color<PREC>(sh, i, k.deg, dir, b, nb);
  if (raw.x < 0.0f) dcol.x = 0.0f;
  if (raw.y < 0.0f) dcol.y = 0.0f;
  if (raw.z < 0.0f) dcol.z = 0.0f;
  if (dcol.x != 0.0f || dcol.y != 0.0f || dcol.z != 0.0f) {
    float3 bg[16];
    sh_basis_grad(k.deg, dir, bg);
    float3 ddir = f3(0, 0, 0);
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      if (kk < nb) {
        o.sh[3 * kk] += dcol.x * b[kk];
        o.sh[3 * kk + 1] += dcol.y * b[kk];
        o.sh[3 * kk + 2] += dcol.z * b[kk];
        ddir += bg[kk] * dot3(sh_coeff<PREC>(sh, i, kk), dcol);
      }
    }
    const float3 dv = (ddir - dir * dot3(dir, ddir)) * (1.0f / lx);
    o.pos += dv;
    dcenter -= dv;
  }
  o.opacity += G[14];
#pragma unroll
  for (int kk = 0; kk < 9; ++kk) o.cam[kk] += dR[kk];
  o.cam[9] += dcenter.x; o.cam[10] += dcenter.y; o.cam[11] += dcenter.z;
  o.cam[12] += dfocal;
}

__device__ __forceinline__ void zero_grads(ParamGrads& o) {
  o.pos = f3(0, 0, 0); o.scales = make_float2(0, 0); o.quat = make_float4(0, 0, 0, 0); o.opacity = 0;
#pragma unroll
  for (int k = 0; k < 48; ++k) o.sh[k] = 0;
#pragma unroll
  for (int k = 0; k < 13; ++k) o.cam[k] = 0;
}

// Reads the record gradient of item `item` (atomic mode) or sums its ordered
// per-entry partials (deterministic mode). Returns false when all zero.
template <bool AUX>
__device__ __forceinline__ bool load_G(const ProjectBwdArgs& a, uint32_t item, float G[GG_STRIDE]) {
  const int NG = AUX ? GG_STRIDE : 16;
#pragma unroll
  for (int k = 0; k < GG_STRIDE; ++k) G[k] = 0.0f;
  if (a.partials == nullptr) {
    const float4* gp = reinterpret_cast<const float4*>(a.grad_geom + (size_t)item * GG_STRIDE);
#pragma unroll
    for (int k = 0; k < NG / 4; ++k) {
      float4 t = gp[k];
      G[4 * k] = t.x; G[4 * k + 1] = t.y; G[4 * k + 2] = t.z; G[4 * k + 3] = t.w;
    }
  } else {
    const uint32_t beg = a.entry_offset[item], cnt = a.counts[item];
    if ((unsigned long long)beg + cnt > *a.entry_total) return false;  // stale offset after an overflow
    for (uint32_t e = beg; e < beg + cnt; ++e) {
      const float4* gp = reinterpret_cast<const float4*>(a.partials + (size_t)e * GG_STRIDE);
#pragma unroll
      for (int k = 0; k < NG / 4; ++k) {
        float4 t = gp[k];
        G[4 * k] += t.x; G[4 * k + 1] += t.y; G[4 * k + 2] += t.z; G[4 * k + 3] += t.w;
      }
    }
  }
  bool nz = false;
#pragma unroll
  for (int k = 0; k < GG_STRIDE; ++k) nz |= (G[k] != 0.0f);
  return nz;
}

// Camera gradient of the view: warp sums, one vector reduction per warp.
__device__ __forceinline__ void flush_cam(float* grad_cam_view, const float cam[13]) {
  float v[16];
#pragma unroll
  for (int k = 0; k < 13; ++k) v[k] = cam[k];
  v[13] = v[14] = v[15] = 0.0f;
  float r = warp_reduce16(v);
  const int lane = threadIdx.x & 31;
  // lanes 2c hold component c; gather the 16 sums to lanes 0..3 as float4s.
  float s[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) s[c] = __shfl_sync(0xffffffffu, r, 2 * c);
  if (lane == 0) {
    red_add_v4(grad_cam_view, s[0], s[1], s[2], s[3]);
    red_add_v4(grad_cam_view + 4, s[4], s[5], s[6], s[7]);
    red_add_v4(grad_cam_view + 8, s[8], s[9], s[10], s[11]);
    atomicAdd(grad_cam_view + 12, s[12]);
  }
}

// Plain form: one view per launch, gradients ADDED into the grad buffers.
template <int PREC, bool AUX>
__global__ void __launch_bounds__(256) k_project_bwd(ProjectBwdArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < a.n;
  const int v = a.view;
  ParamGrads o;
  zero_grads(o);
  bool any = false;
  if (valid) {
    float G[GG_STRIDE];
    const uint32_t item = (uint32_t)v * a.n + i;
    if (load_G<AUX>(a, item, G)) {
      const Cam k = load_cam(a.views, v);
      chain_one<PREC, AUX>(k, __ldg(a.pos + i), __ldg(a.scales + i), __ldg(a.quats + i), a.sh, i, G, o);
      any = true;
    }
  }
  if (a.grad_cam && __any_sync(0xffffffffu, any)) flush_cam(a.grad_cam + 16 * v, o.cam);
  if (!any) return;
  float4* gp = a.grad_pos + i;
  float4 t = *gp;
  *gp = make_float4(t.x + o.pos.x, t.y + o.pos.y, t.z + o.pos.z, t.w);
  float2 ts = a.grad_scales[i];
  a.grad_scales[i] = make_float2(ts.x + o.scales.x, ts.y + o.scales.y);
  float4 tq = a.grad_quat[i];
  a.grad_quat[i] = make_float4(tq.x + o.quat.x, tq.y + o.quat.y, tq.z + o.quat.z, tq.w + o.quat.w);
  a.grad_opacity[i] += o.opacity;
  float4* sh = reinterpret_cast<float4*>(a.grad_sh + (size_t)i * SH_FLOATS);
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    float4 u = sh[k];
    sh[k] = make_float4(u.x + o.sh[4 * k], u.y + o.sh[4 * k + 1], u.z + o.sh[4 * k + 2], u.w + o.sh[4 * k + 3]);
  }
}

// Adam on one raw value (first_attempt/crates/gs-train/src/shaders/adam.wgsl:45-58).
__device__ __forceinline__ float adam1(float& raw, float& m, float& v, float g, const AdamClass& c, float b1, float b2,
                                       float eps, float bc1, float bc2) {
  m = b1 * m + (1.0f - b1) * g;
  v = b2 * v + (1.0f - b2) * g * g;
  raw -= c.lr * (m * bc1) / (sqrtf(v * bc2) + eps);
  return raw;
}

// Chosen form: projection backward over all views of the step fused with the
// Adam step and the activation refresh, one thread per surfel. Parameter
// gradients never leave registers.
template <int PREC, bool AUX>
__global__ void __launch_bounds__(256) k_project_bwd_adam(ProjectBwdArgs a, AdamFusedArgs opt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < a.n;
  ParamGrads o;
  zero_grads(o);
  float4 p = make_float4(0, 0, 0, 0), q = p;
  float2 s = make_float2(0, 0);
  if (valid) { p = __ldg(a.pos + i); s = __ldg(a.scales + i); q = __ldg(a.quats + i); }
  for (int v = 0; v < a.n_views; ++v) {
    float cam_before[13];
#pragma unroll
    for (int k = 0; k < 13; ++k) { cam_before[k] = o.cam[k]; o.cam[k] = 0.0f; }
    bool any = false;
    if (valid) {
      float G[GG_STRIDE];
      if (load_G<AUX>(a, (uint32_t)v * a.n + i, G)) {
        const Cam k = load_cam(a.views, v);
        chain_one<PREC, AUX>(k, p, s, q, a.sh, i, G, o);
        any = true;
      }
    }
    if (a.grad_cam && __any_sync(0xffffffffu, any)) flush_cam(a.grad_cam + 16 * v, o.cam);
#pragma unroll
    for (int k = 0; k < 13; ++k) o.cam[k] = cam_before[k];
  }
  if (!valid) return;
  if (opt.accum_grad_norm) opt.accum_grad_norm[i] += sqrtf(o.pos.x * o.pos.x + o.pos.y * o.pos.y + o.pos.z * o.pos.z);
  const float b1 = opt.beta1, b2 = opt.beta2, eps = opt.eps;
  float bc1 = opt.bc1_inv, bc2 = opt.bc2_inv;
  AdamClass cls[5];
#pragma unroll
  for (int c = 0; c < 5; ++c) cls[c] = opt.cls[c];
  if (opt.dyn) {
    // {lr[5], reg[5], bc1_inv, bc2_inv} written by the host before a graph replay.
#pragma unroll
    for (int c = 0; c < 5; ++c) { cls[c].lr = __ldg(opt.dyn + c); cls[c].reg = __ldg(opt.dyn + 5 + c); }
    bc1 = __ldg(opt.dyn + 10);
    bc2 = __ldg(opt.dyn + 11);
  }
  // pos (identity; the w lane has zero gradient and never moves)
  {
    const AdamClass& c = cls[0];
    float4 r = reinterpret_cast<float4*>(c.raw)[i], m = reinterpret_cast<float4*>(c.m)[i],
           vv = reinterpret_cast<float4*>(c.v)[i];
    float gx = o.pos.x + c.reg, gy = o.pos.y + c.reg, gz = o.pos.z + c.reg;
    adam1(r.x, m.x, vv.x, gx, c, b1, b2, eps, bc1, bc2);
    adam1(r.y, m.y, vv.y, gy, c, b1, b2, eps, bc1, bc2);
    adam1(r.z, m.z, vv.z, gz, c, b1, b2, eps, bc1, bc2);
    adam1(r.w, m.w, vv.w, c.reg, c, b1, b2, eps, bc1, bc2);
    reinterpret_cast<float4*>(c.raw)[i] = r; reinterpret_cast<float4*>(c.m)[i] = m; reinterpret_cast<float4*>(c.v)[i] = vv;
    reinterpret_cast<float4*>(c.act)[i] = r;
  }
  // scales (exp)
  {
    const AdamClass& c = cls[1];
    float2 r = reinterpret_cast<float2*>(c.raw)[i], m = reinterpret_cast<float2*>(c.m)[i],
           vv = reinterpret_cast<float2*>(c.v)[i];
    float ex = __expf(r.x), ey = __expf(r.y);
    adam1(r.x, m.x, vv.x, (o.scales.x + c.reg) * ex, c, b1, b2, eps, bc1, bc2);
    adam1(r.y, m.y, vv.y, (o.scales.y + c.reg) * ey, c, b1, b2, eps, bc1, bc2);
    reinterpret_cast<float2*>(c.raw)[i] = r; reinterpret_cast<float2*>(c.m)[i] = m; reinterpret_cast<float2*>(c.v)[i] = vv;
    reinterpret_cast<float2*>(c.act)[i] = make_float2(__expf(r.x), __expf(r.y));
  }
  // quat (identity)
  {
    const AdamClass& c = cls[2];
    float4 r = reinterpret_cast<float4*>(c.raw)[i], m = reinterpret_cast<float4*>(c.m)[i],
           vv = reinterpret_cast<float4*>(c.v)[i];
    adam1(r.x, m.x, vv.x, o.quat.x + c.reg, c, b1, b2, eps, bc1, bc2);
    adam1(r.y, m.y, vv.y, o.quat.y + c.reg, c, b1, b2, eps, bc1, bc2);
    adam1(r.z, m.z, vv.z, o.quat.z + c.reg, c, b1, b2, eps, bc1, bc2);
    adam1(r.w, m.w, vv.w, o.quat.w + c.reg, c, b1, b2, eps, bc1, bc2);
    reinterpret_cast<float4*>(c.raw)[i] = r; reinterpret_cast<float4*>(c.m)[i] = m; reinterpret_cast<float4*>(c.v)[i] = vv;
    reinterpret_cast<float4*>(c.act)[i] = r;
  }
  // opacity (sigmoid)
  {
    const AdamClass& c = cls[3];
    float r = c.raw[i], m = c.m[i], vv = c.v[i];
    float sg = 1.0f / (1.0f + __expf(-r));
    adam1(r, m, vv, (o.opacity + c.reg) * (sg * (1.0f - sg)), c, b1, b2, eps, bc1, bc2);
    c.raw[i] = r; c.m[i] = m; c.v[i] = vv;
    c.act[i] = 1.0f / (1.0f + __expf(-r));
  }
  // sh (identity), 48 per surfel
  {
    const AdamClass& c = cls[4];
    float4* rr = reinterpret_cast<float4*>(c.raw) + (size_t)i * 12;
    float4* mm = reinterpret_cast<float4*>(c.m) + (size_t)i * 12;
    float4* vp = reinterpret_cast<float4*>(c.v) + (size_t)i * 12;
    float4* ap = reinterpret_cast<float4*>(c.act) + (size_t)i * 12;
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      float4 r = rr[k], m = mm[k], vv = vp[k];
      adam1(r.x, m.x, vv.x, o.sh[4 * k] + c.reg, c, b1, b2, eps, bc1, bc2);
      adam1(r.y, m.y, vv.y, o.sh[4 * k + 1] + c.reg, c, b1, b2, eps, bc1, bc2);
      adam1(r.z, m.z, vv.z, o.sh[4 * k + 2] + c.reg, c, b1, b2, eps, bc1, bc2);
      adam1(r.w, m.w, vv.w, o.sh[4 * k + 3] + c.reg, c, b1, b2, eps, bc1, bc2);
      rr[k] = r; mm[k] = m; vp[k] = vv; ap[k] = r;
      if (opt.sh_half) {
        if (opt.sh_half_is_bf16) {
          __nv_bfloat162* hp = reinterpret_cast<__nv_bfloat162*>(opt.sh_half) + ((size_t)i * 48 + 4 * k) / 2;
          hp[0] = __floats2bfloat162_rn(r.x, r.y);
          hp[1] = __floats2bfloat162_rn(r.z, r.w);
        } else {
          __half2* hp = reinterpret_cast<__half2*>(opt.sh_half) + ((size_t)i * 48 + 4 * k) / 2;
          hp[0] = __floats2half2_rn(r.x, r.y);
          hp[1] = __floats2half2_rn(r.z, r.w);
        }
      }
    }
  }
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

int launch_project_bwd(const ProjectBwdArgs& a, int prec, bool aux, cudaStream_t st) {
  if (a.n == 0) return 0;
  dim3 grid((a.n + 255) / 256);
#define GS_PB(P, X) k_project_bwd<P, X><<<grid, 256, 0, st>>>(a)
  if (prec == 0) { if (aux) GS_PB(0, true); else GS_PB(0, false); }
  else if (prec == 1) { if (aux) GS_PB(1, true); else GS_PB(1, false); }
  else { if (aux) GS_PB(2, true); else GS_PB(2, false); }
#undef GS_PB
  return (int)cudaGetLastError();
}

int launch_project_bwd_adam(const ProjectBwdArgs& a, const AdamFusedArgs& opt, int prec, bool aux, cudaStream_t st) {
  if (a.n == 0) return 0;
  dim3 grid((a.n + 255) / 256);
#define GS_PBA(P, X) k_project_bwd_adam<P, X><<<grid, 256, 0, st>>>(a, opt)
  if (prec == 0) { if (aux) GS_PBA(0, true); else GS_PBA(0, false); }
  else if (prec == 1) { if (aux) GS_PBA(1, true); else GS_PBA(1, false); }
  else { if (aux) GS_PBA(2, true); else GS_PBA(2, false); }
#undef GS_PBA
  return (int)cudaGetLastError();
}

}  // namespace gs
