// Shared device helpers of the projection and its adjoint: SH constants and
// basis, camera and surfel geometry. Included by gs_project.cu (compiled
// without FMA contraction so the forward rect/key arithmetic matches its f32
// restatement bit for bit) and gs_project_bwd.cu (normal contraction).
#pragma once
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
  int W, H, tiles_x, tiles_y, tile, deg;
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
  c.tile = __ldg(&V->tile);
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

// Raw SH colour 0.5 + Σ b_k sh_k (surfel_prep_fwd.wgsl:121-147); `coeff(k)`
// returns coefficient k (rgb).
template <class Coeff>
__device__ __forceinline__ float3 sh_raw_color_with(Coeff coeff, int deg, float3 dir, float b[16], int& nb) {
  nb = sh_basis(deg, dir, b);
  // Explicit FMAs: the projection (built without contraction) and its
  // adjoint (built with it) then round the raw colour identically, so they
  // agree on its clamp at zero.
  float3 acc = f3(0, 0, 0);
#pragma unroll
  for (int k = 0; k < 16; ++k) {  // constant indices keep b[] in registers
    if (k < nb) {
      const float3 c = coeff(k);
      acc = f3(fmaf(c.x, b[k], acc.x), fmaf(c.y, b[k], acc.y), fmaf(c.z, b[k], acc.z));
    }
  }
  return acc + f3(0.5f, 0.5f, 0.5f);
}
template <int PREC>
__device__ __forceinline__ float3 sh_raw_color(const void* sh, size_t i, int deg, float3 dir, float b[16], int& nb) {
  return sh_raw_color_with([&](int k) { return sh_coeff<PREC>(sh, i, k); }, deg, dir, b, nb);
}

// A surfel's 48 SH values held in registers, fetched with 16-byte loads
// (12 for f32 storage, 6 for 16-bit); value j is taken from word j (f32) or
// half j (16-bit). With compile-time j (unrolled loops) the selection is free.
template <int PREC>
struct ShRow {
  static constexpr int Q = PREC == 0 ? SH_FLOATS / 4 : SH_FLOATS / 8;
  uint4 q[Q];
  __device__ __forceinline__ void load(const void* sh, size_t i) {
    const uint4* p = reinterpret_cast<const uint4*>(sh) + i * Q;
#pragma unroll
    for (int k = 0; k < Q; ++k) q[k] = __ldg(p + k);
  }
  __device__ __forceinline__ uint32_t word(int w) const {
    const uint4& u = q[w >> 2];
    const int c = w & 3;
    return c == 0 ? u.x : (c == 1 ? u.y : (c == 2 ? u.z : u.w));
  }
  __device__ __forceinline__ float value(int j) const {
    if constexpr (PREC == 0) {
      return __uint_as_float(word(j));
    } else {
      using H = typename std::conditional<PREC == 1, __half, __nv_bfloat16>::type;
      const uint32_t w = word(j >> 1);
      const unsigned short bits = (unsigned short)((j & 1) ? (w >> 16) : (w & 0xffffu));
      H h;
      memcpy(&h, &bits, 2);
      return h2f<H>(h);
    }
  }
  __device__ __forceinline__ float3 coeff(int k) const { return f3(value(3 * k), value(3 * k + 1), value(3 * k + 2)); }
};

}  // namespace
}  // namespace gs
