// Shared device-side definitions of the surfel training step.
//
// Conventions follow the reference renderer (crates/gs-cpu-ref/src/scene.rs:4-13
// and crates/gs-kernels/src/shaders/raster_common.wgsl:5-95): right-handed
// camera looking down its local -z, x_cam = Rᵀ(p − C) with R camera-to-world,
// pixel ray d = ((x+.5−cx)/f, −(y+.5−cy)/f, −1) with the principal point at
// the image centre, surfel tangent axes τu = Rᵀ R_q e0 s_u, τv = Rᵀ R_q e1 s_v.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace gs {

// raster_common.wgsl:34-39 / scene.rs:17-21
constexpr float LOWPASS_SIGMA2 = 0.5f;
constexpr float ALPHA_SKIP = 0.0039215686f;  // 1/255
constexpr float ALPHA_CLAMP = 0.995f;
constexpr float T_TERMINATE = 1e-4f;
constexpr float NEAR_DEPTH = 0.05f;
constexpr int TILE = 16;  // the reference tile size (rasterizer.rs:13); 8 and 32 are also built
constexpr int SH_FLOATS = 48;

// Sticky device error word bits.
constexpr uint32_t ERR_ENTRY_CAPACITY = 1u << 0;
constexpr uint32_t ERR_TIMEOUT = 1u << 1;

// Per-view camera and image layout, one entry per view of a step.
struct ViewInfo {
  float rot[9];       // camera-to-world R, column-major: rot[3*k + j] = R[j][k]
  float center[3];
  float focal;
  float cx, cy;       // width/2, height/2
  int width, height;
  int tiles_x, tiles_y;
  int tile;           // tile edge in pixels: 8, 16 or 32
  int tile_base;      // first global tile id of this view
  int sh_degree;
  long long pix_base; // first pixel of this view in per-pixel buffers
  double rot64[9];    // R again in double (accurate projected centres, see the record below)
};

// Projected surfel record ("SurfelCam"), one per (view, surfel). The ray–splat
// intersection of crates/gs-cpu-ref/src/forward.rs:136-169 solves
// [τu τv −d](u,v,t)ᵀ = −c by Cramer's rule; with s = −d every triple product
// is linear in s:  det = s·M,  u·det = s·Bu,  v·det = s·Bv,  t·det = tn, where
// M = τu×τv, Bu = τv×c, Bv = c×τu, tn = −c·M. The ray s_c through the
// surfel's centre is parallel to c, so Bu·s_c = Bv·s_c = 0 and, for a pixel
// ray s = s_c + Δs with Δs = (−dx/f, dy/f, 0) (dx, dy: the pixel centre minus
// the projected centre, in pixels), u·det = Bu·Δs and v·det = Bv·Δs exactly.
// Evaluating them from the screen offsets avoids the cancellation of s·Bu
// (|Bu| ~ |c||τ| against u·det ~ |τ|² cosθ for a surfel seen at angle θ to
// its normal), which in FP32 costs up to ~10 % of a nearly edge-on surfel's
// gradient; the projected centre is computed in double and kept as hi + lo.
//   r0 = (M, tn)  r1 = (−Bu.x/f, Bu.y/f, px_lo, px_hi)  r2 = (−Bv.x/f, Bv.y/f, py_lo, py_hi)
//   r3 = (colour rgb, opacity)  r4 = (normal xyz, centre depth)
//   bb = pixel box (x0, x1, y0, y1) outside which α < 1/255 for certain
// Per pixel: det = M·s, u·det = r1.x·dx + r1.y·dy, v·det = r2.x·dx + r2.y·dy,
// t·det = tn, with dx = (pxc − px_hi) − px_lo, dy = (pyc − py_hi) − py_lo.
// FP32 record: 6 float4 = 96 B. Mixed-precision record (80 B, 5 float4):
// geometry r0..r2 and colour/opacity r3 stay FP32 (the geometry feeds a ratio
// of nearly cancelling dot products; colour and opacity rounded to 16 bits
// dominate the gradient error, about 6e-4 and 2e-4 relative at 200k surfels
// x 720p), normal and depth are 16-bit, and the α-box is stored as int16
// pixel bounds: the smallest and largest pixel index whose centre lies inside
// the float box, per axis. Pixel x's centre x + 0.5 lies in [b.x, b.y] exactly
// when lo <= x <= hi, so the loader returns (lo + 0.5, hi + 0.5, ...) and every
// box test selects the same pixels as with the float box. Images up to 32766
// pixels per side.
constexpr int REC_F4_F32 = 6;
constexpr int REC_F4_H = 5;
constexpr int REC_MAX_SIDE_H = 32766;

template <typename H> __device__ __forceinline__ float h2f(H x);
template <> __device__ __forceinline__ float h2f<__half>(__half x) { return __half2float(x); }
template <> __device__ __forceinline__ float h2f<__nv_bfloat16>(__nv_bfloat16 x) { return __bfloat162float(x); }
template <typename H> __device__ __forceinline__ H f2h(float x);
template <> __device__ __forceinline__ __half f2h<__half>(float x) { return __float2half_rn(x); }
template <> __device__ __forceinline__ __nv_bfloat16 f2h<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }

// Smallest integer k with k + 0.5 >= z, and largest k with k + 0.5 <= z,
// clamped to [-5, 32767] (beyond every pixel of an image of at most 32766
// pixels per side). The float estimate is corrected with the exact
// comparisons the raster's per-pixel test makes.
__device__ __forceinline__ int pix_lo(float z) {
  const float zc = fminf(fmaxf(z, -4.0f), 32767.0f);
  int k = (int)ceilf(zc - 0.5f);
  if ((float)k + 0.5f < zc) ++k;
  if ((float)(k - 1) + 0.5f >= zc) --k;
  return k;
}
__device__ __forceinline__ int pix_hi(float z) {
  const float zc = fminf(fmaxf(z, -4.0f), 32767.0f);
  int k = (int)floorf(zc - 0.5f);
  if ((float)k + 0.5f > zc) --k;
  if ((float)(k + 1) + 0.5f <= zc) ++k;
  return k;
}

template <int PREC>
__device__ __forceinline__ const float4* record_ptr(const void* recs, uint32_t idx) {
  return reinterpret_cast<const float4*>(recs) + (size_t)idx * (PREC == 0 ? REC_F4_F32 : REC_F4_H);
}

// The α box of record `idx` (read first, so culled entries cost one load).
template <int PREC>
__device__ __forceinline__ float4 load_record_box(const void* recs, uint32_t idx) {
  if constexpr (PREC == 0) {
    return __ldg(record_ptr<PREC>(recs, idx) + 5);
  } else {
    const int4 raw = __ldg(reinterpret_cast<const int4*>(record_ptr<PREC>(recs, idx) + 4));
    // int16 pairs (lo, hi) of x in raw.z, of y in raw.w (little endian)
    const int x0 = (int)(short)(raw.z & 0xffff), x1 = raw.z >> 16;
    const int y0 = (int)(short)(raw.w & 0xffff), y1 = raw.w >> 16;
    return make_float4((float)x0 + 0.5f, (float)x1 + 0.5f, (float)y0 + 0.5f, (float)y1 + 0.5f);
  }
}

// Loads the geometry and appearance of record `idx` as five float4
// (converting 16-bit fields).
template <int PREC>
__device__ __forceinline__ void load_record(const void* recs, uint32_t idx, float4& r0, float4& r1, float4& r2,
                                            float4& r3, float4& r4) {
  const float4* p = record_ptr<PREC>(recs, idx);
  r0 = __ldg(p); r1 = __ldg(p + 1); r2 = __ldg(p + 2); r3 = __ldg(p + 3);
  if constexpr (PREC == 0) {
    r4 = __ldg(p + 4);
  } else {
    using H = typename std::conditional<PREC == 1, __half, __nv_bfloat16>::type;
    const float4 raw = __ldg(p + 4);
    const H* h = reinterpret_cast<const H*>(&raw);
    r4 = make_float4(h2f<H>(h[0]), h2f<H>(h[1]), h2f<H>(h[2]), h2f<H>(h[3]));
  }
}

// The geometry and colour/opacity alone (r0..r3): what the colour-only
// kernels read.
template <int PREC>
__device__ __forceinline__ void load_record4(const void* recs, uint32_t idx, float4& r0, float4& r1, float4& r2,
                                             float4& r3) {
  const float4* p = record_ptr<PREC>(recs, idx);
  r0 = __ldg(p); r1 = __ldg(p + 1); r2 = __ldg(p + 2); r3 = __ldg(p + 3);
}

template <int PREC>
__device__ __forceinline__ void store_record(void* recs, uint32_t idx, float4 r0, float4 r1, float4 r2, float4 r3,
                                             float4 r4, float4 box) {
  float4* p = reinterpret_cast<float4*>(recs) + (size_t)idx * (PREC == 0 ? REC_F4_F32 : REC_F4_H);
  p[0] = r0; p[1] = r1; p[2] = r2; p[3] = r3;
  if constexpr (PREC == 0) {
    p[4] = r4; p[5] = box;
  } else {
    using H = typename std::conditional<PREC == 1, __half, __nv_bfloat16>::type;
    int4 raw;
    H* h = reinterpret_cast<H*>(&raw);
    h[0] = f2h<H>(r4.x); h[1] = f2h<H>(r4.y); h[2] = f2h<H>(r4.z); h[3] = f2h<H>(r4.w);
    raw.z = (int)(((uint32_t)pix_hi(box.y) << 16) | ((uint32_t)pix_lo(box.x) & 0xffffu));
    raw.w = (int)(((uint32_t)pix_hi(box.w) << 16) | ((uint32_t)pix_lo(box.z) & 0xffffu));
    reinterpret_cast<int4*>(p)[4] = raw;
  }
}

inline size_t record_bytes(int prec) { return prec == 0 ? 96 : 80; }

// Per-surfel camera-space gradient layout written by the backward raster and
// consumed by the projection backward ("grad_geom"). The backward raster
// reduces gradients with respect to the record fields, not (c, τu, τv): the
// chain through M, Bu, Bv, tn is linear, so it is applied once per surfel.
//   0-2 dL/dM   3-5 dL/dBu   6-8 dL/dBv   9 dL/dpx   10 dL/dpy
//   11-13 dL/dcolour   14 dL/dopacity   15 dL/dtn
//   16 dL/ddepth (screen-branch t)   17-19 dL/dnormal   (aux losses only)
constexpr int GG_STRIDE = 20;

__device__ __forceinline__ void red_add_v4(float* p, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1,%2,%3,%4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Warp "transpose" reduction of 16 per-lane values: after it, lanes 2c and
// 2c+1 hold the warp-wide sum of value c. 16 shuffles instead of the 80 of
// sixteen independent butterflies.
__device__ __forceinline__ float warp_reduce16(float (&v)[16]) {
  const unsigned FULL = 0xffffffffu;
  int lane = threadIdx.x & 31;
  float a[8];
  bool hi = lane & 16;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    float send = hi ? v[k] : v[k + 8];
    float keep = hi ? v[k + 8] : v[k];
    a[k] = keep + __shfl_xor_sync(FULL, send, 16);
  }
  float b[4];
  hi = lane & 8;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float send = hi ? a[k] : a[k + 4];
    float keep = hi ? a[k + 4] : a[k];
    b[k] = keep + __shfl_xor_sync(FULL, send, 8);
  }
  float c[2];
  hi = lane & 4;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    float send = hi ? b[k] : b[k + 2];
    float keep = hi ? b[k + 2] : b[k];
    c[k] = keep + __shfl_xor_sync(FULL, send, 4);
  }
  hi = lane & 2;
  float d = (hi ? c[1] : c[0]) + __shfl_xor_sync(FULL, hi ? c[0] : c[1], 2);
  return d + __shfl_xor_sync(FULL, d, 1);
}
// Component held by this lane after warp_reduce16: bits 4..1 of the lane id.
__device__ __forceinline__ int reduce16_component(int lane) {
  return ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace gs

#define GS_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) return ::gs::cuda_fail(_e, #expr, __FILE__, __LINE__); \
  } while (0)

namespace gs {
int cuda_fail(cudaError_t e, const char* expr, const char* file, int line);
}
