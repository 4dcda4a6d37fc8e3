// Fused L1 + D-SSIM loss and its analytic gradient
// (first_attempt/crates/gs-train/src/shaders/ssim.wgsl:41-143,
// first_attempt/crates/gs-train/src/ssim.rs:236-280).
//
// The reference runs 19 full-image passes (products, 8 separable blurs of
// two dispatches each, partials, combine) through ~17 image-sized buffers.
// Here two tiled kernels cover every view of a step:
//   k_ssim_moments: per 16×16 tile, stage x and y with a 5-pixel halo in
//     shared memory, blur the five moments (μx, μy, x², y², xy) of the three
//     channels separably, form SSIM and the three coefficient maps Cμ, Cx²,
//     Cxy per channel (ssim.wgsl:94-126), stored as four float2 planes and
//     one float plane, and accumulate the per-view loss sums.
//   k_ssim_grad: stage the nine coefficient planes with a halo, blur them
//     (the zero-padded symmetric window is self-adjoint) and combine with the
//     L1 term into dL/dx (ssim.wgsl:130-143).
// L = w_l1·mean|x−y| + w_ssim·mean(1−S) over pixels × rgb of each view.
#include <algorithm>

#include "gs_common.cuh"
#include "gs_kernels.h"

namespace gs {
namespace {

// Output tiles of 16×16 pixels, inputs staged with a 5-pixel halo (26×26).
// Separable 11-tap blurs run as sliding windows in registers: a horizontal
// pass where each thread owns one (row, channel or plane) and slides along x,
// then a vertical pass where each thread owns one (column, channel or plane)
// and slides along y, so every staged value is read from shared memory once
// per pass. Pairs of maps blur together in the packed two-wide FP32
// instructions of sm_100 (FFMA2/FADD2/FMUL2): (μx, μy) and (E[x²], E[y²]) per
// channel in the moments kernel, two coefficient planes at a time in the
// gradient kernel; each component rounds as the scalar operation would.
constexpr int T16 = 16, HALO = 5, EXT = T16 + 2 * HALO;  // 26
constexpr int TAPS = 2 * HALO + 1;                       // 11
// Staged rows use an odd pitch (read by lanes holding consecutive rows; for
// 8-byte elements the two 16-lane phases then hit distinct banks), horizontal
// results an odd row pitch, vertical results dense 16×16 planes.
constexpr int IN_PITCH = EXT + 1;                        // 27
constexpr int H_ROW = T16 + 1;                           // 17
constexpr int H_PLANE = EXT * H_ROW;                     // 442
constexpr int V_PLANE = T16 * T16;                       // 256

struct TileLoc {
  int v, x0, y0, W, H;
  long long pix_base;
};

__device__ __forceinline__ TileLoc locate(const SsimArgs& a, int t) {
  TileLoc L;
  int v = 0, base = 0;
  for (;;) {
    const ViewInfo* V = a.views + v;
    const int W = __ldg(&V->width), H = __ldg(&V->height);
    const int nt = ((W + T16 - 1) / T16) * ((H + T16 - 1) / T16);
    if (t < base + nt || v + 1 == a.n_views) {
      const int lt = t - base, tx = (W + T16 - 1) / T16;
      L.v = v; L.W = W; L.H = H;
      L.x0 = (lt % tx) * T16; L.y0 = (lt / tx) * T16;
      L.pix_base = __ldg(&V->pix_base);
      return L;
    }
    base += nt;
    ++v;
  }
}

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// Asynchronous copy of B bytes (4, 8 or 16; both addresses B-aligned) from
// global to shared memory; when !valid nothing is read and the B bytes are
// zero-filled. Completion: cp.async.wait_all, then a barrier for other threads.
template <int B>
__device__ __forceinline__ void cp_async_zfill(void* smem, const void* gmem, bool valid) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(s), "l"(gmem), "n"(B), "r"(valid ? B : 0)
               : "memory");
}

// Slides an 11-tap window along `N_OUT` outputs: out[o] = Σ_d w[|d−5|]·in(o+d)
// (w[k] is the weight at offset ±k), for a scalar map.
template <int N_OUT, class In, class Out>
__device__ __forceinline__ void slide11(const float (&w)[6], In in, Out out) {
  float win[TAPS];
#pragma unroll
  for (int i = 0; i < TAPS - 1; ++i) win[i] = in(i);
#pragma unroll
  for (int o = 0; o < N_OUT; ++o) {
    win[TAPS - 1] = in(o + TAPS - 1);
    float acc = w[0] * win[HALO];
#pragma unroll
    for (int d = 0; d < HALO; ++d) acc += w[HALO - d] * (win[d] + win[TAPS - 1 - d]);
    out(o, acc);
#pragma unroll
    for (int i = 0; i < TAPS - 1; ++i) win[i] = win[i + 1];
  }
}

// The same for two maps at once (float2 windows, packed instructions).
template <int N_OUT, class In, class Out>
__device__ __forceinline__ void slide11x2(const float (&w)[6], In in, Out out) {
  float2 win[TAPS];
#pragma unroll
  for (int i = 0; i < TAPS - 1; ++i) win[i] = in(i);
#pragma unroll
  for (int o = 0; o < N_OUT; ++o) {
    win[TAPS - 1] = in(o + TAPS - 1);
    float2 acc = __fmul2_rn(f2(w[0]), win[HALO]);
#pragma unroll
    for (int d = 0; d < HALO; ++d) acc = __ffma2_rn(f2(w[HALO - d]), __fadd2_rn(win[d], win[TAPS - 1 - d]), acc);
    out(o, acc);
#pragma unroll
    for (int i = 0; i < TAPS - 1; ++i) win[i] = win[i + 1];
  }
}

// Moments → SSIM, its coefficient maps and the per-view loss sums.
// Eight blurred maps, seven of them packed pairs: per channel (μx, μy) and
// (E[x²], E[y²]), then (E[xy]_r, E[xy]_g), and E[xy]_b scalar. Eight maps
// give 208 horizontal row items and 256 vertical items (16 columns, two
// halves of 8 rows), so both passes occupy the block in a single round.
// Coefficient planes (scratch, coef_stride pixels each): float2 planes
// (Cμ_r, Cμ_g), (Cx²_r, Cx²_g), (Cxy_r, Cxy_g), (Cμ_b, Cx²_b) at
// coef + 2k·stride, and Cxy_b at coef + 8·stride.
constexpr int NM2 = 7;  // packed maps
__global__ void __launch_bounds__(256) k_ssim_moments(SsimArgs a) {
  __shared__ float2 s_in[3][EXT][IN_PITCH];     // (x, y) per channel, with halo
  __shared__ float2 s_h2[NM2][EXT * H_ROW];     // horizontal results of the packed maps [map][row][col]
  __shared__ float s_h1[EXT * H_ROW];           // horizontal E[xy]_b
  __shared__ double s_red[2][8];
  // Vertical results reuse s_in after the horizontal pass.
  float2* s_v2 = &s_in[0][0][0];                          // [map][16×16]
  float* s_v1 = reinterpret_cast<float*>(s_v2 + NM2 * V_PLANE);  // [16×16]
  static_assert(NM2 * V_PLANE * 2 + V_PLANE <= 3 * EXT * IN_PITCH * 2, "vertical results fit in s_in");
  const int tid = threadIdx.x;
  const TileLoc L = locate(a, blockIdx.x);
  for (int k = tid; k < EXT * EXT; k += 256) {
    const int ly = k / EXT, lx = k % EXT;
    const int gx = L.x0 + lx - HALO, gy = L.y0 + ly - HALO;
    float4 xv = make_float4(0, 0, 0, 0), yv = xv;
    if (gx >= 0 && gy >= 0 && gx < L.W && gy < L.H) {
      const long long p = L.pix_base + (long long)gy * L.W + gx;
      xv = a.img[p];
      yv = a.target[p];
    }
    s_in[0][ly][lx] = make_float2(xv.x, yv.x);
    s_in[1][ly][lx] = make_float2(xv.y, yv.y);
    s_in[2][ly][lx] = make_float2(xv.z, yv.z);
  }
  float w[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) w[k] = a.w[k];
  __syncthreads();
  // Horizontal: warp m blurs map m, lane r < EXT row r, so each warp runs one
  // of the four code paths (an item order that put two maps in a warp ran
  // both paths with half the lanes each).
  static_assert(NM2 + 1 == 8 && EXT <= 32, "one warp per map, one lane per staged row");
  if ((tid & 31) < EXT) {
    const int m = tid >> 5, r = tid & 31;
    if (m < 6) {
      const float2* XY = &s_in[m >> 1][r][0];
      float2* O = &s_h2[m][r * H_ROW];
      if (m & 1)
        slide11x2<T16>(w, [&](int i) { const float2 v = XY[i]; return __fmul2_rn(v, v); }, [&](int o, float2 v) { O[o] = v; });
      else
        slide11x2<T16>(w, [&](int i) { return XY[i]; }, [&](int o, float2 v) { O[o] = v; });
    } else if (m == 6) {
      const float2* R = &s_in[0][r][0];
      const float2* G = &s_in[1][r][0];
      float2* O = &s_h2[6][r * H_ROW];
      slide11x2<T16>(w, [&](int i) { const float2 u = R[i], v = G[i]; return make_float2(u.x * u.y, v.x * v.y); },
                     [&](int o, float2 v) { O[o] = v; });
    } else {
      const float2* B = &s_in[2][r][0];
      float* O = &s_h1[r * H_ROW];
      slide11<T16>(w, [&](int i) { const float2 v = B[i]; return v.x * v.y; }, [&](int o, float v) { O[o] = v; });
    }
  }
  // L1 of this thread's pixel, read before s_in is reused.
  const int ox = tid & 15, oy = tid >> 4;
  const int gx = L.x0 + ox, gy = L.y0 + oy;
  const bool inside = gx < L.W && gy < L.H;
  float l1 = 0.f;
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const float2 v = s_in[ch][oy + HALO][ox + HALO];
    if (inside) l1 += fabsf(v.x - v.y);
  }
  __syncthreads();
  // Vertical: item = (map, column, half): rows 8h..8h+7 from input rows 8h..8h+17.
  {
    const int m = tid >> 5, c = tid & 15, h = (tid >> 4) & 1;
    if (m < NM2) {
      const float2* I = &s_h2[m][c + 8 * h * H_ROW];
      float2* O = s_v2 + m * V_PLANE + c + 8 * h * T16;
      slide11x2<8>(w, [&](int i) { return I[i * H_ROW]; }, [&](int o, float2 v) { O[o * T16] = v; });
    } else {
      const float* I = &s_h1[c + 8 * h * H_ROW];
      float* O = s_v1 + c + 8 * h * T16;
      slide11<8>(w, [&](int i) { return I[i * H_ROW]; }, [&](int o, float v) { O[o * T16] = v; });
    }
  }
  __syncthreads();
  float ss = 0.f;
  if (inside) {
    const long long pix = L.pix_base + (long long)gy * L.W + gx;
    const float inv_n3 = 1.0f / (3.0f * (float)L.W * (float)L.H);
    const float C1 = 1e-4f, C2 = 9e-4f;
    const float dw = -a.w_ssim * inv_n3;
    float cm[3], cx2[3], cxy[3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      const int q = oy * T16 + ox;
      const float2 mu = s_v2[(ch * 2) * V_PLANE + q], b2 = s_v2[(ch * 2 + 1) * V_PLANE + q];
      const float bxy = ch == 0 ? s_v2[6 * V_PLANE + q].x : (ch == 1 ? s_v2[6 * V_PLANE + q].y : s_v1[q]);
      const float mu_x = mu.x, mu_y = mu.y;
      const float sx2 = b2.x - mu_x * mu_x, sy2 = b2.y - mu_y * mu_y, sxy = bxy - mu_x * mu_y;
      const float p = mu_x * mu_x + mu_y * mu_y + C1;
      const float qd = sx2 + sy2 + C2;
      // p >= C1 and qd ~>= C2: one approximate reciprocal each (about 1 ulp)
      // replaces the four IEEE divisions of the expressions.
      const float ip = __fdividef(1.0f, p), iq = __fdividef(1.0f, qd);
      const float l = (2.0f * mu_x * mu_y + C1) * ip;
      const float cs = (2.0f * sxy + C2) * iq;
      ss += l * cs;
      cm[ch] = (cs * (2.0f * mu_y - 2.0f * mu_x * l) * ip + l * (-2.0f * mu_y + 2.0f * mu_x * cs) * iq) * dw;
      cx2[ch] = (-l * cs * iq) * dw;
      cxy[ch] = (2.0f * l * iq) * dw;
    }
    float2* P2 = reinterpret_cast<float2*>(a.coef);
    const size_t st2 = a.coef_stride;  // float2 plane k starts at float offset 2k·stride
    P2[0 * st2 + pix] = make_float2(cm[0], cm[1]);
    P2[1 * st2 + pix] = make_float2(cx2[0], cx2[1]);
    P2[2 * st2 + pix] = make_float2(cxy[0], cxy[1]);
    P2[3 * st2 + pix] = make_float2(cm[2], cx2[2]);
    a.coef[8 * a.coef_stride + pix] = cxy[2];
  }
  // Per-view loss sums: warp, then block, then one double atomic each.
  double dl1 = warp_sum(l1), dss = warp_sum(ss);
  if ((tid & 31) == 0) { s_red[0][tid >> 5] = dl1; s_red[1][tid >> 5] = dss; }
  __syncthreads();
  if (tid == 0) {
    double t0 = 0, t1 = 0;
    for (int k = 0; k < 8; ++k) { t0 += s_red[0][k]; t1 += s_red[1][k]; }
    atomicAdd(a.loss_sums + 2 * L.v, t0);
    atomicAdd(a.loss_sums + 2 * L.v + 1, t1);
  }
}

// Blur of the nine coefficient maps (the zero-padded symmetric window is
// self-adjoint) combined with the L1 term into dL/dx: four float2 planes
// blurred as packed pairs and one scalar plane.
#ifndef GS_SSIM_GRAD_INPLACE
#define GS_SSIM_GRAD_INPLACE 1
#endif
__global__ void __launch_bounds__(256, GS_SSIM_GRAD_INPLACE ? 6 : 1) k_ssim_grad(SsimArgs a) {
  __shared__ float2 s_c2[4][EXT][IN_PITCH];
  __shared__ float s_c1[EXT][IN_PITCH];
  // In place, the horizontal pass writes each row's 16 results over the row's
  // first 16 staged values (a row belongs to one thread, and output o is
  // written after input o + 10 has been read), so the vertical results get a
  // buffer of their own and the block needs 34.5 KB of shared memory instead
  // of 41.2 KB: 6 resident blocks per SM instead of 5.
  constexpr bool INPL = GS_SSIM_GRAD_INPLACE;
  constexpr int HP = INPL ? IN_PITCH : H_ROW;  // row pitch of the horizontal results
  __shared__ float2 s_h2b[INPL ? 1 : 4][INPL ? 1 : EXT * H_ROW];
  __shared__ float s_h1b[INPL ? 1 : EXT * H_ROW];
  __shared__ float2 s_vb[INPL ? 4 * V_PLANE + V_PLANE / 2 : 1];
  auto s_h2 = [&](int m) -> float2* { return INPL ? &s_c2[m][0][0] : &s_h2b[INPL ? 0 : m][0]; };
  float* s_h1 = INPL ? &s_c1[0][0] : s_h1b;
  float2* s_v2 = INPL ? s_vb : &s_c2[0][0][0];                      // [4][16×16]
  float* s_v1 = reinterpret_cast<float*>(s_v2 + 4 * V_PLANE);        // [16×16]
  static_assert(4 * V_PLANE * 2 + V_PLANE <= 4 * EXT * IN_PITCH * 2, "vertical results fit in s_c2");
  const int tid = threadIdx.x;
  const TileLoc L = locate(a, blockIdx.x);
  // This thread's pixel of the image and target, loaded now so the loads are
  // in flight during the blurs.
  const int ox = tid & 15, oy = tid >> 4;
  const int gx = L.x0 + ox, gy = L.y0 + oy;
  const bool inside = gx < L.W && gy < L.H;
  const long long pix = inside ? L.pix_base + (long long)gy * L.W + gx : 0;
  float4 x = make_float4(0.f, 0.f, 0.f, 0.f), y = x;
  if (inside) {
    x = a.img[pix];
    y = a.target[pix];
  }
  const float2* P2 = reinterpret_cast<const float2*>(a.coef);
  const size_t st2 = a.coef_stride;
  // Staged with asynchronous copies (global -> shared, no registers), so all
  // of a thread's loads are in flight at once; pixels outside the view are
  // zero-filled by the copy (source size 0).
  for (int k = tid; k < EXT * EXT; k += 256) {
    const int ly = k / EXT, lx = k % EXT;
    const int gx = L.x0 + lx - HALO, gy = L.y0 + ly - HALO;
    const bool in = gx >= 0 && gy >= 0 && gx < L.W && gy < L.H;
    const size_t p = in ? (size_t)(L.pix_base + (long long)gy * L.W + gx) : 0;
#pragma unroll
    for (int m = 0; m < 4; ++m) cp_async_zfill<8>(&s_c2[m][ly][lx], P2 + m * st2 + p, in);
    cp_async_zfill<4>(&s_c1[ly][lx], a.coef + 8 * a.coef_stride + p, in);
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  float w[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) w[k] = a.w[k];
  __syncthreads();
  // Horizontal: warp m < 5 blurs plane m, lane r < EXT row r (one code path per warp).
  if (tid < 5 * 32 && (tid & 31) < EXT) {
    const int m = tid >> 5, r = tid & 31;
    if (m < 4) {
      const float2* X = &s_c2[m][r][0];
      float2* O = s_h2(m) + r * HP;
      slide11x2<T16>(w, [&](int i) { return X[i]; }, [&](int o, float2 v) { O[o] = v; });
    } else {
      const float* X = &s_c1[r][0];
      float* O = s_h1 + r * HP;
      slide11<T16>(w, [&](int i) { return X[i]; }, [&](int o, float v) { O[o] = v; });
    }
  }
  __syncthreads();
  // Vertical: item = (map, column, segment), segments of 6 rows starting at
  // rows 0, 5 and 10 (rows 5 and 10 are computed twice, identically).
  if (tid < 5 * T16 * 3) {
    const int m = tid / (3 * T16), rem = tid - m * 3 * T16, sg = rem / T16, c = rem - sg * T16;
    const int r0 = 5 * sg;
    if (m < 4) {
      const float2* I = s_h2(m) + c + r0 * HP;
      float2* O = s_v2 + m * V_PLANE + c + r0 * T16;
      slide11x2<6>(w, [&](int i) { return I[i * HP]; }, [&](int o, float2 v) { O[o * T16] = v; });
    } else {
      const float* I = s_h1 + c + r0 * HP;
      float* O = s_v1 + c + r0 * T16;
      slide11<6>(w, [&](int i) { return I[i * HP]; }, [&](int o, float v) { O[o * T16] = v; });
    }
  }
  __syncthreads();
  if (!inside) return;
  const float k1 = a.w_l1 / (3.0f * (float)L.W * (float)L.H);
  const int q = oy * T16 + ox;
  const float2 vm = s_v2[0 * V_PLANE + q], vx2 = s_v2[1 * V_PLANE + q], vxy = s_v2[2 * V_PLANE + q];
  const float2 vb = s_v2[3 * V_PLANE + q];
  const float vxy_b = s_v1[q];
  const float cmu[3] = {vm.x, vm.y, vb.x}, cx2[3] = {vx2.x, vx2.y, vb.y}, cxy[3] = {vxy.x, vxy.y, vxy_b};
  const float xs[3] = {x.x, x.y, x.z}, ys[3] = {y.x, y.y, y.z};
  float out[3];
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const float diff = xs[ch] - ys[ch];
    const float sg = diff > 0.f ? 1.f : (diff < 0.f ? -1.f : 0.f);
    out[ch] = sg * k1 + cmu[ch] + 2.0f * xs[ch] * cx2[ch] + ys[ch] * cxy[ch];
  }
  a.dl_dcolor[pix] = make_float4(out[0], out[1], out[2], 0.f);
}

// ---- normal-consistency loss (first_attempt/crates/gs-train/src/shaders/normal_loss.wgsl) ----
// Per pixel q with mean depth t̄ = depth_acc/α (0 below alpha_min): P(q) = t̄·ray(q),
// N_d = ±normalize((P(q+x) − P(q)) × (P(q+y) − P(q))) facing the camera,
// L = λ/(W·H) Σ α_q (1 − n̂_q·N_d) with α and the orientation sign detached.
// pass 1 writes dL/dnormal and the stencil coefficients dL/d(dPx), dL/d(dPy);
// pass 2 gathers the forward-difference adjoint into dL/d(depth_acc) = dl_dcolor.w.
__device__ __forceinline__ int view_of(const NormalArgs& a, uint64_t i) {
  int v = 0;
  while (v + 1 < a.n_views && (long long)i >= __ldg(&a.views[v + 1].pix_base)) ++v;
  return v;
}
__device__ __forceinline__ float3 ray_at(const ViewInfo* V, int x, int y) {
  const float cx = (float)__ldg(&V->width) * 0.5f, cy = (float)__ldg(&V->height) * 0.5f, f = __ldg(&V->focal);
  return make_float3(((float)x + 0.5f - cx) / f, -((float)y + 0.5f - cy) / f, -1.0f);
}
__device__ __forceinline__ float3 f3s(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 f3sub(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float f3dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 f3cross(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

__global__ void __launch_bounds__(256) k_normal_pass1(NormalArgs a) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.total_px;
       i += (uint64_t)gridDim.x * blockDim.x) {
    float* cp = a.cp;
    for (int k = 0; k < 6; ++k) cp[(size_t)k * a.stride + i] = 0.f;
    a.dl_dnormal[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (a.lambda == 0.f) continue;
    const int v = view_of(a, i);
    const ViewInfo* V = a.views + v;
    const int W = __ldg(&V->width), H = __ldg(&V->height);
    const uint64_t li = i - (uint64_t)__ldg(&V->pix_base);
    const int x = (int)(li % (uint64_t)W), y = (int)(li / (uint64_t)W);
    if (x + 1 >= W || y + 1 >= H) continue;
    const uint64_t ix = i + 1, iy = i + (uint64_t)W;
    const float aq = a.color[i].w, ax = a.color[ix].w, ay = a.color[iy].w;
    if (aq < a.alpha_min || ax < a.alpha_min || ay < a.alpha_min) continue;
    const float3 p = f3s(ray_at(V, x, y), a.aux[i].y / aq);
    const float3 dpx = f3sub(f3s(ray_at(V, x + 1, y), a.aux[ix].y / ax), p);
    const float3 dpy = f3sub(f3s(ray_at(V, x, y + 1), a.aux[iy].y / ay), p);
    const float3 m = f3cross(dpx, dpy);
    const float len2 = f3dot(m, m);
    if (len2 < 1e-18f) continue;
    const float len = sqrtf(len2);
    const float3 mhat = f3s(m, 1.0f / len);
    const float sign = f3dot(mhat, p) > 0.0f ? -1.0f : 1.0f;
    const float3 nd = f3s(mhat, sign);
    const float4 nv = a.normal[i];
    const float3 av = make_float3(nv.x, nv.y, nv.z);
    const float la2 = f3dot(av, av);
    if (la2 < 1e-18f) continue;
    const float la = sqrtf(la2);
    const float3 nhat = f3s(av, 1.0f / la);
    const float lam = a.lambda / ((float)W * (float)H);
    atomicAdd(a.loss + v, (double)((1.0f - f3dot(nhat, nd)) * aq));
    const float3 dl_dnd = f3s(nhat, -lam * aq);
    const float3 dl_dnhat = f3s(nd, -lam * aq);
    const float3 dl_da = f3s(f3sub(dl_dnhat, f3s(nhat, f3dot(nhat, dl_dnhat))), 1.0f / la);
    a.dl_dnormal[i] = make_float4(dl_da.x, dl_da.y, dl_da.z, 0.f);
    const float3 dl_dm = f3s(f3sub(dl_dnd, f3s(mhat, f3dot(mhat, dl_dnd))), sign / len);
    const float3 cx3 = f3cross(dpy, dl_dm), cy3 = f3cross(dl_dm, dpx);
    cp[0 * a.stride + i] = cx3.x; cp[1 * a.stride + i] = cx3.y; cp[2 * a.stride + i] = cx3.z;
    cp[3 * a.stride + i] = cy3.x; cp[4 * a.stride + i] = cy3.y; cp[5 * a.stride + i] = cy3.z;
  }
}

__global__ void __launch_bounds__(256) k_normal_pass2(NormalArgs a) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.total_px;
       i += (uint64_t)gridDim.x * blockDim.x) {
    float4 c = a.dl_dcolor[i];
    c.w = 0.f;
    if (a.lambda != 0.f) {
      const int v = view_of(a, i);
      const ViewInfo* V = a.views + v;
      const int W = __ldg(&V->width);
      const uint64_t li = i - (uint64_t)__ldg(&V->pix_base);
      const int x = (int)(li % (uint64_t)W), y = (int)(li / (uint64_t)W);
      const float* cp = a.cp;
      // Adjoint of the forward differences: the centre gives −cpx −cpy, the
      // left neighbour's cpx and the upper neighbour's cpy give +.
      float3 acc = make_float3(-cp[0 * a.stride + i] - cp[3 * a.stride + i],
                               -cp[1 * a.stride + i] - cp[4 * a.stride + i],
                               -cp[2 * a.stride + i] - cp[5 * a.stride + i]);
      if (x > 0) {
        acc.x += cp[0 * a.stride + i - 1]; acc.y += cp[1 * a.stride + i - 1]; acc.z += cp[2 * a.stride + i - 1];
      }
      if (y > 0) {
        const uint64_t u = i - (uint64_t)W;
        acc.x += cp[3 * a.stride + u]; acc.y += cp[4 * a.stride + u]; acc.z += cp[5 * a.stride + u];
      }
      const float aq = a.color[i].w;
      if (aq >= a.alpha_min) c.w = f3dot(ray_at(V, x, y), acc) / aq;  // dL/d(depth_acc), α detached
    }
    a.dl_dcolor[i] = c;
  }
}

}  // namespace

int launch_normal_loss(const NormalArgs& a, cudaStream_t st) {
  if (a.total_px == 0) return 0;
  const int grid = (int)std::min<uint64_t>((a.total_px + 255) / 256, 148 * 16);
  k_normal_pass1<<<grid, 256, 0, st>>>(a);
  k_normal_pass2<<<grid, 256, 0, st>>>(a);
  return (int)cudaGetLastError();
}

int launch_ssim(const SsimArgs& a_in, cudaStream_t st) {
  if (a_in.total_tiles16 == 0) return 0;
  SsimArgs a = a_in;
  // Normalised 11-tap Gaussian, sigma 1.5 (ssim.wgsl:32-34 lists its f32 values).
  double g[6], s = 0;
  for (int k = 0; k <= 5; ++k) g[k] = exp(-(double)(k * k) / (2.0 * 1.5 * 1.5));
  s = g[0];
  for (int k = 1; k <= 5; ++k) s += 2 * g[k];
  for (int k = 0; k <= 5; ++k) a.w[k] = (float)(g[k] / s);
  k_ssim_moments<<<a.total_tiles16, 256, 0, st>>>(a);
  k_ssim_grad<<<a.total_tiles16, 256, 0, st>>>(a);
  return (int)cudaGetLastError();
}

}  // namespace gs
