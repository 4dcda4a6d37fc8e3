// Fused L1 + D-SSIM loss and its analytic gradient
// (first_attempt/crates/gs-train/src/shaders/ssim.wgsl:41-143,
// first_attempt/crates/gs-train/src/ssim.rs:236-280).
//
// The reference runs 19 full-image passes (products, 8 separable blurs of
// two dispatches each, partials, combine) through ~17 image-sized buffers.
// Here two tiled kernels cover every view of a step:
//   k_ssim_moments: per 16×16 tile, stage x and y with a 5-pixel halo in
//     shared memory, blur the five moments (μx, μy, x², y², xy) separably,
//     form SSIM and the three coefficient maps Cμ, Cx², Cxy per channel
//     (ssim.wgsl:94-126), and accumulate the per-view loss sums.
//   k_ssim_grad: stage the nine coefficient maps with a halo, blur them
//     (the zero-padded symmetric window is self-adjoint) and combine with the
//     L1 term into dL/dx (ssim.wgsl:130-143).
// L = w_l1·mean|x−y| + w_ssim·mean(1−S) over pixels × rgb of each view.
#include "gs_common.cuh"
#include "gs_kernels.h"

namespace gs {
namespace {

constexpr int T16 = 16, HALO = 5, EXT = T16 + 2 * HALO;  // 26

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

__global__ void __launch_bounds__(256) k_ssim_moments(SsimArgs a) {
  __shared__ float s_x[3][EXT][EXT], s_y[3][EXT][EXT];
  __shared__ float s_h[5][EXT][T16];
  __shared__ double s_red[2][8];
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
    s_x[0][ly][lx] = xv.x; s_x[1][ly][lx] = xv.y; s_x[2][ly][lx] = xv.z;
    s_y[0][ly][lx] = yv.x; s_y[1][ly][lx] = yv.y; s_y[2][ly][lx] = yv.z;
  }
  const int ox = tid & 15, oy = tid >> 4;
  const int gx = L.x0 + ox, gy = L.y0 + oy;
  const bool inside = gx < L.W && gy < L.H;
  const long long pix = L.pix_base + (long long)gy * L.W + gx;
  const float C1 = 1e-4f, C2 = 9e-4f;
  float l1 = 0.f, ss = 0.f;
  for (int ch = 0; ch < 3; ++ch) {
    __syncthreads();
    for (int k = tid; k < EXT * T16; k += 256) {
      const int r = k / T16, c = k % T16;
      float m0 = 0, m1 = 0, m2 = 0, m3 = 0, m4 = 0;
#pragma unroll
      for (int d = -HALO; d <= HALO; ++d) {
        const float w = a.w[d < 0 ? -d : d];
        const float xv = s_x[ch][r][c + HALO + d], yv = s_y[ch][r][c + HALO + d];
        m0 += w * xv; m1 += w * yv; m2 += w * xv * xv; m3 += w * yv * yv; m4 += w * xv * yv;
      }
      s_h[0][r][c] = m0; s_h[1][r][c] = m1; s_h[2][r][c] = m2; s_h[3][r][c] = m3; s_h[4][r][c] = m4;
    }
    __syncthreads();
    float mu_x = 0, mu_y = 0, bx2 = 0, by2 = 0, bxy = 0;
#pragma unroll
    for (int d = -HALO; d <= HALO; ++d) {
      const float w = a.w[d < 0 ? -d : d];
      const int r = oy + HALO + d;
      mu_x += w * s_h[0][r][ox]; mu_y += w * s_h[1][r][ox]; bx2 += w * s_h[2][r][ox];
      by2 += w * s_h[3][r][ox]; bxy += w * s_h[4][r][ox];
    }
    if (inside) {
      const float inv_n3 = 1.0f / (3.0f * (float)L.W * (float)L.H);
      const float sx2 = bx2 - mu_x * mu_x, sy2 = by2 - mu_y * mu_y, sxy = bxy - mu_x * mu_y;
      const float p = mu_x * mu_x + mu_y * mu_y + C1;
      const float q = sx2 + sy2 + C2;
      const float l = (2.0f * mu_x * mu_y + C1) / p;
      const float cs = (2.0f * sxy + C2) / q;
      const float S = l * cs;
      const float dw = -a.w_ssim * inv_n3;
      const float ds_dmux = cs * (2.0f * mu_y - 2.0f * mu_x * l) / p + l * (-2.0f * mu_y + 2.0f * mu_x * cs) / q;
      const float ds_dbx2 = -l * cs / q;
      const float ds_dbxy = 2.0f * l / q;
      float* cf = a.coef + (size_t)pix * 9 + ch * 3;
      cf[0] = ds_dmux * dw; cf[1] = ds_dbx2 * dw; cf[2] = ds_dbxy * dw;
      ss += S;
      l1 += fabsf(s_x[ch][oy + HALO][ox + HALO] - s_y[ch][oy + HALO][ox + HALO]);
    }
  }
  // Per-view loss sums: warp, then block, then one double atomic each.
  double dl1 = warp_sum(l1), dss = warp_sum(ss);
  if ((tid & 31) == 0) { s_red[0][tid >> 5] = dl1; s_red[1][tid >> 5] = dss; }
  __syncthreads();
  if (tid == 0) {
    double t0 = 0, t1 = 0;
    for (int w = 0; w < 8; ++w) { t0 += s_red[0][w]; t1 += s_red[1][w]; }
    atomicAdd(a.loss_sums + 2 * L.v, t0);
    atomicAdd(a.loss_sums + 2 * L.v + 1, t1);
  }
}

__global__ void __launch_bounds__(256) k_ssim_grad(SsimArgs a) {
  __shared__ float s_c[9][EXT][EXT];
  __shared__ float s_h[9][EXT][T16];
  const int tid = threadIdx.x;
  const TileLoc L = locate(a, blockIdx.x);
  for (int k = tid; k < EXT * EXT; k += 256) {
    const int ly = k / EXT, lx = k % EXT;
    const int gx = L.x0 + lx - HALO, gy = L.y0 + ly - HALO;
    const bool in = gx >= 0 && gy >= 0 && gx < L.W && gy < L.H;
    if (in) {
      const float* cf = a.coef + (size_t)(L.pix_base + (long long)gy * L.W + gx) * 9;
#pragma unroll
      for (int m = 0; m < 9; ++m) s_c[m][ly][lx] = cf[m];
    } else {
#pragma unroll
      for (int m = 0; m < 9; ++m) s_c[m][ly][lx] = 0.f;
    }
  }
  __syncthreads();
  for (int k = tid; k < EXT * T16; k += 256) {
    const int r = k / T16, c = k % T16;
    float acc[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) acc[m] = 0.f;
#pragma unroll
    for (int d = -HALO; d <= HALO; ++d) {
      const float w = a.w[d < 0 ? -d : d];
#pragma unroll
      for (int m = 0; m < 9; ++m) acc[m] += w * s_c[m][r][c + HALO + d];
    }
#pragma unroll
    for (int m = 0; m < 9; ++m) s_h[m][r][c] = acc[m];
  }
  __syncthreads();
  const int ox = tid & 15, oy = tid >> 4;
  const int gx = L.x0 + ox, gy = L.y0 + oy;
  if (gx >= L.W || gy >= L.H) return;
  float acc[9];
#pragma unroll
  for (int m = 0; m < 9; ++m) acc[m] = 0.f;
#pragma unroll
  for (int d = -HALO; d <= HALO; ++d) {
    const float w = a.w[d < 0 ? -d : d];
#pragma unroll
    for (int m = 0; m < 9; ++m) acc[m] += w * s_h[m][oy + HALO + d][ox];
  }
  const long long pix = L.pix_base + (long long)gy * L.W + gx;
  const float4 x = a.img[pix], y = a.target[pix];
  const float k1 = a.w_l1 / (3.0f * (float)L.W * (float)L.H);
  const float xs[3] = {x.x, x.y, x.z}, ys[3] = {y.x, y.y, y.z};
  float out[3];
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const float diff = xs[ch] - ys[ch];
    const float sg = diff > 0.f ? 1.f : (diff < 0.f ? -1.f : 0.f);
    out[ch] = sg * k1 + acc[3 * ch] + 2.0f * xs[ch] * acc[3 * ch + 1] + ys[ch] * acc[3 * ch + 2];
  }
  a.dl_dcolor[pix] = make_float4(out[0], out[1], out[2], 0.f);
}

}  // namespace

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
