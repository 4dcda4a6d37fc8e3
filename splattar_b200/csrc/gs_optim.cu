// Adam over raw parameters with the raw→activated chain rule
// (first_attempt/crates/gs-train/src/shaders/adam.wgsl:33-74; bias
// corrections computed on the host as first_attempt/crates/gs-train/src/
// optim.rs:179-197 does), the raw-parameter initialisation of
// first_attempt/crates/gs-train/src/trainer.rs:763-791, the 16-bit renderer
// copy of SH for mixed precision, and the densify/prune compaction.
#include "gs_common.cuh"
#include "gs_kernels.h"

namespace gs {
namespace {

__device__ __forceinline__ float act_fn(float x, int a) {
  return a == 1 ? __expf(x) : (a == 2 ? 1.0f / (1.0f + __expf(-x)) : x);
}
__device__ __forceinline__ float dact_fn(float x, int a) {
  if (a == 1) return __expf(x);
  if (a == 2) {
    const float s = 1.0f / (1.0f + __expf(-x));
    return s * (1.0f - s);
  }
  return 1.0f;
}

__device__ __forceinline__ void adam_el(float& r, float& m, float& v, float g, float lr, float b1, float b2, float eps,
                                        float bc1, float bc2) {
  m = b1 * m + (1.0f - b1) * g;
  v = b2 * v + (1.0f - b2) * g * g;
  r -= lr * (m * bc1) / (sqrtf(v * bc2) + eps);
}

// One class, float4-vectorised when n % 4 == 0 (every class of the trainer
// except a non-multiple-of-4 opacity count).
__global__ void __launch_bounds__(256) k_adam(AdamClass c, uint64_t n, const float* grad, int activation, float b1,
                                              float b2, float eps, float bc1, float bc2) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  if ((n & 3) == 0) {
    float4* R = reinterpret_cast<float4*>(c.raw);
    float4* M = reinterpret_cast<float4*>(c.m);
    float4* V = reinterpret_cast<float4*>(c.v);
    float4* A = reinterpret_cast<float4*>(c.act);
    const float4* G = reinterpret_cast<const float4*>(grad);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n / 4; i += stride) {
      float4 r = R[i], m = M[i], v = V[i];
      const float4 g = G[i];
      adam_el(r.x, m.x, v.x, (g.x + c.reg) * dact_fn(r.x, activation), c.lr, b1, b2, eps, bc1, bc2);
      adam_el(r.y, m.y, v.y, (g.y + c.reg) * dact_fn(r.y, activation), c.lr, b1, b2, eps, bc1, bc2);
      adam_el(r.z, m.z, v.z, (g.z + c.reg) * dact_fn(r.z, activation), c.lr, b1, b2, eps, bc1, bc2);
      adam_el(r.w, m.w, v.w, (g.w + c.reg) * dact_fn(r.w, activation), c.lr, b1, b2, eps, bc1, bc2);
      R[i] = r; M[i] = m; V[i] = v;
      if (A) A[i] = make_float4(act_fn(r.x, activation), act_fn(r.y, activation), act_fn(r.z, activation),
                                act_fn(r.w, activation));
    }
  } else {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      float r = c.raw[i], m = c.m[i], v = c.v[i];
      adam_el(r, m, v, (grad[i] + c.reg) * dact_fn(r, activation), c.lr, b1, b2, eps, bc1, bc2);
      c.raw[i] = r; c.m[i] = m; c.v[i] = v;
      if (c.act) c.act[i] = act_fn(r, activation);
    }
  }
}

// raw = inverse activation of act (log of scales ≥ 1e-6, logit of opacity
// clamped to [1e-4, 1−1e-4]), then act = activation(raw); zero moments.
__global__ void __launch_bounds__(256) k_activate_init(AdamClass c, uint64_t n, int activation) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float a = c.act[i];
    float r = a;
    if (activation == 1) r = logf(fmaxf(a, 1e-6f));
    else if (activation == 2) {
      const float o = fminf(fmaxf(a, 1e-4f), 1.0f - 1e-4f);
      r = logf(o / (1.0f - o));
    }
    c.raw[i] = r;
    c.m[i] = 0.f;
    c.v[i] = 0.f;
    c.act[i] = activation == 0 ? r : act_fn(r, activation);
  }
}

__global__ void __launch_bounds__(256) k_to_half(const float* src, void* dst, uint64_t n, bool bf16) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    if (bf16) reinterpret_cast<__nv_bfloat16*>(dst)[i] = __float2bfloat16_rn(src[i]);
    else reinterpret_cast<__half*>(dst)[i] = __float2half_rn(src[i]);
  }
}

int grid_of(uint64_t n) {
  uint64_t g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  return g < 1 ? 1 : (int)g;
}

// ---- densify / prune (no reference counterpart) ----
__global__ void __launch_bounds__(256) k_densify_flags(DensifyArgs a, uint32_t* keep, uint32_t* clone) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const bool k = a.opacity_act[i] >= a.opacity_threshold;
    const bool c = k && a.accum[i] * a.inv_steps > a.grad_threshold;
    keep[i] = k ? 1u : 0u;
    clone[i] = c ? 1u : 0u;
  }
}

// Gathers one per-surfel array (width floats each) into tmp at its new slots.
// Clones copy the source values, except moment arrays which start at zero.
__global__ void __launch_bounds__(256) k_densify_scatter(const float* src, float* tmp, int width, bool zero_clone,
                                                         uint32_t n, uint32_t capacity, const uint32_t* keep,
                                                         const uint32_t* keep_off, const uint32_t* clone,
                                                         const uint32_t* clone_off, const uint32_t* n_keep) {
  const uint32_t nk = *n_keep;
  const uint64_t total = (uint64_t)n * width;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t i = (uint32_t)(e / width), k = (uint32_t)(e % width);
    const float x = src[e];
    if (keep[i]) tmp[(uint64_t)keep_off[i] * width + k] = x;
    if (clone[i]) {
      const uint64_t slot = (uint64_t)nk + clone_off[i];
      if (slot < capacity) tmp[slot * width + k] = zero_clone ? 0.f : x;
    }
  }
}

__global__ void k_densify_count(const uint32_t* n_keep, const uint32_t* n_clone, uint32_t capacity, uint32_t* n_out) {
  const uint64_t t = (uint64_t)*n_keep + *n_clone;
  *n_out = t > capacity ? capacity : (uint32_t)t;
}

__global__ void __launch_bounds__(256) k_accum_norm(const float4* grad_pos, float* accum, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 g = grad_pos[i];
    accum[i] += sqrtf(g.x * g.x + g.y * g.y + g.z * g.z);
  }
}

}  // namespace

int launch_accum_norm(const float4* grad_pos, float* accum, uint32_t n, cudaStream_t st) {
  if (n == 0) return 0;
  k_accum_norm<<<grid_of(n), 256, 0, st>>>(grad_pos, accum, n);
  return (int)cudaGetLastError();
}

int launch_adam_grad(const AdamClass& c, const float* grad, uint64_t n, int activation, float beta1, float beta2,
                     float eps, float bc1_inv, float bc2_inv, cudaStream_t st) {
  if (n == 0) return 0;
  const uint64_t work = (n & 3) == 0 ? n / 4 : n;
  k_adam<<<grid_of(work), 256, 0, st>>>(c, n, grad, activation, beta1, beta2, eps, bc1_inv, bc2_inv);
  return (int)cudaGetLastError();
}

int launch_activate_init(const AdamClass& c, uint64_t n, int activation, cudaStream_t st) {
  if (n == 0) return 0;
  k_activate_init<<<grid_of(n), 256, 0, st>>>(c, n, activation);
  return (int)cudaGetLastError();
}

int launch_to_half(const float* src, void* dst, uint64_t n, bool bf16, cudaStream_t st) {
  if (n == 0) return 0;
  k_to_half<<<grid_of(n), 256, 0, st>>>(src, dst, n, bf16);
  return (int)cudaGetLastError();
}

int launch_densify(DensifyArgs& a, void* scan_scratch, cudaStream_t st) {
  if (a.n == 0) return 0;
  uint32_t* keep = a.flags;
  uint32_t* clone = a.flags + a.capacity;
  uint32_t* keep_off = a.slots;
  uint32_t* clone_off = a.slots + a.capacity;
  uint32_t* n_keep = a.n_out_dev + 1;
  uint32_t* n_clone = a.n_out_dev + 2;
  k_densify_flags<<<grid_of(a.n), 256, 0, st>>>(a, keep, clone);
  int e = launch_scan(keep, nullptr, keep_off, a.n, nullptr, n_keep, nullptr, scan_scratch, st);
  if (e) return e;
  e = launch_scan(clone, nullptr, clone_off, a.n, nullptr, n_clone, nullptr, scan_scratch, st);
  if (e) return e;
  k_densify_count<<<1, 1, 0, st>>>(n_keep, n_clone, a.capacity, a.n_out_dev);
  for (int k = 0; k < a.n_arrays; ++k) {
    const int w = a.widths[k] > 0 ? a.widths[k] : -a.widths[k];
    const bool zero_clone = a.widths[k] < 0;  // negative width marks a moment array
    const uint64_t total = (uint64_t)a.n * w;
    k_densify_scatter<<<grid_of(total), 256, 0, st>>>(a.arrays[k], a.tmp, w, zero_clone, a.n, a.capacity, keep,
                                                     keep_off, clone, clone_off, n_keep);
    // Copy the whole capacity range back: slots past the new count hold
    // stale values nobody reads.
    cudaMemcpyAsync(a.arrays[k], a.tmp, sizeof(float) * (size_t)a.capacity * w, cudaMemcpyDeviceToDevice, st);
  }
  return (int)cudaGetLastError();
}

}  // namespace gs
