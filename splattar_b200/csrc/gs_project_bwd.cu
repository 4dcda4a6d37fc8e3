// Adjoint of the surfel projection: crates/gs-kernels/src/shaders/surfel_prep_bwd.wgsl:129-284 —
// chains the per-surfel record gradients (see GG_STRIDE in gs_common.cuh)
// into position, scales, quaternion (through normalisation), opacity, SH
// (clamp-masked, with the view-direction path) and the camera accumulators
// dL/dR, dL/dC, dL/dfocal; and the chosen form's fusion of that chain with
// Adam. Compiled with normal FMA contraction (gradients are compared within
// tolerance, not bit for bit).
#include <cstring>
#include <type_traits>

#include "gs_geom.cuh"

namespace gs {
namespace {

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
// `O` holds pos, scales, quat, opacity and cam[13]; `sink(kk, g)` receives the
// gradient g (rgb) of SH coefficient kk.
template <int PREC, bool AUX, class O, class Sink, class Coeff>
__device__ __forceinline__ void chain_core(const Cam& k, const float4 p, const float2 s, const float4 q, Coeff coeff,
                                           const float* G, O& o, Sink sink) {
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
  const float3 raw = sh_raw_color_with(coeff, k.deg, dir, b, nb);
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
        sink(kk, dcol * b[kk]);
        ddir += bg[kk] * dot3(coeff(kk), dcol);
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

template <int PREC, bool AUX>
__device__ __forceinline__ void chain_one(const Cam& k, const float4 p, const float2 s, const float4 q, const void* sh,
                                          size_t i, const float* G, ParamGrads& o) {
  chain_core<PREC, AUX>(k, p, s, q, [&](int kk) { return sh_coeff<PREC>(sh, i, kk); }, G, o, [&](int kk, float3 g) {
    o.sh[3 * kk] += g.x;
    o.sh[3 * kk + 1] += g.y;
    o.sh[3 * kk + 2] += g.z;
  });
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

// Deterministic mode: the warp's camera gradient summed in a fixed order
// (the transpose reduction) and stored, 16 floats (13 used), at dst. All 32
// lanes must call.
__device__ __forceinline__ void store_cam_warp(float* dst, const float cam[13]) {
  float v[16];
#pragma unroll
  for (int k = 0; k < 13; ++k) v[k] = cam[k];
  v[13] = v[14] = v[15] = 0.0f;
  const float r = warp_reduce16(v);
  const int lane = threadIdx.x & 31;
  if (!(lane & 1)) dst[reduce16_component(lane)] = r;
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
  if (a.cam_partials) {
    store_cam_warp(a.cam_partials + ((size_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 16, o.cam);
  } else if (a.grad_cam && __any_sync(0xffffffffu, any)) {
    flush_cam(a.grad_cam + 16 * v, o.cam);
  }
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

// The same update with the hardware's approximate square root and division
// (relative error ~1e-7, far inside Adam's tolerance), for the fused kernel.
__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void adam1_fast(float& raw, float& m, float& v, float g, float lr, float b1, float b2,
                                           float eps, float bc1, float bc2) {
  m = b1 * m + (1.0f - b1) * g;
  v = b2 * v + (1.0f - b2) * g * g;
  raw -= lr * __fdividef(m * bc1, sqrt_approx(v * bc2) + eps);
}

// Chosen form: projection backward over all views of the step fused with the
// Adam step and the activation refresh. A block owns S surfels (S = 32, or the
// largest power of two with S·V ≤ 256 for more than 8 views) and V·S threads
// rounded up to whole warps.
//   Prologue: one thread starts bulk copies (cp.async.bulk, completion on an
//     mbarrier) of the block's rows of the five classes' raw, m and v arrays
//     into shared memory; they land while phase 1 computes.
//   Phase 1: thread (v, s) chains the record gradient of item v·n + i into
//     the 58 parameter gradients of surfel i for view v (pos 3, scales 2,
//     quat 4, opacity 1, SH 48), kept in shared memory, and the view's camera
//     gradient, summed over the block's surfels and added with one vector
//     reduction per group of lanes.
//   Phase 2: after a bounded wait on the copies, each thread updates floats
//     of the block's parameter rows: gradient = sum over views (in view order
//     in deterministic mode, else accumulated by shared-memory atomics in
//     phase 1), then Adam and the activation, stored coalesced.
// Parameter gradients never reach global memory. The optimizer arrays are
// allocated in whole multiples of 64 surfels so the last block's copies stay
// inside them.
constexpr int PBA_MAX_THREADS = 256;
constexpr int PBA_SLOTS = 58;
constexpr int PBA_PARAMS = 59;           // floats per surfel over the five classes
constexpr int PBA_MAX_SURFELS = 32;
// Floats per surfel and first gradient slot of the classes pos, scales, quat, opacity, SH.
__host__ __device__ constexpr int pba_w(int c) { return c == 0 ? 4 : c == 1 ? 2 : c == 2 ? 4 : c == 3 ? 1 : 48; }
__host__ __device__ constexpr int pba_slot(int c) { return c == 0 ? 0 : c == 1 ? 3 : c == 2 ? 5 : c == 3 ? 9 : 10; }

__host__ __device__ constexpr int pba_surfels(int views) {
  int s = 1;
  while (s < PBA_MAX_SURFELS && s * 2 * views <= PBA_MAX_THREADS) s *= 2;
  return s;
}
__host__ __device__ constexpr int pba_threads(int views) { return (views * pba_surfels(views) + 31) / 32 * 32; }
// Gradient slots: per (view, surfel) thread (ordered: summed over views in
// view order in phase 2) or per surfel (atomic: views add into one slot).
__host__ __device__ constexpr size_t pba_smem(int views, bool ordered) {
  return sizeof(float) * ((size_t)PBA_PARAMS * 3 * pba_surfels(views) + (size_t)SH_FLOATS * (pba_surfels(views) + 1) +
                          (size_t)PBA_SLOTS * (ordered ? pba_threads(views) + 1 : pba_surfels(views) + 1));
}

struct GeoGrads {
  float3 pos;
  float2 scales;
  float4 quat;
  float opacity;
  float cam[13];
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// 1-D bulk copy global -> shared (both 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for phase 0 of the barrier for at most ~max_cycles SM cycles (a limit
// of 0 or less gives up at once, without looking).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, long long max_cycles) {
  if (max_cycles <= 0) return false;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, 0)) {
    if (clock64() - t0 > max_cycles) return false;
  }
  return true;
}

// Camera gradient of one view summed over groups of `group` lanes (a power of
// two ≤ 32 holding the same view); the first lane of each group adds it when
// `write` (false for groups past the last view). All 32 lanes must call.
__device__ __forceinline__ void flush_cam_group(float* grad_cam_view, const float cam[13], int group, bool write) {
  if (group >= 32) {
    if (__any_sync(0xffffffffu, write)) flush_cam(grad_cam_view, cam);
    return;
  }
  float v[13];
#pragma unroll
  for (int k = 0; k < 13; ++k) v[k] = cam[k];
  for (int o = group >> 1; o > 0; o >>= 1) {
#pragma unroll
    for (int k = 0; k < 13; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  }
  if (write && (threadIdx.x & (group - 1)) == 0) {
    red_add_v4(grad_cam_view, v[0], v[1], v[2], v[3]);
    red_add_v4(grad_cam_view + 4, v[4], v[5], v[6], v[7]);
    red_add_v4(grad_cam_view + 8, v[8], v[9], v[10], v[11]);
    atomicAdd(grad_cam_view + 12, v[12]);
  }
}

// Deterministic mode: the camera gradient of one view summed over groups of
// `group` lanes in a fixed order and stored (16 floats, 13 used) at dst by
// the group's first lane when `write`. All 32 lanes must call.
__device__ __forceinline__ void store_cam_group(float* dst, const float cam[13], int group, bool write) {
  if (group >= 32) {
    if (__any_sync(0xffffffffu, write)) store_cam_warp(dst, cam);
    return;
  }
  float v[13];
#pragma unroll
  for (int k = 0; k < 13; ++k) v[k] = cam[k];
  for (int o = group >> 1; o > 0; o >>= 1) {
#pragma unroll
    for (int k = 0; k < 13; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  }
  if (write && (threadIdx.x & (group - 1)) == 0) {
#pragma unroll
    for (int k = 0; k < 13; ++k) dst[k] = v[k];
    dst[13] = dst[14] = dst[15] = 0.0f;
  }
}

// ORD (deterministic mode): every (view, surfel) thread keeps its own
// gradient slots and phase 2 sums them in view order (88 KB of shared memory
// at 8 views, 2 blocks per SM). Otherwise the views of a surfel add into one
// slot with shared-memory atomics (36 KB, 3 blocks per SM at ≤ 80 registers).
template <int PREC, bool AUX, bool ORD>
__global__ void __launch_bounds__(PBA_MAX_THREADS, ORD ? 2 : 3) k_project_bwd_adam(ProjectBwdArgs a, AdamFusedArgs opt) {
  extern __shared__ __align__(16) float s_dyn[];
  __shared__ uint64_t s_bar;
  const int tid = threadIdx.x;
  const int V = a.n_views, S = pba_surfels(V), NT = blockDim.x;
  // Slot and SH strides are one more than a multiple of 32 floats, so the
  // threads of a warp that walk consecutive slots (or coefficients) of one
  // surfel hit distinct banks.
  const int PITCH = ORD ? NT + 1 : S + 1;              // slot stride
  const int SHP = S + 1;                               // SH coefficient stride
  float* s_stage = s_dyn;                              // [class][raw|m|v][S*W]
  float* s_sh = s_stage + PBA_PARAMS * 3 * S;          // [SH_FLOATS][SHP]: the block's activated SH, transposed
  float* s_g = s_sh + SH_FLOATS * SHP;                 // [PBA_SLOTS][PITCH]
  const uint32_t i0 = blockIdx.x * (uint32_t)S;
  // This thread's (view, surfel) item and its record gradient, loaded first
  // so the loads are in flight while the block stages its SH rows.
  const int v1 = tid / S, sl1 = tid % S;
  const uint32_t i1 = i0 + (uint32_t)sl1;
  const bool active1 = v1 < V && i1 < a.n;
  float G[GG_STRIDE];
  const bool gnz = active1 && load_G<AUX>(a, (uint32_t)v1 * a.n + i1, G);
  if (tid == 0) mbar_init(&s_bar);
  __syncthreads();
  if (tid == 0) {
    mbar_expect_tx(&s_bar, (uint32_t)(sizeof(float) * PBA_PARAMS * 3 * S));
    float* dst = s_stage;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const uint32_t rowb = (uint32_t)(sizeof(float) * S * pba_w(c));
      const size_t off = (size_t)i0 * pba_w(c);
      bulk_g2s(dst, opt.cls[c].raw + off, rowb, &s_bar); dst += S * pba_w(c);
      bulk_g2s(dst, opt.cls[c].m + off, rowb, &s_bar); dst += S * pba_w(c);
      bulk_g2s(dst, opt.cls[c].v + off, rowb, &s_bar); dst += S * pba_w(c);
    }
  }
  {  // the block's SH rows, coalesced 16-byte loads, converted and transposed for conflict-free reads
    const uint32_t ns = min((uint32_t)S, a.n - i0);
    constexpr int PER = PREC == 0 ? 4 : 8;          // values per 16-byte load
    constexpr int QROW = SH_FLOATS / PER;           // loads per surfel row
    const uint4* src = reinterpret_cast<const uint4*>(a.sh) + (size_t)i0 * QROW;
    for (int L = tid; L < (int)ns * QROW; L += NT) {
      const int sl = L / QROW, f0 = (L - sl * QROW) * PER;
      const uint4 u = __ldg(src + L);
      const uint32_t w[4] = {u.x, u.y, u.z, u.w};
      if constexpr (PREC == 0) {
#pragma unroll
        for (int j = 0; j < 4; ++j) s_sh[(f0 + j) * SHP + sl] = __uint_as_float(w[j]);
      } else {
        using H = typename std::conditional<PREC == 1, __half, __nv_bfloat16>::type;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          H lo, hi;
          const unsigned short bl = (unsigned short)(w[j] & 0xffffu), bh = (unsigned short)(w[j] >> 16);
          memcpy(&lo, &bl, 2);
          memcpy(&hi, &bh, 2);
          s_sh[(f0 + 2 * j) * SHP + sl] = h2f<H>(lo);
          s_sh[(f0 + 2 * j + 1) * SHP + sl] = h2f<H>(hi);
        }
      }
    }
  }
  if (!ORD)
    for (int k = tid; k < PBA_SLOTS * PITCH; k += NT) s_g[k] = 0.0f;
  __syncthreads();
  // ---- phase 1
  {
    const int v = v1, sl = sl1;
    const uint32_t i = i1;
    const bool active = active1;
    // ORD: this thread's column; atomic: the surfel's column, shared by its views.
    float* col = s_g + (ORD ? tid : sl);
    auto put = [&](int slot, float g) {
      if (ORD) col[slot * PITCH] = g;
      else atomicAdd(col + slot * PITCH, g);  // unconditional: a branch per slot cost more than adding zeros
    };
    GeoGrads o;
    o.pos = f3(0, 0, 0); o.scales = make_float2(0, 0); o.quat = make_float4(0, 0, 0, 0); o.opacity = 0;
#pragma unroll
    for (int k = 0; k < 13; ++k) o.cam[k] = 0.0f;
    bool any = false;
    uint32_t written = 0;  // SH coefficients whose gradient slots the chain wrote
    if (active) {
      if (gnz) {
        const Cam k = load_cam(a.views, v);
        const float* shc = s_sh + sl;
        chain_core<PREC, AUX>(k, __ldg(a.pos + i), __ldg(a.scales + i), __ldg(a.quats + i),
                              [&](int kk) { return f3(shc[(3 * kk) * SHP], shc[(3 * kk + 1) * SHP], shc[(3 * kk + 2) * SHP]); },
                              G, o, [&](int kk, float3 g) {
                                put(10 + 3 * kk, g.x);
                                put(11 + 3 * kk, g.y);
                                put(12 + 3 * kk, g.z);
                                written |= 1u << kk;
                              });
        any = true;
        if (ORD) {
#pragma unroll
          for (int kk = 0; kk < 16; ++kk) {
            if (!(written >> kk & 1u)) {
              col[(10 + 3 * kk) * PITCH] = 0.0f;
              col[(11 + 3 * kk) * PITCH] = 0.0f;
              col[(12 + 3 * kk) * PITCH] = 0.0f;
            }
          }
        }
        put(0, o.pos.x); put(1, o.pos.y); put(2, o.pos.z);
        put(3, o.scales.x); put(4, o.scales.y);
        put(5, o.quat.x); put(6, o.quat.y); put(7, o.quat.z); put(8, o.quat.w);
        put(9, o.opacity);
      }
    }
    if (ORD && !any) {
#pragma unroll 2
      for (int j = 0; j < PBA_SLOTS; ++j) col[j * PITCH] = 0.0f;
    }
    // Every lane of a group holds the same view (S is a power of two, V·S a
    // multiple of S); lanes past the last view hold zeros and write nothing.
    if (a.cam_partials)
      store_cam_group(a.cam_partials + ((size_t)blockIdx.x * V + (v < V ? v : V - 1)) * 16, o.cam, S < 32 ? S : 32,
                      v < V);
    else if (a.grad_cam && __any_sync(0xffffffffu, any))
      flush_cam_group(a.grad_cam + 16 * (v < V ? v : V - 1), o.cam, S < 32 ? S : 32, v < V);
  }
  __syncthreads();
  // ---- phase 2
  if (!mbar_wait_bounded(&s_bar, opt.wait_cycles[0])) {
    // The block's optimizer rows are not (known to be) in shared memory: flag
    // the expiry, skip this block's update, and give the copies in flight the
    // drain limit to land before the block exits. Should the drain wait expire
    // too, the block exits with copies in flight, which may then land in
    // shared memory a later block of the SM uses: the error word reports the
    // launch as failed and its results must be discarded.
    if (tid == 0 && opt.error_word) atomicOr(opt.error_word, ERR_TIMEOUT);
    mbar_wait_bounded(&s_bar, opt.wait_cycles[1]);
    return;
  }
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
  const uint32_t ns = min((uint32_t)S, a.n - i0);
  auto grad_sum = [&](int slot, int sl) {
    const float* p = s_g + slot * PITCH + sl;
    if (!ORD) return *p;
    float g = 0.0f;
#pragma unroll 8
    for (int v = 0; v < V; ++v) g += p[v * S];
    return g;
  };
  if (opt.accum_grad_norm && tid < (int)ns) {
    const float gx = grad_sum(0, tid), gy = grad_sum(1, tid), gz = grad_sum(2, tid);
    opt.accum_grad_norm[i0 + tid] += sqrtf(gx * gx + gy * gy + gz * gz);
  }
  const float* stage = s_stage;
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    const AdamClass& C = cls[c];
    const int W = pba_w(c);
    const size_t base = (size_t)i0 * W;
    const float* sr = stage;
    const float* sm = stage + S * W;
    const float* sv = stage + 2 * S * W;
    stage += 3 * S * W;
    for (int L = tid; L < (int)ns * W; L += NT) {
      const int sl = L / W, w = L - sl * W;
      const float g = (c == 0 && w == 3) ? 0.0f : grad_sum(pba_slot(c) + w, sl);
      float r = sr[L], m = sm[L], vv = sv[L];
      float gr = g + C.reg;
      if (c == 1) gr *= __expf(r);                                                                // scales: exp
      if (c == 3) { const float sg = __fdividef(1.0f, 1.0f + __expf(-r)); gr *= sg * (1.0f - sg); }  // opacity
      adam1_fast(r, m, vv, gr, C.lr, b1, b2, eps, bc1, bc2);
      C.raw[base + L] = r; C.m[base + L] = m; C.v[base + L] = vv;
      float act = r;
      if (c == 1) act = __expf(r);
      if (c == 3) act = __fdividef(1.0f, 1.0f + __expf(-r));
      C.act[base + L] = act;
      if (c == 4 && opt.sh_half) {
        if (opt.sh_half_is_bf16) reinterpret_cast<__nv_bfloat16*>(opt.sh_half)[base + L] = __float2bfloat16_rn(r);
        else reinterpret_cast<__half*>(opt.sh_half)[base + L] = __float2half_rn(r);
      }
    }
  }
}

}  // namespace

// Opts the kernels that need more than 48 KB of dynamic shared memory in, on
// the current device. Called when a handle is created (outside any capture).
int prepare_project_kernels() {
  size_t big = 0;
  for (int v = 1; v <= 64; ++v) big = pba_smem(v, true) > big ? pba_smem(v, true) : big;
  const int smem = (int)big;
  const void* fns[12] = {
      (const void*)k_project_bwd_adam<0, false, true>, (const void*)k_project_bwd_adam<0, true, true>,
      (const void*)k_project_bwd_adam<1, false, true>, (const void*)k_project_bwd_adam<1, true, true>,
      (const void*)k_project_bwd_adam<2, false, true>, (const void*)k_project_bwd_adam<2, true, true>,
      (const void*)k_project_bwd_adam<0, false, false>, (const void*)k_project_bwd_adam<0, true, false>,
      (const void*)k_project_bwd_adam<1, false, false>, (const void*)k_project_bwd_adam<1, true, false>,
      (const void*)k_project_bwd_adam<2, false, false>, (const void*)k_project_bwd_adam<2, true, false>};
  for (const void* f : fns) {
    const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return (int)e;
  }
  return 0;
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

namespace {

// One block per view: 16 unit-lanes × 16 components, each unit-lane summing
// a fixed stride of units in order, then the 16 lanes in order.
__global__ void __launch_bounds__(256) k_cam_reduce(const float* part, uint64_t units, int V, float* grad_cam) {
  __shared__ float s_sum[16][17];
  const int v = blockIdx.x, c = threadIdx.x & 15, ul = threadIdx.x >> 4;
  float acc = 0.0f;
  for (uint64_t u = (uint64_t)ul; u < units; u += 16) acc += __ldg(part + (u * (uint64_t)V + (uint64_t)v) * 16 + c);
  s_sum[ul][c] = acc;
  __syncthreads();
  if (threadIdx.x < 13) {
    float t = 0.0f;
#pragma unroll
    for (int l = 0; l < 16; ++l) t += s_sum[l][threadIdx.x];
    grad_cam[16 * v + threadIdx.x] = t;
  }
}

}  // namespace

uint64_t cam_partial_units(uint32_t n, int n_views) {
  if (n_views <= 0) return (uint64_t)((n + 255) / 256) * 8;  // plain kernel: 8 warps per 256-thread block
  const uint32_t S = (uint32_t)pba_surfels(n_views);
  return (uint64_t)((n + S - 1) / S);
}

int launch_cam_reduce(const float* partials, uint64_t units, int n_views, float* grad_cam, cudaStream_t st) {
  if (n_views <= 0) return 0;
  k_cam_reduce<<<n_views, 256, 0, st>>>(partials, units, n_views, grad_cam);
  return (int)cudaGetLastError();
}

int launch_project_bwd_adam(const ProjectBwdArgs& a, const AdamFusedArgs& opt, int prec, bool aux, cudaStream_t st) {
  if (a.n == 0) return 0;
  if (a.n_views < 1 || a.n_views > PBA_MAX_THREADS) return (int)cudaErrorInvalidValue;
  const int S = pba_surfels(a.n_views);
  dim3 grid((a.n + S - 1) / S);
  // Deterministic mode (per-entry partials) keeps the view-ordered sum.
  const bool ord = a.partials != nullptr;
  const size_t smem = pba_smem(a.n_views, ord);
#define GS_PBA(P, X)                                                                              \
  do {                                                                                            \
    if (ord) k_project_bwd_adam<P, X, true><<<grid, pba_threads(a.n_views), smem, st>>>(a, opt);  \
    else k_project_bwd_adam<P, X, false><<<grid, pba_threads(a.n_views), smem, st>>>(a, opt);     \
  } while (0)
  if (prec == 0) { if (aux) GS_PBA(0, true); else GS_PBA(0, false); }
  else if (prec == 1) { if (aux) GS_PBA(1, true); else GS_PBA(1, false); }
  else { if (aux) GS_PBA(2, true); else GS_PBA(2, false); }
#undef GS_PBA
  return (int)cudaGetLastError();
}

}  // namespace gs
