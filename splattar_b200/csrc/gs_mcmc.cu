// MCMC dead-surfel relocation and exploration noise, entirely on the device
// (first_attempt/crates/gs-train/src/trainer.rs:1558-1689 with
// shaders/relocate.wgsl; shaders/mcmc.wgsl).
//
// The reference reads the activated opacities back to the host, samples an
// alive target for every dead surfel (opacity-proportional, through a
// cumulative f64 table and one xorshift64 draw per dead surfel in index
// order; a target already taken defers the dead surfel), pairs leftover dead
// slots with oversized alive surfels, uploads the pairs and runs the copy
// kernels. Here every step stays on the GPU and reproduces those choices:
//   * alive opacities (f32 ≥ 2^-8) are exact multiples of 2^-31, so their
//     prefix sum in 64-bit fixed point equals the reference's f64 table
//     exactly while it stays below 2^22 (4,194,304 opacity units);
//   * the k-th dead surfel's draw is the xorshift64 state after k+1 steps,
//     computed by jumping ahead with precomputed powers of the generator's
//     GF(2) matrix;
//   * a target picked by several dead surfels goes to the lowest dead rank
//     (atomicMin), exactly the sequential "earlier dead surfel wins";
//   * the median alive size and the size-descending order of oversized
//     surfels come from stable radix sorts (ties by index, as Rust's stable
//     sort).
// Nothing is read back; the generator state lives on the device.
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include <algorithm>

#include "gs_common.cuh"
#include "gs_kernels.h"

namespace gs {
namespace {

constexpr uint32_t NONE = 0xffffffffu;

__device__ __forceinline__ uint64_t gf2_apply(const uint64_t* rows, uint64_t x) {
  uint64_t y = 0;
#pragma unroll 8
  for (int i = 0; i < 64; ++i) y |= (uint64_t)(__popcll(rows[i] & x) & 1) << i;
  return y;
}
// State after `steps` xorshift64 steps from x (jump[j] = rows of M^(2^j)).
__device__ uint64_t xs_jump(const uint64_t* jump, uint64_t x, uint64_t steps) {
  for (int j = 0; j < MCMC_JUMP_LEVELS && steps; ++j, steps >>= 1)
    if (steps & 1) x = gf2_apply(jump + 64 * j, x);
  return x;
}

__global__ void __launch_bounds__(256) k_mcmc_flags(McmcArgs a) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const float o = a.opac_act[i];
    const bool dead = o < a.dead_threshold;
    a.dead[i] = dead ? 1u : 0u;
    // Alive opacities ≥ threshold > 2^-8 are integers in units of 2^-31.
    a.weight[i] = dead ? 0ull : (unsigned long long)(o * 2147483648.0f);
    a.owner[i] = NONE;
    a.used[i] = 0u;
    const float2 s = a.scales_act[i];
    a.size_key[i] = dead ? NONE : __float_as_uint(fmaxf(s.x, s.y));
    a.size_val[i] = i;
  }
}

// Exclusive prefix of 64-bit weights (chunked, as the 32-bit scan).
__global__ void __launch_bounds__(256) k_scan64_reduce(const unsigned long long* in, uint32_t n,
                                                       unsigned long long* bsum) {
  const uint32_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const uint32_t beg = blockIdx.x * chunk, end = min(n, beg + chunk);
  unsigned long long s = 0;
  for (uint32_t i = beg + threadIdx.x; i < end; i += blockDim.x) s += in[i];
  using BR = cub::BlockReduce<unsigned long long, 256>;
  __shared__ typename BR::TempStorage tmp;
  s = BR(tmp).Sum(s);
  if (threadIdx.x == 0) bsum[blockIdx.x] = s;
}
__global__ void __launch_bounds__(SCAN_GRID) k_scan64_blocks(unsigned long long* bsum, unsigned long long* total) {
  using BS = cub::BlockScan<unsigned long long, SCAN_GRID>;
  __shared__ typename BS::TempStorage tmp;
  unsigned long long v = bsum[threadIdx.x], excl, agg;
  BS(tmp).ExclusiveSum(v, excl, agg);
  bsum[threadIdx.x] = excl;
  if (threadIdx.x == 0) *total = agg;
}
__global__ void __launch_bounds__(256) k_scan64_down(const unsigned long long* in, unsigned long long* out, uint32_t n,
                                                     const unsigned long long* boff) {
  const uint32_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const uint32_t beg = blockIdx.x * chunk, end = min(n, beg + chunk);
  using BS = cub::BlockScan<unsigned long long, 256>;
  __shared__ typename BS::TempStorage tmp;
  unsigned long long running = boff[blockIdx.x];
  for (uint32_t t0 = beg; t0 < end; t0 += 256) {
    const uint32_t i = t0 + threadIdx.x;
    const unsigned long long v = i < end ? in[i] : 0ull;
    unsigned long long excl, agg;
    BS(tmp).ExclusiveSum(v, excl, agg);
    if (i < end) out[i] = running + excl;
    running += agg;
    __syncthreads();
  }
}

// One draw per dead surfel (rank k = draw k); records its pick and bids for
// the target with its rank.
__global__ void __launch_bounds__(256) k_mcmc_pick(McmcArgs a) {
  const unsigned long long total = *a.total_weight;
  if (total == 0) return;
  const double total_f = (double)total * 0x1p-31;
  const uint64_t x0 = *a.rng_state;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    if (!a.dead[i]) continue;
    const uint32_t k = a.dead_rank[i];
    a.dead_idx[k] = i;
    const uint64_t x = xs_jump(a.jump, x0, (uint64_t)k + 1);
    const double r = (double)(x >> 11) / 9007199254740992.0 * total_f;
    // partition_point(cum, c < r): first j whose inclusive sum ≥ r.
    uint32_t lo = 0, hi = a.n;
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo) / 2;
      const double c = (double)(a.cum[mid] + a.weight[mid]) * 0x1p-31;
      if (c < r) lo = mid + 1;
      else hi = mid;
    }
    const uint32_t t = lo < a.n ? lo : a.n - 1;
    if (t == i) {
      a.pick[k] = NONE;
      continue;
    }
    a.pick[k] = t;
    atomicMin(&a.owner[t], k);
  }
}

__global__ void __launch_bounds__(256) k_mcmc_claim(McmcArgs a) {
  const uint32_t n_dead = a.counters[0];
  const bool run = *a.total_weight != 0;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_dead; k += gridDim.x * blockDim.x) {
    const uint32_t t = run ? a.pick[k] : NONE;
    const bool won = t != NONE && a.owner[t] == k;
    if (!won) a.pick[k] = NONE;
    else a.used[t] = 1u;
    a.leftover_flag[k] = won ? 0u : 1u;
    if (won) atomicAdd(a.counters + 1, 1u);
    else atomicAdd(a.counters + 3, 1u);
  }
}

__global__ void k_mcmc_advance(McmcArgs a) {
  if (*a.total_weight != 0 && a.counters[0] != 0) *a.rng_state = xs_jump(a.jump, *a.rng_state, a.counters[0]);
}

// Oversized alive surfels still unused: size > split_ratio × median alive size.
__global__ void __launch_bounds__(256) k_mcmc_over_flags(McmcArgs a) {
  const uint32_t n_alive = a.n - a.counters[0];
  const bool run = a.split_ratio > 0.f && *a.total_weight != 0 && a.counters[0] != 0 && n_alive >= 16;
  const float cap = run ? a.split_ratio * __uint_as_float(a.sorted_size_key[n_alive / 2]) : 0.f;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    bool over = false;
    if (run && !a.dead[i] && !a.used[i]) {
      const float2 s = a.scales_act[i];
      over = fmaxf(s.x, s.y) > cap;
    }
    a.over_flag[i] = over ? 1u : 0u;
  }
}

__global__ void __launch_bounds__(256) k_mcmc_over_list(McmcArgs a) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    if (!a.over_flag[i]) continue;
    const uint32_t r = a.over_rank[i];
    const float2 s = a.scales_act[i];
    a.over_key[r] = ~__float_as_uint(fmaxf(s.x, s.y));  // descending size
    a.over_val[r] = i;
  }
}

__global__ void __launch_bounds__(256) k_mcmc_left_list(McmcArgs a) {
  const uint32_t n_dead = a.counters[0];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_dead; k += gridDim.x * blockDim.x)
    if (a.leftover_flag[k]) a.left_idx[a.left_rank[k]] = a.dead_idx[k];
}

__global__ void k_mcmc_split_count(McmcArgs a) {
  const uint32_t n_over = a.counters[5], n_left = a.counters[6];
  a.counters[2] = n_over < n_left ? n_over : n_left;
}

__device__ __forceinline__ float sigmoidf(float x) { return 1.0f / (1.0f + expf(-x)); }

template <int PREC>
__device__ __forceinline__ void store_sh_half(void* sh_half, size_t idx, float v) {
  if constexpr (PREC == 1) reinterpret_cast<__half*>(sh_half)[idx] = __float2half_rn(v);
  else if constexpr (PREC == 2) reinterpret_cast<__nv_bfloat16*>(sh_half)[idx] = __float2bfloat16_rn(v);
}

// relocate_params + relocate_moments (relocate.wgsl) for pair p, plus the
// activated copies of both surfels (the reference re-activates every class
// afterwards).
template <int PREC>
__global__ void __launch_bounds__(256) k_mcmc_relocate(McmcArgs a) {
  const uint32_t n_dead = a.counters[0], n_split = a.counters[2];
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n_dead + n_split; p += gridDim.x * blockDim.x) {
    uint32_t d, s;
    bool split;
    if (p < n_dead) {
      s = a.pick[p];
      if (s == NONE) continue;
      d = a.dead_idx[p];
      split = false;
    } else {
      d = a.left_idx[p - n_dead];
      s = a.over_sorted_val[p - n_dead];
      split = true;
    }
    // Split opacity α' = 1 − √(1−α) for both, in logit space.
    const float alpha = fminf(fmaxf(a.opac_act[s], 1e-4f), 0.999f);
    const float alpha_new = fminf(fmaxf(1.0f - sqrtf(1.0f - alpha), 1e-4f), 0.999f);
    const float logit = logf(alpha_new / (1.0f - alpha_new));
    a.opac_raw[d] = logit;
    a.opac_raw[s] = logit;
    const float4 q = a.quat_raw[s];
    a.quat_raw[d] = q;
    float2 sc = a.scales_raw[s];
    if (split) {
      // Halves displaced ±0.6σ along the major in-plane axis, scales ×0.6.
      const float ql = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
      const float x = q.x / ql, y = q.y / ql, z = q.z / ql, w = q.w / ql;
      const float3 col0 = make_float3(1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + w * z), 2.0f * (x * z - w * y));
      const float3 col1 = make_float3(2.0f * (x * y - w * z), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + w * x));
      const float sx = expf(sc.x), sy = expf(sc.y);
      float3 axis = make_float3(col0.x * sx, col0.y * sx, col0.z * sx);
      if (sy > sx) axis = make_float3(col1.x * sy, col1.y * sy, col1.z * sy);
      const float4 c = a.pos_raw[s];
      a.pos_raw[d] = make_float4(c.x + 0.6f * axis.x, c.y + 0.6f * axis.y, c.z + 0.6f * axis.z, c.w);
      a.pos_raw[s] = make_float4(c.x - 0.6f * axis.x, c.y - 0.6f * axis.y, c.z - 0.6f * axis.z, c.w);
      sc = make_float2(sc.x - 0.51f, sc.y - 0.51f);
    } else {
      a.pos_raw[d] = a.pos_raw[s];
      sc = make_float2(sc.x - 0.16f, sc.y - 0.16f);
    }
    a.scales_raw[s] = sc;
    a.scales_raw[d] = sc;
    for (int k = 0; k < SH_FLOATS; ++k) a.sh_raw[(size_t)d * SH_FLOATS + k] = a.sh_raw[(size_t)s * SH_FLOATS + k];
    // Zero the Adam moments of both.
    const uint32_t both[2] = {d, s};
    for (int b = 0; b < 2; ++b) {
      const size_t i = both[b];
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        const int W = c == 0 ? 4 : c == 1 ? 2 : c == 2 ? 4 : c == 3 ? 1 : SH_FLOATS;
        for (int k = 0; k < W; ++k) {
          a.m[c][i * W + k] = 0.f;
          a.v[c][i * W + k] = 0.f;
        }
      }
      // Activated copies.
      a.pos_act[i] = a.pos_raw[i];
      const float2 r = a.scales_raw[i];
      a.scales_act_w[i] = make_float2(expf(r.x), expf(r.y));
      a.quat_act[i] = a.quat_raw[i];
      a.opac_act_w[i] = sigmoidf(a.opac_raw[i]);
      for (int k = 0; k < SH_FLOATS; ++k) {
        const float v = a.sh_raw[i * SH_FLOATS + k];
        a.sh_act[i * SH_FLOATS + k] = v;
        if (PREC != 0 && a.sh_half) store_sh_half<PREC>(a.sh_half, i * SH_FLOATS + k, v);
      }
    }
  }
}

// Exploration noise (mcmc.wgsl:39-58): PCG-hashed sums of four uniforms.
__device__ __forceinline__ uint32_t pcg_hash(uint32_t v) {
  const uint32_t state = v * 747796405u + 2891336453u;
  const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}
__device__ __forceinline__ float noise1(uint32_t seed) {
  float acc = 0.f;
  uint32_t s = seed;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    s = pcg_hash(s);
    acc += (float)(s & 0x00ffffffu) / 16777216.0f;
  }
  return acc - 2.0f;
}

__global__ void __launch_bounds__(256) k_mcmc_noise(float4* pos_raw, const float2* scales_act, const float* opac_act,
                                                    uint32_t n, uint32_t seed, float sigma, float opacity_k) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float2 s = scales_act[i];
    const float mean_scale = 0.5f * (s.x + s.y);
    const float gate = expf(-opacity_k * opac_act[i]);
    const float amp = sigma * mean_scale * gate;
    if (amp <= 0.f) continue;
    const uint32_t base = pcg_hash(i ^ seed);
    float4 p = pos_raw[i];
    p.x += amp * noise1(base ^ 0x68bc21ebu);
    p.y += amp * noise1(base ^ 0x2c1b3c6du);
    p.z += amp * noise1(base ^ 0x1f123bb5u);
    pos_raw[i] = p;
  }
}

__global__ void k_copy_pos(const float4* raw, float4* act, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) act[i] = raw[i];
}

inline int grid_n(uint64_t n) { return (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 148 * 16)); }

}  // namespace

// Rows of M^(2^j), j < MCMC_JUMP_LEVELS, for the xorshift64 (13, 7, 17) step.
void mcmc_jump_tables(uint64_t* out) {
  auto step = [](uint64_t x) {
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    return x;
  };
  uint64_t m[64];  // rows
  for (int i = 0; i < 64; ++i) m[i] = 0;
  for (int j = 0; j < 64; ++j) {
    const uint64_t col = step(1ull << j);
    for (int i = 0; i < 64; ++i)
      if (col >> i & 1ull) m[i] |= 1ull << j;
  }
  for (int lvl = 0; lvl < MCMC_JUMP_LEVELS; ++lvl) {
    for (int i = 0; i < 64; ++i) out[64 * lvl + i] = m[i];
    uint64_t sq[64];  // m·m: row_i = XOR of rows m[j] for bits j of m[i]
    for (int i = 0; i < 64; ++i) {
      uint64_t r = 0;
      for (int j = 0; j < 64; ++j)
        if (m[i] >> j & 1ull) r ^= m[j];
      sq[i] = r;
    }
    for (int i = 0; i < 64; ++i) m[i] = sq[i];
  }
}

int launch_mcmc_relocate(McmcArgs& a, int prec, void* scan_scratch, void* sort_scratch, cudaStream_t st) {
  if (a.n == 0) return 0;
  const int g = grid_n(a.n);
  cudaMemsetAsync(a.counters, 0, sizeof(uint32_t) * 8, st);
  k_mcmc_flags<<<g, 256, 0, st>>>(a);
  int e = launch_scan(a.dead, nullptr, a.dead_rank, a.n, nullptr, a.counters + 0, nullptr, scan_scratch, st);
  if (e) return e;
  auto* bsum = reinterpret_cast<unsigned long long*>(scan_scratch);
  k_scan64_reduce<<<SCAN_GRID, 256, 0, st>>>(a.weight, a.n, bsum);
  k_scan64_blocks<<<1, SCAN_GRID, 0, st>>>(bsum, a.total_weight);
  k_scan64_down<<<SCAN_GRID, 256, 0, st>>>(a.weight, a.cum, a.n, bsum);
  k_mcmc_pick<<<g, 256, 0, st>>>(a);
  k_mcmc_claim<<<g, 256, 0, st>>>(a);
  k_mcmc_advance<<<1, 1, 0, st>>>(a);
  if (a.split_ratio > 0.f) {
    int in1 = 0;
    e = launch_radix_sort(a.size_key, a.size_val, a.key2, a.val2, a.n, nullptr, 32, sort_scratch, &in1, st);
    if (e) return e;
    a.sorted_size_key = in1 ? a.key2 : a.size_key;
    k_mcmc_over_flags<<<g, 256, 0, st>>>(a);
    e = launch_scan(a.over_flag, nullptr, a.over_rank, a.n, nullptr, a.counters + 5, nullptr, scan_scratch, st);
    if (e) return e;
    k_mcmc_over_list<<<g, 256, 0, st>>>(a);
    // The size keys are consumed; their buffers take the second sort.
    e = launch_radix_sort(a.over_key, a.over_val, a.key2, a.val2, a.n, a.counters + 5, 32, sort_scratch, &in1, st);
    if (e) return e;
    a.over_sorted_val = in1 ? a.val2 : a.over_val;
    e = launch_scan(a.leftover_flag, nullptr, a.left_rank, a.n, a.counters + 0, a.counters + 6, nullptr, scan_scratch,
                    st);
    if (e) return e;
    k_mcmc_left_list<<<g, 256, 0, st>>>(a);
    k_mcmc_split_count<<<1, 1, 0, st>>>(a);
  }
  if (prec == 0) k_mcmc_relocate<0><<<g, 256, 0, st>>>(a);
  else if (prec == 1) k_mcmc_relocate<1><<<g, 256, 0, st>>>(a);
  else k_mcmc_relocate<2><<<g, 256, 0, st>>>(a);
  return (int)cudaGetLastError();
}

int launch_mcmc_noise(float4* pos_raw, float4* pos_act, const float2* scales_act, const float* opac_act, uint32_t n,
                      uint32_t seed, float sigma, float opacity_k, cudaStream_t st) {
  if (n == 0) return 0;
  k_mcmc_noise<<<grid_n(n), 256, 0, st>>>(pos_raw, scales_act, opac_act, n, seed, sigma, opacity_k);
  k_copy_pos<<<grid_n(n), 256, 0, st>>>(pos_raw, pos_act, n);
  return (int)cudaGetLastError();
}

}  // namespace gs
