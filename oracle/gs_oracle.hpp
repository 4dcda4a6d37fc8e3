// Test infrastructure only: the correctness oracle for the 2D-Gaussian-surfel
// training step. Nothing in the shipped library links or calls this code; it is
// used by tests/, the smoke check and the CPU-baseline leg of the benchmark.
//
// PARITY STATUS: unpinned against golden vectors. The reference ships no
// known-answer files for this path (its tests regenerate scenes from seeds and
// compare against its own Rust oracle, crates/gs-cpu-ref, which cannot be built
// here: no Rust toolchain). This file restates that oracle in C++ line by line
// and is certified instead by central finite differences (the reference's own
// gate, crates/gs-cpu-ref/tests/gradcheck.rs) and by analytic known-answer
// cases derived from the reference's camera and surfel conventions.
//
// Restated from (paths inside the reference project):
//   constants           crates/gs-cpu-ref/src/scene.rs:17-21
//   quat_to_mat          crates/gs-cpu-ref/src/math.rs:14-34
//   quat_grad            crates/gs-cpu-ref/src/math.rs:38-88
//   triple, triple_grads crates/gs-cpu-ref/src/math.rs:93-99
//   sh_basis[_grad]      crates/gs-cpu-ref/src/math.rs:127-191
//   pixel_ray            crates/gs-cpu-ref/src/forward.rs:32-40
//   prepare              crates/gs-cpu-ref/src/forward.rs:44-97
//   covers_pixel         crates/gs-cpu-ref/src/forward.rs:104-123
//   evaluate             crates/gs-cpu-ref/src/forward.rs:136-169
//   distortion_loss      crates/gs-cpu-ref/src/forward.rs:174-205
//   render               crates/gs-cpu-ref/src/forward.rs:207-246
//   gradients_full       crates/gs-cpu-ref/src/backward.rs:57-249
//   chain_ray_branch     crates/gs-cpu-ref/src/backward.rs:262-308
//   chain_screen_branch  crates/gs-cpu-ref/src/backward.rs:312-337
//
// Two additions beyond the reference oracle, both needed to compare against a
// tile-binned GPU rasterizer:
//   * n_contrib is reported the way the GPU kernel reports it
//     (crates/gs-kernels/src/shaders/rasterize_fwd.wgsl:172): the position,
//     inside the pixel's tile list, just past the last contributor.
//   * every pixel carries a "marginal" flag set when an alpha, transmittance,
//     branch or tile-rect decision lies so close to its threshold that float
//     and double evaluation may legitimately disagree.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace orc {

constexpr double LOWPASS_SIGMA2 = 0.5;
constexpr double ALPHA_SKIP = 1.0 / 255.0;
constexpr double ALPHA_CLAMP = 0.995;
constexpr double T_TERMINATE = 1e-4;
constexpr double NEAR_DEPTH = 0.05;

// Relative widths of the "marginal" bands (see header comment).
constexpr double MARGIN_ALPHA = 2e-5;  // absolute, on alpha in [0,1]
constexpr double MARGIN_T = 1e-3;      // relative, on transmittance vs T_TERMINATE
constexpr double MARGIN_RECT = 1e-5;   // absolute, in tile units
constexpr double MARGIN_BRANCH = 1e-6; // absolute, on g_ray - g_scr
// Conditioning of the float32 evaluation: a float32 rasterizer computes M =
// τu×τv, Bu = τv×c, Bv = c×τu, tn = −c·M and the dot products with s in
// single precision, so each carries an absolute error up to about
// COND_K·ε32 times the product of its factors' magnitudes. Propagated through
// u = (s·Bu)/det, v = (s·Bv)/det, t = tn/det, that gives a bound δq on the
// exponent the hit uses. Decisions within δq of a threshold, and hits whose
// δq exceeds COND_MAX_DQ (near-grazing surfels, where det ≈ 0), make the
// pixel marginal.
constexpr double EPS32 = 5.9604644775390625e-8;  // 2^-24
constexpr double COND_K = 16.0;
constexpr double COND_MAX_DQ = 1e-2;

struct V3 {
  double x = 0, y = 0, z = 0;
  V3() = default;
  V3(double a, double b, double c) : x(a), y(b), z(c) {}
  double& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  V3 operator+(const V3& o) const { return {x + o.x, y + o.y, z + o.z}; }
  V3 operator-(const V3& o) const { return {x - o.x, y - o.y, z - o.z}; }
  V3 operator-() const { return {-x, -y, -z}; }
  V3 operator*(double s) const { return {x * s, y * s, z * s}; }
  V3 operator/(double s) const { return {x / s, y / s, z / s}; }
  V3& operator+=(const V3& o) { x += o.x; y += o.y; z += o.z; return *this; }
  V3& operator-=(const V3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  bool is_zero() const { return x == 0 && y == 0 && z == 0; }
};
inline V3 operator*(double s, const V3& v) { return v * s; }
inline double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(const V3& a, const V3& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double length(const V3& a) { return std::sqrt(dot(a, a)); }
inline V3 normalize(const V3& a) { return a / length(a); }
inline V3 vmax0(const V3& a) { return {std::max(a.x, 0.0), std::max(a.y, 0.0), std::max(a.z, 0.0)}; }

// Column-major 3x3: c[k] is column k.
struct M3 {
  V3 c[3];
  V3 mul(const V3& v) const { return c[0] * v.x + c[1] * v.y + c[2] * v.z; }
  V3 mul_t(const V3& v) const { return {dot(c[0], v), dot(c[1], v), dot(c[2], v)}; }
};

// ------------------------------------------------------------------ math.rs
inline M3 quat_to_mat(const double q[4]) {
  double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  double x = q[0] / n, y = q[1] / n, z = q[2] / n, w = q[3] / n;
  M3 m;
  m.c[0] = {1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y)};
  m.c[1] = {2 * (x * y - w * z), 1 - 2 * (x * x + z * z), 2 * (y * z + w * x)};
  m.c[2] = {2 * (x * z + w * y), 2 * (y * z - w * x), 1 - 2 * (x * x + y * y)};
  return m;
}

// dL/dq for an unnormalised quaternion given dL/dR (Frobenius pairing),
// chained through the normalisation Jacobian (I - q̂q̂ᵀ)/n.
inline void quat_grad(const double q[4], const M3& dl_dr, double out[4]) {
  double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  double qh[4] = {q[0] / n, q[1] / n, q[2] / n, q[3] / n};
  double x = qh[0], y = qh[1], z = qh[2], w = qh[3];
  M3 d[4];
  d[0].c[0] = {0, 2 * y, 2 * z};     d[0].c[1] = {2 * y, -4 * x, 2 * w};  d[0].c[2] = {2 * z, -2 * w, -4 * x};
  d[1].c[0] = {-4 * y, 2 * x, -2 * w}; d[1].c[1] = {2 * x, 0, 2 * z};   d[1].c[2] = {2 * w, 2 * z, -4 * y};
  d[2].c[0] = {-4 * z, 2 * w, 2 * x}; d[2].c[1] = {-2 * w, -4 * z, 2 * y}; d[2].c[2] = {2 * x, 2 * y, 0};
  d[3].c[0] = {0, 2 * z, -2 * y};     d[3].c[1] = {-2 * z, 0, 2 * x};   d[3].c[2] = {2 * y, -2 * x, 0};
  double dqh[4] = {0, 0, 0, 0};
  for (int k = 0; k < 4; ++k)
    for (int col = 0; col < 3; ++col) dqh[k] += dot(dl_dr.c[col], d[k].c[col]);
  double dt = dqh[0] * qh[0] + dqh[1] * qh[1] + dqh[2] * qh[2] + dqh[3] * qh[3];
  for (int i = 0; i < 4; ++i) out[i] = (dqh[i] - qh[i] * dt) / n;
}

inline double triple(const V3& a, const V3& b, const V3& c) { return dot(a, cross(b, c)); }
inline void triple_grads(const V3& a, const V3& b, const V3& c, V3& ga, V3& gb, V3& gc) {
  ga = cross(b, c);
  gb = cross(c, a);
  gc = cross(a, b);
}

constexpr double SH_C0 = 0.28209479177387814;
constexpr double SH_C1 = 0.4886025119029199;
constexpr double SH_C2[5] = {1.0925484305920792, -1.0925484305920792, 0.31539156525252005,
                             -1.0925484305920792, 0.5462742152960396};
constexpr double SH_C3[7] = {-0.5900435899266435, 2.890611442640554, -0.4570457994644658,
                             0.3731763325901154,  -0.4570457994644658, 1.445305721320277,
                             -0.5900435899266435};

inline int num_coeffs(int degree) { return (degree + 1) * (degree + 1); }

inline int sh_basis(int degree, const V3& d, double b[16]) {
  double x = d.x, y = d.y, z = d.z;
  int k = 0;
  b[k++] = SH_C0;
  if (degree >= 1) {
    b[k++] = -SH_C1 * y;
    b[k++] = SH_C1 * z;
    b[k++] = -SH_C1 * x;
  }
  if (degree >= 2) {
    double xx = x * x, yy = y * y, zz = z * z;
    b[k++] = SH_C2[0] * x * y;
    b[k++] = SH_C2[1] * y * z;
    b[k++] = SH_C2[2] * (2 * zz - xx - yy);
    b[k++] = SH_C2[3] * x * z;
    b[k++] = SH_C2[4] * (xx - yy);
  }
  if (degree >= 3) {
    double xx = x * x, yy = y * y, zz = z * z;
    b[k++] = SH_C3[0] * y * (3 * xx - yy);
    b[k++] = SH_C3[1] * x * y * z;
    b[k++] = SH_C3[2] * y * (4 * zz - xx - yy);
    b[k++] = SH_C3[3] * z * (2 * zz - 3 * xx - 3 * yy);
    b[k++] = SH_C3[4] * x * (4 * zz - xx - yy);
    b[k++] = SH_C3[5] * z * (xx - yy);
    b[k++] = SH_C3[6] * x * (xx - 3 * yy);
  }
  return k;
}

inline int sh_basis_grad(int degree, const V3& d, V3 g[16]) {
  double x = d.x, y = d.y, z = d.z;
  int k = 0;
  g[k++] = V3();
  if (degree >= 1) {
    g[k++] = {0, -SH_C1, 0};
    g[k++] = {0, 0, SH_C1};
    g[k++] = {-SH_C1, 0, 0};
  }
  if (degree >= 2) {
    g[k++] = SH_C2[0] * V3(y, x, 0);
    g[k++] = SH_C2[1] * V3(0, z, y);
    g[k++] = SH_C2[2] * V3(-2 * x, -2 * y, 4 * z);
    g[k++] = SH_C2[3] * V3(z, 0, x);
    g[k++] = SH_C2[4] * V3(2 * x, -2 * y, 0);
  }
  if (degree >= 3) {
    double xx = x * x, yy = y * y, zz = z * z;
    g[k++] = SH_C3[0] * V3(6 * x * y, 3 * xx - 3 * yy, 0);
    g[k++] = SH_C3[1] * V3(y * z, x * z, x * y);
    g[k++] = SH_C3[2] * V3(-2 * x * y, 4 * zz - xx - 3 * yy, 8 * y * z);
    g[k++] = SH_C3[3] * V3(-6 * x * z, -6 * y * z, 6 * zz - 3 * xx - 3 * yy);
    g[k++] = SH_C3[4] * V3(4 * zz - 3 * xx - yy, -2 * x * y, 8 * x * z);
    g[k++] = SH_C3[5] * V3(2 * x * z, -2 * y * z, xx - yy);
    g[k++] = SH_C3[6] * V3(3 * xx - 3 * yy, -6 * x * y, 0);
  }
  return k;
}

// View-dependent colour of one surfel: max(0.5 + sum_k sh_k * basis_k(dir), 0)
// per channel, with the clamp mask (crates/gs-cpu-ref/src/forward.rs
// prepare; crates/gs-core/src/sh.rs sh_to_color). sh is coefficient-major rgb.
inline V3 sh_color(int degree, const double* sh, const V3& dir, bool clamped[3]) {
  double b[16];
  const int nb = sh_basis(degree, dir, b);
  V3 raw(0.5, 0.5, 0.5);
  for (int k = 0; k < nb; ++k) raw += V3(sh[3 * k], sh[3 * k + 1], sh[3 * k + 2]) * b[k];
  clamped[0] = raw.x < 0; clamped[1] = raw.y < 0; clamped[2] = raw.z < 0;
  return vmax0(raw);
}

// ------------------------------------------------------------------ scene.rs
// Surfels are stored SoA. SH is always padded to 16 coefficients (48 doubles
// per surfel, coefficient-major rgb), the same padding the GPU uses.
struct Scene {
  int n = 0;
  int sh_degree = 0;
  const double* pos = nullptr;     // n*3
  const double* scales = nullptr;  // n*2 activated
  const double* quat = nullptr;    // n*4 xyzw unnormalised
  const double* opacity = nullptr; // n activated
  const double* sh = nullptr;      // n*48
};

struct Camera {
  double center[3];
  double quat[4];  // camera-to-world xyzw
  double focal;
  int width, height;
};

struct SurfelCam {
  int idx;
  V3 c, tu, tv, color;
  bool clamped[3];
  double opacity;
  V3 normal;
  double depth, px, py;
  // Tile rect (inclusive), visibility, and whether any of its truncation or
  // visibility decisions is marginal.
  int x0, y0, x1, y1;
  bool visible;
  bool rect_marginal;
};

inline V3 pixel_ray(const Camera& cam, int x, int y) {
  double cx = cam.width * 0.5, cy = cam.height * 0.5;
  return {(x + 0.5 - cx) / cam.focal, -(y + 0.5 - cy) / cam.focal, -1.0};
}

// Tile rect exactly as covers_pixel computes it, plus marginal detection.
inline void tile_rect(SurfelCam& sc, const Camera& cam, int tile) {
  double r = std::min(3.0 * cam.focal * (length(sc.tu) + length(sc.tv)) / sc.depth + 3.0, 64.0);
  double T = tile;
  sc.visible = sc.px + r >= 0.0 && sc.px - r < cam.width && sc.py + r >= 0.0 && sc.py - r < cam.height;
  int tiles_x = (cam.width + tile - 1) / tile, tiles_y = (cam.height + tile - 1) / tile;
  double max_tx = tiles_x - 1, max_ty = tiles_y - 1;
  double a[4] = {(sc.px - r) / T, (sc.py - r) / T, (sc.px + r) / T, (sc.py + r) / T};
  double lim[4] = {max_tx, max_ty, max_tx, max_ty};
  int out[4];
  bool marg = false;
  for (int k = 0; k < 4; ++k) {
    double v = std::min(std::max(a[k], 0.0), lim[k]);
    out[k] = (int)v;
    if (a[k] > -MARGIN_RECT && a[k] < lim[k] + MARGIN_RECT) {
      double fr = a[k] - std::floor(a[k]);
      if (fr < MARGIN_RECT || fr > 1.0 - MARGIN_RECT) marg = true;
    }
  }
  double vis_terms[4] = {sc.px + r, cam.width - (sc.px - r), sc.py + r, cam.height - (sc.py - r)};
  for (double v : vis_terms)
    if (std::fabs(v) < MARGIN_RECT * T) marg = true;
  sc.x0 = out[0]; sc.y0 = out[1]; sc.x1 = out[2]; sc.y1 = out[3];
  sc.rect_marginal = marg;
}

inline float f32_of(double v) { return (float)v; }
inline uint32_t f32_bits(double v) {
  float f = (float)v;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

// forward.rs:44-97 — transform, SH colour, normal, projection; culled when
// depth < NEAR; sorted by (f32 depth bits, index).
inline std::vector<SurfelCam> prepare(const Scene& s, const Camera& cam, int tile) {
  M3 r_cam = quat_to_mat(cam.quat);
  V3 C(cam.center[0], cam.center[1], cam.center[2]);
  double cx = cam.width * 0.5, cy = cam.height * 0.5;
  std::vector<SurfelCam> out;
  out.reserve(s.n);
  for (int i = 0; i < s.n; ++i) {
    V3 p(s.pos[3 * i], s.pos[3 * i + 1], s.pos[3 * i + 2]);
    V3 x = p - C;
    V3 c = r_cam.mul_t(x);
    double depth = -c.z;
    if (depth < NEAR_DEPTH) continue;
    M3 rs = quat_to_mat(s.quat + 4 * i);
    V3 tu = r_cam.mul_t(rs.c[0] * s.scales[2 * i]);
    V3 tv = r_cam.mul_t(rs.c[1] * s.scales[2 * i + 1]);
    V3 dir = normalize(p - C);
    SurfelCam sc;
    sc.idx = i;
    sc.c = c; sc.tu = tu; sc.tv = tv;
    sc.color = sh_color(s.sh_degree, s.sh + 48 * i, dir, sc.clamped);
    V3 nrm = cross(tu, tv);
    if (dot(nrm, nrm) > 0.0) {
      nrm = normalize(nrm);
      if (dot(nrm, c) > 0.0) nrm = -nrm;
    }
    sc.normal = nrm;
    sc.opacity = s.opacity[i];
    sc.depth = depth;
    double w = -c.z;
    sc.px = cx + cam.focal * c.x / w;
    sc.py = cy - cam.focal * c.y / w;
    tile_rect(sc, cam, tile);
    out.push_back(sc);
  }
  std::stable_sort(out.begin(), out.end(), [](const SurfelCam& a, const SurfelCam& b) {
    uint32_t ka = f32_bits(a.depth), kb = f32_bits(b.depth);
    if (ka != kb) return ka < kb;
    return a.idx < b.idx;
  });
  return out;
}

inline bool covers_tile(const SurfelCam& sc, int tx, int ty) {
  return sc.visible && tx >= sc.x0 && tx <= sc.x1 && ty >= sc.y0 && ty <= sc.y1;
}

struct Hit {
  double ghat;
  bool ray_branch;
  double u, v, t;
  bool branch_marginal;
  double q, dq;  // exponent of ghat (ghat = exp(−q)) and its float32 error bound
};

// forward.rs:136-169
inline Hit evaluate(const SurfelCam& sc, const V3& d, double pix_x, double pix_y) {
  V3 s = -d;
  double det = triple(sc.tu, sc.tv, s);
  double g_ray = 0, u = 0, v = 0, t = 0;
  double q_ray = INFINITY, dq_ray = 0.0;
  bool marg = false;
  const double e = COND_K * EPS32;
  if (std::fabs(det) > 1e-12) {
    u = triple(-sc.c, sc.tv, s) / det;
    v = triple(sc.tu, -sc.c, s) / det;
    t = triple(sc.tu, sc.tv, -sc.c) / det;
    const double ns = length(s), ntu = length(sc.tu), ntv = length(sc.tv), nc = length(sc.c);
    const double ddet = e * ns * ntu * ntv, adet = std::fabs(det);
    const double du = (e * ns * ntv * nc + std::fabs(u) * ddet) / adet;
    const double dv = (e * ns * nc * ntu + std::fabs(v) * ddet) / adet;
    const double dt = (e * nc * ntu * ntv + std::fabs(t) * ddet) / adet;
    if (t > NEAR_DEPTH) {
      q_ray = (u * u + v * v) * 0.5;
      dq_ray = std::fabs(u) * du + std::fabs(v) * dv;
      g_ray = std::exp(-q_ray);
    }
    if (std::fabs(t - NEAR_DEPTH) < 1e-6 + dt) marg = true;
  }
  double dx = pix_x - sc.px, dy = pix_y - sc.py;
  const double q_scr = (dx * dx + dy * dy) / (2.0 * LOWPASS_SIGMA2);
  const double dq_scr = (std::fabs(dx) * e * (std::fabs(sc.px) + pix_x) + std::fabs(dy) * e * (std::fabs(sc.py) + pix_y)) /
                        LOWPASS_SIGMA2;
  double g_scr = std::exp(-q_scr);
  if (std::fabs(g_ray - g_scr) < MARGIN_BRANCH * std::max(1.0, g_scr) && (g_ray > 0 || g_scr > 0)) marg = true;
  if (std::fabs(q_ray - q_scr) < dq_ray + dq_scr) marg = true;
  if (g_ray >= g_scr) return {g_ray, true, u, v, t, marg, q_ray, dq_ray};
  return {g_scr, false, u, v, sc.depth, marg, q_scr, dq_scr};
}

// Per-tile entry lists in depth order: list[tile] = indices into the sorted
// SurfelCam vector. Identical to filtering the sorted vector with
// covers_pixel, which is what the reference's render loop does. With
// stride > 1 only the tiles t with t % stride == offset (row-major tile ids)
// get their lists; the others stay empty (a bounded sample of the image).
inline std::vector<std::vector<int>> tile_lists(const std::vector<SurfelCam>& sc, const Camera& cam, int tile,
                                                int stride = 1, int offset = 0) {
  int tiles_x = (cam.width + tile - 1) / tile, tiles_y = (cam.height + tile - 1) / tile;
  std::vector<std::vector<int>> lists((size_t)tiles_x * tiles_y);
  for (int k = 0; k < (int)sc.size(); ++k) {
    const SurfelCam& s = sc[k];
    if (!s.visible) continue;
    for (int ty = s.y0; ty <= s.y1; ++ty)
      for (int tx = s.x0; tx <= s.x1; ++tx) {
        const int t = ty * tiles_x + tx;
        if (stride > 1 && t % stride != offset) continue;
        lists[(size_t)t].push_back(k);
      }
  }
  return lists;
}

struct RenderOut {
  double* color;      // P*3
  double* alpha;      // P
  double* depth;      // P
  double* normal;     // P*3
  double* trans;      // P final transmittance (may be null)
  int32_t* ncontrib;  // P (may be null)
  uint8_t* marginal;  // P (may be null)
  int32_t* last_idx = nullptr;  // P: input index of the last contributing surfel, -1 if none (may be null)
  int32_t* count = nullptr;     // P: number of contributing surfels (alpha >= 1/255) (may be null)
};

// One pixel's forward walk over its tile list (forward.rs:218-244).
inline void render_pixel(const std::vector<SurfelCam>& sc, const std::vector<int>& list, const Camera& cam,
                         int x, int y, size_t i, const RenderOut& o) {
  V3 d = pixel_ray(cam, x, y);
  double pix_x = x + 0.5, pix_y = y + 0.5;
  double T = 1.0;
  V3 col, nrm;
  double a = 0, dep = 0;
  int nc = 0, last = -1, cnt = 0;
  bool marg = false;
  for (int li = 0; li < (int)list.size(); ++li) {
    const SurfelCam& s = sc[list[li]];
    if (s.rect_marginal) marg = true;
    Hit h = evaluate(s, d, pix_x, pix_y);
    double raw = s.opacity * h.ghat;
    double alpha = std::min(raw, ALPHA_CLAMP);
    if (std::fabs(alpha - ALPHA_SKIP) < MARGIN_ALPHA) marg = true;
    if (std::fabs(raw - ALPHA_CLAMP) < MARGIN_ALPHA) marg = true;
    if (s.opacity > 0.0) {  // the skip and clamp decisions in exponent space, within the float32 bound
      if (std::fabs(h.q - std::log(255.0 * s.opacity)) < h.dq) marg = true;
      if (s.opacity > ALPHA_CLAMP && std::fabs(h.q - std::log(s.opacity / ALPHA_CLAMP)) < h.dq) marg = true;
    }
    if (alpha < ALPHA_SKIP) continue;
    if (h.branch_marginal) marg = true;
    if (h.dq > COND_MAX_DQ) marg = true;  // an ill-conditioned contribution
    double w = T * alpha;
    col += s.color * w;
    a += w;
    dep += h.t * w;
    nrm += s.normal * w;
    T *= 1.0 - alpha;
    nc = li + 1;
    last = s.idx;
    ++cnt;
    if (std::fabs(T - T_TERMINATE) < MARGIN_T * T_TERMINATE) marg = true;
    if (T < T_TERMINATE) break;
  }
  o.color[3 * i] = col.x; o.color[3 * i + 1] = col.y; o.color[3 * i + 2] = col.z;
  o.alpha[i] = a;
  o.depth[i] = dep;
  o.normal[3 * i] = nrm.x; o.normal[3 * i + 1] = nrm.y; o.normal[3 * i + 2] = nrm.z;
  if (o.trans) o.trans[i] = T;
  if (o.ncontrib) o.ncontrib[i] = nc;
  if (o.marginal) o.marginal[i] = marg ? 1 : 0;
  if (o.last_idx) o.last_idx[i] = last;
  if (o.count) o.count[i] = cnt;
}

// forward.rs:174-205 — Σ_rays Σ_i Σ_j w_i w_j |t_i − t_j|.
inline double distortion_loss(const Scene& s, const Camera& cam, int tile) {
  auto sc = prepare(s, cam, tile);
  auto lists = tile_lists(sc, cam, tile);
  int tiles_x = (cam.width + tile - 1) / tile;
  double total = 0;
  for (int y = 0; y < cam.height; ++y)
    for (int x = 0; x < cam.width; ++x) {
      const auto& list = lists[(size_t)(y / tile) * tiles_x + x / tile];
      V3 d = pixel_ray(cam, x, y);
      double T = 1.0, a_pre = 0, b_pre = 0;
      for (int k : list) {
        const SurfelCam& s2 = sc[k];
        Hit h = evaluate(s2, d, x + 0.5, y + 0.5);
        double alpha = std::min(s2.opacity * h.ghat, ALPHA_CLAMP);
        if (alpha < ALPHA_SKIP) continue;
        double w = T * alpha;
        total += 2.0 * w * (h.t * a_pre - b_pre);
        a_pre += w;
        b_pre += w * h.t;
        T *= 1.0 - alpha;
        if (T < T_TERMINATE) break;
      }
    }
  return total;
}

// ------------------------------------------------------------- backward.rs
struct CamAcc {
  V3 dc, dtu, dtv, dcolor, dnormal;
  double dopacity = 0;
};

struct Grads {
  double* pos;      // n*3
  double* scales;   // n*2
  double* quat;     // n*4
  double* opacity;  // n
  double* sh;       // n*48
  double* cam_center; // 3
  double* cam_quat;   // 4
  double* focal;      // 1
  double* dl_dr_cam;  // 9, column-major dL/dR (the GPU's grad_cam[0..9])
};

inline void add_transpose_chain(M3& dl_dr, const V3& y, const V3& dl_da) {
  for (int k = 0; k < 3; ++k) dl_dr.c[k] += y * dl_da[k];
}

// backward.rs:262-308
inline void chain_ray_branch(const SurfelCam& sc, const V3& d, const Hit& hit, double dl_dghat, double dl_dt,
                             CamAcc& a, double& dfocal, double focal) {
  V3 s = -d;
  double det = triple(sc.tu, sc.tv, s);
  double u = hit.u, v = hit.v, t = hit.t;
  double dl_du = -u * hit.ghat * dl_dghat;
  double dl_dv = -v * hit.ghat * dl_dghat;
  double dl_dnu = dl_du / det, dl_dnv = dl_dv / det, dl_dnt = dl_dt / det;
  double dl_ddet = -(u * dl_du + v * dl_dv + t * dl_dt) / det;
  V3 ds, ga, gb, gc;
  triple_grads(-sc.c, sc.tv, s, ga, gb, gc);
  a.dc -= ga * dl_dnu; a.dtv += gb * dl_dnu; ds += gc * dl_dnu;
  triple_grads(sc.tu, -sc.c, s, ga, gb, gc);
  a.dtu += ga * dl_dnv; a.dc -= gb * dl_dnv; ds += gc * dl_dnv;
  triple_grads(sc.tu, sc.tv, -sc.c, ga, gb, gc);
  a.dtu += ga * dl_dnt; a.dtv += gb * dl_dnt; a.dc -= gc * dl_dnt;
  triple_grads(sc.tu, sc.tv, s, ga, gb, gc);
  a.dtu += ga * dl_ddet; a.dtv += gb * dl_ddet; ds += gc * dl_ddet;
  V3 dd = -ds;
  dfocal += dd.x * (-d.x / focal) + dd.y * (-d.y / focal);
}

// backward.rs:312-337
inline void chain_screen_branch(const SurfelCam& sc, double pix_x, double pix_y, double dl_dghat, CamAcc& a,
                                double& dfocal, const Camera& cam) {
  double dx = pix_x - sc.px, dy = pix_y - sc.py;
  double g = std::exp(-(dx * dx + dy * dy) / (2.0 * LOWPASS_SIGMA2));
  double dl_ddx = -(dx / LOWPASS_SIGMA2) * g * dl_dghat;
  double dl_ddy = -(dy / LOWPASS_SIGMA2) * g * dl_dghat;
  double dpx = -dl_ddx, dpy = -dl_ddy;
  double f = cam.focal, w = -sc.c.z;
  a.dc.x += dpx * f / w;
  a.dc.z += dpx * f * sc.c.x / (w * w);
  a.dc.y += dpy * (-f / w);
  a.dc.z += dpy * (-f * sc.c.y / (w * w));
  dfocal += dpx * sc.c.x / w + dpy * (-sc.c.y / w);
}

struct Contribution {
  int list_idx;  // index into the sorted SurfelCam vector
  double alpha;
  bool clamped_alpha;
  double t_before;
  Hit hit;
};

struct LossIn {
  const double* dl_dcolor;  // P*3
  const double* dl_ddepth;  // P or null
  const double* dl_dnormal; // P*3 or null
  double lambda_dist;
};

// Per-pixel replay + reverse walk (backward.rs:67-173), accumulating into
// per-sorted-surfel camera-space accumulators.
inline void backward_pixel(const std::vector<SurfelCam>& sc, const std::vector<int>& list, const Camera& cam,
                           int x, int y, const LossIn& L, CamAcc* acc, double& dfocal,
                           std::vector<Contribution>& contribs) {
  size_t pix = (size_t)y * cam.width + x;
  V3 dlc(L.dl_dcolor[3 * pix], L.dl_dcolor[3 * pix + 1], L.dl_dcolor[3 * pix + 2]);
  double dld = L.dl_ddepth ? L.dl_ddepth[pix] : 0.0;
  V3 dln = L.dl_dnormal ? V3(L.dl_dnormal[3 * pix], L.dl_dnormal[3 * pix + 1], L.dl_dnormal[3 * pix + 2]) : V3();
  bool any_image = !dlc.is_zero() || dld != 0.0 || !dln.is_zero();
  if (!any_image && L.lambda_dist == 0.0) return;
  V3 d = pixel_ray(cam, x, y);
  double pix_x = x + 0.5, pix_y = y + 0.5;
  contribs.clear();
  double T = 1.0, w_total = 0, wt_total = 0;
  for (int k : list) {
    const SurfelCam& s = sc[k];
    Hit h = evaluate(s, d, pix_x, pix_y);
    double raw = s.opacity * h.ghat;
    double alpha = std::min(raw, ALPHA_CLAMP);
    if (alpha < ALPHA_SKIP) continue;
    double w = T * alpha;
    w_total += w;
    wt_total += w * h.t;
    contribs.push_back({k, alpha, raw > ALPHA_CLAMP, T, h});
    T *= 1.0 - alpha;
    if (T < T_TERMINATE) break;
  }
  V3 suf_c, suf_n;
  double suf_d = 0, suf_w = 0, suf_cw = 0;
  for (int ci = (int)contribs.size() - 1; ci >= 0; --ci) {
    const Contribution& cb = contribs[ci];
    const SurfelCam& s = sc[cb.list_idx];
    CamAcc& a = acc[cb.list_idx];
    double t_i = cb.t_before, alpha = cb.alpha, w = t_i * alpha, t_hit = cb.hit.t;
    double dt_dist = 0, coef = 0;
    if (L.lambda_dist != 0.0) {
      double a_pre = w_total - suf_w - w;
      double b_pre = wt_total - suf_d - w * t_hit;
      dt_dist = L.lambda_dist * 2.0 * w * (a_pre - suf_w);
      coef = L.lambda_dist * (2.0 * (t_hit * a_pre - b_pre) + 2.0 * (suf_d - t_hit * suf_w));
    }
    a.dcolor += dlc * w;
    a.dnormal += dln * w;
    double dl_dt = dld * w + dt_dist;
    double dl_dalpha = dot(dlc, s.color) * t_i - dot(dlc, suf_c) / (1.0 - alpha) +
                       dld * (t_hit * t_i - suf_d / (1.0 - alpha)) + dot(dln, s.normal) * t_i -
                       dot(dln, suf_n) / (1.0 - alpha) + coef * t_i - suf_cw / (1.0 - alpha);
    suf_c += s.color * w;
    suf_d += t_hit * w;
    suf_n += s.normal * w;
    suf_w += w;
    suf_cw += coef * w;
    if (cb.clamped_alpha) continue;
    a.dopacity += dl_dalpha * cb.hit.ghat;
    double dl_dghat = dl_dalpha * s.opacity;
    if (cb.hit.ray_branch) {
      chain_ray_branch(s, d, cb.hit, dl_dghat, dl_dt, a, dfocal, cam.focal);
    } else {
      a.dc.z -= dl_dt;
      chain_screen_branch(s, pix_x, pix_y, dl_dghat, a, dfocal, cam);
    }
  }
}

// backward.rs:176-248 — camera-space accumulators → parameter gradients.
inline void chain_to_params(const Scene& scn, const Camera& cam, const std::vector<SurfelCam>& sc,
                            const std::vector<CamAcc>& acc, double dfocal, const Grads& g) {
  M3 r_cam = quat_to_mat(cam.quat);
  V3 C(cam.center[0], cam.center[1], cam.center[2]);
  M3 dl_dr_cam;
  V3 dcenter;
  for (size_t k = 0; k < sc.size(); ++k) {
    const SurfelCam& s = sc[k];
    const CamAcc& a = acc[k];
    int i = s.idx;
    V3 a_dtu = a.dtu, a_dtv = a.dtv;
    if (!a.dnormal.is_zero()) {
      V3 m = cross(s.tu, s.tv);
      double len = length(m);
      if (len > 1e-12) {
        V3 mhat = m / len;
        double sign = dot(mhat, s.c) > 0.0 ? -1.0 : 1.0;
        V3 dl_dm = (a.dnormal - mhat * dot(mhat, a.dnormal)) * (sign / len);
        a_dtu += cross(s.tv, dl_dm);
        a_dtv += cross(dl_dm, s.tu);
      }
    }
    V3 p(scn.pos[3 * i], scn.pos[3 * i + 1], scn.pos[3 * i + 2]);
    V3 x = p - C;
    V3 dx = r_cam.mul(a.dc);
    g.pos[3 * i] += dx.x; g.pos[3 * i + 1] += dx.y; g.pos[3 * i + 2] += dx.z;
    dcenter -= dx;
    add_transpose_chain(dl_dr_cam, x, a.dc);
    M3 rs = quat_to_mat(scn.quat + 4 * i);
    for (int axis = 0; axis < 2; ++axis) {
      V3 dtau = axis == 0 ? a_dtu : a_dtv;
      double scale = scn.scales[2 * i + axis];
      V3 axis_world = rs.c[axis];
      V3 yv = axis_world * scale;
      V3 dy = r_cam.mul(dtau);
      g.scales[2 * i + axis] += dot(dy, axis_world);
      M3 dl_drs;
      dl_drs.c[axis] = dy * scale;
      double dq[4];
      quat_grad(scn.quat + 4 * i, dl_drs, dq);
      for (int j = 0; j < 4; ++j) g.quat[4 * i + j] += dq[j];
      add_transpose_chain(dl_dr_cam, yv, dtau);
    }
    V3 dlc = a.dcolor;
    for (int ch = 0; ch < 3; ++ch)
      if (s.clamped[ch]) dlc[ch] = 0.0;
    if (!dlc.is_zero()) {
      V3 v = p - C;
      double len = length(v);
      V3 dir = v / len;
      double b[16];
      V3 bg[16];
      int nb = sh_basis(scn.sh_degree, dir, b);
      sh_basis_grad(scn.sh_degree, dir, bg);
      V3 ddir;
      const double* sh = scn.sh + 48 * i;
      for (int kk = 0; kk < nb; ++kk) {
        g.sh[48 * i + 3 * kk] += dlc.x * b[kk];
        g.sh[48 * i + 3 * kk + 1] += dlc.y * b[kk];
        g.sh[48 * i + 3 * kk + 2] += dlc.z * b[kk];
        ddir += bg[kk] * dot(V3(sh[3 * kk], sh[3 * kk + 1], sh[3 * kk + 2]), dlc);
      }
      V3 dv = (ddir - dir * dot(dir, ddir)) / len;
      g.pos[3 * i] += dv.x; g.pos[3 * i + 1] += dv.y; g.pos[3 * i + 2] += dv.z;
      dcenter -= dv;
    }
    g.opacity[i] += a.dopacity;
  }
  g.cam_center[0] += dcenter.x; g.cam_center[1] += dcenter.y; g.cam_center[2] += dcenter.z;
  double dq[4];
  quat_grad(cam.quat, dl_dr_cam, dq);
  for (int j = 0; j < 4; ++j) g.cam_quat[j] += dq[j];
  g.focal[0] += dfocal;
  if (g.dl_dr_cam)
    for (int k = 0; k < 3; ++k) {
      g.dl_dr_cam[3 * k] += dl_dr_cam.c[k].x;
      g.dl_dr_cam[3 * k + 1] += dl_dr_cam.c[k].y;
      g.dl_dr_cam[3 * k + 2] += dl_dr_cam.c[k].z;
    }
}

}  // namespace orc
