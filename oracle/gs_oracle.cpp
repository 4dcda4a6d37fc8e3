// Test infrastructure only (see gs_oracle.hpp): C entry points of the oracle
// for ctypes. Never linked into the shipped library.
//
// PARITY STATUS: unpinned against golden vectors (none exist in the
// reference); certified by finite differences and analytic known answers.
#include "gs_oracle.hpp"

#include <chrono>
#include <cstdio>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace orc;

extern "C" {

struct orc_scene {
  int n;
  int sh_degree;
  const double* pos;
  const double* scales;
  const double* quat;
  const double* opacity;
  const double* sh;  // n*48
};

struct orc_camera {
  double center[3];
  double quat[4];
  double focal;
  int width;
  int height;
};

static Scene to_scene(const orc_scene* s) {
  Scene o;
  o.n = s->n; o.sh_degree = s->sh_degree; o.pos = s->pos; o.scales = s->scales;
  o.quat = s->quat; o.opacity = s->opacity; o.sh = s->sh;
  return o;
}
static Camera to_cam(const orc_camera* c) {
  Camera o;
  for (int k = 0; k < 3; ++k) o.center[k] = c->center[k];
  for (int k = 0; k < 4; ++k) o.quat[k] = c->quat[k];
  o.focal = c->focal; o.width = c->width; o.height = c->height;
  return o;
}

static void set_threads(int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
}

int orc_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// Projection summary per input surfel (unsorted index order): rect (x0,y0,x1,y1)
// with culled/invisible items reported as (1,1,0,0), f32 depth-key bits,
// rect-marginal flag, sorted position (or -1 when depth-culled).
int orc_project(const orc_scene* s_, const orc_camera* c_, int tile, int32_t* rects, uint32_t* keys,
                uint8_t* rect_marginal, int32_t* sorted_pos) {
  Scene s = to_scene(s_);
  Camera cam = to_cam(c_);
  auto sc = prepare(s, cam, tile);
  for (int i = 0; i < s.n; ++i) {
    rects[4 * i] = 1; rects[4 * i + 1] = 1; rects[4 * i + 2] = 0; rects[4 * i + 3] = 0;
    keys[i] = 0; rect_marginal[i] = 0; sorted_pos[i] = -1;
  }
  for (int k = 0; k < (int)sc.size(); ++k) {
    const SurfelCam& x = sc[k];
    int i = x.idx;
    if (x.visible) {
      rects[4 * i] = x.x0; rects[4 * i + 1] = x.y0; rects[4 * i + 2] = x.x1; rects[4 * i + 3] = x.y1;
    }
    keys[i] = f32_bits(x.depth);
    rect_marginal[i] = x.rect_marginal ? 1 : 0;
    sorted_pos[i] = k;
  }
  return (int)sc.size();
}

// Forward render. literal=1 walks every sorted surfel per pixel through the
// tile-rect test, exactly as crates/gs-cpu-ref/src/forward.rs:218-244 does
// (O(P·N), single thread); literal=0 walks the per-tile lists (same result)
// in parallel over pixel rows.
int orc_render(const orc_scene* s_, const orc_camera* c_, int tile, int literal, int nthreads, double* color,
               double* alpha, double* depth, double* normal, double* trans, int32_t* ncontrib, uint8_t* marginal) {
  Scene s = to_scene(s_);
  Camera cam = to_cam(c_);
  auto sc = prepare(s, cam, tile);
  RenderOut o{color, alpha, depth, normal, trans, ncontrib, marginal};
  int tiles_x = (cam.width + tile - 1) / tile;
  if (literal) {
    std::vector<int> list;
    list.reserve(sc.size());
    for (int y = 0; y < cam.height; ++y)
      for (int x = 0; x < cam.width; ++x) {
        list.clear();
        for (int k = 0; k < (int)sc.size(); ++k)
          if (covers_tile(sc[k], x / tile, y / tile)) list.push_back(k);
        render_pixel(sc, list, cam, x, y, (size_t)y * cam.width + x, o);
      }
    return 0;
  }
  auto lists = tile_lists(sc, cam, tile);
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
  for (int y = 0; y < cam.height; ++y)
    for (int x = 0; x < cam.width; ++x)
      render_pixel(sc, lists[(size_t)(y / tile) * tiles_x + x / tile], cam, x, y, (size_t)y * cam.width + x, o);
  return 0;
}

// Forward render of a bounded sample of the image: only the pixels of tiles t
// with t % stride == offset (row-major tile ids of this camera) are written;
// the arrays are full-size and the other pixels are left as the caller set
// them. last_idx receives the input index of each pixel's last contributing
// surfel (-1 if none), which identifies the contributor independently of how
// a tile list was binned, and count its number of contributing surfels.
int orc_render_sampled(const orc_scene* s_, const orc_camera* c_, int tile, int stride, int offset, int nthreads,
                       double* color, double* alpha, double* depth, double* normal, double* trans, int32_t* ncontrib,
                       uint8_t* marginal, int32_t* last_idx, int32_t* count) {
  Scene s = to_scene(s_);
  Camera cam = to_cam(c_);
  if (stride < 1 || offset < 0 || offset >= stride) return -1;
  auto sc = prepare(s, cam, tile);
  RenderOut o{color, alpha, depth, normal, trans, ncontrib, marginal, last_idx, count};
  const int tiles_x = (cam.width + tile - 1) / tile, tiles_y = (cam.height + tile - 1) / tile;
  auto lists = tile_lists(sc, cam, tile, stride, offset);
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = offset; t < tiles_x * tiles_y; t += stride) {
    const int tx = t % tiles_x, ty = t / tiles_x;
    for (int y = ty * tile; y < std::min(cam.height, (ty + 1) * tile); ++y)
      for (int x = tx * tile; x < std::min(cam.width, (tx + 1) * tile); ++x)
        render_pixel(sc, lists[(size_t)t], cam, x, y, (size_t)y * cam.width + x, o);
  }
  return 0;
}

struct orc_grads {
  double* pos;
  double* scales;
  double* quat;
  double* opacity;
  double* sh;
  double* cam_center;
  double* cam_quat;
  double* focal;
  double* dl_dr_cam;
};

// Full analytic backward (crates/gs-cpu-ref/src/backward.rs:57-249). Gradients
// are ACCUMULATED into the caller's (zeroed) arrays. Per-tile partial
// accumulators are merged in tile order, so the result is deterministic for
// any thread count.
static int gradients_tiles(const orc_scene* s_, const orc_camera* c_, int tile, int stride, int offset,
                           const double* dl_dcolor, const double* dl_ddepth, const double* dl_dnormal,
                           double lambda_dist, int nthreads, const orc_grads* g_) {
  Scene s = to_scene(s_);
  Camera cam = to_cam(c_);
  if (stride < 1 || offset < 0 || offset >= stride) return -1;
  auto sc = prepare(s, cam, tile);
  auto lists = tile_lists(sc, cam, tile, stride, offset);
  int tiles_x = (cam.width + tile - 1) / tile, tiles_y = (cam.height + tile - 1) / tile;
  LossIn L{dl_dcolor, dl_ddepth, dl_dnormal, lambda_dist};
  int n_tiles = tiles_x * tiles_y;
  std::vector<std::vector<CamAcc>> partial(n_tiles);
  std::vector<double> tile_dfocal(n_tiles, 0.0);
  set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = offset; t < n_tiles; t += stride) {
    const auto& list = lists[t];
    if (list.empty()) continue;
    // Local accumulators indexed by position in the tile list: backward_pixel
    // sees the tile's surfels as a dense sub-vector.
    std::vector<CamAcc> local(list.size());
    std::vector<SurfelCam> sub;
    sub.reserve(list.size());
    for (int k : list) sub.push_back(sc[k]);
    std::vector<int> sub_list(list.size());
    for (size_t j = 0; j < list.size(); ++j) sub_list[j] = (int)j;
    std::vector<Contribution> contribs;
    double dfocal = 0;
    int tx = t % tiles_x, ty = t / tiles_x;
    for (int y = ty * tile; y < std::min(cam.height, (ty + 1) * tile); ++y)
      for (int x = tx * tile; x < std::min(cam.width, (tx + 1) * tile); ++x)
        backward_pixel(sub, sub_list, cam, x, y, L, local.data(), dfocal, contribs);
    partial[t] = std::move(local);
    tile_dfocal[t] = dfocal;
  }
  std::vector<CamAcc> acc(sc.size());
  double dfocal = 0;
  for (int t = 0; t < n_tiles; ++t) {
    const auto& list = lists[t];
    if (partial[t].empty()) continue;
    for (size_t j = 0; j < list.size(); ++j) {
      CamAcc& a = acc[list[j]];
      const CamAcc& p = partial[t][j];
      a.dc += p.dc; a.dtu += p.dtu; a.dtv += p.dtv; a.dcolor += p.dcolor; a.dnormal += p.dnormal;
      a.dopacity += p.dopacity;
    }
    dfocal += tile_dfocal[t];
  }
  Grads g{g_->pos, g_->scales, g_->quat, g_->opacity, g_->sh, g_->cam_center, g_->cam_quat, g_->focal, g_->dl_dr_cam};
  chain_to_params(s, cam, sc, acc, dfocal, g);
  return 0;
}

int orc_gradients(const orc_scene* s_, const orc_camera* c_, int tile, const double* dl_dcolor,
                  const double* dl_ddepth, const double* dl_dnormal, double lambda_dist, int nthreads,
                  const orc_grads* g_) {
  return gradients_tiles(s_, c_, tile, 1, 0, dl_dcolor, dl_ddepth, dl_dnormal, lambda_dist, nthreads, g_);
}

// The backward restricted to the pixels of tiles t with t % stride == offset:
// the exact gradient of a loss whose image gradient is zero on every other
// pixel (the caller's dl_* arrays are full-size; other pixels are not read).
int orc_gradients_sampled(const orc_scene* s_, const orc_camera* c_, int tile, int stride, int offset,
                          const double* dl_dcolor, const double* dl_ddepth, const double* dl_dnormal,
                          double lambda_dist, int nthreads, const orc_grads* g_) {
  return gradients_tiles(s_, c_, tile, stride, offset, dl_dcolor, dl_ddepth, dl_dnormal, lambda_dist, nthreads, g_);
}

double orc_distortion_loss(const orc_scene* s_, const orc_camera* c_, int tile) {
  return distortion_loss(to_scene(s_), to_cam(c_), tile);
}

// ------------------------------------------------------------------------
// f32 restatement of the projection arithmetic of
// crates/gs-kernels/src/shaders/surfel_prep_fwd.wgsl:64-132, evaluated in the
// same operation order with no contraction (this file is compiled with
// -ffp-contract=off). Used for bit-exact checks of tile rects and depth keys.
// R is column-major (rot[3*k + j] = column k, row j), the camera-to-world
// rotation already normalised.
static inline float dot3f(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

int orc_project_f32(int n, const float* pos4, const float* scales2, const float* quats4, const float* rot9,
                    const float* center3, float focal, int width, int height, int tile, uint32_t* rects4,
                    uint32_t* keys, float* cam_out /* n*12: c.xyz, depth, tu.xyz, px, tv.xyz, py */) {
  int tiles_x = (width + tile - 1) / tile, tiles_y = (height + tile - 1) / tile;
  const float* r0 = rot9;
  const float* r1 = rot9 + 3;
  const float* r2 = rot9 + 6;
  for (int i = 0; i < n; ++i) {
    uint32_t rect[4] = {1u, 1u, 0u, 0u};
    float x[3] = {pos4[4 * i] - center3[0], pos4[4 * i + 1] - center3[1], pos4[4 * i + 2] - center3[2]};
    float c[3] = {dot3f(r0, x), dot3f(r1, x), dot3f(r2, x)};
    float depth = -c[2];
    float* co = cam_out ? cam_out + 12 * i : nullptr;
    if (depth < 0.05f) {
      for (int k = 0; k < 4; ++k) rects4[4 * i + k] = rect[k];
      keys[i] = 0;
      if (co)
        for (int k = 0; k < 12; ++k) co[k] = 0.f;
      continue;
    }
    const float* q = quats4 + 4 * i;
    float qn = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    float qx = q[0] / qn, qy = q[1] / qn, qz = q[2] / qn, qw = q[3] / qn;
    float col0[3] = {1.0f - 2.0f * (qy * qy + qz * qz), 2.0f * (qx * qy + qw * qz), 2.0f * (qx * qz - qw * qy)};
    float col1[3] = {2.0f * (qx * qy - qw * qz), 1.0f - 2.0f * (qx * qx + qz * qz), 2.0f * (qy * qz + qw * qx)};
    float su = scales2[2 * i], sv = scales2[2 * i + 1];
    float yu[3] = {col0[0] * su, col0[1] * su, col0[2] * su};
    float yv[3] = {col1[0] * sv, col1[1] * sv, col1[2] * sv};
    float tu[3] = {dot3f(r0, yu), dot3f(r1, yu), dot3f(r2, yu)};
    float tv[3] = {dot3f(r0, yv), dot3f(r1, yv), dot3f(r2, yv)};
    float cx = (float)width * 0.5f, cy = (float)height * 0.5f;
    float px = cx + focal * c[0] / depth;
    float py = cy - focal * c[1] / depth;
    float lu = std::sqrt(dot3f(tu, tu)), lv = std::sqrt(dot3f(tv, tv));
    float r = std::min(3.0f * focal * (lu + lv) / depth + 3.0f, 64.0f);
    float tf = (float)tile;
    float mx = (float)(tiles_x - 1), my = (float)(tiles_y - 1);
    auto clampf = [](float v, float lo, float hi) { return std::min(std::max(v, lo), hi); };
    uint32_t x0 = (uint32_t)clampf((px - r) / tf, 0.0f, mx);
    uint32_t y0 = (uint32_t)clampf((py - r) / tf, 0.0f, my);
    uint32_t x1 = (uint32_t)clampf((px + r) / tf, 0.0f, mx);
    uint32_t y1 = (uint32_t)clampf((py + r) / tf, 0.0f, my);
    if (px + r >= 0.0f && px - r < (float)width && py + r >= 0.0f && py - r < (float)height) {
      rect[0] = x0; rect[1] = y0; rect[2] = x1; rect[3] = y1;
    }
    for (int k = 0; k < 4; ++k) rects4[4 * i + k] = rect[k];
    uint32_t kb;
    std::memcpy(&kb, &depth, 4);
    keys[i] = kb;
    if (co) {
      co[0] = c[0]; co[1] = c[1]; co[2] = c[2]; co[3] = depth;
      co[4] = tu[0]; co[5] = tu[1]; co[6] = tu[2]; co[7] = px;
      co[8] = tv[0]; co[9] = tv[1]; co[10] = tv[2]; co[11] = py;
    }
  }
  return 0;
}

// Camera-to-world rotation from an xyzw quaternion in f32, normalised first
// (the host-side conversion crates/gs-kernels/src/rasterizer.rs:410 performs
// with glam before writing the camera uniform). Column-major output.
void orc_camera_rotation_f32(const float* q_in, float* rot9) {
  float inv = 1.0f / std::sqrt(q_in[0] * q_in[0] + q_in[1] * q_in[1] + q_in[2] * q_in[2] + q_in[3] * q_in[3]);
  float x = q_in[0] * inv, y = q_in[1] * inv, z = q_in[2] * inv, w = q_in[3] * inv;
  float x2 = x + x, y2 = y + y, z2 = z + z;
  float xx = x * x2, xy = x * y2, xz = x * z2;
  float yy = y * y2, yz = y * z2, zz = z * z2;
  float wx = w * x2, wy = w * y2, wz = w * z2;
  rot9[0] = 1.0f - (yy + zz); rot9[1] = xy + wz; rot9[2] = xz - wy;
  rot9[3] = xy - wz; rot9[4] = 1.0f - (xx + zz); rot9[5] = yz + wx;
  rot9[6] = xz + wy; rot9[7] = yz - wx; rot9[8] = 1.0f - (xx + yy);
}

// ------------------------------------------------------------------------
// L1 + D-SSIM in f64, restating first_attempt/crates/gs-train/src/shaders/
// ssim.wgsl:41-143 (products, separable 11-tap sigma=1.5 blur with zero
// padding, partials, combine). Loss = w_l1·mean|x−y| + w_ssim·mean(1−S), means
// over pixels×3 channels. The reference form (1−λ)·L1 + λ·(1−S)/2 is
// w_l1 = 1−λ, w_ssim = λ/2; the benchmark form 0.8·L1 + 0.2·(1−S) is
// w_l1 = 0.8, w_ssim = 0.2. Images are rgba (4 doubles per pixel); alpha is
// ignored. Writes dL/dx (rgb, w = 0) and returns the loss; l1_sum/ssim_sum get
// the channel sums of |x−y| and S.
static void blur_sep(const std::vector<double>& src, std::vector<double>& dst, int W, int H, const double* w) {
  std::vector<double> tmp(src.size());
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      double a = src[(size_t)y * W + x] * w[0];
      for (int k = 1; k <= 5; ++k) {
        if (x >= k) a += src[(size_t)y * W + x - k] * w[k];
        if (x + k < W) a += src[(size_t)y * W + x + k] * w[k];
      }
      tmp[(size_t)y * W + x] = a;
    }
  dst.resize(src.size());
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      double a = tmp[(size_t)y * W + x] * w[0];
      for (int k = 1; k <= 5; ++k) {
        if (y >= k) a += tmp[(size_t)(y - k) * W + x] * w[k];
        if (y + k < H) a += tmp[(size_t)(y + k) * W + x] * w[k];
      }
      dst[(size_t)y * W + x] = a;
    }
}

// SH colour of one surfel seen along dir (coefficient-major rgb, up to 16
// coefficients); clamped[3] receives the clamp mask. Returns the number of
// basis functions of the degree.
int orc_sh_color(int degree, const double* sh, const double* dir, double* rgb, int* clamped) {
  bool cm[3];
  V3 c = sh_color(degree, sh, V3(dir[0], dir[1], dir[2]), cm);
  rgb[0] = c.x; rgb[1] = c.y; rgb[2] = c.z;
  for (int k = 0; k < 3; ++k) clamped[k] = cm[k] ? 1 : 0;
  return (degree + 1) * (degree + 1);
}

// Rotation of a (not necessarily unit) xyzw quaternion, column-major 3x3.
void orc_quat_to_mat(const double* q, double* r9) {
  M3 m = quat_to_mat(q);
  for (int c = 0; c < 3; ++c) { r9[3 * c] = m.c[c].x; r9[3 * c + 1] = m.c[c].y; r9[3 * c + 2] = m.c[c].z; }
}

// dL/dq through the normalisation for dL/dR given column-major.
void orc_quat_grad(const double* q, const double* dl_dr9, double* out4) {
  M3 w;
  for (int c = 0; c < 3; ++c) w.c[c] = V3(dl_dr9[3 * c], dl_dr9[3 * c + 1], dl_dr9[3 * c + 2]);
  quat_grad(q, w, out4);
}

// SH basis values (b[16]) and their gradients w.r.t. the direction (g[48],
// xyz per basis function); returns the number of basis functions.
int orc_sh_basis(int degree, const double* d, double* b, double* g) {
  V3 dir(d[0], d[1], d[2]), gg[16];
  const int nb = sh_basis(degree, dir, b);
  sh_basis_grad(degree, dir, gg);
  for (int k = 0; k < nb; ++k) { g[3 * k] = gg[k].x; g[3 * k + 1] = gg[k].y; g[3 * k + 2] = gg[k].z; }
  return nb;
}

// Scalar triple product a . (b x c) and its gradients (math.rs triple_grads).
double orc_triple(const double* a, const double* b, const double* c, double* ga, double* gb, double* gc) {
  V3 A(a[0], a[1], a[2]), B(b[0], b[1], b[2]), Cc(c[0], c[1], c[2]), GA, GB, GC;
  triple_grads(A, B, Cc, GA, GB, GC);
  const V3* g[3] = {&GA, &GB, &GC};
  double* o[3] = {ga, gb, gc};
  for (int k = 0; k < 3; ++k) { o[k][0] = g[k]->x; o[k][1] = g[k]->y; o[k][2] = g[k]->z; }
  return triple(A, B, Cc);
}

void orc_gauss_weights(double* w6) {
  double s = 0, g[6];
  for (int k = 0; k <= 5; ++k) g[k] = std::exp(-(double)(k * k) / (2.0 * 1.5 * 1.5));
  s = g[0];
  for (int k = 1; k <= 5; ++k) s += 2 * g[k];
  for (int k = 0; k <= 5; ++k) w6[k] = g[k] / s;
}

double orc_l1_ssim(const double* img, const double* ref, int W, int H, double w_l1, double w_ssim,
                   double* dl_out /* rgba */, double* l1_sum, double* ssim_sum) {
  const double C1 = 1e-4, C2 = 9e-4;
  double wts[6];
  orc_gauss_weights(wts);
  size_t P = (size_t)W * H;
  double inv_n3 = 1.0 / (double)(P * 3);
  double loss = 0, l1s = 0, ss = 0;
  for (int ch = 0; ch < 3; ++ch) {
    std::vector<double> x(P), y(P), xx(P), yy(P), xy(P);
    for (size_t i = 0; i < P; ++i) {
      x[i] = img[4 * i + ch]; y[i] = ref[4 * i + ch];
      xx[i] = x[i] * x[i]; yy[i] = y[i] * y[i]; xy[i] = x[i] * y[i];
    }
    std::vector<double> mx, my, bx2, by2, bxy;
    blur_sep(x, mx, W, H, wts);
    blur_sep(y, my, W, H, wts);
    blur_sep(xx, bx2, W, H, wts);
    blur_sep(yy, by2, W, H, wts);
    blur_sep(xy, bxy, W, H, wts);
    std::vector<double> cmu(P), cx2(P), cxy(P);
    double dw = -w_ssim * inv_n3;
    for (size_t i = 0; i < P; ++i) {
      double sx2 = bx2[i] - mx[i] * mx[i], sy2 = by2[i] - my[i] * my[i], sxy = bxy[i] - mx[i] * my[i];
      double p = mx[i] * mx[i] + my[i] * my[i] + C1;
      double q = sx2 + sy2 + C2;
      double l = (2 * mx[i] * my[i] + C1) / p;
      double cs = (2 * sxy + C2) / q;
      double S = l * cs;
      ss += S;
      double ds_dmux = cs * (2 * my[i] - 2 * mx[i] * l) / p + l * (-2 * my[i] + 2 * mx[i] * cs) / q;
      double ds_dbx2 = -l * cs / q;
      double ds_dbxy = 2 * l / q;
      cmu[i] = ds_dmux * dw; cx2[i] = ds_dbx2 * dw; cxy[i] = ds_dbxy * dw;
    }
    std::vector<double> bcmu, bcx2, bcxy;
    blur_sep(cmu, bcmu, W, H, wts);
    blur_sep(cx2, bcx2, W, H, wts);
    blur_sep(cxy, bcxy, W, H, wts);
    for (size_t i = 0; i < P; ++i) {
      double diff = x[i] - y[i];
      double sg = diff > 0 ? 1.0 : (diff < 0 ? -1.0 : 0.0);
      l1s += std::fabs(diff);
      if (dl_out) dl_out[4 * i + ch] = sg * w_l1 * inv_n3 + bcmu[i] + 2 * x[i] * bcx2[i] + y[i] * bcxy[i];
    }
  }
  if (dl_out)
    for (size_t i = 0; i < P; ++i) dl_out[4 * i + 3] = 0.0;
  loss = w_l1 * l1s * inv_n3 + w_ssim * (1.0 - ss * inv_n3);
  if (l1_sum) *l1_sum = l1s;
  if (ssim_sum) *ssim_sum = ss;
  return loss;
}

// ------------------------------------------------------------------------
// Adam over raw parameters with the raw→activated chain rule, restating
// first_attempt/crates/gs-train/src/shaders/adam.wgsl:33-74 with host bias
// corrections (first_attempt/crates/gs-train/src/optim.rs:179-197).
// activation: 0 identity, 1 exp, 2 sigmoid. In-place on raw/m/v; writes act.
void orc_adam(int n, double* raw, const double* grad_act, double* m, double* v, double* act, int activation,
              double lr, double beta1, double beta2, double eps, double reg, int t) {
  double bc1_inv = 1.0 / (1.0 - std::pow(beta1, t));
  double bc2_inv = 1.0 / (1.0 - std::pow(beta2, t));
  for (int i = 0; i < n; ++i) {
    double x = raw[i];
    double da = 1.0;
    if (activation == 1) da = std::exp(x);
    else if (activation == 2) { double s = 1.0 / (1.0 + std::exp(-x)); da = s * (1.0 - s); }
    double g = (grad_act[i] + reg) * da;
    m[i] = beta1 * m[i] + (1.0 - beta1) * g;
    v[i] = beta2 * v[i] + (1.0 - beta2) * g * g;
    raw[i] -= lr * (m[i] * bc1_inv) / (std::sqrt(v[i] * bc2_inv) + eps);
    double y = raw[i];
    act[i] = activation == 1 ? std::exp(y) : (activation == 2 ? 1.0 / (1.0 + std::exp(-y)) : y);
  }
}

// ------------------------------------------------------------------------
// Timed CPU step for the benchmark's baseline leg: projection + per-tile lists
// + forward + L1/SSIM + backward + parameter chain + Adam on one view, with the
// raster phases restricted to every `tile_stride`-th tile (a bounded sample).
// Returns seconds per phase in times[6]: prep+bin, fwd, loss, bwd, chain, adam.
int orc_cpu_step_timed(const orc_scene* s_, const orc_camera* c_, int tile, int tile_stride, int nthreads,
                       const double* target_rgba, double* times) {
  using clk = std::chrono::steady_clock;
  auto sec = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
  Scene s = to_scene(s_);
  Camera cam = to_cam(c_);
  set_threads(nthreads);
  auto t0 = clk::now();
  auto sc = prepare(s, cam, tile);
  auto lists = tile_lists(sc, cam, tile);
  auto t1 = clk::now();
  int tiles_x = (cam.width + tile - 1) / tile, tiles_y = (cam.height + tile - 1) / tile;
  int n_tiles = tiles_x * tiles_y;
  size_t P = (size_t)cam.width * cam.height;
  std::vector<double> color(P * 3, 0.0), alpha(P, 0.0), depth(P, 0.0), normal(P * 3, 0.0);
  RenderOut o{color.data(), alpha.data(), depth.data(), normal.data(), nullptr, nullptr, nullptr};
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = 0; t < n_tiles; t += tile_stride) {
    int tx = t % tiles_x, ty = t / tiles_x;
    for (int y = ty * tile; y < std::min(cam.height, (ty + 1) * tile); ++y)
      for (int x = tx * tile; x < std::min(cam.width, (tx + 1) * tile); ++x)
        render_pixel(sc, lists[t], cam, x, y, (size_t)y * cam.width + x, o);
  }
  auto t2 = clk::now();
  std::vector<double> img(P * 4), dl(P * 4);
  for (size_t i = 0; i < P; ++i) {
    img[4 * i] = color[3 * i]; img[4 * i + 1] = color[3 * i + 1]; img[4 * i + 2] = color[3 * i + 2]; img[4 * i + 3] = 1;
  }
  orc_l1_ssim(img.data(), target_rgba, cam.width, cam.height, 0.8, 0.2, dl.data(), nullptr, nullptr);
  auto t3 = clk::now();
  std::vector<double> dlc(P * 3);
  for (size_t i = 0; i < P; ++i)
    for (int ch = 0; ch < 3; ++ch) dlc[3 * i + ch] = dl[4 * i + ch];
  LossIn L{dlc.data(), nullptr, nullptr, 0.0};
  std::vector<std::vector<CamAcc>> partial(n_tiles);
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = 0; t < n_tiles; t += tile_stride) {
    const auto& list = lists[t];
    if (list.empty()) continue;
    std::vector<SurfelCam> sub;
    sub.reserve(list.size());
    for (int k : list) sub.push_back(sc[k]);
    std::vector<int> sub_list(list.size());
    for (size_t j = 0; j < list.size(); ++j) sub_list[j] = (int)j;
    std::vector<CamAcc> local(list.size());
    std::vector<Contribution> contribs;
    double df = 0;
    int tx = t % tiles_x, ty = t / tiles_x;
    for (int y = ty * tile; y < std::min(cam.height, (ty + 1) * tile); ++y)
      for (int x = tx * tile; x < std::min(cam.width, (tx + 1) * tile); ++x)
        backward_pixel(sub, sub_list, cam, x, y, L, local.data(), df, contribs);
    partial[t] = std::move(local);
  }
  std::vector<CamAcc> acc(sc.size());
  for (int t = 0; t < n_tiles; ++t) {
    if (partial[t].empty()) continue;
    const auto& list = lists[t];
    for (size_t j = 0; j < list.size(); ++j) {
      CamAcc& a = acc[list[j]];
      const CamAcc& p = partial[t][j];
      a.dc += p.dc; a.dtu += p.dtu; a.dtv += p.dtv; a.dcolor += p.dcolor; a.dnormal += p.dnormal;
      a.dopacity += p.dopacity;
    }
  }
  auto t4 = clk::now();
  std::vector<double> gpos(s.n * 3, 0.0), gsc(s.n * 2, 0.0), gq(s.n * 4, 0.0), gop(s.n, 0.0), gsh((size_t)s.n * 48, 0.0);
  double gcc[3] = {0, 0, 0}, gcq[4] = {0, 0, 0, 0}, gf = 0, gr[9] = {0};
  Grads g{gpos.data(), gsc.data(), gq.data(), gop.data(), gsh.data(), gcc, gcq, &gf, gr};
  chain_to_params(s, cam, sc, acc, 0.0, g);
  auto t5 = clk::now();
  // Adam over the 59 floats per surfel (pos 4 incl. pad lane, scales 2, quat
  // 4, opacity 1, SH 48), parallel over chunks.
  size_t np = (size_t)s.n * 59;
  std::vector<double> raw(np, 0.1), m(np, 0.0), v(np, 0.0), act(np, 0.0), gr2(np, 0.0);
  for (size_t i = 0; i < (size_t)s.n * 48; ++i) gr2[i] = gsh[i];
  int chunks = 64;
#pragma omp parallel for
  for (int c = 0; c < chunks; ++c) {
    size_t lo = np * c / chunks, hi = np * (c + 1) / chunks;
    orc_adam((int)(hi - lo), raw.data() + lo, gr2.data() + lo, m.data() + lo, v.data() + lo, act.data() + lo, 0,
             1e-3, 0.9, 0.999, 1e-15, 0.0, 1);
  }
  auto t6 = clk::now();
  times[0] = sec(t0, t1); times[1] = sec(t1, t2); times[2] = sec(t2, t3);
  times[3] = sec(t3, t4); times[4] = sec(t4, t5); times[5] = sec(t5, t6);
  return (int)sc.size();
}

}  // extern "C"
