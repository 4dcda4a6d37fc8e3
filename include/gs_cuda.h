/*
 * gs_cuda — B200 (sm_100a) implementation of splattar's differentiable
 * 2D-Gaussian-surfel training step behind a plain C ABI.
 *
 * The reference exposes this path as concrete Rust structs holding public GPU
 * buffers that callers bind directly (no trait exists):
 *   gs_kernels::Rasterizer   crates/gs-kernels/src/rasterizer.rs:56-98
 *   gs_kernels::TileBinner   crates/gs-kernels/src/binning.rs:22-43
 *   gs_wgpu::RadixSorter     crates/gs-wgpu/src/sort.rs:17-327
 *   gs_wgpu::PrefixSum       crates/gs-wgpu/src/prefix_sum.rs:19-165
 *   gs_train::SsimLoss       first_attempt/crates/gs-train/src/ssim.rs:26-299
 *   gs_train::Optimizer      first_attempt/crates/gs-train/src/optim.rs:50-242
 *   gs_train::Trainer::step  first_attempt/crates/gs-train/src/trainer.rs:1139-1332
 * Each entry point below names the reference item it replaces. Every call
 * returns a gs_status. Work is stream-ordered on the caller's cudaStream_t
 * (passed as void*; NULL = legacy default stream). Handles are not
 * thread-safe; several handles may coexist. Device buffers are owned by the
 * handle unless a function takes caller pointers.
 *
 * Device errors that cannot be returned synchronously (entry-capacity
 * overflow, a bounded wait that expired) set a sticky error word on the
 * device; gs_rasterizer_check() synchronises and reports it.
 */
#ifndef GS_CUDA_H
#define GS_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  GS_OK = 0,
  GS_ERR_INVALID_ARG = 1,
  GS_ERR_CAPACITY = 2,       /* surfels, views, pixels or tile entries exceed the config */
  GS_ERR_CUDA = 3,           /* a CUDA runtime call failed */
  GS_ERR_DEVICE_TIMEOUT = 4, /* a bounded device-side wait expired */
  GS_ERR_NONFINITE = 5,
  GS_ERR_STATE = 6,          /* call out of order (e.g. backward before forward) */
  GS_ERR_IO = 7,             /* a file could not be opened, read or written */
  GS_ERR_FORMAT = 8          /* a file is not in a supported format (text in gs_last_error(NULL)) */
} gs_status;

/* Storage precision of the renderer-facing copies (projected records, SH). */
typedef enum { GS_PREC_F32 = 0, GS_PREC_F16 = 1, GS_PREC_BF16 = 2 } gs_precision;

enum {
  GS_FLAG_DETERMINISTIC = 1u << 0, /* ordered reductions, no float atomics on any gradient: per-entry record
                                      gradients summed in entry order, parameter gradients in view order, camera
                                      gradients as per-block partials summed in block order; results are bitwise
                                      reproducible run to run */
  GS_FLAG_PERSISTENT = 1u << 1,    /* persistent raster kernels over a global tile queue */
  GS_FLAG_COLOR_ONLY = 1u << 2,    /* backward ignores dl_dcolor.w, dl_dnormal and lambda_dist; the chosen-form
                                      training step's forward writes colour, alpha and final T only (OUT_NORMAL and
                                      the depth in OUT_AUX.y are left as they were) */
  GS_FLAG_TIGHT_BINNING = 1u << 3, /* bin a surfel only into the tiles its alpha >= 1/255 box overlaps: images and
                                      gradients are unchanged; tile lists, ranges and OUT_NCONTRIB then refer to the
                                      shorter lists instead of the reference's conservative rects */
  GS_FLAG_STORED_STATE = 1u << 4,  /* stored-state backward for the chosen-form step (with GS_FLAG_COLOR_ONLY): the
                                      forward records which tile entries composited into each pixel (one bit per
                                      pixel and entry, 32 bytes per entry of max_entries held by the handle) and
                                      the backward evaluates only those; results are identical */
  GS_FLAG_FULL_LISTS = 1u << 5     /* turn off the chosen-form step's occlusion cut. With the cut (the default,
                                      except in deterministic and stored-state modes) each tile is binned only down
                                      to the depth its pixels needed in the previous step with the same views, plus
                                      a margin (GS_BUF_TILE_CUT); a tile whose truncated list runs out before all its
                                      pixels terminate is binned and rendered again in full within the same step
                                      (counted in GS_BUF_INCOMPLETE_TILES). Images, contributor indices and
                                      gradients are those of the full lists; tile lists, ranges and the entry
                                      count then cover the truncated lists, and the full lists of completed
                                      tiles follow them in GS_BUF_SORTED_ITEMS (find a tile's list through
                                      GS_BUF_RANGES) */
};

/* Rasterizer::new(ctx, capacity, width, height, max_entries)
 * (crates/gs-kernels/src/rasterizer.rs:108). Adds a view count and pixel
 * budget for the batched multi-view form. Zero fields take defaults:
 * max_views 1, max_pixels width*height*max_views, max_entries
 * 64*capacity*max_views (the reference trainer's entries_per_surfel,
 * first_attempt/crates/gs-train/src/trainer.rs:474), tile 16. */
typedef struct {
  uint32_t capacity;
  uint32_t width;
  uint32_t height;
  uint32_t max_views;
  uint64_t max_pixels;
  uint64_t max_entries;
  uint32_t tile;        /* tile edge in pixels: 8, 16 or 32 (0 = 16, the reference's); see gs_set_tile_size */
  uint32_t batch;       /* shared-memory staging depth of the forward raster: 64, 128 or 256 (0 = 128) */
  uint32_t precision;   /* gs_precision */
  uint32_t flags;       /* GS_FLAG_* */
  uint32_t pixels_per_thread; /* forward raster: vertically adjacent pixels per thread; (batch, pixels_per_thread)
                                 must be a forward shape built for the tile (table at gs_autotune); 0 = 1 (4 for
                                 tile 32) */
} gs_raster_config;

/* RasterCamera (crates/gs-kernels/src/rasterizer.rs:34-41) plus the image
 * size, which the reference fixes per Rasterizer. quat is camera-to-world
 * xyzw, normalised on upload; principal point is the image centre; fx = fy. */
typedef struct {
  float quat[4];
  float center[3];
  float focal;
  uint32_t width;
  uint32_t height;
  uint32_t sh_degree;
} gs_camera;

/* SceneInput (crates/gs-kernels/src/rasterizer.rs:44-54): host SoA arrays of
 * ACTIVATED parameters. sh is coefficient-major rgb, sh_coeffs*3 floats per
 * surfel, padded to 48 on upload. */
typedef struct {
  const float* positions; /* n*3 */
  const float* scales;    /* n*2 */
  const float* quats;     /* n*4 xyzw */
  const float* opacities; /* n */
  const float* sh;        /* n*sh_coeffs*3 */
  uint32_t sh_coeffs;
  uint32_t n;
} gs_scene_input;

/* Public buffers of Rasterizer (rasterizer.rs:66-93), TileBinner and SsimLoss.
 * Per-pixel buffers hold all views back to back (gs_rasterizer_view_offset). */
typedef enum {
  GS_BUF_POSITIONS = 0,   /* float4 per surfel (w = 1) */
  GS_BUF_SCALES = 1,      /* float2 */
  GS_BUF_QUATS = 2,       /* float4 */
  GS_BUF_OPACITIES = 3,   /* float */
  GS_BUF_SH = 4,          /* 48 floats */
  GS_BUF_OUT_COLOR = 5,   /* float4: rgb + accumulated alpha */
  GS_BUF_OUT_AUX = 6,     /* float4: final T, alpha-weighted depth, 0, 0 */
  GS_BUF_OUT_NORMAL = 7,  /* float4 */
  GS_BUF_OUT_NCONTRIB = 8,/* u32: tile-list position just past the last contributor */
  GS_BUF_DL_DCOLOR = 9,   /* float4: rgb loss gradient + depth-loss gradient in w */
  GS_BUF_DL_DNORMAL = 10, /* float4 */
  GS_BUF_GRAD_POS = 11,   /* float4 */
  GS_BUF_GRAD_SCALES = 12,/* float2 */
  GS_BUF_GRAD_QUAT = 13,  /* float4 */
  GS_BUF_GRAD_OPACITY = 14,/* float */
  GS_BUF_GRAD_SH = 15,    /* 48 floats */
  GS_BUF_GRAD_CAM = 16,   /* 16 floats per view: dL/dR (column-major 9), dL/dC 3, dL/dfocal, pad 3 */
  GS_BUF_TARGET = 17,     /* float4 loss target per pixel (SsimLoss::target) */
  GS_BUF_RANGES = 18,     /* uint2 per tile (all views' tiles back to back): [start, end) */
  GS_BUF_SORTED_ITEMS = 19,/* uint2 per entry, tile-major, depth-ascending: (tile id counted from the first view's
                              first tile, item view*num_surfels + surfel; the expansion index in deterministic mode) */
  GS_BUF_ENTRY_COUNT = 20,/* u64: total tile entries of the last forward */
  GS_BUF_LOSS = 21,       /* double per view x2: sum |x-y| over rgb, sum SSIM over rgb */
  GS_BUF_RAW_POS = 22,    /* optimizer raw parameters (Optimizer ParamClass::raw) */
  GS_BUF_RAW_SCALES = 23,
  GS_BUF_RAW_QUAT = 24,
  GS_BUF_RAW_OPACITY = 25,
  GS_BUF_RAW_SH = 26,
  GS_BUF_RECTS = 27,      /* uint4 tile rect per item (x0,y0,x1,y1 inclusive; culled or off-screen = 1,1,0,0) */
  GS_BUF_DEPTH_KEYS = 28, /* u32 per item after the depth sort: f32 bits of the centre depth, ascending */
  GS_BUF_DEPTH_ORDER = 29,/* u32 per item after the depth sort: item index (stable, ties by index) */
  GS_BUF_GRAD_NORM_SUM = 30,/* float per surfel: sum over optimizer steps since the last densify (or init) of
                               |dL/dpos|, the densify statistic */
  GS_BUF_M_POS = 31,      /* Adam first moments (Optimizer ParamClass::m), layout of the raw buffers */
  GS_BUF_M_SCALES = 32,
  GS_BUF_M_QUAT = 33,
  GS_BUF_M_OPACITY = 34,
  GS_BUF_M_SH = 35,
  GS_BUF_V_POS = 36,      /* Adam second moments (Optimizer ParamClass::v) */
  GS_BUF_V_SCALES = 37,
  GS_BUF_V_QUAT = 38,
  GS_BUF_V_OPACITY = 39,
  GS_BUF_V_SH = 40,
  GS_BUF_NORMAL_LOSS = 41,/* double per view: sum over pixels of alpha (1 - n.N_d) of the last gs_loss_normal */
  GS_BUF_INCOMPLETE_TILES = 42,/* u32: tiles the last chosen-form step rendered again with full lists (occlusion cut) */
  GS_BUF_TILE_CUT = 43    /* u32 per tile: f32 bits of the deepest centre depth the next chosen-form step bins into
                             the tile (all ones: no cut); reset when the step's views or shape change */
} gs_buffer_id;

typedef struct gs_rasterizer gs_rasterizer;

/* Rasterizer::new */
gs_status gs_rasterizer_create(const gs_raster_config* cfg, gs_rasterizer** out);
gs_status gs_rasterizer_destroy(gs_rasterizer* r);
/* Rasterizer::upload_scene (rasterizer.rs:359-386). Blocking copy. */
gs_status gs_rasterizer_upload_scene(gs_rasterizer* r, const gs_scene_input* scene, void* stream);
/* Rasterizer::lambda_dist (rasterizer.rs:60) */
gs_status gs_rasterizer_set_lambda_dist(gs_rasterizer* r, float lambda_dist);
/* No reference counterpart (the reference's device code has no waits). The
 * chosen-form step's fused projection backward + Adam kernel copies each
 * block's optimizer rows into shared memory with bulk copies and waits for
 * them with two bounded waits: copy_wait_cycles before the block's Adam update
 * (on expiry the block skips its update and sets the sticky error word, which
 * gs_rasterizer_check reports as GS_ERR_DEVICE_TIMEOUT; 0 gives up at once)
 * and drain_wait_cycles for the copies to land before an expired block exits
 * (at least 1e8 cycles, else GS_ERR_INVALID_ARG). Defaults 2e9 and 2e9 SM
 * cycles (about 1 s each at 1.965 GHz). Host-only; later steps use them. */
gs_status gs_rasterizer_set_wait_limits(gs_rasterizer* r, uint64_t copy_wait_cycles, uint64_t drain_wait_cycles);
/* Rasterizer::forward (rasterizer.rs:389-448): projection, binning, forward
 * raster for n_views cameras (1 = the reference's single-view call). */
gs_status gs_rasterizer_forward(gs_rasterizer* r, const gs_camera* cams, uint32_t n_views, uint32_t num_surfels,
                                void* stream);
/* Rasterizer::backward (rasterizer.rs:320-356): clears the gradient buffers,
 * then backward raster and projection backward, summing over the views of the
 * last forward. Reads dl_dcolor (+ w depth gradient) and dl_dnormal. */
gs_status gs_rasterizer_backward(gs_rasterizer* r, uint32_t num_surfels, void* stream);
/* Buffer address and size in bytes. */
gs_status gs_rasterizer_buffer(gs_rasterizer* r, gs_buffer_id id, void** dptr, size_t* bytes);
/* First pixel (in per-pixel buffers) and first tile of a view of the last forward. */
gs_status gs_rasterizer_view_offset(gs_rasterizer* r, uint32_t view, uint64_t* pixel_offset, uint32_t* tile_offset);
/* Stream-ordered copies between host memory and a handle buffer; blocking. */
gs_status gs_rasterizer_read(gs_rasterizer* r, gs_buffer_id id, uint64_t byte_offset, void* host, size_t bytes,
                             void* stream);
gs_status gs_rasterizer_write(gs_rasterizer* r, gs_buffer_id id, uint64_t byte_offset, const void* host, size_t bytes,
                              void* stream);
/* Asynchronous variants: the other side may be pinned host memory or device
 * memory (the direction follows from the pointer, cudaMemcpyDefault), and
 * must stay valid until the stream reaches the copy. A device source lets a
 * caller prefetch the next step's input on another stream and move it into
 * the handle with a device-to-device copy. */
gs_status gs_rasterizer_read_async(gs_rasterizer* r, gs_buffer_id id, uint64_t byte_offset, void* host, size_t bytes,
                                   void* stream);
gs_status gs_rasterizer_write_async(gs_rasterizer* r, gs_buffer_id id, uint64_t byte_offset, const void* host,
                                    size_t bytes, void* stream);
/* Synchronises the stream and reports (and clears) the sticky device error word. */
gs_status gs_rasterizer_check(gs_rasterizer* r, void* stream);
/* Text of the last error on this handle (or of the last failed create when r is NULL). */
gs_status gs_last_error(gs_rasterizer* r, char* msg, size_t cap);

/* SsimLoss::encode (first_attempt/crates/gs-train/src/ssim.rs:236-280):
 * L = w_l1*mean|x-y| + w_ssim*mean(1-SSIM) per view, rgb channels, 11-tap
 * sigma 1.5 Gaussian window with zero padding. Reads OUT_COLOR and TARGET,
 * writes DL_DCOLOR (w = 0) and the per-view sums into GS_BUF_LOSS. The
 * reference's own form (1-lambda)*L1 + lambda*(1-SSIM)/2 is w_l1 = 1-lambda,
 * w_ssim = lambda/2. */
gs_status gs_loss_l1_ssim(gs_rasterizer* r, float w_l1, float w_ssim, void* stream);

/* NormalLoss (first_attempt/crates/gs-train/src/normal_loss.rs,
 * shaders/normal_loss.wgsl:52-145), for every view of the last forward (which
 * must have written depth and normals, i.e. not the colour-only training
 * step): with mean depth tbar = depth_acc/alpha (pixels with alpha below
 * alpha_min are skipped; 0.2 in the reference), P = tbar * ray and
 * N_d = normalize(dP/dx x dP/dy) facing the camera,
 * L = lambda/(W*H) * sum_q alpha_q (1 - n_q . N_d), alpha and the orientation
 * detached (the W*H division is NormalLoss::set_lambda's). Writes
 * DL_DNORMAL and the depth-gradient channel DL_DCOLOR.w (rgb untouched; run
 * after gs_loss_l1_ssim) and the per-view sums into GS_BUF_NORMAL_LOSS. */
gs_status gs_loss_normal(gs_rasterizer* r, float lambda, float alpha_min, void* stream);

/* Camera pose refinement (crates/gs-track/src/lib.rs:289-337), host-only:
 * gs_camera_step_grad = camera_step_grad (the antisymmetric part of
 * R^T dL/dR as a rotation gradient, then dL/dC; GS_ERR_NONFINITE for a
 * non-finite input); gs_camera_adam6 = adam6 (betas 0.9/0.999, eps 1e-10,
 * separate rotation and centre rates; t is the 1-based step);
 * gs_camera_apply_step = apply_camera_step (q <- normalize(q * exp(-step[0..3])),
 * C <- C - step[3..6]). */
gs_status gs_camera_step_grad(const float grad_cam[16], const float quat[4], float out6[6]);
gs_status gs_camera_adam6(float m[6], float v[6], uint32_t t, const float grad[6], float lr_rot, float lr_center,
                          float step[6]);
gs_status gs_camera_apply_step(gs_camera* cam, const float step[6]);

/* Trainer schedule (first_attempt/crates/gs-train/src/trainer.rs), host-only.
 * gs_scene_extent = the position-LR scale of trainer.rs:740-746: half the
 * diagonal of the bounding box of n positions (stride floats apart, xyz
 * first), at least 1e-3. gs_schedule_t = schedule_t (trainer.rs:407-416):
 * iter/iters, or with an anneal (start, len, t0) t0 + (1 − t0)·min(1,
 * (iter − start)/len) (iter before start counts as start). gs_position_lr =
 * the exponential decay of trainer.rs:1150: lr_pos·extent·final_factor^t
 * (the defaults are lr_pos 1.6e-4, final_factor 0.01, trainer.rs:470-471). */
typedef struct {
  uint32_t start;
  uint32_t len;
  float t0;
} gs_anneal;
gs_status gs_scene_extent(const float* positions, uint32_t n, uint32_t stride, float* extent);
gs_status gs_schedule_t(uint32_t iter, uint32_t iters, const gs_anneal* anneal, float* t);
gs_status gs_position_lr(float lr_pos, float extent, float final_factor, float t, float* lr);

/* Optimizer (first_attempt/crates/gs-train/src/optim.rs:50-242) over the five
 * classes the trainer registers (trainer.rs:757-761): pos (identity, 4 per
 * surfel incl. pad lane), scales (exp), quat (identity), opacity (sigmoid),
 * sh (identity, 48). */
typedef struct {
  float lr[5];      /* pos, scales, quat, opacity, sh */
  float reg[5];     /* constant added to dL/d(activated) (optim.rs:37) */
  float beta1;
  float beta2;
  float eps;        /* the reference uses 1e-8 (optim.rs:187) */
} gs_adam_config;

/* Trainer::new raw upload (trainer.rs:763-791): raw = inverse activation of
 * the current activated buffers (log scales, logit opacity); zero moments, t = 0. */
gs_status gs_optimizer_init(gs_rasterizer* r, uint32_t num_surfels, void* stream);
/* Optimizer::encode_step (optim.rs:205-227): t += 1, Adam on every class,
 * then refresh the activated buffers. */
gs_status gs_optimizer_step(gs_rasterizer* r, const gs_adam_config* cfg, uint32_t num_surfels, void* stream);

/* One Adam step on caller device arrays (adam.wgsl:45-74): activation 0
 * identity, 1 exp, 2 sigmoid; t is the 1-based step for bias correction.
 * act may be NULL. */
gs_status gs_adam_flat(float* raw, const float* grad_act, float* m, float* v, float* act, uint64_t n,
                       uint32_t activation, float lr, float beta1, float beta2, float eps, float reg, uint32_t t,
                       void* stream);

/* One training iteration (Trainer::step, trainer.rs:1139-1332, without the
 * out-of-scope appearance, pose and noise stages): forward over n_views
 * cameras, L1+SSIM against TARGET, backward summing over views, Adam.
 * form 0 = plain: views one at a time, FP32, separate kernels per stage.
 * form 1 = chosen: all views batched in one pass per stage, tight binning
 *          (GS_FLAG_TIGHT_BINNING), persistent raster kernels, projection
 *          backward fused with Adam, storage precision from the config, the
 *          whole step replayed as one CUDA graph.
 * loss 0 = L1+SSIM against TARGET with weights w_l1, w_ssim (Trainer::step).
 * loss 1 = the image gradient the caller wrote into DL_DCOLOR (rgb; the
 *          depth channel and DL_DNORMAL are not read) is used as it is: no
 *          loss kernel runs and GS_BUF_LOSS is zero. This is the reference's
 *          split between a loss producer that writes dl_dcolor (SsimLoss,
 *          NormalLoss, the tracker's photometric loss,
 *          crates/gs-track/src/lib.rs:134-142) and Rasterizer::backward. */
enum { GS_LOSS_L1_SSIM = 0, GS_LOSS_GIVEN = 1 };
typedef struct {
  float w_l1;
  float w_ssim;
  gs_adam_config adam;
  uint32_t form;
  uint32_t loss;  /* GS_LOSS_* */
} gs_step_config;
gs_status gs_train_step(gs_rasterizer* r, const gs_camera* cams, uint32_t n_views, uint32_t num_surfels,
                        const gs_step_config* cfg, void* stream);

/* The same step with CUDA events recorded on the stream between its stages
 * (not graph-replayed); blocking. stage_ms receives milliseconds per stage,
 * summed over views: 0 projection, 1 depth sort + entry scan, 2 tile-entry
 * expansion, 3 tile sort, 4 tile ranges, 5 forward raster, 6 L1+SSIM,
 * 7 backward raster, 8 projection backward + Adam. */
gs_status gs_train_step_profiled(gs_rasterizer* r, const gs_camera* cams, uint32_t n_views, uint32_t num_surfels,
                                 const gs_step_config* cfg, void* stream, float stage_ms[9], uint32_t* n_stages);

/* No reference counterpart: the work of the raster kernels on the last
 * forward, counted on the device by replaying each pixel's walk (for the
 * compute side of their roofline; not meant for a timed region). out =
 * {forward hit evaluations (list entries whose alpha box holds the pixel,
 * up to the pixel's termination), contributing pairs (alpha >= 1/255, the
 * forward's own decisions), backward hit evaluations (entries before the
 * pixel's last contributor that the backward evaluates), pixels}. Blocking. */
gs_status gs_raster_work(gs_rasterizer* r, uint64_t out[4], void* stream);

/* Raster launch shapes (staging batch, pixels per thread) built per tile size:
 *   forward   tile 8:  ppt 1 or 2 with batch 64/128/256
 *             tile 16: (64,1) (128,1) (256,1) (64,2) (128,2) (64,4) (64,8) (128,8) (32,0)
 *             tile 32: ppt 2 or 4 with batch 64/128/256, and (128,8)
 *   backward  tile 8:  (64,1) (64,2) (128,2)
 *             tile 16: (64,1) (64,2) (128,2) (64,4) (32,8) (64,8) (128,8) (32,0)
 *             tile 32: (64,4) (64,8)
 * (32,0) selects the pixel-compacted kernels (one warp per tile spreading each
 * entry's box pixels over its lanes) for the colour-only persistent passes of
 * the training step; other passes fall back to (64,4) forward and (64,8)
 * backward. The backward with aux losses uses its own fixed shape.
 *
 * Autotuner (config-2 sweep of the batched form): at the handle's current
 * tile size, times the forward (projection + binning + raster) over every
 * forward shape and the colour-only backward raster over every backward
 * shape on these cameras (tight binning, the config's precision) and keeps
 * the fastest. out = {fwd batch, fwd pixels/thread, bwd batch, bwd
 * pixels/thread}. Blocking. GS_ERR_CAPACITY if the tile entries exceed
 * max_entries. */
gs_status gs_autotune(gs_rasterizer* r, const gs_camera* cams, uint32_t n_views, uint32_t num_surfels, void* stream,
                      uint32_t out[4]);
/* The same sweep over tile sizes 8, 16 and 32 (the reference fixes 16,
 * crates/gs-kernels/src/rasterizer.rs:13): each tile size's shapes are timed
 * as above, tile sizes whose entries exceed max_entries (or whose tile count
 * exceeds the handle's tile budget) are skipped, and the fastest forward +
 * backward total is kept. out = {tile, fwd batch, fwd pixels/thread, bwd
 * batch, bwd pixels/thread}; times_ms (optional, 6 floats) = {fwd, bwd} ms
 * per launch of the winning shapes for tiles 8, 16, 32 (-1 where skipped).
 * The stored-state handle stays at tile 16. Blocking. */
gs_status gs_autotune_tiles(gs_rasterizer* r, const gs_camera* cams, uint32_t n_views, uint32_t num_surfels,
                            void* stream, uint32_t out[5], float times_ms[6]);
/* Applies launch shapes (the layout of gs_autotune's out, e.g. a stored
 * result) without timing. Each pair must be built for the handle's tile
 * size (table above), else GS_ERR_INVALID_ARG and nothing changes. Host-only. */
gs_status gs_set_launch_shapes(gs_rasterizer* r, const uint32_t shapes[4]);
/* Changes the tile edge (8, 16 or 32 pixels) of later forwards. Launch
 * shapes not built for the new size fall back to its first forward shape and
 * its default backward shape ((128,2) where built, else (64,4)). Tile rects,
 * entry lists, ranges and contributor indices of later forwards refer to the
 * new tiling (the oracle's rect arithmetic takes the tile size as a
 * parameter). GS_ERR_INVALID_ARG for other sizes, or for a tile other than
 * 16 on a stored-state handle. Host-only. */
gs_status gs_set_tile_size(gs_rasterizer* r, uint32_t tile);
/* The handle's current tile edge in pixels (0 for a null handle). */
uint32_t gs_tile_size(const gs_rasterizer* r);

/* Densify/prune compaction (no reference counterpart; the reference only
 * relocates at fixed budget, trainer.rs:1558-1689): surfels whose mean
 * accumulated position-gradient norm exceeds grad_threshold are cloned
 * (copy with zeroed moments, appended while capacity allows), surfels whose
 * activated opacity is below opacity_threshold are removed, and survivors are
 * compacted in index order. Resets the gradient accumulators. */
typedef struct {
  float grad_threshold;     /* 2e-4 in the 6M-surfel workload */
  float opacity_threshold;  /* 0.005 */
} gs_densify_config;
gs_status gs_densify_prune(gs_rasterizer* r, const gs_densify_config* cfg, uint32_t num_surfels,
                           uint32_t* num_out, void* stream);

/* ---- MCMC relocation (first_attempt/crates/gs-train/src/trainer.rs:1558-1689,
 * shaders/relocate.wgsl, shaders/mcmc.wgsl) -------------------------------
 * Dead surfels (activated opacity below dead_threshold) move onto alive
 * surfels sampled in proportion to opacity (one xorshift64 draw per dead
 * surfel in index order; a target already taken by a lower-indexed dead
 * surfel defers this one); with split_ratio > 0, leftover dead slots then
 * split the alive surfels larger than split_ratio x the median alive size
 * (largest first). Both surfels of a pair get the opacity 1 - sqrt(1 - a),
 * shrunk scales (x0.85, or x0.6 and +-0.6 sigma offsets for splits) and zero
 * Adam moments. The same choices as the reference's host sampler for the same
 * generator state, computed on the device without a readback; the generator
 * state lives on the device and advances by one step per dead surfel.
 * Requires gs_optimizer_init. Stream-ordered. */
typedef struct {
  float dead_threshold; /* 0.005 in the reference trainer (trainer.rs:487) */
  float split_ratio;    /* 8.0 (trainer.rs:488); 0 disables splits */
} gs_mcmc_config;
gs_status gs_mcmc_seed(gs_rasterizer* r, uint64_t xorshift_state, void* stream);  /* nonzero; blocking */
gs_status gs_mcmc_relocate(gs_rasterizer* r, const gs_mcmc_config* cfg, uint32_t num_surfels, void* stream);
/* Blocking: out = {dead, relocated, split, deferred} of the last relocation, and the generator state. */
gs_status gs_mcmc_stats(gs_rasterizer* r, uint32_t out[4], uint64_t* xorshift_state, void* stream);
/* Exploration noise on positions (mcmc.wgsl:39-58): each coordinate moves by
 * sigma * mean(scale) * exp(-opacity_k * opacity) * (sum of 4 uniforms - 2),
 * uniforms from a PCG hash of (index ^ seed); the activated positions follow. */
gs_status gs_mcmc_noise(gs_rasterizer* r, uint32_t num_surfels, uint32_t seed, float sigma, float opacity_k,
                        void* stream);

/* ---- TileBinner (crates/gs-kernels/src/binning.rs:22-238) ---------------
 * Items are tile-space AABBs (uint4 min_x, min_y, max_x, max_y inclusive;
 * max < min = culled) with u32 depth keys. After encode, sorted_entries holds
 * entry indices in the reference's expansion order (item-major, row-major
 * within the rect) grouped by tile and depth-ascending, ties by entry index;
 * entry_items maps entry -> item; ranges holds [start, end) per tile. */
typedef struct gs_binner gs_binner;
gs_status gs_binner_create(uint32_t max_items, uint64_t max_entries, uint32_t num_tiles, gs_binner** out);
gs_status gs_binner_destroy(gs_binner* b);
gs_status gs_binner_encode(gs_binner* b, const uint32_t* rects_dev, const uint32_t* depths_dev, uint32_t num_items,
                           uint32_t tiles_x, void* stream);
/* which: 0 sorted_entries (u32), 1 entry_items (u32), 2 ranges (uint2), 3 entry count (u64) */
gs_status gs_binner_buffer(gs_binner* b, uint32_t which, void** dptr, size_t* bytes);

/* ---- RadixSorter / PrefixSum (crates/gs-wgpu/src/{sort,prefix_sum}.rs) ----
 * Stable LSD sort of n (key, value) u32 pairs on bits [0, key_bits), in
 * place; and an exclusive u32 scan with the total written to *total_dev.
 * Both take caller device pointers and allocate their scratch on first use
 * per size class (held until gs_shutdown). */
gs_status gs_radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint64_t n, uint32_t key_bits, void* stream);
gs_status gs_exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* total_dev, void* stream);

/* No counterpart in the reference. The same stable LSD sort as
 * gs_radix_sort_pairs for callers that cannot let the library allocate device
 * memory (a host that owns all device memory through its own pool, a loop
 * that must not pay an allocation's latency or implicit synchronisation, a
 * binding that forbids hidden allocations): it calls no allocator. Its
 * scratch is a fixed array in the library's device image sized for at most
 * 1,048,576 pairs (about 8.6 MB, held by every GPU that loads the library
 * until exit); larger n returns GS_ERR_CAPACITY. The first call on a device
 * looks up that array's device address and keeps it for the process, so make
 * it before any stream capture, and do not call this entry point after
 * resetting the device (cudaDeviceReset), which invalidates that address.
 * Calls share the array: calls that overlap on the GPU (different streams,
 * or different host threads) race and corrupt each other's results.
 * Stream-ordered, does not synchronise. */
gs_status gs_radix_sort_pairs_noalloc(uint32_t* keys, uint32_t* vals, uint64_t n, uint32_t key_bits, void* stream);

/* ---- Surfel PLY files (first_attempt/crates/gs-io/src/ply) ---------------
 * The 3DGS binary little-endian layout: x y z | f_dc_0..2 | f_rest_0..44
 * (channel-major) | opacity (logit) | scale_0..2 (log) | rot_0..3 (w first).
 * gs_ply_write is write_3dgs_ply (ply/writer.rs): activated inputs
 * (positions 4 floats per surfel, scales 2, quats xyzw, opacities, SH 48
 * coefficient-major); the third log-scale is written as -10 (flattened).
 * gs_ply_info / gs_ply_read are load_ply for splat files (ply/reader.rs):
 * properties located by name, f_rest counts 0/9/24/45, activated outputs
 * (positions 3, scales 3 = exp, quats xyzw normalised or identity when
 * degenerate, opacities = sigmoid, SH sh_coeffs*3 coefficient-major).
 * Errors: GS_ERR_IO (open/read/write), GS_ERR_FORMAT (not a ply, not
 * binary_little_endian 1.0, unknown layout, non-float property, wrong f_rest
 * count, payload shorter than the header's count, more surfels than
 * capacity); the text is in gs_last_error(NULL). Host-only. */
gs_status gs_ply_write(const char* path, uint32_t count, const float* positions4, const float* scales2,
                       const float* quats4, const float* opacities, const float* sh48);
gs_status gs_ply_info(const char* path, uint32_t* count, uint32_t* sh_coeffs);
gs_status gs_ply_read(const char* path, uint32_t capacity, float* positions3, float* scales3, float* quats4,
                      float* opacities, float* sh, uint32_t* count);
/* The handle's activated surfels [0, num_surfels) to a PLY file (blocking). */
gs_status gs_rasterizer_save_ply(gs_rasterizer* r, const char* path, uint32_t num_surfels, void* stream);
/* A splat PLY file into the handle (gs_rasterizer_upload_scene of its
 * activated values; the third scale is dropped). *num_surfels = its count. */
gs_status gs_rasterizer_load_ply(gs_rasterizer* r, const char* path, uint32_t* num_surfels, void* stream);

/* Camera-to-world rotation (column-major 3x3) exactly as the forward computes
 * it from gs_camera.quat (glam Mat3::from_quat of the normalised quaternion,
 * rasterizer.rs:410). Host-only, no GPU needed. */
gs_status gs_camera_rotation(const gs_camera* cam, float rot9[9]);

/* Library version string and build flags; host-only. */
const char* gs_version(void);
/* Frees the library's global scratch (sort/scan) on the current device. */
gs_status gs_shutdown(void);

#ifdef __cplusplus
}
#endif
#endif /* GS_CUDA_H */
