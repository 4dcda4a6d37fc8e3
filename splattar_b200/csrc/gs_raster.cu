// Raster kernels for 16-pixel tiles (the reference's tile size) and the
// launchers that dispatch on the tile size; the kernels themselves are in
// gs_raster.cuh, and gs_raster_t8.cu / gs_raster_t32.cu instantiate them for
// 8- and 32-pixel tiles.
#include "gs_raster.cuh"

namespace gs {

GS_RASTER_INSTANTIATE(16)

extern template int raster_fwd_occupancy_t<8>(int, int, int, bool, bool, bool);
extern template int raster_fwd_occupancy_t<32>(int, int, int, bool, bool, bool);
extern template int raster_bwd_occupancy_t<8>(int, bool, int, int, bool, bool);
extern template int raster_bwd_occupancy_t<32>(int, bool, int, int, bool, bool);
extern template int launch_raster_fwd_t<8>(const RasterArgs&, int, int, int, bool, bool, bool, int, cudaStream_t);
extern template int launch_raster_fwd_t<32>(const RasterArgs&, int, int, int, bool, bool, bool, int, cudaStream_t);
extern template int launch_raster_bwd_t<8>(const RasterArgs&, int, bool, int, int, bool, bool, int, cudaStream_t);
extern template int launch_raster_bwd_t<32>(const RasterArgs&, int, bool, int, int, bool, bool, int, cudaStream_t);

namespace {
const RasterShape FWD8[] = {{64, 1}, {128, 1}, {256, 1}, {64, 2}, {128, 2}, {256, 2}};
// (32, 0): the pixel-compacted kernels (colour-only persistent passes)
const RasterShape FWD16[] = {{64, 1}, {128, 1}, {256, 1}, {64, 2}, {128, 2}, {64, 4}, {64, 8}, {128, 8}, {32, 0}};
const RasterShape FWD32[] = {{64, 2}, {128, 2}, {256, 2}, {64, 4}, {128, 4}, {256, 4}, {128, 8}};
const RasterShape BWD8[] = {{64, 1}, {64, 2}, {128, 2}};
const RasterShape BWD16[] = {{64, 1}, {64, 2}, {128, 2}, {64, 4}, {32, 8}, {64, 8}, {128, 8}, {32, 0}};
const RasterShape BWD32[] = {{64, 4}, {64, 8}};
}  // namespace

int raster_fwd_shapes(int tile, const RasterShape** out) {
  switch (tile) {
    case 8: *out = FWD8; return 6;
    case 16: *out = FWD16; return 9;
    case 32: *out = FWD32; return 7;
    default: *out = nullptr; return 0;
  }
}

int raster_bwd_shapes(int tile, const RasterShape** out) {
  switch (tile) {
    case 8: *out = BWD8; return 3;
    case 16: *out = BWD16; return 8;
    case 32: *out = BWD32; return 2;
    default: *out = nullptr; return 0;
  }
}

int raster_fwd_occupancy(int tile, int prec, int batch, int ppt, bool det, bool color, bool mask) {
  if (tile == 8) return raster_fwd_occupancy_t<8>(prec, batch, ppt, det, color, mask);
  if (tile == 32) return raster_fwd_occupancy_t<32>(prec, batch, ppt, det, color, mask);
  return raster_fwd_occupancy_t<16>(prec, batch, ppt, det, color, mask);
}

int raster_bwd_occupancy(int tile, int prec, bool aux, int ppt, int batch, bool det, bool mask) {
  if (tile == 8) return raster_bwd_occupancy_t<8>(prec, aux, ppt, batch, det, mask);
  if (tile == 32) return raster_bwd_occupancy_t<32>(prec, aux, ppt, batch, det, mask);
  return raster_bwd_occupancy_t<16>(prec, aux, ppt, batch, det, mask);
}

int launch_raster_fwd(const RasterArgs& a, int tile, int prec, int batch, int ppt, bool det, bool persistent,
                      bool color, int grid, cudaStream_t st) {
  if (tile == 8) return launch_raster_fwd_t<8>(a, prec, batch, ppt, det, persistent, color, grid, st);
  if (tile == 16) return launch_raster_fwd_t<16>(a, prec, batch, ppt, det, persistent, color, grid, st);
  if (tile == 32) return launch_raster_fwd_t<32>(a, prec, batch, ppt, det, persistent, color, grid, st);
  return (int)cudaErrorInvalidValue;
}

int launch_raster_work(const RasterArgs& a, int tile, int prec, unsigned long long* out4, cudaStream_t st) {
  if (a.total_tiles == 0) return 0;
  auto go = [&](auto kernel, int threads) { kernel<<<a.total_tiles, threads, 0, st>>>(a, out4); };
  if (tile == 8) {
    if (prec == 0) go(k_raster_work<8, 0>, 64); else if (prec == 1) go(k_raster_work<8, 1>, 64); else go(k_raster_work<8, 2>, 64);
  } else if (tile == 16) {
    if (prec == 0) go(k_raster_work<16, 0>, 256); else if (prec == 1) go(k_raster_work<16, 1>, 256); else go(k_raster_work<16, 2>, 256);
  } else if (tile == 32) {
    if (prec == 0) go(k_raster_work<32, 0>, 256); else if (prec == 1) go(k_raster_work<32, 1>, 256); else go(k_raster_work<32, 2>, 256);
  } else {
    return (int)cudaErrorInvalidValue;
  }
  return (int)cudaGetLastError();
}

int launch_raster_bwd(const RasterArgs& a, int tile, int prec, bool aux, int ppt, int batch, bool det,
                      bool persistent, int grid, cudaStream_t st) {
  if (tile == 8) return launch_raster_bwd_t<8>(a, prec, aux, ppt, batch, det, persistent, grid, st);
  if (tile == 16) return launch_raster_bwd_t<16>(a, prec, aux, ppt, batch, det, persistent, grid, st);
  if (tile == 32) return launch_raster_bwd_t<32>(a, prec, aux, ppt, batch, det, persistent, grid, st);
  return (int)cudaErrorInvalidValue;
}

}  // namespace gs
