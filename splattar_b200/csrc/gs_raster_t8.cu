// Raster kernels (gs_raster.cuh) instantiated for 8-pixel tiles.
#include "gs_raster.cuh"

namespace gs {
GS_RASTER_INSTANTIATE(8)
}  // namespace gs
