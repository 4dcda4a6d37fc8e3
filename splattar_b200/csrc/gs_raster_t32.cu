// Raster kernels (gs_raster.cuh) instantiated for 32-pixel tiles.
#include "gs_raster.cuh"

namespace gs {
GS_RASTER_INSTANTIATE(32)
}  // namespace gs
