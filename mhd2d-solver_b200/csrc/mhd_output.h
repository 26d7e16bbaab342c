// Device packing of the reference's binary grid dump (mhd_grid_pack).
#pragma once
#include <cuda_runtime.h>

#include "mhd_common.cuh"

namespace mhd {
namespace output {

// Values per cell record: x, y, rho, [u, v, w, p], Bx, By, Bz, div B,
// [mx, my, mz, e].
inline int grid_fields(bool natural, bool conservation) {
  return 7 + (natural ? 4 : 0) + (conservation ? 4 : 0);
}

// Writes the nx * ny records of state U (device, Grid layout) to out
// (device): doubles, or floats when single.
void launch_grid_pack(const Grid& g, const double* U, bool natural, bool conservation,
                      bool single, double start_x, double start_y, void* out,
                      cudaStream_t st);

}  // namespace output
}  // namespace mhd
