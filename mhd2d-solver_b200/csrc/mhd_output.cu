// Device packing of the reference's binary grid dump: the records of
// outputGridDataBinary (file_access.cpp:1193-1325) for the natural data of
// toNaturalData (conversions.cpp:37-57), with the div B ranges and B ghost
// substitutions of outputGridData (file_access.cpp:1530-1677).  Compiled
// without FMA contraction, so every value rounds as the reference computes
// it; the host only writes the block to its file.
#include "mhd_output.h"

#include <algorithm>

namespace mhd {
namespace output {
namespace {

struct PackArgs {
  int natural, conservation;
  double start_x, start_y;
  int x0, x1, y0, y1;  // cells whose div B is computed: [x0, x1) x [y0, y1)
  int per_l, per_r, per_b, per_t;  // periodic sides: their B ghosts are periodic copies
};

// One record per interior cell, cells in i-major order, values in the
// writer's order.
template <typename T>
__global__ void __launch_bounds__(256) k_grid_pack(Grid g, const double* __restrict__ U,
                                                   PackArgs a, T* __restrict__ out) {
  const long long n = (long long)g.nx * g.ny;
  const int nf = 7 + (a.natural ? 4 : 0) + (a.conservation ? 4 : 0);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int ii = int(e / g.ny), jj = int(e % g.ny);
    const int i = 2 + ii, j = 2 + jj;
    const double r = U[g.at(0, i, j)], mx = U[g.at(1, i, j)], my = U[g.at(2, i, j)];
    const double mz = U[g.at(3, i, j)], bx = U[g.at(4, i, j)], by = U[g.at(5, i, j)];
    const double bz = U[g.at(6, i, j)], en = U[g.at(7, i, j)];
    double divb = 0.0;
    if (i >= a.x0 && i < a.x1 && j >= a.y0 && j < a.y1) {
      // a periodic side's ghost layer holds the copy outputGridData writes
      const double bxm = (i == 2 && a.per_l) ? U[g.at(4, g.nx + 1, j)] : U[g.at(4, i - 1, j)];
      const double bxp = (i == g.nx + 1 && a.per_r) ? U[g.at(4, 2, j)] : U[g.at(4, i + 1, j)];
      const double bym = (j == 2 && a.per_b) ? U[g.at(5, i, g.ny + 1)] : U[g.at(5, i, j - 1)];
      const double byp = (j == g.ny + 1 && a.per_t) ? U[g.at(5, i, 2)] : U[g.at(5, i, j + 1)];
      divb = fabs((bxp - bxm) / (2.0 * g.dx) + (byp - bym) / (2.0 * g.dy));
    }
    T* o = out + e * nf;
    int f = 0;
    o[f++] = T(a.start_x + ii * g.dx);
    o[f++] = T(a.start_y + jj * g.dy);
    o[f++] = T(r);
    if (a.natural) {
      const double mm = mx * mx + my * my + mz * mz;
      const double bb = bx * bx + by * by + bz * bz;
      o[f++] = T(mx / r);
      o[f++] = T(my / r);
      o[f++] = T(mz / r);
      o[f++] = T((g.gamma - 1.0) * (en - 0.5 * mm / r - 0.5 * bb));
    }
    o[f++] = T(bx);
    o[f++] = T(by);
    o[f++] = T(bz);
    o[f++] = T(divb);
    if (a.conservation) {
      o[f++] = T(mx);
      o[f++] = T(my);
      o[f++] = T(mz);
      o[f++] = T(en);
    }
  }
}

}  // namespace

void launch_grid_pack(const Grid& g, const double* U, bool natural, bool conservation,
                      bool single, double start_x, double start_y, void* out,
                      cudaStream_t st) {
  PackArgs a{};
  a.natural = natural ? 1 : 0;
  a.conservation = conservation ? 1 : 0;
  a.start_x = start_x;
  a.start_y = start_y;
  // Neumann and open sides leave their edge cells out of div B
  const auto edge_out = [](int b) { return b == NEUMANN || b == OPEN; };
  a.x0 = edge_out(g.bc[LEFT]) ? 3 : 2;
  a.x1 = edge_out(g.bc[RIGHT]) ? g.nx + 1 : g.nx + 2;
  a.y0 = edge_out(g.bc[BOTTOM]) ? 3 : 2;
  a.y1 = edge_out(g.bc[TOP]) ? g.ny + 1 : g.ny + 2;
  a.per_l = g.bc[LEFT] == PERIODIC;
  a.per_r = g.bc[RIGHT] == PERIODIC;
  a.per_b = g.bc[BOTTOM] == PERIODIC;
  a.per_t = g.bc[TOP] == PERIODIC;
  const long long n = (long long)g.nx * g.ny;
  const int blocks = int(std::min<long long>((n + 255) / 256, 148LL * 8));
  if (single)
    k_grid_pack<float><<<blocks, 256, 0, st>>>(g, U, a, static_cast<float*>(out));
  else
    k_grid_pack<double><<<blocks, 256, 0, st>>>(g, U, a, static_cast<double*>(out));
}

}  // namespace output
}  // namespace mhd
