// Second-order central finite differences: SpatialMethodCentralFD2::integrate
// (spatialmethodcentralfd2.cpp:44-160).
//
// The reference forms the physical fluxes F, G on the interior and on the
// ring of ghost cells around it, takes the maxima of the signed wave speeds
// for dtIdeal, and then UL = -(F_{i+1} - F_{i-1}) / (2 dx) - (G_{j+1} -
// G_{j-1}) / (2 dy).  Here that is two HBM-bound passes over the state and
// no flux arrays:
//   k_cfd_check  one thread per ring cell: the density / pressure checks and
//                the wave-speed maxima (warp shuffles, one atomic per warp);
//   k_cfd_ul     one thread per interior cell: the fluxes of its four
//                neighbours, recomputed from U, and UL.  It stands down when
//                a density was non-positive: the reference returns before
//                forming UL.
// Reference behaviour kept:
//   * the four ring corners are skipped with nxFirst / nxLast for BOTH
//     indices (lines 60-64), so with ny < nx the ring cells (1, ny+2) and
//     (nx+2, ny+2) are evaluated (their ghost values take part in the checks
//     and maxima), and with ny > nx the ring cells (1, j), (nx+2, j),
//     j >= nx+2, are skipped.  The reference then reads its never-written
//     flux arrays there (uninitialised memory); these kernels use 0, what a
//     freshly mapped allocation holds;
//   * max over u - cf ... u + cf of the SIGNED speeds, starting from 0, a NaN
//     never entering (std::max over an initialiser list);
//   * a non-positive density is fatal and reported at the first such cell in
//     loop order (i outer, j inner); a non-positive pressure is fatal too,
//     reported at the last such cell, after UL and dtIdeal are formed.
// Both kernels keep every expression in the reference's order (parity build:
// bit-identical).
#pragma once

#include "mhd_flux.cuh"

#ifndef MHD_KNS
#define MHD_KNS exact
#endif

namespace mhd {
namespace MHD_KNS {

// The reference's corner test: nxFirst = 2 and nxLast = nx + 2 for i and j.
__device__ __forceinline__ bool cfd_skip(const Grid& g, int i, int j) {
  const int f = 2, l = g.nx + 2;
  return (i < f && j < f) || (i < f && j >= l) || (i >= l && j < f) || (i >= l && j >= l);
}

// std::max({m, u - cf, u - ca, u - cs, u, u + cs, u + ca, u + cf}): the
// first largest, so a NaN candidate never replaces the running value.
__device__ __forceinline__ double cfd_max_speeds(double m, double u, double cf, double ca,
                                                 double cs) {
  const double v[7] = {u - cf, u - ca, u - cs, u, u + cs, u + ca, u + cf};
#pragma unroll
  for (int n = 0; n < 7; n++)
    if (m < v[n]) m = v[n];
  return m;
}

// Signed wave-speed maximum of one direction with normal field bn and
// normal velocity un (spatialmethodcentralfd2.cpp:118-137).
__device__ __forceinline__ double cfd_dir_max(double m, double r, double bn, double un, double bb,
                                              double c2) {
  const double ca2 = bn * bn / r;
  const double ca = sqrt(ca2);
  const double ct2 = 0.5 * (bb / r + c2);
  double ctemp = ct2 * ct2 - c2 * ca2;
  if (ctemp < 0.0) ctemp = 0.0;
  double cs2 = ct2 - sqrt(ctemp);
  if (cs2 < 0.0) cs2 = 0.0;
  const double cs = sqrt(cs2);
  double cf2 = ct2 + sqrt(ctemp);
  if (cf2 < 0.0) cf2 = 0.0;
  const double cf = sqrt(cf2);
  return cfd_max_speeds(m, un, cf, ca, cs);
}

// Checks and wave-speed maxima over the ring domain [1, nx+3) x [1, ny+3).
// Block: 32 (j) x 8 (i) cells.  ctl->cfd_first keeps kCfdFirstBase - (i*NY + j)
// of the first non-positive density (max = smallest index), ctl->cfd_last
// 1 + (i*NY + j) of the last non-positive pressure; 0 means none.
__global__ void __launch_bounds__(256) k_cfd_check(Grid g, const double* __restrict__ U, Ctl* ctl) {
  if (ctl->skip) return;
  const int j = 1 + blockIdx.x * 32 + (threadIdx.x & 31), i = 1 + blockIdx.y * 8 + (threadIdx.x >> 5);
  double cx = 0.0, cy = 0.0;
  if (i < g.nx + 3 && j < g.ny + 3 && !cfd_skip(g, i, j)) {
    const double gm = g.gamma;
    const double r = U[g.at(0, i, j)];
    const double mx = U[g.at(1, i, j)], u = mx / r;
    const double my = U[g.at(2, i, j)], v = my / r;
    const double mz = U[g.at(3, i, j)], w = mz / r;
    const double bx = U[g.at(4, i, j)], by = U[g.at(5, i, j)], bz = U[g.at(6, i, j)];
    const double e = U[g.at(7, i, j)];
    const double uu = u * u + v * v + w * w;
    const double bb = bx * bx + by * by + bz * bz;
    const double p = (gm - 1.0) * (e - 0.5 * r * uu - 0.5 * bb);
    const unsigned long long lin = (unsigned long long)i * g.NY + j;
    if (r <= 0.0) {
      atomicMax(&ctl->cfd_first, kCfdFirstBase - lin);
    } else {
      if (p <= 0.0) atomicMax(&ctl->cfd_last, lin + 1);
      double c2 = gm * p / r;
      if (c2 < 0.0) c2 = 0.0;
      cx = cfd_dir_max(0.0, r, bx, u, bb, c2);
      cy = cfd_dir_max(0.0, r, by, v, bb, c2);
    }
  }
  cx = warp_max(cx);
  cy = warp_max(cy);
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(&ctl->maxX, cx);
    atomic_max_pos(&ctl->maxY, cy);
  }
}

// x (X = true) or y physical flux of cell (i, j), 0 for a skipped ring cell
// (the same expressions as spatialmethodcentralfd2.cpp:80-98).
template <bool X>
__device__ __forceinline__ void cfd_flux(const Grid& g, const double* __restrict__ U, int i, int j,
                                         double* out) {
  if (cfd_skip(g, i, j)) {
#pragma unroll
    for (int k = 0; k < NF; k++) out[k] = 0.0;
    return;
  }
  double q[NF], F[NF], G[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) q[k] = U[g.at(k, i, j)];
  phys_flux(g.gamma, q, F, G);
  F[4] = 0.0;
  G[5] = 0.0;
#pragma unroll
  for (int k = 0; k < NF; k++) out[k] = X ? F[k] : G[k];
}

// UL of the interior cells; cxf = 1/(2 dx), cyf = 1/(2 dy) as the host forms
// them.  Block: 32 (j) x 8 (i) cells.
__global__ void __launch_bounds__(256) k_cfd_ul(Grid g, const double* __restrict__ U,
                                                double* __restrict__ UL, double cxf, double cyf,
                                                const Ctl* ctl) {
  if (ctl->skip || ctl->cfd_first) return;
  const int j = 2 + blockIdx.x * 32 + (threadIdx.x & 31), i = 2 + blockIdx.y * 8 + (threadIdx.x >> 5);
  if (i >= g.nx + 2 || j >= g.ny + 2) return;
  double fp[NF], fm[NF], gp[NF], gq[NF];
  cfd_flux<true>(g, U, i + 1, j, fp);
  cfd_flux<true>(g, U, i - 1, j, fm);
  cfd_flux<false>(g, U, i, j + 1, gp);
  cfd_flux<false>(g, U, i, j - 1, gq);
#pragma unroll
  for (int k = 0; k < NF; k++)
    UL[g.at(k, i, j)] = -(cxf) * (fp[k] - fm[k]) - (cyf) * (gp[k] - gq[k]);
}

}  // namespace MHD_KNS
}  // namespace mhd
