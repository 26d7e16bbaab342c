// Second-order central finite differences: SpatialMethodCentralFD2::integrate
// (spatialmethodcentralfd2.cpp:44-160).
//
// The reference forms the physical fluxes F, G on the interior and on the
// ring of ghost cells around it, takes the maxima of the signed wave speeds
// for dtIdeal, and then UL = -(F_{i+1} - F_{i-1}) / (2 dx) - (G_{j+1} -
// G_{j-1}) / (2 dy).  Here that is two HBM-bound passes over the state and
// no flux arrays:
//   k_cfd_check  a grid-stride loop over the ring domain: the density /
//                pressure checks and the wave-speed maxima (warp shuffles,
//                one atomic per block);
//   k_cfd_ul     8 x 32 interior cells per block: the fluxes of the block's
//                cells and its one-cell rim once, into shared memory, then
//                UL.  It stands down when a density was non-positive: the
//                reference returns before forming UL.
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

// Checks and wave-speed maxima over the ring domain [1, nx+3) x [1, ny+3),
// a grid-stride loop over its cells (j fastest).  ctl->cfd_first keeps
// kCfdFirstBase - (i*NY + j) of the first non-positive density (max =
// smallest index), ctl->cfd_last 1 + (i*NY + j) of the last non-positive
// pressure; 0 means none.  One pair of maxima atomics per block.
__global__ void __launch_bounds__(256) k_cfd_check(Grid g, const double* __restrict__ U, Ctl* ctl) {
  if (ctl->skip) return;
  const int W = g.ny + 2;
  const long long n = (long long)(g.nx + 2) * W;
  double cx = 0.0, cy = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = 1 + int(e / W), j = 1 + int(e % W);
    if (cfd_skip(g, i, j)) continue;
    const double gm = g.gamma;
    const double r = U[g.at(0, i, j)];
    const double mx = U[g.at(1, i, j)], u = mx / r;
    const double my = U[g.at(2, i, j)], v = my / r;
    const double mz = U[g.at(3, i, j)], w = mz / r;
    const double bx = U[g.at(4, i, j)], by = U[g.at(5, i, j)], bz = U[g.at(6, i, j)];
    const double en = U[g.at(7, i, j)];
    const double uu = u * u + v * v + w * w;
    const double bb = bx * bx + by * by + bz * bz;
    const double p = (gm - 1.0) * (en - 0.5 * r * uu - 0.5 * bb);
    const unsigned long long lin = (unsigned long long)i * g.NY + j;
    if (r <= 0.0) {
      atomicMax(&ctl->cfd_first, kCfdFirstBase - lin);
      continue;
    }
    if (p <= 0.0) atomicMax(&ctl->cfd_last, lin + 1);
    double c2 = gm * p / r;
    if (c2 < 0.0) c2 = 0.0;
    cx = cfd_dir_max(cx, r, bx, u, bb, c2);
    cy = cfd_dir_max(cy, r, by, v, bb, c2);
  }
  __shared__ double red[2][8];
  cx = warp_max(cx);
  cy = warp_max(cy);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { red[0][wid] = cx; red[1][wid] = cy; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < int(blockDim.x >> 5); q++) {
      cx = take_max(cx, red[0][q]);
      cy = take_max(cy, red[1][q]);
    }
    atomic_max_pos(&ctl->maxX, cx);
    atomic_max_pos(&ctl->maxY, cy);
  }
}

// UL of a 8 (i) x 32 (j) block of interior cells; cxf = 1/(2 dx),
// cyf = 1/(2 dy) as the host forms them.  The block first evaluates the
// physical fluxes of its cells once, into shared memory: F on rows i0-1 ..
// i0+8, G on columns j0-1 .. j0+32 (336 cells, the same expressions as
// spatialmethodcentralfd2.cpp:80-98; 0 for a skipped ring cell or a cell
// past the ring), then forms UL from them.
constexpr int CFD_TI = 8, CFD_TJ = 32;

__global__ void __launch_bounds__(256) k_cfd_ul(Grid g, const double* __restrict__ U,
                                                double* __restrict__ UL, double cxf, double cyf,
                                                const Ctl* ctl) {
  if (ctl->skip || ctl->cfd_first) return;
  __shared__ double sF[7][CFD_TI + 2][CFD_TJ];  // x fluxes, component 4 (= 0) not stored
  __shared__ double sG[7][CFD_TI][CFD_TJ + 2];  // y fluxes, component 5 (= 0) not stored
  const int i0 = 2 + blockIdx.y * CFD_TI, j0 = 2 + blockIdx.x * CFD_TJ;
  constexpr int NIN = CFD_TI * CFD_TJ, NROW = 2 * CFD_TJ, NCOL = 2 * CFD_TI;
  for (int e = threadIdx.x; e < NIN + NROW + NCOL; e += blockDim.x) {
    int r, c;  // tile coordinates: cell (i0 + r, j0 + c)
    if (e < NIN) { r = e / CFD_TJ; c = e % CFD_TJ; }
    else if (e < NIN + NROW) { const int q = e - NIN; r = q < CFD_TJ ? -1 : CFD_TI; c = q % CFD_TJ; }
    else { const int q = e - NIN - NROW; r = q % CFD_TI; c = q < CFD_TI ? -1 : CFD_TJ; }
    const int i = i0 + r, j = j0 + c;
    double F[NF], G[NF];
    if (i <= g.nx + 2 && j <= g.ny + 2 && !cfd_skip(g, i, j)) {
      double q[NF];
#pragma unroll
      for (int k = 0; k < NF; k++) q[k] = U[g.at(k, i, j)];
      phys_flux(g.gamma, q, F, G);
    } else {
#pragma unroll
      for (int k = 0; k < NF; k++) { F[k] = 0.0; G[k] = 0.0; }
    }
    if (c >= 0 && c < CFD_TJ) {
#pragma unroll
      for (int m = 0; m < NF; m++)
        if (m != 4) sF[slot_of(m)][r + 1][c] = F[m];
    }
    if (r >= 0 && r < CFD_TI) {
#pragma unroll
      for (int m = 0; m < NF; m++)
        if (m != 5) sG[m < 5 ? m : m - 1][r][c + 1] = G[m];
    }
  }
  __syncthreads();
  const int r = threadIdx.x / CFD_TJ, c = threadIdx.x % CFD_TJ;
  const int i = i0 + r, j = j0 + c;
  if (i >= g.nx + 2 || j >= g.ny + 2) return;
#pragma unroll
  for (int k = 0; k < NF; k++) {
    const double fp = k == 4 ? 0.0 : sF[slot_of(k)][r + 2][c];
    const double fm = k == 4 ? 0.0 : sF[slot_of(k)][r][c];
    const double gp = k == 5 ? 0.0 : sG[k < 5 ? k : k - 1][r][c + 2];
    const double gq = k == 5 ? 0.0 : sG[k < 5 ? k : k - 1][r][c];
    UL[g.at(k, i, j)] = -(cxf) * (fp - fm) - (cyf) * (gp - gq);
  }
}

}  // namespace MHD_KNS
}  // namespace mhd
