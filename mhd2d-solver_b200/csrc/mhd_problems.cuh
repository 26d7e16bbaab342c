// Device-side initial states (problem setups of file_access.cpp) for the
// batched runs and the adjoint.  Kinds and parameter lists are those of
// mhd_batch_init_problem in include/mhd2d_b200.h.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/mhd2d_b200.h"
#include "mhd_eigen.cuh"

namespace mhd {
namespace MHD_KNS {

// Device-side initial states (interior cells; ghosts are filled by the
// first boundary pass).  Conversions follow conversions.cpp:20-35.
__device__ __forceinline__ void to_conserved(double gm, double rho, double u, double v, double w,
                                             double bx, double by, double bz, double p,
                                             double* q) {
  q[0] = rho;
  q[1] = u * rho;
  q[2] = v * rho;
  q[3] = w * rho;
  q[4] = bx;
  q[5] = by;
  q[6] = bz;
  const double uu = u * u + v * v + w * w;
  const double bb = bx * bx + by * by + bz * bz;
  q[7] = p / (gm - 1.0) + 0.5 * rho * uu + 0.5 * bb;
}

struct ProblemArgs {
  int kind;
  int K;
  double p[48];
  double ev[NF];  // wave: the chosen right eigenvector
  double avg[NF]; // wave: conserved background state
  // lobe plasma sheet: rows [lim_dn, lim_up) hold the sheet, tp transition
  // points; aux (device, freed by release_problem): sheet start column per
  // row [NY], tanh profile factor per row [NY], transition weights [tp]
  int lim_dn, lim_up, tp;
  double* aux;
};

constexpr int kShockTubeParams = 19;  // Lx, Ly, angle, left[8], right[8]
constexpr int kSheetLobesParams = 42; // Lx, Ly, x0, y0, head, foot, thickness, profile,
                                      // transition, points, left, right, up, down [8 each]

__global__ void kb_problem(Grid g, double* __restrict__ U, ProblemArgs a) {
  const long long n = (long long)g.nx * g.ny;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int ii = int(e / g.ny), jj = int(e - (long long)ii * g.ny);
    const int i = ii + 2, j = jj + 2;
    double q[NF];
    const double gm = g.gamma;
    if (a.kind == MHD_PROBLEM_EXPLOSION) {
      // readProblemExplosion (file_access.cpp:398-470): centre at index (NX/2, NY/2)
      const double di = double(i - g.NX / 2), dj = double(j - g.NY / 2);
      const double r = a.p[2];
      const bool inside = di * di * g.dx * g.dx + dj * dj * g.dy * g.dy < r * r;
      const double rho = inside ? a.p[3] : a.p[5];
      const double p = inside ? a.p[4] : a.p[6];
      to_conserved(gm, rho, 0.0, 0.0, 0.0, a.p[7], a.p[8], 0.0, p, q);
    } else if (a.kind == MHD_PROBLEM_WAVE) {
      // readProblemWaveTest (file_access.cpp:922-1045)
      const double x = a.p[0] + ii * g.dx, y = a.p[1] + jj * g.dy;
      const double kx = a.p[14], ky = a.p[15];
      const double sx = 2.0 * M_PI / a.p[2], sy = 2.0 * M_PI / a.p[3];
      const double cphase = cos(sx * kx * x + sy * ky * y);
      double c[NF];
#pragma unroll
      for (int k = 0; k < NF; k++) c[k] = a.avg[k] + a.p[12] * a.ev[k] * cphase;
      // natural variables, rotation by atan2(ky, kx), back to conserved
      const double u = c[1] / c[0], v = c[2] / c[0], w = c[3] / c[0];
      const double mm = c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
      const double bb = c[4] * c[4] + c[5] * c[5] + c[6] * c[6];
      const double p = (gm - 1.0) * (c[7] - 0.5 * mm / c[0] - 0.5 * bb);
      const double ang = atan2(ky, kx), ct = cos(ang), st = sin(ang);
      const double ru = ct * u - st * v, rv = st * u + ct * v;
      const double rbx = ct * c[4] - st * c[5], rby = st * c[4] + ct * c[5];
      to_conserved(gm, c[0], ru, rv, w, rbx, rby, c[6], p, q);
    } else if (a.kind == MHD_PROBLEM_ORSZAG_TANG) {
      // readProblemOTVortex (file_access.cpp:578-613)
      const double x = ii * g.dx, y = jj * g.dy;
      to_conserved(gm, gm * gm, -sin(y), sin(x), 0.0, -sin(y), sin(2 * x), 0.0, gm, q);
    } else if (a.kind == MHD_PROBLEM_SHOCK_TUBE) {
      // readProblemShockTube (file_access.cpp:300-395): the interface line
      // through the domain centre at the given angle; cells below the row
      // "jump" of their column get the left state.  p[19] = x0, p[20] = y0,
      // p[21] = slope, computed on the host as the reference computes them.
      const double line_y = a.p[20] - a.p[21] * (double(i - 2) * g.dx - a.p[19]);
      const double line_j = 2 + (line_y / g.dy + 0.5);
      const double last = double(g.ny + 2);
      const int jump = int(line_j < 2 ? 2.0 : (line_j > last ? last : line_j));
      const double* s = j < jump ? a.p + 3 : a.p + 11;
      to_conserved(gm, s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7], q);
    } else {
      // plasma sheet: By = tanh(x/delta), T = 0.5, p = 1.25 - By^2/2, rho = p/T,
      // v = sum_k a_k sin(k pi y) exp(-x^2/0.04)
      const double x = a.p[0] + ii * g.dx, y = a.p[1] + jj * g.dy;
      const double by = tanh(x / a.p[2]);
      const double p = 1.25 - 0.5 * by * by;
      const double rho = p / 0.5;
      double v = 0.0;
      const double env = exp(-x * x / 0.04);
      for (int k = 1; k <= a.K; k++) v += a.p[3 + k] * sin(k * M_PI * y) * env;
      to_conserved(gm, rho, 0.0, v, 0.0, 0.0, by, 0.0, p, q);
    }
#pragma unroll
    for (int k = 0; k < NF; k++) U[g.at(k, i, j)] = q[k];
  }
}

// The reference's plasma sheet (readProblemPlasmaSheet, file_access.cpp:
// 614-919), in four passes over natural variables kept in the state block
// (rho, u, v, w, Bx, By, Bz, p in planes 0..7) and converted at the end:
// the lobes and the two sheet halves, the transitions across the
// sheet-lobe rows (per column i, in the reference's order), the transitions
// across the sheet's start (per row j), then toConservationData.
__device__ __forceinline__ double& nat(const Grid& g, double* U, int k, int i, int j) {
  return U[g.at(k, i, j)];
}

__global__ void kb_sheet_base(Grid g, double* __restrict__ U, ProblemArgs a) {
  const long long n = (long long)g.nx * g.ny;
  const double* left = a.p + 10;
  const double* right = a.p + 18;
  const double* up = a.p + 26;
  const double* down = a.p + 34;
  const bool tanh_profile = a.p[7] != 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = 2 + int(e / g.ny), j = 2 + int(e % g.ny);
    double v[NF];
    if (j < a.lim_dn || j >= a.lim_up) {
      const double* s = j < a.lim_dn ? down : up;
#pragma unroll
      for (int k = 0; k < NF; k++) v[k] = s[k];
    } else {
      const double* s = double(i) < a.aux[j] ? left : right;
#pragma unroll
      for (int k = 0; k < NF; k++) v[k] = s[k];
      if (tanh_profile) {
        const double cb = a.aux[g.NY + j];
        const double bb = s[4] * s[4] + s[5] * s[5] + s[6] * s[6];
        v[4] = s[4] * cb;
        v[5] = s[5] * cb;
        v[6] = s[6] * cb;
        v[7] = s[7] + 0.5 * bb * (1.0 - cb * cb);  // total pressure kept constant
      }
    }
#pragma unroll
    for (int k = 0; k < NF; k++) nat(g, U, k, i, j) = v[k];
  }
}

__device__ __forceinline__ double mag_p(const Grid& g, double* U, int i, int j) {
  const double bx = nat(g, U, 4, i, j), by = nat(g, U, 5, i, j), bz = nat(g, U, 6, i, j);
  return 0.5 * (bx * bx + by * by + bz * bz);
}

// coef * first + (1 - coef) * second, the reference's blend
__device__ __forceinline__ double blend(double c, double first, double second) {
  return c * first + (1.0 - c) * second;
}

// One blended point at (i, j) between (ia, ja) and (ib, jb), pressure fixed
// so that the total pressure is the blend of the two totals.
__device__ __forceinline__ void sheet_blend(const Grid& g, double* U, double c, int i, int j,
                                            int ia, int ja, int ib, int jb, double pta,
                                            double ptb) {
#pragma unroll
  for (int k = 0; k < NF; k++)
    nat(g, U, k, i, j) = blend(c, nat(g, U, k, ia, ja), nat(g, U, k, ib, jb));
  nat(g, U, 7, i, j) = blend(c, pta, ptb) - mag_p(g, U, i, j);
}

__global__ void kb_sheet_rows(Grid g, double* __restrict__ U, ProblemArgs a) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.nx + 2) return;
  const int tp = a.tp, half = tp / 2;
  const double* w = a.aux + 2 * g.NY;
  const int dn_btm = a.lim_dn - tp - 1, dn_top = a.lim_dn + tp;
  const int up_btm = a.lim_up - tp - 1, up_top = a.lim_up + tp;
  const double pdb = nat(g, U, 7, i, dn_btm) + mag_p(g, U, i, dn_btm);
  const double pdt = nat(g, U, 7, i, dn_top) + mag_p(g, U, i, dn_top);
  const double pub = nat(g, U, 7, i, up_btm) + mag_p(g, U, i, up_btm);
  const double put = nat(g, U, 7, i, up_top) + mag_p(g, U, i, up_top);
  for (int p = 0; p < tp; p++)
    sheet_blend(g, U, w[p], i, a.lim_dn - half + p, i, dn_btm, i, dn_top, pdb, pdt);
  for (int p = 0; p < tp; p++)
    sheet_blend(g, U, w[p], i, a.lim_up - half + p, i, up_btm, i, up_top, pub, put);
}

__global__ void kb_sheet_cols(Grid g, double* __restrict__ U, ProblemArgs a) {
  const int j = a.lim_dn + blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.lim_up) return;
  const int tp = a.tp, half = tp / 2;
  const double* w = a.aux + 2 * g.NY;
  const int s = int(a.aux[j]);
  const int il = s - half - 1, ir = s + half;
  for (int p = 0; p < tp; p++) {
    const double pl = nat(g, U, 7, il, j) + mag_p(g, U, il, j);
    const double pr = nat(g, U, 7, ir, j) + mag_p(g, U, ir, j);
    sheet_blend(g, U, w[p], s - half + p, j, il, j, ir, j, pl, pr);
  }
}

__global__ void kb_natural_to_conserved(Grid g, double* __restrict__ U) {
  const long long n = (long long)g.nx * g.ny;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = 2 + int(e / g.ny), j = 2 + int(e % g.ny);
    double v[NF], q[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) v[k] = nat(g, U, k, i, j);
    to_conserved(g.gamma, v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], q);
#pragma unroll
    for (int k = 0; k < NF; k++) nat(g, U, k, i, j) = q[k];
  }
}

// Right eigenvector `wave` at the state (avg, avg) (getEigens_F with
// break_on_neg_pressure = true, as readProblemWaveTest calls it).
__global__ void kb_wave_eigen(double gamma, const double* avg, int wave, double* out, int* err) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const Gas G{gamma, gamma - 1.0, (gamma - 2.0) / (gamma - 1.0), 1.0 / sqrt(2.0)};
  double U[NF];
  for (int k = 0; k < NF; k++) U[k] = avg[k];
  Mid e;
  if (!midpoint(G, U, U, e) || e.negp) { *err = 1; return; }
  double q[NF];
  for (int k = 0; k < NF; k++) q[k] = 0.0;
  rv_row(e, G, wave, q);
  for (int k = 0; k < NF; k++) out[k] = q[k];
  *err = 0;
}

// Host side: checks (kind, p, np) and fills a; a wave's right eigenvector is
// computed on the device (kb_wave_eigen, synchronised on `stream`).
// Returns MHD_OK or MHD_ERR_WRONG_PARAMETER (with `err`); a CUDA failure is
// reported in `ce`.
// Host side of the lobe plasma sheet: the reference's index arithmetic
// (lobe width, sheet rows, the elliptic sheet start per row, the tanh
// profile and the linear transition weights) in the reference's own double
// and int expressions, so the device passes only copy and blend.
inline int sheet_lobes_args(const Grid& g, const double* p, ProblemArgs& a, std::string& err,
                            cudaStream_t stream, cudaError_t& ce) {
  const double Ly = p[1], start_x = p[2];
  const double head = p[4], foot = p[5], thickness = p[6];
  const int profile = int(p[7]), transition = int(p[8]);
  const double dx = g.dx, dy = g.dy;
  const int NYF = 2, NYL = g.ny + 2, NXF = 2;
  const int lobe_width = (Ly - thickness) / 2.0 / dy;
  a.lim_up = NYL - lobe_width;
  a.lim_dn = NYF + lobe_width;
  a.tp = transition ? 2 * int(p[9]) : 0;
  if (profile < 0 || profile > 1 || transition < 0 || transition > 1 || a.tp < 0 ||
      a.lim_dn < NYF || a.lim_up > NYL || a.lim_dn > a.lim_up) {
    err = "sheet: lobe width, profile or transition outside the grid";
    return MHD_ERR_WRONG_PARAMETER;
  }
  std::vector<double> aux(2 * size_t(g.NY) + size_t(a.tp), 0.0);
  const double ea = head - foot, eb = 0.5 * (thickness - dy), eb2 = eb * eb;
  for (int j = a.lim_dn; j < a.lim_up; j++) {
    const double ey = (j - 1.5) * dy - Ly / 2;
    const double rad = 1.0 - (ey * ey / eb2);
    if (!(rad >= 0.0)) {  // the reference would convert a NaN column to int here
      err = "sheet: the sheet rows reach past the sheet thickness (choose Ly - thickness "
            "as an even number of cells)";
      return MHD_ERR_WRONG_PARAMETER;
    }
    const double ex = foot + ea * std::sqrt(rad);
    const int s = (-start_x + ex) / dx + NXF;
    aux[j] = s;
    if (profile == 1)
      aux[g.NY + j] = std::tanh(2.0 * (j - a.lim_dn) / ((a.lim_up - 1) - a.lim_dn) - 1.0);
    // the transition columns must stay inside the block
    if (a.tp && (s - a.tp / 2 - 1 < 0 || s + a.tp / 2 > g.NX - 1)) {
      err = "sheet: transition across the sheet start leaves the grid";
      return MHD_ERR_WRONG_PARAMETER;
    }
  }
  if (a.tp) {
    if (a.lim_dn - a.tp - 1 < 0 || a.lim_up + a.tp > g.NY - 1) {
      err = "sheet: transition across the lobes leaves the grid";
      return MHD_ERR_WRONG_PARAMETER;
    }
    const double diff = 1.0 / a.tp;
    for (int q = 0; q < a.tp; q++) aux[2 * size_t(g.NY) + q] = (a.tp - q - 0.5) * diff;
  }
  if ((ce = cudaMalloc(&a.aux, aux.size() * sizeof(double))) != cudaSuccess) return MHD_ERR_CUDA;
  ce = cudaMemcpyAsync(a.aux, aux.data(), aux.size() * sizeof(double), cudaMemcpyHostToDevice,
                       stream);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(stream);  // the host vector goes away
  return ce == cudaSuccess ? MHD_OK : MHD_ERR_CUDA;
}

inline int problem_args(int kind, const double* p, int np, double gamma, cudaStream_t stream,
                        ProblemArgs& a, std::string& err, cudaError_t& ce,
                        const Grid* grid = nullptr) {
  a = ProblemArgs{};
  a.kind = kind;
  ce = cudaSuccess;
  if (kind == MHD_PROBLEM_SHOCK_TUBE) {
    if (!p || np < kShockTubeParams || !grid) return MHD_ERR_WRONG_PARAMETER;
    for (int q = 0; q < kShockTubeParams; q++) a.p[q] = p[q];
    const double Lx = p[0], Ly = p[1], angle = p[2];
    a.p[19] = 0.5 * Lx - 0.5 * grid->dx;
    a.p[20] = 0.5 * Ly - 0.5 * grid->dy;
    a.p[21] = std::tan((90.0 - angle) * M_PI / 180.0);
    return MHD_OK;
  }
  if (kind == MHD_PROBLEM_SHEET_LOBES) {
    if (!p || np < kSheetLobesParams || !grid) return MHD_ERR_WRONG_PARAMETER;
    for (int q = 0; q < kSheetLobesParams; q++) a.p[q] = p[q];
    return sheet_lobes_args(*grid, p, a, err, stream, ce);
  }
  if (kind == MHD_PROBLEM_EXPLOSION) {
    if (!p || np < 9) return MHD_ERR_WRONG_PARAMETER;
  } else if (kind == MHD_PROBLEM_WAVE) {
    if (!p || np < 16) return MHD_ERR_WRONG_PARAMETER;
    const int wave = int(p[13]);
    if (wave < 0 || wave > 6 || p[14] < 0 || p[15] < 0) return MHD_ERR_WRONG_PARAMETER;
  } else if (kind == MHD_PROBLEM_PLASMA_SHEET) {
    if (!p || np < 4 || int(p[3]) < 0 || 4 + int(p[3]) > np || 4 + int(p[3]) > 40)
      return MHD_ERR_WRONG_PARAMETER;
    a.K = int(p[3]);
  } else if (kind != MHD_PROBLEM_ORSZAG_TANG) {
    return MHD_ERR_WRONG_PARAMETER;
  }
  for (int q = 0; q < np && q < 40; q++) a.p[q] = p[q];
  if (kind == MHD_PROBLEM_WAVE) {
    // conserved background (toConservationPoint), then its right eigenvector
    const double rho = p[4], u = p[5], v = p[6], w = p[7], bx = p[8], by = p[9], bz = p[10];
    const double pr = p[11], gm = gamma;
    a.avg[0] = rho;
    a.avg[1] = u * rho; a.avg[2] = v * rho; a.avg[3] = w * rho;
    a.avg[4] = bx; a.avg[5] = by; a.avg[6] = bz;
    const double uu = u * u + v * v + w * w, bb = bx * bx + by * by + bz * bz;
    a.avg[7] = pr / (gm - 1.0) + 0.5 * rho * uu + 0.5 * bb;
    double* dtmp = nullptr;
    if ((ce = cudaMalloc(&dtmp, 2 * NF * sizeof(double) + sizeof(int))) != cudaSuccess)
      return MHD_ERR_CUDA;
    int* derr = reinterpret_cast<int*>(dtmp + 2 * NF);
    int herr = 0;
    cudaMemcpyAsync(dtmp, a.avg, NF * sizeof(double), cudaMemcpyHostToDevice, stream);
    kb_wave_eigen<<<1, 32, 0, stream>>>(gm, dtmp, int(p[13]), dtmp + NF, derr);
    cudaMemcpyAsync(a.ev, dtmp + NF, NF * sizeof(double), cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, stream);
    ce = cudaStreamSynchronize(stream);
    cudaFree(dtmp);
    if (ce != cudaSuccess) return MHD_ERR_CUDA;
    if (herr) {
      err = "readProblemWaveTest: failed to calculate eigensystem from average values.";
      return MHD_ERR_WRONG_PARAMETER;
    }
  }
  return MHD_OK;
}

// Number of launches enqueue_problem issues for a.
inline int problem_launches(const ProblemArgs& a) {
  return a.kind == MHD_PROBLEM_SHEET_LOBES ? (a.tp ? 4 : 2) : 1;
}

inline void enqueue_problem(const Grid& g, double* U, const ProblemArgs& a, cudaStream_t stream) {
  const long long cells = (long long)g.nx * g.ny;
  const long long b = (cells + 255) / 256;
  const int grid = int(b < 148LL * 16 ? b : 148LL * 16);
  if (a.kind != MHD_PROBLEM_SHEET_LOBES) {
    kb_problem<<<grid, 256, 0, stream>>>(g, U, a);
    return;
  }
  kb_sheet_base<<<grid, 256, 0, stream>>>(g, U, a);
  if (a.tp) {
    kb_sheet_rows<<<(g.nx + 127) / 128, 128, 0, stream>>>(g, U, a);
    if (a.lim_up > a.lim_dn)
      kb_sheet_cols<<<(a.lim_up - a.lim_dn + 127) / 128, 128, 0, stream>>>(g, U, a);
  }
  kb_natural_to_conserved<<<grid, 256, 0, stream>>>(g, U);
}

// Waits for the setup launches and frees what problem_args allocated.
inline cudaError_t release_problem(ProblemArgs& a, cudaStream_t stream) {
  if (!a.aux) return cudaSuccess;
  cudaError_t e = cudaStreamSynchronize(stream);
  cudaFree(a.aux);
  a.aux = nullptr;
  return e;
}

}  // namespace MHD_KNS
}  // namespace mhd
