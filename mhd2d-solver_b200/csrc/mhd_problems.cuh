// Device-side initial states (problem setups of file_access.cpp) for the
// batched runs and the adjoint.  Kinds and parameter lists are those of
// mhd_batch_init_problem in include/mhd2d_b200.h.
#pragma once

#include <cuda_runtime.h>

#include <string>

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
  double p[40];
  double ev[NF];  // wave: the chosen right eigenvector
  double avg[NF]; // wave: conserved background state
};

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
inline int problem_args(int kind, const double* p, int np, double gamma, cudaStream_t stream,
                        ProblemArgs& a, std::string& err, cudaError_t& ce) {
  a = ProblemArgs{};
  a.kind = kind;
  ce = cudaSuccess;
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

inline void enqueue_problem(const Grid& g, double* U, const ProblemArgs& a, cudaStream_t stream) {
  const long long cells = (long long)g.nx * g.ny;
  const long long b = (cells + 255) / 256;
  kb_problem<<<int(b < 148LL * 16 ? b : 148LL * 16), 256, 0, stream>>>(g, U, a);
}

}  // namespace MHD_KNS
}  // namespace mhd
