// Boundary fill, RK3 / Euler stage updates, the time-step controller and
// the div-B kernels.  All arithmetic keeps the reference's association
// order (the parity build uses -fmad=false).
#pragma once

#include "mhd_common.cuh"

#ifndef MHD_KNS
#define MHD_KNS exact
#endif

namespace mhd {
namespace MHD_KNS {

// ---------------------------------------------------------------------------
// Ghost-cell fill, SpatialIntegrationMethod::applyBoundaryConditions
// (spatialintegrationmethod.cpp:85-300).  The reference fills the sides in
// the order left, right, bottom, top, each reading only interior cells or
// its own freshly mirrored ghosts; every ghost value is therefore a function
// of interior cells alone and all four sides are filled in one pass here.
// Neumann adds the div B = 0 extrapolation of the normal field component
// (lines 122-130, 174-182, 226-234, 278-286), written below in terms of the
// interior cells its mirrored operands came from.  Corners are not touched.
struct Snap {
  const double *l, *r, *b, *t;  // Dirichlet edge snapshots [8][NY], [8][NX]
};

// Number of ghost values one fill writes: 2 layers x 8 fields on 4 sides.
__host__ __device__ __forceinline__ long long bc_count(const Grid& g) {
  return 4LL * NF * g.ny + 4LL * NF * g.nx;
}

// Ghost value e in [0, bc_count(g)).
__device__ __forceinline__ void bc_elem(const Grid& g, double* __restrict__ U, const Snap& d,
                                        long long e) {
  const int nx = g.nx, ny = g.ny;
  const long long nlr = 2LL * 2 * NF * ny;
  const double rxy = g.dx / g.dy, ryx = g.dy / g.dx;
  {
    if (e < nlr) {  // left / right: side, layer, field, row j (fastest)
      const int j = 2 + int(e % ny);
      long long q = e / ny;
      const int k = int(q % NF); q /= NF;
      const int gl = 1 + int(q % 2);
      const int side = int(q / 2);  // 0 left, 1 right
      const int b = g.bc_of(side);
      if (side == 0) {
        const int it = 2 - gl;
        double v;
        if (b == PERIODIC) v = U[g.at(k, nx + 2 - gl, j)];
        else if (b == DIRICHLET) v = d.l[k * g.NY + j];
        else v = U[g.at(k, 2 + gl, j)];
        if (b == NEUMANN && k == 4 && j >= 3 && j < ny + 1) {
          // it = 1: U4[1] = U4[3] - rxy*(U5[2][j-1] - U5[2][j+1])
          // it = 0: U4[0] = U4[2] - rxy*(U5[1][j-1] - U5[1][j+1]), U5[1] mirrors U5[3]
          const int s5 = (it == 1) ? 2 : 3;
          v = U[g.at(4, it + 2, j)] - rxy * (U[g.at(5, s5, j - 1)] - U[g.at(5, s5, j + 1)]);
        }
        U[g.at(k, it, j)] = v;
      } else {
        const int it = nx + 1 + gl;
        double v;
        if (b == PERIODIC) v = U[g.at(k, 1 + gl, j)];
        else if (b == DIRICHLET) v = d.r[k * g.NY + j];
        else v = U[g.at(k, nx + 1 - gl, j)];
        if (b == NEUMANN && k == 4 && j >= 3 && j < ny + 1) {
          // it = nx+2: U4[nx]   - rxy*(U5[nx+1][j+1] - U5[nx+1][j-1])
          // it = nx+3: U4[nx+1] - rxy*(U5[nx+2][j+1] - U5[nx+2][j-1]), U5[nx+2] mirrors U5[nx]
          const int s5 = (it == nx + 2) ? nx + 1 : nx;
          v = U[g.at(4, it - 2, j)] - rxy * (U[g.at(5, s5, j + 1)] - U[g.at(5, s5, j - 1)]);
        }
        U[g.at(k, it, j)] = v;
      }
    } else {  // bottom / top: side, field, column i, layer (fastest)
      long long q = e - nlr;
      const int gl = 1 + int(q % 2); q /= 2;
      const int i = 2 + int(q % nx); q /= nx;
      const int k = int(q % NF);
      const int side = int(q / NF);  // 0 bottom, 1 top
      const int b = g.bc_of(2 + side);
      if (side == 0) {
        const int jt = 2 - gl;
        double v;
        if (b == PERIODIC) v = U[g.at(k, i, ny + 2 - gl)];
        else if (b == DIRICHLET) v = d.b[k * g.NX + i];
        else v = U[g.at(k, i, 2 + gl)];
        if (b == NEUMANN && k == 5 && i >= 3 && i < nx + 1) {
          // jt = 1: U5[i][3] - ryx*(U4[i-1][2] - U4[i+1][2])
          // jt = 0: U5[i][2] - ryx*(U4[i-1][1] - U4[i+1][1]), U4[.][1] mirrors U4[.][3]
          const int s4 = (jt == 1) ? 2 : 3;
          v = U[g.at(5, i, jt + 2)] - ryx * (U[g.at(4, i - 1, s4)] - U[g.at(4, i + 1, s4)]);
        }
        U[g.at(k, i, jt)] = v;
      } else {
        const int jt = ny + 1 + gl;
        double v;
        if (b == PERIODIC) v = U[g.at(k, i, 1 + gl)];
        else if (b == DIRICHLET) v = d.t[k * g.NX + i];
        else v = U[g.at(k, i, ny + 1 - gl)];
        if (b == NEUMANN && k == 5 && i >= 3 && i < nx + 1) {
          // jt = ny+2: U5[i][ny]   - ryx*(U4[i+1][ny+1] - U4[i-1][ny+1])
          // jt = ny+3: U5[i][ny+1] - ryx*(U4[i+1][ny+2] - U4[i-1][ny+2]), U4[.][ny+2] mirrors U4[.][ny]
          const int s4 = (jt == ny + 2) ? ny + 1 : ny;
          v = U[g.at(5, i, jt - 2)] - ryx * (U[g.at(4, i + 1, s4)] - U[g.at(4, i - 1, s4)]);
        }
        U[g.at(k, i, jt)] = v;
      }
    }
  }
}

__global__ void k_bc(Grid g, double* __restrict__ U, Snap d, const Ctl* ctl) {
  if (ctl->skip) return;
  const long long n = bc_count(g);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    bc_elem(g, U, d, e);
}

// Part of the boundary fill, the same elements as k_bc: part 1 the left /
// right sides (every field, row and layer); part 2 the bottom / top sides of
// rows [i0, i1) only.  The two sides' values depend on interior cells only
// (never on another side's ghosts), so the parts of a fill can run in any
// order and at different times.
__global__ void k_bc_part(Grid g, double* __restrict__ U, Snap d, const Ctl* ctl, int part,
                          int i0, int i1) {
  if (ctl->skip) return;
  const long long nlr = 2LL * 2 * NF * g.ny;  // left / right elements come first
  const long long n = part == 1 ? nlr : 2LL * NF * (i1 - i0) * 2;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    if (part == 1) {
      bc_elem(g, U, d, q);
      continue;
    }
    // q -> (side, field, row i, layer) with i in [i0, i1), layer fastest
    long long r = q;
    const int gl = int(r % 2); r /= 2;
    const int ii = int(r % (i1 - i0)); r /= (i1 - i0);
    const int k = int(r % NF);
    const int side = int(r / NF);
    const long long e = nlr + (((long long)side * NF + k) * g.nx + (i0 + ii - 2)) * 2 + gl;
    bc_elem(g, U, d, e);
  }
}

// Dirichlet edge snapshot (spatialintegrationmethod.cpp:39-59).
__global__ void k_snapshot(Grid g, const double* __restrict__ U, double* l, double* r, double* b,
                           double* t) {
  const int n = NF * (g.nx > g.ny ? g.nx : g.ny);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int m = g.nx > g.ny ? g.nx : g.ny;
    const int k = e / m, p = 2 + e % m;
    if (p < g.nx + 2) {
      b[k * g.NX + p] = U[g.at(k, p, 2)];
      t[k * g.NX + p] = U[g.at(k, p, g.ny + 1)];
    }
    if (p < g.ny + 2) {
      l[k * g.NY + p] = U[g.at(k, 2, p)];
      r[k * g.NY + p] = U[g.at(k, g.nx + 1, p)];
    }
  }
}

// ---------------------------------------------------------------------------
// Stage updates on the interior (timeintegrationrk3.cpp:85-88, 108-111,
// 131-134; timeintegrationeuler.cpp:55-58).  dt comes from the control block.
//   mode 0: U  = U + dt*UL                           (Euler)
//   mode 1: U1 = U + dt*UL
//   mode 2: U2 = (3/4)U + (1/4)U1 + (1/4)dt*UL
//   mode 3: U  = (1/3)U + (2/3)U2 + (2/3)dt*UL
__device__ __forceinline__ void combine_at(int mode, double dt, long long a,
                                           double* __restrict__ U, double* __restrict__ U1,
                                           double* __restrict__ U2,
                                           const double* __restrict__ UL) {
  switch (mode) {
    case 0: U[a] = U[a] + dt * UL[a]; break;
    case 1: U1[a] = U[a] + dt * UL[a]; break;
    case 2: U2[a] = (3.0 / 4.0) * U[a] + (1.0 / 4.0) * U1[a] + (1.0 / 4.0) * dt * UL[a]; break;
    case 4: U1[a] = (1.0 / 3.0) * U[a] + (2.0 / 3.0) * U2[a] + (2.0 / 3.0) * dt * UL[a]; break;
    default: U[a] = (1.0 / 3.0) * U[a] + (2.0 / 3.0) * U2[a] + (2.0 / 3.0) * dt * UL[a]; break;
  }
}

__global__ void k_combine(Grid g, int mode, double* __restrict__ U, double* __restrict__ U1,
                          double* __restrict__ U2, const double* __restrict__ UL, const Ctl* ctl) {
  if (ctl->skip) return;
  const double dt = ctl->dt;
  const int j = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = 2 + blockIdx.y;
  const int k = blockIdx.z;
  if (j >= g.ny + 2) return;
  combine_at(mode, dt, g.at(k, i, j), U, U1, U2, UL);
}

// The last RK3 stage update of rows [i0, i1) (ghost rows included) written
// to U1 instead of U: the interior gets the same update as mode 3 (mode 4 of
// combine_at), the ghost cells a copy of U's.  The rows of U1 then hold what
// U holds after the in-place update, while U keeps the step's start state
// for a retry.
__global__ void k_combine_final_rows(Grid g, int i0, int i1, double* __restrict__ U,
                                     double* __restrict__ U1, double* __restrict__ U2,
                                     const double* __restrict__ UL, const Ctl* ctl) {
  if (ctl->skip) return;
  const double dt = ctl->dt;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = i0 + blockIdx.y;
  const int k = blockIdx.z;
  if (j >= g.NY || i >= i1) return;
  const long long a = g.at(k, i, j);
  if (i >= 2 && i < g.nx + 2 && j >= 2 && j < g.ny + 2) combine_at(4, dt, a, U, U1, U2, UL);
  else U1[a] = U[a];
}

// ---------------------------------------------------------------------------
// Time-step control (timeintegrationmethod.cpp:35-90 and the retry logic of
// timeintegrationrk3.cpp:48-156), one thread.
struct StepParams {
  double dx, dy, dt_min, dt_max, cfl;
};

// updateDt: returns the ReturnStatus value; 10 (WrongParameter) stands for
// the inputs on which the reference's doubling / halving loops never end
// (dt = 0 with a positive target, or a negative target).
__device__ __forceinline__ int update_dt(const StepParams& p, double& cur, double ideal) {
  if (p.cfl == 0.0) return 1;  // NoChange: constant time mode
  double dt = cur;
  int n = 0;
  while (dt < 0.5 * p.cfl * ideal) {
    dt *= 2.0;
    if (++n > 4200) return 10;
  }
  n = 0;
  while (dt > p.cfl * ideal) {
    dt /= 2.0;
    if (++n > 4200) return 10;
  }
  if (dt > p.dt_max) dt = p.dt_max;
  if (dt < p.dt_min) return 4;  // ErrorTimeUnderflow
  if (dt == cur) return 1;
  cur = dt;
  return 2;
}

__device__ __forceinline__ double min3(double a, double b, double c) {
  double m = a;          // std::min({a, b, c}): the first smallest
  if (b < m) m = b;
  if (c < m) m = c;
  return m;
}


__device__ __forceinline__ void control_step(Ctl* c, const StepParams& p, int phase, double arg) {
  if (phase == PH_RESET_CARRY) {  // the next step of a device-side step loop
    arg = c->dt;
    phase = PH_RESET_STEP;
  }
  if (phase == PH_RESET_STEP || phase == PH_RESET_INTEGRATE) {
    c->skip = 0; c->retry = 0; c->error = 0; c->neg_last = 0; c->step_done = 0;
    c->maxX = 0ull; c->maxY = 0ull;
    c->neg_count = 0ull; c->negd_count = 0ull;
    c->cfd_first = 0ull; c->cfd_last = 0ull;
    if (phase == PH_RESET_STEP) {
      c->dt1 = arg; c->dt = arg; c->dt2 = p.dt_max; c->dt3 = p.dt_max;
    }
    return;
  }
  if (phase == PH_RK_RETRY) {
    if (!c->retry || c->error) return;
    c->skip = 0; c->retry = 0;
    c->dt = min3(c->dt1, c->dt2, c->dt3);
    return;
  }
  if (phase == PH_DONE) {
    if (!c->skip && !c->error) c->step_done = 1;
    return;
  }
  if (c->skip) return;
  // central FD: a non-positive density (6) ends the integration before
  // dtIdeal; a non-positive pressure (7) is fatal after dtIdeal and UL
  // (spatialmethodcentralfd2.cpp:71-77, 139-159)
  if (!c->error) c->error = c->cfd_first ? 6 : (c->cfd_last ? 7 : 0);
  if (c->error && c->error != 7) { c->skip = 1; return; }
  const double ax = p.dx / bits_to_double(c->maxX), ay = p.dy / bits_to_double(c->maxY);
  const double ideal = (ay < ax) ? ay : ax;  // std::min(a, b)
  c->dtIdeal = ideal;
  c->maxX = 0ull; c->maxY = 0ull;
  if (c->error) { c->skip = 1; return; }
  int st = 1;
  switch (phase) {
    case PH_RK_FIRST:
      st = update_dt(p, c->dt1, ideal);
      if (st == 4 || st == 10) break;
      c->dt = min3(c->dt1, c->dt2, c->dt3);
      break;
    case PH_RK_SECOND:
      st = update_dt(p, c->dt2, ideal);
      if (st == 4 || st == 10) break;
      if (c->dt2 < c->dt) { c->retry = 1; c->skip = 1; }
      break;
    case PH_RK_FINAL:
      st = update_dt(p, c->dt3, ideal);
      if (st == 4 || st == 10) break;
      if (c->dt3 < c->dt) { c->retry = 1; c->skip = 1; }
      break;
    case PH_EULER:
      st = update_dt(p, c->dt, ideal);
      break;
    default:
      break;
  }
  c->upd_status = st;
  if (st == 4 || st == 10) { c->error = st; c->skip = 1; }
}

__global__ void k_control(Ctl* c, StepParams p, int phase, double arg) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  control_step(c, p, phase, arg);
}

// ---------------------------------------------------------------------------
// div B (div_b_fix.cpp).  Range [x0,x1) x [y0,y1): one cell in from every
// non-periodic side; periodic sides first wrap the Bx, By ghost layers.
struct DivRange {
  int x0, x1, y0, y1;
};

__global__ void k_divb_wrap(Grid g, double* __restrict__ U) {
  const int nx = g.nx, ny = g.ny;
  const int n = 2 * 2 * (nx > ny ? nx : ny);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int m = nx > ny ? nx : ny;
    const int k = 4 + (e / m) % 2, which = e / (2 * m), p = 2 + e % m;
    if (which == 0 && p < ny + 2) {
      if (g.bc[LEFT] == PERIODIC) {
        U[g.at(k, 0, p)] = U[g.at(k, nx, p)];
        U[g.at(k, 1, p)] = U[g.at(k, nx + 1, p)];
      }
      if (g.bc[RIGHT] == PERIODIC) {
        U[g.at(k, nx + 2, p)] = U[g.at(k, 2, p)];
        U[g.at(k, nx + 3, p)] = U[g.at(k, 3, p)];
      }
    }
    if (which == 1 && p < nx + 2) {
      if (g.bc[BOTTOM] == PERIODIC) {
        U[g.at(k, p, 0)] = U[g.at(k, p, ny)];
        U[g.at(k, p, 1)] = U[g.at(k, p, ny + 1)];
      }
      if (g.bc[TOP] == PERIODIC) {
        U[g.at(k, p, ny + 2)] = U[g.at(k, p, 2)];
        U[g.at(k, p, ny + 3)] = U[g.at(k, p, 3)];
      }
    }
  }
}

// max and sum of |central div B|; sums go to per-block partials, reduced in
// a fixed order by k_divb_finish so repeated runs give identical totals.
__global__ void __launch_bounds__(256) k_divb_reduce(Grid g, const double* __restrict__ U,
                                                     DivRange R, double* partial, Ctl* c) {
  const int w = R.y1 - R.y0, h = R.x1 - R.x0;
  const long long n = (long long)w * h;
  double mx = 0.0, sum = 0.0;
  const double d2x = 2.0 * g.dx, d2y = 2.0 * g.dy;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = R.x0 + int(e / w), j = R.y0 + int(e % w);
    const double d = fabs((U[g.at(4, i + 1, j)] - U[g.at(4, i - 1, j)]) / d2x +
                          (U[g.at(5, i, j + 1)] - U[g.at(5, i, j - 1)]) / d2y);
    mx = take_max(mx, d);
    sum += d;
  }
  __shared__ double sm[2][8];
  mx = warp_max(mx);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { sm[0][wid] = mx; sm[1][wid] = sum; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0, s = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) { m = take_max(m, sm[0][q]); s += sm[1][q]; }
    partial[blockIdx.x] = s;
    atomic_max_pos(&c->divb_max, m);
  }
}

__global__ void k_divb_finish(double* partial, int nb, double dxdy, Ctl* c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int b = 0; b < nb; b++) s += partial[b];
  c->divb_sum = s * dxdy;
}

// Totals of the reference's non-grid output (outputNonGridData,
// file_access.cpp:1680-1712, on the primitives of toNaturalData,
// conversions.cpp:37-57): per block of the interior, the sums of entropy
// log(p rho^-gamma), energy, mass and rho |u|, and the max of |u|^2, as 5
// partials per block (partial[5 b + q]); the host adds the blocks in order.
constexpr int TOT_THREADS = 256;
__global__ void __launch_bounds__(TOT_THREADS) k_totals(Grid g, const double* __restrict__ U,
                                                         double* __restrict__ partial) {
  const long long n = (long long)g.nx * g.ny;
  const double gm = g.gamma;
  double s_ent = 0.0, s_en = 0.0, s_mass = 0.0, s_mom = 0.0, uumax = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = 2 + int(e / g.ny), j = 2 + int(e % g.ny);
    const double r = U[g.at(0, i, j)], mx = U[g.at(1, i, j)], my = U[g.at(2, i, j)];
    const double mz = U[g.at(3, i, j)], bx = U[g.at(4, i, j)], by = U[g.at(5, i, j)];
    const double bz = U[g.at(6, i, j)], en = U[g.at(7, i, j)];
    const double u0 = mx / r, u1 = my / r, u2 = mz / r;
    const double mm = mx * mx + my * my + mz * mz;
    const double bb = bx * bx + by * by + bz * bz;
    const double p = (gm - 1.0) * (en - 0.5 * mm / r - 0.5 * bb);
    const double uu = u0 * u0 + u1 * u1 + u2 * u2;
    uumax = take_max(uumax, uu);
    s_ent += log(p * pow(r, -gm));
    s_en += en;
    s_mass += r;
    s_mom += r * sqrt(uu);
  }
  double v[5] = {s_ent, s_en, s_mass, s_mom, uumax};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int q = 0; q < 4; q++) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    v[4] = take_max(v[4], __shfl_xor_sync(0xffffffffu, v[4], o));
  }
  __shared__ double sm[5][TOT_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    for (int q = 0; q < 5; q++) sm[q][wid] = v[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int w = 0; w < TOT_THREADS / 32; w++) {
      for (int q = 0; q < 4; q++) t[q] += sm[q][w];
      t[4] = take_max(t[4], sm[4][w]);
    }
    for (int q = 0; q < 5; q++) partial[5 * blockIdx.x + q] = t[q];
  }
}

// One colour of a red-black sweep of the reference's SOR update
// (div_b_fix.cpp:262-280).  The stride-2 Laplacian couples (i, j) only to
// (i+-2, j) and (i, j+-2), so colour ((i>>1) + (j>>1)) & 1 makes every
// point's neighbours the other colour: a half sweep updates its points in
// any order with the same result.  Each thread owns one same-colour pair
// j, j+1 (j even) of one row.
struct SorCoef {
  double pxf, pyf, bxf, byf, coef, omega;
};

// Rows per block of k_sor_half (at most): each block reduces its update /
// potential maxima over its rows before its two atomics.  Small grids take
// fewer rows per block so that the half sweep still spreads over the SMs.
constexpr int SOR_ROWS = 8;
constexpr int SOR_THREADS = 128;

// Same-colour column pairs per row: thread q of a row owns columns
// jb = 2*(2q + b), jb + 1 with b = (colour + (i>>1)) & 1.
__host__ __device__ __forceinline__ int sor_pairs(const DivRange& R) { return (R.y1 + 3) / 4 + 1; }


// The divergence source terms of the SOR update are fixed during a solve:
// X = bxf*(Bx[i+1][j] - Bx[i-1][j]), Y = byf*(By[i][j+1] - By[i][j-1]), the
// same products the per-point update forms (so it stays bit-identical).  They
// are stored once per solve, per colour and pair, as {X(jb), X(jb+1), Y(jb),
// Y(jb+1)}: a warp's half sweep reads them as contiguous 32-byte items.
__global__ void k_sor_rhs(Grid g, const double* __restrict__ U, DivRange R, SorCoef s,
                          double4* __restrict__ xy) {
  const int Q = sor_pairs(R), H = R.x1 - R.x0;
  const long long n = 2LL * H * Q;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int q = int(e % Q);
    const int ir = int((e / Q) % H);
    const int color = int(e / ((long long)Q * H));
    const int i = R.x0 + ir;
    const int jb = 2 * (2 * q + ((color + (i >> 1)) & 1));
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int t = 0; t < 2; t++) {
      const int j = jb + t;
      if (j >= R.y0 && j < R.y1) {
        v[t] = s.bxf * (U[g.at(4, i + 1, j)] - U[g.at(4, i - 1, j)]);
        v[2 + t] = s.byf * (U[g.at(5, i, j + 1)] - U[g.at(5, i, j - 1)]);
      }
    }
    xy[e] = make_double4(v[0], v[1], v[2], v[3]);
  }
}

// Row read in place of periodic ghost row r (fused sweeps).
__device__ __forceinline__ int sor_src_row(const Grid& g, int r) {
  if (g.bc[LEFT] == PERIODIC && r < 2) return r + g.nx;
  if (g.bc[RIGHT] == PERIODIC && r >= g.nx + 2) return r - g.nx;
  return r;
}

// Convergence test after a sweep (div_b_fix.cpp:370-373): stop when
// max|update| / max|phi| <= rmax.  The ratio of the last sweep is kept for
// the final verdict, which the host evaluates as the reference does.
__device__ __forceinline__ void sor_check(Ctl* c, double rtol, double max_sweeps,
                                          double* last_ratio) {
  const double ratio = bits_to_double(c->rmax) / bits_to_double(c->pmax);
  *last_ratio = ratio;
  c->rmax = 0ull; c->pmax = 0ull;
  c->sor_sweeps += 1;
  if (ratio <= rtol || c->sor_sweeps >= max_sweeps) c->sor_done = 1;
}

// One row of a half sweep in registers (k_sor_half): the thread's pair of
// the row, its four neighbour pairs and its source terms.
struct SorRow {
  double2 up, dn, lf, rt, me;
  double4 f;
  double* pme;
  int jb;
  bool ok;
};

// The previous row of a chain (k_sor_half): addresses and values of its
// other-colour loads.
struct SorChain {
  const double* up = nullptr;
  const double* lf = nullptr;
  const double* rt = nullptr;
  double2 vup, vlf, vrt;
};

// Loads row offset ir of a half sweep (when it is in the range and holds
// points of the thread's pair); REUSE: takes the values the chain's
// previous row loaded from the same addresses.
template <bool FUSED, bool REUSE>
__device__ __forceinline__ void sor_row_load(const Grid& g, const double* __restrict__ phi,
                                             const double4* __restrict__ xy, const DivRange& R,
                                             int color, int q, int Q, int H, long long P, int ir,
                                             SorChain& c, SorRow& o) {
  const int i = R.x0 + ir;
  const int jb = 2 * (2 * q + ((color + (i >> 1)) & 1));
  o.ok = i < R.x1 && !(jb + 1 < R.y0 || jb >= R.y1);
  if (!o.ok) {
    c.up = c.lf = c.rt = nullptr;
    return;
  }
  const double* prow = phi + (long long)i * P + g.off;
  const double* urow = prow + 2 * P;
  const double* drow = prow - 2 * P;
  int jl = jb - 2, jr = jb + 2;
  if (FUSED) {
    urow = phi + (long long)sor_src_row(g, i + 2) * P + g.off;
    drow = phi + (long long)sor_src_row(g, i - 2) * P + g.off;
    if (g.bc[BOTTOM] == PERIODIC && jl < 2) jl += g.ny;
    if (g.bc[TOP] == PERIODIC && jr >= g.ny + 2) jr -= g.ny;
  }
  const double* pu = urow + jb;
  const double* pd = drow + jb;
  const double* pl = prow + jl;
  const double* pr = prow + jr;
  o.f = xy[((long long)color * H + ir) * Q + q];
  o.up = *reinterpret_cast<const double2*>(pu);
  if (REUSE) {
    o.dn = pd == c.lf ? c.vlf : (pd == c.rt ? c.vrt : *reinterpret_cast<const double2*>(pd));
    o.lf = pl == c.up ? c.vup : *reinterpret_cast<const double2*>(pl);
    o.rt = pr == c.up ? c.vup : *reinterpret_cast<const double2*>(pr);
    c.up = pu; c.vup = o.up;
    c.lf = pl; c.vlf = o.lf;
    c.rt = pr; c.vrt = o.rt;
  } else {
    o.dn = *reinterpret_cast<const double2*>(pd);
    o.lf = *reinterpret_cast<const double2*>(pl);
    o.rt = *reinterpret_cast<const double2*>(pr);
  }
  o.me = *reinterpret_cast<const double2*>(prow + jb);
  o.pme = const_cast<double*>(prow) + jb;
  o.jb = jb;
}

// The reference's per-point update (div_b_fix.cpp:262-280) of a loaded row's
// pair, its maxima, and the store of the pair.
__device__ __forceinline__ void sor_row_update(const SorCoef& s, const DivRange& R,
                                               const SorRow& o, double& rmax, double& pmax) {
  const double ax[2] = {o.up.x, o.up.y}, bx[2] = {o.dn.x, o.dn.y};
  const double ay[2] = {o.rt.x, o.rt.y}, by[2] = {o.lf.x, o.lf.y};
  const double X[2] = {o.f.x, o.f.y}, Y[2] = {o.f.z, o.f.w};
  double out[2] = {o.me.x, o.me.y};
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const int j = o.jb + t;
    if (j >= R.y0 && j < R.y1) {
      double r = s.pxf * (ax[t] + bx[t]);
      r += s.pyf * (ay[t] + by[t]);
      r += X[t];
      r += Y[t];
      r *= s.coef;
      r -= out[t];
      out[t] += s.omega * r;
      rmax = take_max(rmax, fabs(r));
      pmax = take_max(pmax, fabs(out[t]));
    }
  }
  *reinterpret_cast<double2*>(o.pme) = make_double2(out[0], out[1]);
}

// One colour of a red-black sweep.  The potential pairs are read and written
// as 16-byte items (jb is even, the padded row offset is even).  FUSED:
// periodic ghosts are read at their source points, and the last block of the
// colour-1 launch runs the convergence test.  PAIRS: two rows' loads in
// flight per thread (large grids); otherwise one row at a time, with the
// loads its chain's previous row made reused (sor_pairs_ok picks).
template <bool FUSED, bool PAIRS>
__global__ void __launch_bounds__(SOR_THREADS) k_sor_half(Grid g, double* __restrict__ phi,
                                                          const double4* __restrict__ xy,
                                                          DivRange R, SorCoef s, int color,
                                                          Ctl* c, double rtol, double max_sweeps,
                                                          double* last_ratio, int rpb) {
  if (c->sor_done) return;
  __shared__ double red[2][SOR_THREADS / 32];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int Q = sor_pairs(R), H = R.x1 - R.x0;
  const long long P = g.pitch;
  double rmax = 0.0, pmax = 0.0;
  if (q < Q) {
    // The block's rows form two chains, offsets 0, 2, 4, ... and 1, 3, 5, ...
    // Rows are independent within a half sweep: a row writes only its own
    // pair, and its neighbour pairs are points of the other colour, which the
    // half sweep does not change.  So any order reads the same values.
    const int half = (rpb + 1) / 2;
    if (PAIRS) {
      // one row of each chain per iteration, both rows' loads issued before
      // either row is updated: twice as many loads in flight
      SorChain none;
      for (int k = 0; k < half; k++) {
        SorRow a, b;
        sor_row_load<FUSED, false>(g, phi, xy, R, color, q, Q, H, P, blockIdx.y * rpb + 2 * k,
                                   none, a);
        if (2 * k + 1 < rpb)
          sor_row_load<FUSED, false>(g, phi, xy, R, color, q, Q, H, P,
                                     blockIdx.y * rpb + 2 * k + 1, none, b);
        else
          b.ok = false;
        if (a.ok) sor_row_update(s, R, a, rmax, pmax);
        if (b.ok) sor_row_update(s, R, b, rmax, pmax);
      }
    } else {
      // one chain after the other.  Row i + 2's pair sits two columns from
      // row i's: the pair row i reads above it is the one row i + 2 reads at
      // its left or right, and the one row i reads at its right or left is
      // the one row i + 2 reads below it.  A load whose address equals one
      // of the chain's previous row's takes that value (3 loads of the
      // potential per row instead of 5).
      SorChain c;
      for (int k = 0; k < rpb; k++) {
        const int rr = k < half ? 2 * k : 2 * (k - half) + 1;
        if (k == half) c = SorChain();  // the second chain starts
        SorRow a;
        sor_row_load<FUSED, true>(g, phi, xy, R, color, q, Q, H, P, blockIdx.y * rpb + rr, c, a);
        if (a.ok) sor_row_update(s, R, a, rmax, pmax);
      }
    }
  }
  rmax = warp_max(rmax);
  pmax = warp_max(pmax);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][w] = rmax;
    red[1][w] = pmax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q2 = 1; q2 < SOR_THREADS / 32; q2++) {
      rmax = take_max(rmax, red[0][q2]);
      pmax = take_max(pmax, red[1][q2]);
    }
    atomic_max_pos(&c->rmax, rmax);
    atomic_max_pos(&c->pmax, pmax);
    if (FUSED && color == 1) {
      // the last block to finish sees every block's maxima
      __threadfence();
      const unsigned nb = gridDim.x * gridDim.y;
      if (atomicAdd(&c->sor_ticket, 1u) == nb - 1) {
        __threadfence();
        c->sor_ticket = 0u;
        sor_check(c, rtol, max_sweeps, last_ratio);
      }
    }
  }
}

// Potential ghosts after each sweep (div_b_fix.cpp:282-364).  force = 1
// refreshes them whether or not the solve has stopped (fused sweeps: once
// before the first and once after the last sweep).
__global__ void k_phi_bc(Grid g, double* __restrict__ phi, const Ctl* c, int force) {
  if (!force && c->sor_done) return;
  const int nx = g.nx, ny = g.ny, m = nx > ny ? nx : ny;
  const long long P = g.pitch;
  auto PH = [&](int i, int j) -> double& { return phi[(long long)i * P + g.off + j]; };
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 2 * m; e += gridDim.x * blockDim.x) {
    const int which = e / m, p = 2 + e % m;
    if (which == 0 && p < ny + 2) {
      if (g.bc[LEFT] == PERIODIC) { PH(0, p) = PH(nx, p); PH(1, p) = PH(nx + 1, p); }
      else if (g.bc[LEFT] == OPEN) PH(1, p) = PH(2, p);
      if (g.bc[RIGHT] == PERIODIC) { PH(nx + 2, p) = PH(2, p); PH(nx + 3, p) = PH(3, p); }
      else if (g.bc[RIGHT] == OPEN) PH(nx + 2, p) = PH(nx + 1, p);
    }
    if (which == 1 && p < nx + 2) {
      if (g.bc[BOTTOM] == PERIODIC) { PH(p, 0) = PH(p, ny); PH(p, 1) = PH(p, ny + 1); }
      else if (g.bc[BOTTOM] == OPEN) PH(p, 1) = PH(p, 2);
      if (g.bc[TOP] == PERIODIC) { PH(p, ny + 2) = PH(p, 2); PH(p, ny + 3) = PH(p, 3); }
      else if (g.bc[TOP] == OPEN) PH(p, ny + 2) = PH(p, ny + 1);
    }
  }
}

// The convergence test of the unfused sweep, as its own one-thread launch.
__global__ void k_sor_check(Ctl* c, double rtol, double max_sweeps, double* last_ratio) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || c->sor_done) return;
  sor_check(c, rtol, max_sweeps, last_ratio);
}

// B += central gradient of phi over [x0-1, x1+1) x [y0-1, y1+1)
// (div_b_fix.cpp:392-399).
__global__ void k_sor_correct(Grid g, double* __restrict__ U, const double* __restrict__ phi,
                              DivRange R, double bxf, double byf) {
  const int w = R.y1 - R.y0 + 2, h = R.x1 - R.x0 + 2;
  const long long P = g.pitch;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)w * h;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = R.x0 - 1 + int(e / w), j = R.y0 - 1 + int(e % w);
    const double* pr = phi + (long long)i * P + g.off;
    U[g.at(4, i, j)] += (pr[j + P] - pr[j - P]) * bxf;
    U[g.at(5, i, j)] += (pr[j + 1] - pr[j - 1]) * byf;
  }
}

}  // namespace MHD_KNS
}  // namespace mhd
