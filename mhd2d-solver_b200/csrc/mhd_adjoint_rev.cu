// Reverse sweep of the discrete adjoint (mhd_adjoint.cu): the interface
// adjoint, the per-cell gather and the boundary-fill transpose of one stage.
//
// Built twice (MHD_ADJREV names the launchers' namespace): `contracted`
// with FMA contraction, `uncontracted` with the parity build's rounding (the
// forward kernels the adjoint records and replays are uncontracted in
// mhd_adjoint.cu either way).  The reverse sweep recomputes the recording's
// midpoint states; in the contracted build MHD_MIDPOINT_UNFUSED keeps their
// products unfused, so the midpoint takes the recording's branches (pressure
// and speed clamps, the degenerate and sign cases).  The eigenvector rows,
// the physical fluxes and the generated reverse code have no value-dependent
// branches: contraction changes their rounding only.  Where the eigen-system
// is near-degenerate (B_perp ~ 0 in a current sheet) that rounding is
// amplified: the two builds' gradients then differ by ~1e-8 relative.
#include <cuda_runtime.h>

#include "mhd_adjoint_gen.cuh"
#include "mhd_adjoint_rev.h"
#include "mhd_flux.cuh"

namespace mhd {
namespace MHD_KNS {

// Adjoint of one stage update at element a, except its UL term: the adjoint
// of UL is ul_coef(mode, dt) times the adjoint of the update's output
// (stage_out), which ka_adj_iface reads directly.
__device__ __forceinline__ void combine_adj_at(int mode, long long a, double* __restrict__ lU,
                                               double* __restrict__ lU1,
                                               double* __restrict__ lU2) {
  switch (mode) {
    case 0:  // U = U + dt*UL
      break;
    case 1: {  // U1 = U + dt*UL
      const double b = lU1[a];
      lU[a] += b;
      lU1[a] = 0.0;
      break;
    }
    case 2: {  // U2 = (3/4)U + (1/4)U1 + (1/4)dt*UL
      const double b = lU2[a];
      lU[a] += (3.0 / 4.0) * b;
      lU1[a] += (1.0 / 4.0) * b;
      lU2[a] = 0.0;
      break;
    }
    default: {  // U = (1/3)U + (2/3)U2 + (2/3)dt*UL
      const double b = lU[a];
      lU2[a] += (2.0 / 3.0) * b;
      lU[a] = (1.0 / 3.0) * b;
      break;
    }
  }
}

// Stencil of interface f (between cells f and f+1 along the direction) at
// transverse index t: cell of stencil point p.
__device__ __forceinline__ long long cell_at(const Grid& g, bool ydir, int k, int f, int t, int p) {
  return ydir ? g.at(k, t, f - 1 + p) : g.at(k, f - 1 + p, t);
}

constexpr int AIB = 64;  // threads per block of ka_adj_iface (31 KB of shared memory)
constexpr int AIB_MIN = 6;  // resident blocks per SM: 168 registers, 6 x 31 KB shared

// Interface tiles of ka_adj_iface: each warp takes BF consecutive faces
// along the direction times BT transverse cells (BF * BT = 32 threads) and
// sums its faces' contributions per stencil cell before writing them.
// The CL = BF + 3 cells a tile's stencils touch overlap the next tile's by
// 3, so the scratch holds CL / BF cell records of 15 words per face instead
// of the 44 words of every face.  x faces: 8 x 4 (consecutive lanes along
// t, the contiguous j); y faces: 32 x 1 (lanes along f, j again).
struct ITile {
  int bf, bt, cl, ntile, nt;  // tile shape, tiles along the direction, transverse cells
  long long plane;            // doubles per scratch word plane
};
constexpr int BF_X = 4, BF_Y = 32;
// a cell is then touched by the stencils of at most two tiles (the gather reads two records)
static_assert(BF_X >= 3 && BF_Y >= 3 && 32 % BF_X == 0 && 32 % BF_Y == 0, "interface tile shape");
// Stencil cells of one warp's tile (NCW), and the warp's shared-memory
// region: the cells' frame fluxes (7 x NCW), primitives (4 x NCW) and frame
// states (8 x NCW).  Once the warp's interfaces are done with the fluxes and
// primitives, their first 16 x 32 doubles hold the lanes' U1 / U2 adjoints.
constexpr int NCW = (BF_X + 3) * (32 / BF_X) > (BF_Y + 3) * (32 / BF_Y) ? (BF_X + 3) * (32 / BF_X)
                                                                      : (BF_Y + 3) * (32 / BF_Y);
constexpr int WOFF_P = 7 * NCW, WOFF_S = 11 * NCW, WREG = 19 * NCW;
static_assert(16 * 32 <= WOFF_S, "U1 / U2 adjoints fit over the fluxes and primitives");
constexpr int NPW = 15;  // scratch words per cell record: 7 flux-adjoint slots, 8 state adjoints

__host__ __device__ inline ITile itile(const Grid& g, bool ydir) {
  ITile T;
  T.bf = ydir ? BF_Y : BF_X;
  T.bt = 32 / T.bf;
  T.cl = T.bf + 3;
  const int nf = ydir ? g.ny + 1 : g.nx + 1;  // faces 1..n+1 along the direction
  T.nt = ydir ? g.nx : g.ny;                  // interior transverse cells 2..n+1
  T.ntile = (nf + T.bf - 1) / T.bf;
  T.plane = (long long)T.ntile * T.cl * T.nt;
  return T;
}

// Scratch word w of the record of tile tau, touched cell c (cell tau*bf + c
// along the direction) and transverse cell t: x records are ordered
// [w][tau][c][t], y records [w][t][tau][c], so both run along j.
__host__ __device__ inline long long rec_at(const ITile& T, bool ydir, int w, int tau, int c,
                                            int t) {
  const long long r = ydir ? (long long)(t - 2) * T.ntile * T.cl + (long long)tau * T.cl + c
                           : ((long long)tau * T.cl + c) * T.nt + (t - 2);
  return w * T.plane + r;
}

// Adjoint of the numerical flux of one interface f at transverse cell t
// (the interface's frame is the x frame: y interfaces work on x/y-swapped
// states, as the forward does).  The frame fluxes, primitives and states of
// its 4 stencil points come from the warp's cell arrays at wr (point p: cell
// ci0 + p * cstep); the midpoint is formed from the primitives (midpoint_p),
// as the recording's flux kernel forms it.  Leaves in the thread's column of
// sFb the adjoints of the frame fluxes of the 4 stencil points (row 7p +
// slot(m)) and adds the adjoints of the frame states U1, U2 to U1b, U2b.
//
// The characteristics are walked in pairs (0, 6), (2, 4), (1, 5), (3):
// rows k and 6 - k share a symmetric part, so the adjoint of the pair's
// eigenvector rows is one pass (pair_adjoint) over the summed and
// differenced seeds.
template <bool YDIR>
__device__ __forceinline__ void iface_adjoint(const Grid& g, const Gas& G,
                                              const unsigned* __restrict__ mask,
                                              const double* __restrict__ lB, double cL,
                                              double inv_d, int f, int t, int tid,
                                              const double* __restrict__ wr, int ci0,
                                              int cstep, double (*sFb)[AIB], double* U1b,
                                              double* U2b) {
  const double* sC = wr;           // frame fluxes of the warp's cells
  const double* sP = wr + WOFF_P;  // their primitives
  const double* sS = wr + WOFF_S;  // their frame states
  const int ncell = YDIR ? g.ny : g.nx;
  const int lo_bc = YDIR ? BOTTOM : LEFT, hi_bc = YDIR ? TOP : RIGHT;
  const int l1 = (g.bc_of(lo_bc) == OPEN && f < 2) ? 2 : 1;
  const int l2 = (g.bc_of(hi_bc) == OPEN && f > ncell) ? 1 : 2;
#pragma unroll
  for (int c = 0; c < 28; c++) sFb[c][tid] = 0.0;
  // adjoint of the frame numerical flux: UL = -(F_f - F_{f-1}) / d - ...;
  // the adjoint of UL is cL times the adjoint lB of the stage update's output
  double lF[NF];
  const int cell_lo = f, cell_hi = f + 1;  // the two cells sharing the face
#pragma unroll
  for (int m = 0; m < NF; m++) {
    const int kk = YDIR ? swap_xy(m) : m;
    double v = 0.0;
    if (cell_lo >= 2 && cell_lo <= ncell + 1)
      v -= inv_d * (cL * lB[YDIR ? g.at(kk, t, cell_lo) : g.at(kk, cell_lo, t)]);
    if (cell_hi >= 2 && cell_hi <= ncell + 1)
      v += inv_d * (cL * lB[YDIR ? g.at(kk, t, cell_hi) : g.at(kk, cell_hi, t)]);
    lF[m] = v;
  }
  double U1[NF], U2[NF], P1[4], P2[4];
#pragma unroll
  for (int k = 0; k < NF; k++) {
    U1[k] = sS[k * NCW + ci0 + l1 * cstep];
    U2[k] = sS[k * NCW + ci0 + l2 * cstep];
  }
#pragma unroll
  for (int k = 0; k < 4; k++) {
    P1[k] = sP[k * NCW + ci0 + l1 * cstep];
    P2[k] = sP[k * NCW + ci0 + l2 * cstep];
  }
  Mid e0;
  if (!midpoint_p(G, U1, U2, P1, P2, e0)) return;  // sFb, U1b, U2b stay zero
  const unsigned mw = mask[YDIR ? (long long)t * g.NY + f : (long long)f * g.NY + t];
  MidBar mb{};
#pragma unroll 1
  for (int pi = 0; pi < 4; pi++) {
    const int ka = pi == 0 ? 0 : pi == 1 ? 2 : pi == 2 ? 1 : 3;
    // pair seeds: LS / LD = lb_k +- lb_{6-k} (slots 0..6), fS / fD likewise
    double LS[7], LD[7], fS = 0.0, fD = 0.0;
#pragma unroll
    for (int s = 0; s < 7; s++) { LS[s] = 0.0; LD[s] = 0.0; }
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int k = h == 0 ? ka : 6 - ka;
      if (h == 1 && k == ka) break;
      // keeps the row products inside the iteration (fewer live registers)
      opaque(e0);
      const unsigned code = (mw >> (4 * k)) & 0xFu;
      const int up = int(code >> 2);
      // upwind choice "zero": the characteristic's flux is the constant 0 (its
      // row may even be non-finite, as at a midpoint whose pressure was clamped)
      if (up == 2) continue;
      double l[NF], r[NF];
#pragma unroll
      for (int m = 0; m < NF; m++) { l[m] = 0.0; r[m] = 0.0; }
      lv_row(e0, G, k, l);
      rv_row(e0, G, k, r);
      // frozen ENO combination: ca * F[pa] + cb * F[pa + 1] (the other two points have
      // weight 0)
      const int pa = up == 0 ? ((code & 1u) ? 0 : 1) : ((code & 2u) ? 1 : 2);
      const double ca = pa == 0 ? -0.5 : (pa == 1 ? 0.5 : 1.5);
      const double cb = pa == 0 ? 1.5 : (pa == 1 ? 0.5 : -0.5);
      double phi[NF], fw = 0.0, gk = 0.0;
#pragma unroll
      for (int m = 0; m < NF; m++) {
        if (m == 4) { phi[m] = 0.0; continue; }
        const int s = slot_of(m);
        phi[m] = ca * sC[s * NCW + ci0 + pa * cstep] + cb * sC[s * NCW + ci0 + (pa + 1) * cstep];
        fw += l[m] * phi[m];
      }
#pragma unroll
      for (int m = 0; m < NF; m++) gk += lF[m] * r[m];
      const double sg = h == 0 ? 1.0 : -1.0;
#pragma unroll
      for (int m = 0; m < NF; m++) {
        if (m == 4) continue;
        const int s = slot_of(m);
        LS[s] += gk * phi[m];
        LD[s] += sg * (gk * phi[m]);
      }
      fS += fw;
      fD += sg * fw;
      if (gk != 0.0) {
#pragma unroll
        for (int m = 0; m < NF; m++) {
          if (m == 4) continue;
          const int s = slot_of(m);
          const double v = gk * l[m];
          sFb[7 * pa + s][tid] += ca * v;
          sFb[7 * pa + 7 + s][tid] += cb * v;
        }
      }
    }
    opaque(e0);
    pair_adjoint(e0, G, pi, LS, LD, fS, fD, lF, mb);
  }
  // U1, U2 again from shared memory (volatile: not kept live across the loop)
  {
    const volatile double* vq = sS;
#pragma unroll
    for (int k = 0; k < NF; k++) {
      U1[k] = vq[k * NCW + ci0 + l1 * cstep];
      U2[k] = vq[k * NCW + ci0 + l2 * cstep];
    }
  }
  midpoint_adjoint(G, e0, U1, U2, mb, U1b, U2b);
}

// Adjoint of the numerical flux of every interface of one direction, one
// thread per interface (iface_adjoint), one interface tile per warp
// (ITile).  The warp then writes one record per touched cell: the sums of
// its faces' flux adjoints (slot w < 7) and state adjoints (7 + k) at that
// cell, added in the order of the stencil position p = 0..3 (faces
// descending), the adjoint of U1 before that of U2 per face.
template <bool YDIR>
__global__ void __launch_bounds__(AIB, AIB_MIN)
    ka_adj_iface(Grid g, Gas G, const double* __restrict__ X, const unsigned* __restrict__ mask,
                 const double* __restrict__ lB, double cL, double* __restrict__ S,
                 double inv_d) {
  __shared__ double sW[(AIB / 32) * WREG];  // per warp: its cells' fluxes, primitives, states
  __shared__ double sFb[28][AIB];  // per interface: adjoints of its 4 stencil points' fluxes
  const int tid = threadIdx.x, lane = tid & 31;
  double* wr = sW + (tid / 32) * WREG;
  double* sQ = wr;  // [16][32]: the lanes' U1 / U2 adjoints, after the interfaces
  const ITile T = itile(g, YDIR);
  const int nf = YDIR ? g.ny + 1 : g.nx + 1, ncell = nf - 1;
  const long long tile = (long long)blockIdx.x * (AIB / 32) + tid / 32;
  const long long ntiles = (long long)T.ntile * ((T.nt + T.bt - 1) / T.bt);
  const int tau = int(tile % T.ntile), tb = int(tile / T.ntile);
  // the tile's stencil cells (c, tl2), cell tau*bf + c along the direction:
  // states, primitives and fluxes once per cell (each is a stencil point of
  // up to 4 faces)
  if (tile < ntiles) {
    for (int ci = lane; ci < T.cl * T.bt; ci += 32) {
      const int c = YDIR ? ci % T.cl : ci / T.bt, tl2 = YDIR ? ci / T.cl : ci % T.bt;
      const int a = tau * T.bf + c, t2 = 2 + tb * T.bt + tl2;
      if (a > ncell + 3 || t2 > T.nt + 1) continue;  // read by no interface
      double q[NF], F[NF], Gy[NF], P[4];
#pragma unroll
      for (int k = 0; k < NF; k++)
        q[k] = X[YDIR ? g.at(swap_xy(k), t2, a) : g.at(k, a, t2)];
      phys_flux(G.gm, q, F, Gy);
      cell_primitives(G.gm, q, P);
#pragma unroll
      for (int m = 0; m < NF; m++)
        if (m != 4) wr[slot_of(m) * NCW + ci] = F[m];
#pragma unroll
      for (int k = 0; k < 4; k++) wr[WOFF_P + k * NCW + ci] = P[k];
#pragma unroll
      for (int k = 0; k < NF; k++) wr[WOFF_S + k * NCW + ci] = q[k];
    }
  }
  __syncwarp();
  const int fl = YDIR ? lane % T.bf : lane / T.bt, tl = YDIR ? lane / T.bf : lane % T.bt;
  const int f = 1 + tau * T.bf + fl, t = 2 + tb * T.bt + tl;
  double U1b[NF], U2b[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) { U1b[k] = 0.0; U2b[k] = 0.0; }
  if (tile < ntiles && f <= nf && t <= T.nt + 1) {
    // stencil point p of this face is cell (fl + p, tl)
    const int ci0 = YDIR ? tl * T.cl + fl : fl * T.bt + tl;
    const int cstep = YDIR ? 1 : T.bt;
    iface_adjoint<YDIR>(g, G, mask, lB, cL, inv_d, f, t, tid, wr, ci0, cstep, sFb, U1b, U2b);
  } else {
#pragma unroll
    for (int c = 0; c < 28; c++) sFb[c][tid] = 0.0;
  }
  __syncwarp();  // every lane is done with the fluxes and primitives sQ overwrites
#pragma unroll
  for (int k = 0; k < NF; k++) {
    sQ[k * 32 + lane] = U1b[k];
    sQ[(8 + k) * 32 + lane] = U2b[k];
  }
  __syncwarp();
  if (tile >= ntiles) return;
  const int lo_bc = YDIR ? BOTTOM : LEFT, hi_bc = YDIR ? TOP : RIGHT;
  const bool open_lo = g.bc_of(lo_bc) == OPEN, open_hi = g.bc_of(hi_bc) == OPEN;
  for (int it = lane; it < T.cl * T.bt; it += 32) {
    int c, tl2;
    if (YDIR) {
      c = it % T.cl; tl2 = it / T.cl;
    } else {
      tl2 = it % T.bt; c = it / T.bt;
    }
    const int t2 = 2 + tb * T.bt + tl2;
    if (t2 > T.nt + 1) continue;
    double fb[7], qb[NF];
#pragma unroll
    for (int w = 0; w < 7; w++) fb[w] = 0.0;
#pragma unroll
    for (int k = 0; k < NF; k++) qb[k] = 0.0;
#pragma unroll
    for (int p = 0; p < 4; p++) {
      const int fl2 = c - p;
      if (fl2 < 0 || fl2 >= T.bf) continue;
      const int tw = YDIR ? tl2 * T.bf + fl2 : fl2 * T.bt + tl2;  // the face's lane
      const int th = (tid - lane) + tw;
#pragma unroll
      for (int w = 0; w < 7; w++) fb[w] += sFb[7 * p + w][th];
      const int f2 = 1 + tau * T.bf + fl2;
      const int l1 = (open_lo && f2 < 2) ? 2 : 1;
      const int l2 = (open_hi && f2 > ncell) ? 1 : 2;
      if (p == l1) {
#pragma unroll
        for (int k = 0; k < NF; k++) qb[k] += sQ[k * 32 + tw];
      }
      if (p == l2) {
#pragma unroll
        for (int k = 0; k < NF; k++) qb[k] += sQ[(8 + k) * 32 + tw];
      }
    }
    double* r = S + rec_at(T, YDIR, 0, tau, c, t2);
#pragma unroll
    for (int w = 0; w < 7; w++) r[w * T.plane] = fb[w];
#pragma unroll
    for (int k = 0; k < NF; k++) r[(7 + k) * T.plane] = qb[k];
  }
}

// Programmatic dependent launch: a kernel launched with the programmatic
// stream-serialization attribute may be scheduled before the previous kernel
// of its stream has finished; it waits here, before touching memory that
// kernel writes or reads.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Per cell: sum the interface contributions of both directions and apply the
// transposed flux Jacobians.  Two lanes per cell (an even / odd lane pair):
// the even lane takes the x direction, the odd lane the y direction; the
// pair then adds the two parts in the order x, y.  Interior cells first take
// the adjoint of the stage update (combine_adj_at, mode) and then add the
// result to the stage input's adjoint lbuf (one of lU, lU1, lU2, selected by
// in_buf); ghost cells write it to T for the boundary-fill transpose.  The
// even lane writes fields 0-3, the odd lane fields 4-7.
__global__ void __launch_bounds__(128) ka_adj_gather(Grid g, Gas G, const double* __restrict__ X,
                                                     const double* __restrict__ SX,
                                                     const double* __restrict__ SY,
                                                     double* __restrict__ T, int mode,
                                                     int in_buf, double* __restrict__ lU,
                                                     double* __restrict__ lU1,
                                                     double* __restrict__ lU2) {
  const long long NXY = (long long)g.NX * g.NY;
  const long long e2 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long e = e2 >> 1;
  const bool yd = (e2 & 1) != 0;
  const bool valid = e < NXY;
  const int i = valid ? int(e / g.NY) : 0, j = valid ? int(e % g.NY) : 0;
  double part[NF];  // this lane's direction, in the cell's (x) frame
#pragma unroll
  for (int k = 0; k < NF; k++) part[k] = 0.0;
  const int a = yd ? j : i;  // position along the direction
  const int t = yd ? i : j;  // transverse position
  const int ntr = yd ? g.nx : g.ny;
  if (valid && t >= 2 && t <= ntr + 1) {
    const double* S = yd ? SY : SX;
    const ITile TT = itile(g, yd);
    double fb[NF], qb[NF];
#pragma unroll
    for (int m = 0; m < NF; m++) { fb[m] = 0.0; qb[m] = 0.0; }
    // the records of the (one or two) tiles whose stencils touch the cell:
    // the tile of the higher faces first, then the tile below it
    const int tau1 = a / TT.bf, c1 = a % TT.bf;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int tau = tau1 - h, c = c1 + h * TT.bf;
      if (tau < 0 || tau >= TT.ntile || c >= TT.cl) continue;
      const double* r = S + rec_at(TT, yd, 0, tau, c, t);
#pragma unroll
      for (int m = 0; m < NF; m++)
        if (m != 4) fb[m] += r[slot_of(m) * TT.plane];
#pragma unroll
      for (int k = 0; k < NF; k++) qb[k] += r[(7 + k) * TT.plane];
    }
    {
      double q[NF];
#pragma unroll
      for (int k = 0; k < NF; k++) q[k] = X[g.at(yd ? swap_xy(k) : k, i, j)];
      flux_x_adjoint(G.gm, q, fb, qb);
      // constant indices on both branches (a runtime permutation would put part in local memory)
      if (yd) {
#pragma unroll
        for (int k = 0; k < NF; k++) part[swap_xy(k)] = qb[k];
      } else {
#pragma unroll
        for (int k = 0; k < NF; k++) part[k] = qb[k];
      }
    }
  }
  // lu = (0 + x part) + y part on both lanes of the pair
  double lu[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) {
    const double other = __shfl_xor_sync(0xffffffffu, part[k], 1);
    const double px = yd ? other : part[k], py = yd ? part[k] : other;
    lu[k] = (0.0 + px) + py;
  }
  if (!valid) return;
  const int k0 = yd ? 4 : 0;
  if (i >= 2 && i <= g.nx + 1 && j >= 2 && j <= g.ny + 1) {
    double* lbuf = in_buf == 0 ? lU : (in_buf == 1 ? lU1 : lU2);
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      const int k = k0 + kk;
      const long long ad = g.at(k, i, j);
      combine_adj_at(mode, ad, lU, lU1, lU2);
      lbuf[ad] += yd ? lu[4 + kk] : lu[kk];
    }
  } else {
#pragma unroll
    for (int kk = 0; kk < 4; kk++) T[g.at(k0 + kk, i, j)] = yd ? lu[4 + kk] : lu[kk];
  }
}

// Transpose of the boundary fill (k_bc / bc_elem), copy part, for field k
// and boundary cell c of one side: adds the adjoints of the side's two ghost
// layers (in T) to the interior cells of D they were copied from.
// Dirichlet ghosts hold the edge snapshot of the initial state, so their
// adjoints go to lsnap (the side's [8][NY] or [8][NX] array).  Every cell it
// adds to lies in field k, row / column c.
__device__ __forceinline__ void adj_bc_copy(const Grid& g, int side, int k, int c,
                                            const double* __restrict__ T,
                                            double* __restrict__ D,
                                            double* __restrict__ lsnap) {
  const bool xs = side == LEFT || side == RIGHT;
  const int b = g.bc_of(side);
  if (b == DIRICHLET) {
    const int len = xs ? g.NY : g.NX;
    double acc = 0.0;
    for (int gl = 1; gl <= 2; gl++) {
      if (side == LEFT) acc += T[g.at(k, 2 - gl, c)];
      else if (side == RIGHT) acc += T[g.at(k, g.nx + 1 + gl, c)];
      else if (side == BOTTOM) acc += T[g.at(k, c, 2 - gl)];
      else acc += T[g.at(k, c, g.ny + 1 + gl)];
    }
    lsnap[k * len + c] += acc;
    return;
  }
  for (int gl = 1; gl <= 2; gl++) {
    int gi, gj, si, sj;  // ghost cell, its source
    if (side == LEFT) {
      gi = 2 - gl; gj = c; sj = c;
      si = b == PERIODIC ? g.nx + 2 - gl : 2 + gl;
      if (b == NEUMANN && k == 4 && c >= 3 && c < g.ny + 1) si = gi + 2;
    } else if (side == RIGHT) {
      gi = g.nx + 1 + gl; gj = c; sj = c;
      si = b == PERIODIC ? 1 + gl : g.nx + 1 - gl;
      if (b == NEUMANN && k == 4 && c >= 3 && c < g.ny + 1) si = gi - 2;
    } else if (side == BOTTOM) {
      gj = 2 - gl; gi = c; si = c;
      sj = b == PERIODIC ? g.ny + 2 - gl : 2 + gl;
      if (b == NEUMANN && k == 5 && c >= 3 && c < g.nx + 1) sj = gj + 2;
    } else {
      gj = g.ny + 1 + gl; gi = c; si = c;
      sj = b == PERIODIC ? 1 + gl : g.ny + 1 - gl;
      if (b == NEUMANN && k == 5 && c >= 3 && c < g.nx + 1) sj = gj - 2;
    }
    D[g.at(k, si, sj)] += T[g.at(k, gi, gj)];
  }
}

// Transpose of the boundary fill, div B part, for boundary cell c of a
// Neumann side.  A left ghost Bx at row it, column c' reads By at row s5,
// columns c'-1 (coefficient -rxy) and c'+1 (+rxy); the target (By, s5, c)
// therefore collects -rxy * ghost(c+1) and +rxy * ghost(c-1).  The other
// sides mirror this.  The cells it adds to lie in field 5 (x sides) or 4
// (y sides), row / column c.
__device__ __forceinline__ void adj_bc_divb(const Grid& g, int side, int c,
                                            const double* __restrict__ T,
                                            double* __restrict__ D) {
  const bool xs = side == LEFT || side == RIGHT;
  const double rxy = g.dx / g.dy, ryx = g.dy / g.dx;
  for (int layer = 0; layer < 2; layer++) {
    if (xs) {
      int gi, s5;
      double cm, cp;  // coefficients of the ghosts at columns c+1 and c-1
      if (side == LEFT) {
        gi = layer;
        s5 = gi == 1 ? 2 : 3;
        cm = -rxy; cp = rxy;
      } else {  // right: -rxy * (By[j+1] - By[j-1])
        gi = g.nx + 2 + layer;
        s5 = gi == g.nx + 2 ? g.nx + 1 : g.nx;
        cm = rxy; cp = -rxy;
      }
      double acc = 0.0;
      if (c + 1 >= 3 && c + 1 < g.ny + 1) acc += cm * T[g.at(4, gi, c + 1)];
      if (c - 1 >= 3 && c - 1 < g.ny + 1) acc += cp * T[g.at(4, gi, c - 1)];
      D[g.at(5, s5, c)] += acc;
    } else {
      int gj, s4;
      double cm, cp;
      if (side == BOTTOM) {  // -ryx * (Bx[i-1] - Bx[i+1])
        gj = layer;
        s4 = gj == 1 ? 2 : 3;
        cm = -ryx; cp = ryx;
      } else {  // top: -ryx * (Bx[i+1] - Bx[i-1])
        gj = g.ny + 2 + layer;
        s4 = gj == g.ny + 2 ? g.ny + 1 : g.ny;
        cm = ryx; cp = -ryx;
      }
      double acc = 0.0;
      if (c + 1 >= 3 && c + 1 < g.nx + 1) acc += cm * T[g.at(5, c + 1, gj)];
      if (c - 1 >= 3 && c - 1 < g.nx + 1) acc += cp * T[g.at(5, c - 1, gj)];
      D[g.at(4, c, s4)] += acc;
    }
  }
}

// Transpose of the boundary fill for the two sides of one direction (x:
// left then right; y: bottom then top), one thread per field k and boundary
// cell c.  Everything a thread adds lands in field k, row / column c (the
// div B terms of a Neumann side are added by the thread of the field they
// land in), so no two threads add to the same cell, and every cell takes its
// terms in the order: low side copies, low side div B, high side copies,
// high side div B.  The x launch runs before the y launch, which keeps the
// order at the corners.
__global__ void ka_adj_bc(Grid g, int ydir, const double* __restrict__ T, double* __restrict__ D,
                          double* __restrict__ lsnap_lo, double* __restrict__ lsnap_hi) {
  pdl_wait();
  const int nb = ydir ? g.nx : g.ny;  // boundary cells along the sides
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= NF * nb) return;
  const int k = e / nb, c = 2 + e % nb;
  const int lo = ydir ? BOTTOM : LEFT, kdiv = ydir ? 4 : 5;
  for (int h = 0; h < 2; h++) {
    const int side = lo + h;
    adj_bc_copy(g, side, k, c, T, D, h ? lsnap_hi : lsnap_lo);
    if (k == kdiv && g.bc_of(side) == NEUMANN) adj_bc_divb(g, side, c, T, D);
  }
}

}  // namespace MHD_KNS

namespace adjrev {
namespace MHD_ADJREV {

namespace K = MHD_KNS;

size_t record_doubles(const Grid& g, bool ydir) {
  return (size_t)K::NPW * (size_t)K::itile(g, ydir).plane;
}

void launch_iface(const Grid& g, const GasConsts& gc, bool ydir, const double* X,
                  const unsigned* mask, const double* lB, double cL, double* S, double inv_d,
                  cudaStream_t st) {
  const K::Gas G{gc.gm, gc.g1, gc.g21, gc.rs2};
  const K::ITile T = K::itile(g, ydir);
  const int tpb = K::AIB / 32;  // interface tiles per block
  const int nb = int((T.ntile * (long long)((T.nt + T.bt - 1) / T.bt) + tpb - 1) / tpb);
  if (ydir)
    K::ka_adj_iface<true><<<nb, K::AIB, 0, st>>>(g, G, X, mask, lB, cL, S, inv_d);
  else
    K::ka_adj_iface<false><<<nb, K::AIB, 0, st>>>(g, G, X, mask, lB, cL, S, inv_d);
}

void launch_gather(const Grid& g, const GasConsts& gc, const double* X, const double* SX,
                   const double* SY, double* T, int mode, int in_buf, double* lU, double* lU1,
                   double* lU2, cudaStream_t st) {
  const K::Gas G{gc.gm, gc.g1, gc.g21, gc.rs2};
  const long long ncell = (long long)g.NX * g.NY;
  K::ka_adj_gather<<<int((2 * ncell + 127) / 128), 128, 0, st>>>(g, G, X, SX, SY, T, mode,
                                                                  in_buf, lU, lU1, lU2);
}

// The boundary transposes are a few thousand threads each: launched as
// programmatic dependents of the kernel before them (ka_adj_bc waits in
// pdl_wait), their launch latency overlaps that kernel's tail.
void launch_bc(const Grid& g, int ydir, const double* T, double* D, double* lsnap_lo,
               double* lsnap_hi, cudaStream_t st) {
  const int nb = ydir ? g.nx : g.ny;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((NF * nb + 127) / 128);
  cfg.blockDim = dim3(128);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, K::ka_adj_bc, g, ydir, T, D, lsnap_lo, lsnap_hi);
}

}  // namespace MHD_ADJREV
}  // namespace adjrev
}  // namespace mhd
