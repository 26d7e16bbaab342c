// Fused spatial operator L(U) for the ENO-Roe and ENO-LF schemes.
//
// One CTA owns a TI x TJ tile of interior cells (i rows, j columns; j is the
// contiguous direction).  It
//   0. stages the (TI+4) x (TJ+4) box of the 8 fields into shared memory,
//   1. computes the physical fluxes F (x) and G (y) once per cell
//      (SpatialMethodEno::updateFluxes, spatialmethodeno.cpp:89-127),
//   2. evaluates the (TI+1) x TJ x-interfaces and TI x (TJ+1) y-interfaces
//      the tile needs (getNumericalFluxF/G of the Roe and LF schemes), one
//      interface per lane, warp-uniform direction, and keeps the numerical
//      fluxes in shared memory,
//   3. forms UL = -(F_i - F_{i-1})/dx - (G_j - G_{j-1})/dy
//      (spatialmethodenoroe.cpp:169-176) and writes it to HBM,
// and folds max|lambda| of its interfaces into the context's CFL maxima.
// The reference runs these steps as separate full-grid passes with F, G,
// VUF, VUG, F_, G_ arrays in memory; here nothing but U and UL crosses HBM.
//
// Interface work per tile: x rows ii = -1..TI-1 (TI+1 warp tasks of TJ
// lanes), y rows of TJ lanes (TI tasks) plus the TI left-edge y interfaces
// (1 task).  With TI = 8, TJ = 32 that is 18 warp tasks, 3 per warp for 6
// warps.
#pragma once

#include "mhd_eigen.cuh"
#include "mhd_tma.cuh"

// Per-cell primitives in the tile (sP: u, v, w and the midpoint formula's
// total pressure), computed once per cell in phase 1 instead of once per
// interface side.  The fast build forms them with one reciprocal of the
// density; the parity build (MHD_PARITY_CELL_PRIM) with the reference's own
// divisions and operation order, so the midpoint (midpoint_p) is bit-identical.
#if defined(MHD_FAST) || defined(MHD_PARITY_CELL_PRIM)
#define MHD_CELL_PRIM 1
#endif

#ifndef MHD_MINB
#define MHD_MINB 2
#endif

// How pair_flux forms the characteristics of the fast (finite, structural
// zeros skipped) interface flux, per scheme: bit 0 pairs the left rows of
// the mirror waves k and 6 - k, bit 1 pairs their right rows; 0 forms one
// row at a time.  -1 keeps the streamed one-pass loop of interface_flux.
#ifndef MHD_PAIRS_ROE
#define MHD_PAIRS_ROE 3
#endif
#ifndef MHD_PAIRS_LF
#define MHD_PAIRS_LF 3
#endif
// ENO-Roe, streamed loop: 1 projects only the upwind side's stencil (see
// roe_side_flux), 0 all four points and three differences.
#ifndef MHD_ROE_SIDE
#define MHD_ROE_SIDE 1
#endif

#ifndef MHD_KNS
#define MHD_KNS exact
#endif

namespace mhd {
namespace MHD_KNS {

// Component -> slot of a 7-wide flux vector (column 4 is structurally 0).
__host__ __device__ constexpr int slot_of(int m) { return m < 4 ? m : m - 1; }
// x <-> y role swap of a state / flux component.
__host__ __device__ constexpr int swap_xy(int m) {
  return m == 1 ? 2 : m == 2 ? 1 : m == 4 ? 5 : m == 5 ? 4 : m;
}

struct CharOut {
  double *cx, *cy, *LUx, *LUy;  // pitched like U; null when not requested
};

template <int TI_, int TJ_>
struct TileGeom {
  static constexpr int TI = TI_, TJ = TJ_;
  static constexpr int RU = TI + 4, CU = TJ + 4;
  static constexpr int OFF_U = 0;
  static constexpr int OFF_F = OFF_U + NF * RU * CU;       // sF[7][RU][TJ]
  static constexpr int OFF_G = OFF_F + 7 * RU * TJ;        // sG[7][TI][CU], slots in y frame order
  static constexpr int OFF_FX = OFF_G + 7 * TI * CU;       // sFx[8][TI+1][TJ]
  static constexpr int OFF_GY = OFF_FX + 8 * (TI + 1) * TJ;  // sGy[8][TI][TJ+1], y frame order
#ifdef MHD_CELL_PRIM
  // per-cell primitives sP[4][RU][CU] (u, v, w, total pressure)
  static constexpr int OFF_P = OFF_GY + 8 * TI * (TJ + 1);
  static constexpr int TOTAL = OFF_P + 4 * RU * CU;
#else
  static constexpr int TOTAL = OFF_GY + 8 * TI * (TJ + 1);
#endif
  static constexpr size_t BYTES = size_t(TOTAL) * sizeof(double);
  static constexpr size_t TMA_BYTES = BYTES + 128;  // k_flux: room to align the box to 128 B
};

// Physical x / y fluxes of one cell, same arithmetic as updateFluxes.
__device__ __forceinline__ void phys_flux(double gm, const double* q, double* F, double* G) {
  const double r = q[0], mx = q[1], my = q[2], mz = q[3];
  const double bx = q[4], by = q[5], bz = q[6], en = q[7];
  const double u = mx / r, v = my / r, w = mz / r;
  const double uu = u * u + v * v + w * w;
  const double ub = u * bx + v * by + w * bz;
  const double bb = bx * bx + by * by + bz * bz;
  const double p = (gm - 1.0) * (en - 0.5 * r * uu - 0.5 * bb);
  const double pt = p + 0.5 * bb;
  F[0] = mx;
  F[1] = mx * u - bx * bx + pt;
  F[2] = my * u - bx * by;
  F[3] = mz * u - bx * bz;
  F[5] = by * u - bx * v;
  F[6] = bz * u - bx * w;
  F[7] = (en + pt) * u - bx * ub;
  G[0] = my;
  G[1] = mx * v - by * bx;
  G[2] = my * v - by * by + pt;
  G[3] = mz * v - by * bz;
  G[4] = bx * v - by * u;
  G[6] = bz * v - by * w;
  G[7] = (en + pt) * v - by * ub;
}

#ifdef MHD_FAST
// Fast build: the physical fluxes with one reciprocal of the density, and
// the cell's primitives P = (u, v, w, total pressure) for the midpoints of
// its four interfaces (midpoint_fast).
__device__ __forceinline__ void phys_flux_fast(double gm, const double* q, double* F, double* G,
                                               double* P) {
  const double r = q[0], mx = q[1], my = q[2], mz = q[3];
  const double bx = q[4], by = q[5], bz = q[6], en = q[7];
  const double ir = 1.0 / r;
  const double u = mx * ir, v = my * ir, w = mz * ir;
  const double uu = u * u + v * v + w * w;
  const double ub = u * bx + v * by + w * bz;
  const double bb = bx * bx + by * by + bz * bz;
  const double p = (gm - 1.0) * (en - 0.5 * r * uu - 0.5 * bb);
  const double pt = p + 0.5 * bb;
  F[0] = mx;
  F[1] = mx * u - bx * bx + pt;
  F[2] = my * u - bx * by;
  F[3] = mz * u - bx * bz;
  F[5] = by * u - bx * v;
  F[6] = bz * u - bx * w;
  F[7] = (en + pt) * u - bx * ub;
  G[0] = my;
  G[1] = mx * v - by * bx;
  G[2] = my * v - by * by + pt;
  G[3] = mz * v - by * bz;
  G[4] = bx * v - by * u;
  G[6] = bz * v - by * w;
  G[7] = (en + pt) * v - by * ub;
  P[0] = u;
  P[1] = v;
  P[2] = w;
  P[3] = pt;
}
#endif

// ENO-2 stencil choice on one characteristic (spatialmethodenoroe.cpp:240-254).
__device__ __forceinline__ double eno_minus(double w0, double w1, double w2, double v0, double v1) {
  return (fabs(v0) < fabs(v1)) ? (-(1.0 / 2.0) * w0 + (3.0 / 2.0) * w1)
                               : ((1.0 / 2.0) * w1 + (1.0 / 2.0) * w2);
}
__device__ __forceinline__ double eno_plus(double w1, double w2, double w3, double v1, double v2) {
  return (fabs(v1) < fabs(v2)) ? ((1.0 / 2.0) * w1 + (1.0 / 2.0) * w2)
                               : ((3.0 / 2.0) * w2 - (1.0 / 2.0) * w3);
}

// One lane's view of its interface stencil inside the shared tile.
struct Lane {
  const double* f;   // flux stencil point l of slot s at f[s*fplane + l*fstep]
  int fplane, fstep;
  const double* q;   // state stencil point l of field k at q[k*qplane + l*qstep]
  int qplane, qstep;
  bool swp;          // y interface: x/y roles swapped
  int l1, l2;        // stencil points of U1 / U2 (1 / 2, or open-boundary substitutes)
#ifdef MHD_CELL_PRIM
  const double* p;   // primitives (u, v, w, pt) of point l at p[k*qplane + l*qstep]
  __device__ __forceinline__ double P(int k, int l) const {
    return p[(swp && k < 2 ? 1 - k : k) * qplane + l * qstep];
  }
#endif
  // component 4 of a frame flux is identically zero (F[4], G[5]) and not stored
  __device__ __forceinline__ double F(int m, int l) const {
    return m == 4 ? 0.0 : f[slot_of(m) * fplane + l * fstep];
  }
  __device__ __forceinline__ double Q(int k, int l) const {
    return q[(swp ? swap_xy(k) : k) * qplane + l * qstep];
  }
};

// Upwind choice of the ENO-Roe flux of one characteristic from its
// projections w (4 points) and undivided differences vw (3 points)
// (spatialmethodenoroe.cpp:240-264).
__device__ __forceinline__ double roe_upwind(const double* w, const double* vw, double ak) {
  const double wm = eno_minus(w[0], w[1], w[2], vw[0], vw[1]);
  const double wp = eno_plus(w[1], w[2], w[3], vw[1], vw[2]);
  return (ak >= 0 && wm < 1.0e10) ? wm : ((ak <= 0 && wp < 1.0e10) ? wp : 0.0);
}

// ENO-Roe characteristic flux of one stencil side: s0 = 0 the ENO- side
// (differences 0, 1 pick points 0, 1 or 1, 2), s0 = 1 the ENO+ side
// (differences 1, 2 pick points 1, 2 or 2, 3); the same sums in the same
// order as the full projection (spatialmethodenoroe.cpp:240-254).
__device__ __forceinline__ double roe_side_value(const Lane& L, const double* l, unsigned lm,
                                                 int s0) {
#if defined(MHD_FAST) && MHD_FAST_ENO3
  // fast build: project the side's three stencil points once and take the
  // undivided differences of the projections (the reference projects the
  // differences of the fluxes, then two of the points again)
  double w0 = 0.0, w1 = 0.0, w2 = 0.0;
#pragma unroll
  for (int m = 0; m < NF; m++) {
    if (!(lm & (1u << m))) continue;
    w0 += l[m] * L.F(m, s0);
    w1 += l[m] * L.F(m, s0 + 1);
    w2 += l[m] * L.F(m, s0 + 2);
  }
  const bool left = fabs(w1 - w0) < fabs(w2 - w1);
  const int pa = s0 + (left ? 0 : 1);
  const double wa = left ? w0 : w1, wb = left ? w1 : w2;
  return pa == 0 ? (-(1.0 / 2.0) * wa + (3.0 / 2.0) * wb)
       : (pa == 1 ? ((1.0 / 2.0) * wa + (1.0 / 2.0) * wb)
                  : ((3.0 / 2.0) * wa - (1.0 / 2.0) * wb));
#else
  double va = 0.0, vb = 0.0;
#pragma unroll
  for (int m = 0; m < NF; m++) {
    if (!(lm & (1u << m))) continue;
    const double fa = L.F(m, s0), fb = L.F(m, s0 + 1), fc = L.F(m, s0 + 2);
    va += l[m] * (fb - fa);
    vb += l[m] * (fc - fb);
  }
  const int pa = s0 + (fabs(va) < fabs(vb) ? 0 : 1);
  double wa = 0.0, wb = 0.0;
#pragma unroll
  for (int m = 0; m < NF; m++) {
    if (!(lm & (1u << m))) continue;
    wa += l[m] * L.F(m, pa);
    wb += l[m] * L.F(m, pa + 1);
  }
  return pa == 0 ? (-(1.0 / 2.0) * wa + (3.0 / 2.0) * wb)
       : (pa == 1 ? ((1.0 / 2.0) * wa + (1.0 / 2.0) * wb)
                  : ((3.0 / 2.0) * wa - (1.0 / 2.0) * wb));
#endif
}

// ENO-Roe flux of characteristic k with left row l, projecting only what
// the reference's choice keeps (spatialmethodenoroe.cpp:240-264):
// fw = (lambda >= 0 && wm < 1e10) ? wm : ((lambda <= 0 && wp < 1e10) ? wp : 0).
// The reference projects the fluxes at all 4 stencil points and their 3
// undivided differences; here the upwind side is projected alone (4 of the
// 7 dot products): ENO- for lambda >= 0, ENO+ for lambda < 0.  Only lambda
// = 0 with wm >= 1e10 (or NaN) needs ENO+ as well; a NaN lambda gives 0.
__device__ __forceinline__ double roe_side_flux(const Lane& L, const double* l, unsigned lm,
                                                double ak) {
  if (ak != ak) return 0.0;
  const double v = roe_side_value(L, l, lm, ak >= 0.0 ? 0 : 1);
  if (v < 1.0e10) return v;
  if (!(ak == 0.0)) return 0.0;
  const double wp = roe_side_value(L, l, lm, 1);
  return wp < 1.0e10 ? wp : 0.0;
}

// ENO-Roe flux of a characteristic under a recorded choice code c (bits 0-1:
// the ENO- / ENO+ stencil took the left pair, bits 2-3: upwind choice 0 wm,
// 1 wp, 2 zero): the frozen-stencil replay projects only the two stencil
// points of the recorded pair, the same sums in the same order as the
// recording.
__device__ __forceinline__ double roe_frozen_flux(const Lane& L, const double* l, unsigned lm,
                                                  unsigned c) {
  const int up = int(c >> 2);
  if (up == 2) return 0.0;
  // points pa, pa + 1; pa = 0: -(1/2) wa + (3/2) wb, 1: (1/2) wa + (1/2) wb,
  // 2: (3/2) wa - (1/2) wb
  const int pa = up == 0 ? ((c & 1u) ? 0 : 1) : ((c & 2u) ? 1 : 2);
  double wa = 0.0, wb = 0.0;
#pragma unroll
  for (int m = 0; m < NF; m++) {
    if (!(lm & (1u << m))) continue;
    wa += l[m] * L.F(m, pa);
    wb += l[m] * L.F(m, pa + 1);
  }
  return pa == 0 ? (-(1.0 / 2.0) * wa + (3.0 / 2.0) * wb)
       : (pa == 1 ? ((1.0 / 2.0) * wa + (1.0 / 2.0) * wb)
                  : ((3.0 / 2.0) * wa - (1.0 / 2.0) * wb));
}

// ENO-LF flux of one characteristic from its projections of the state (ru)
// and of the flux (rf) at the 4 stencil points and its dissipation
// coefficient al (spatialmethodenolf.cpp:276-326).
__device__ __forceinline__ double lf_split(const double* ru, const double* rf, double al) {
  double w[4];
#pragma unroll
  for (int p = 0; p < 4; p++) w[p] = 0.5 * (rf[p] + al * ru[p]);
  const double wm = eno_minus(w[0], w[1], w[2], w[1] - w[0], w[2] - w[1]);
#pragma unroll
  for (int p = 0; p < 4; p++) w[p] = 0.5 * (rf[p] - al * ru[p]);
  const double wp = eno_plus(w[1], w[2], w[3], w[2] - w[1], w[3] - w[2]);
  return wm + wp;
}

// Left row k of a characteristic projected on the stencil: the ENO-Roe
// projections of the fluxes and their undivided differences, or the ENO-LF
// projections of the state and the fluxes, reduced to the characteristic
// flux fw; LU gets lv.U1 (Roe) or lv.U at point 1 (LF).  Two rows at once
// (TWO) share the stencil reads and the differences.
template <int SCHEME, bool CHARS, bool TWO, int MASK>
__device__ __forceinline__ void project_rows(const Mid& e, const Lane& L, const double* U1,
                                             const double* alpha, int ka, int kb,
                                             const double* la, const double* lb, double* fw,
                                             double* LU, unsigned mw) {
  const unsigned lm = lv_mask(ka);  // == lv_mask(kb)
  if constexpr (SCHEME == 2 && (MASK == 2 || MHD_ROE_SIDE)) {
    if constexpr (MASK == 2) {
      fw[ka] = roe_frozen_flux(L, la, lm, (mw >> (4 * ka)) & 0xFu);
      if (TWO) fw[kb] = roe_frozen_flux(L, lb, lm, (mw >> (4 * kb)) & 0xFu);
    } else {
      fw[ka] = roe_side_flux(L, la, lm, eigenvalue(e, ka));
      if (TWO) fw[kb] = roe_side_flux(L, lb, lm, eigenvalue(e, kb));
    }
    if (CHARS) {
      double acc = 0.0, acb = 0.0;
#pragma unroll
      for (int m = 0; m < NF; m++)
        if (lm & (1u << m)) {
          acc += la[m] * U1[m];
          if (TWO) acb += lb[m] * U1[m];
        }
      LU[ka] = acc;
      if (TWO) LU[kb] = acb;
    }
  } else if constexpr (SCHEME == 2) {
    double wa[4] = {0.0, 0.0, 0.0, 0.0}, va[3] = {0.0, 0.0, 0.0};
    double wb[4] = {0.0, 0.0, 0.0, 0.0}, vb[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int m = 0; m < NF; m++) {
      if (!(lm & (1u << m))) continue;
      const double f0 = L.F(m, 0), f1 = L.F(m, 1), f2 = L.F(m, 2), f3 = L.F(m, 3);
      const double d0 = f1 - f0, d1 = f2 - f1, d2 = f3 - f2;
      wa[0] += la[m] * f0;
      wa[1] += la[m] * f1;
      wa[2] += la[m] * f2;
      wa[3] += la[m] * f3;
      va[0] += la[m] * d0;
      va[1] += la[m] * d1;
      va[2] += la[m] * d2;
      if (TWO) {
        wb[0] += lb[m] * f0;
        wb[1] += lb[m] * f1;
        wb[2] += lb[m] * f2;
        wb[3] += lb[m] * f3;
        vb[0] += lb[m] * d0;
        vb[1] += lb[m] * d1;
        vb[2] += lb[m] * d2;
      }
    }
    fw[ka] = roe_upwind(wa, va, eigenvalue(e, ka));
    if (TWO) fw[kb] = roe_upwind(wb, vb, eigenvalue(e, kb));
    if (CHARS) {
      double acc = 0.0, acb = 0.0;
#pragma unroll
      for (int m = 0; m < NF; m++)
        if (lm & (1u << m)) {
          acc += la[m] * U1[m];
          if (TWO) acb += lb[m] * U1[m];
        }
      LU[ka] = acc;
      if (TWO) LU[kb] = acb;
    }
  } else {
    double rua[4], rfa[4], rub[4], rfb[4];
#pragma unroll
    for (int p = 0; p < 4; p++) {
      double a = 0.0, b = 0.0, c = 0.0, d = 0.0;
#pragma unroll
      for (int m = 0; m < NF; m++)
        if (lm & (1u << m)) {
          const double q = L.Q(m, p), f = L.F(m, p);
          a += la[m] * q;
          b += la[m] * f;
          if (TWO) {
            c += lb[m] * q;
            d += lb[m] * f;
          }
        }
      rua[p] = a; rfa[p] = b; rub[p] = c; rfb[p] = d;
    }
    fw[ka] = lf_split(rua, rfa, alpha[ka]);
    if (TWO) fw[kb] = lf_split(rub, rfb, alpha[kb]);
    if (CHARS) {
      LU[ka] = rua[1];
      if (TWO) LU[kb] = rub[1];
    }
  }
}

// Characteristics 0..6 of one interface (SCHEME 2 ENO-Roe, 3 ENO-LF), fast
// form (finite values, structural zeros skipped), in two passes: the left
// rows give the 7 characteristic fluxes fw, the right rows project them
// back.
//
// The rows of the mirror waves k and 6 - k are sums and differences of the
// same products (spatialmethodeno.cpp:392-552).  LV_PAIRS forms both left
// rows of a pair together, so the shared products are formed once and one
// pass over the stencil serves both.  RV_PAIRS does the same for the right
// rows; the back projection must still add the waves in the order 0..6
// like the reference's loop, so the products of waves 6, 5, 4 (rounded on
// their own, as the unfused build rounds every product) wait in registers
// and are added after wave 3.  Every value is the reference's expression in
// the reference's order, so all forms give the same bits.
template <int SCHEME, bool CHARS, bool LV_PAIRS, bool RV_PAIRS, int MASK>
__device__ __forceinline__ void pair_flux(Mid& e, const Gas& G, const Lane& L, const double* U1,
                                          const double* alpha, double* Fn, double* LU,
                                          bool& nonfinite, unsigned mw) {
  double fw[7];
  if constexpr (LV_PAIRS) {
#pragma unroll
    for (int t = 0; t < 4; t++) {
      opaque(e);
      double la[NF], lb[NF];
      lv_row(e, G, t, la);
      if (t < 3) {
        lv_row(e, G, 6 - t, lb);
        project_rows<SCHEME, CHARS, true, MASK>(e, L, U1, alpha, t, 6 - t, la, lb, fw, LU, mw);
      } else {
        project_rows<SCHEME, CHARS, false, MASK>(e, L, U1, alpha, t, t, la, la, fw, LU, mw);
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < 7; k++) {
      opaque(e);
      double l[NF];
      lv_row(e, G, k, l);
      project_rows<SCHEME, CHARS, false, MASK>(e, L, U1, alpha, k, k, l, l, fw, LU, mw);
    }
  }
#pragma unroll
  for (int k = 0; k < 7; k++)
    if (!isfinite(fw[k])) nonfinite = true;

  if constexpr (RV_PAIRS) {
#ifdef MHD_FAST
    // fast build: the pair's two products go into the sums at once (any
    // order of the seven terms is within the tolerance), with the rows'
    // divisions taken through the midpoint's reciprocals
#pragma unroll
    for (int t = 0; t < 4; t++) {
      opaque(e);
      const bool two = t < 3;
      double qa[NF], qb[NF];
      rv_row<true>(e, G, t, qa);
      if (two) rv_row<true>(e, G, 6 - t, qb);
      const unsigned rm = rv_mask(t);  // == rv_mask(6 - t)
#pragma unroll
      for (int m = 0; m < NF; m++)
        if (rm & (1u << m)) {
          Fn[m] += qa[m] * fw[t];
          if (two) Fn[m] += qb[m] * fw[6 - t];
        }
    }
#else
    double h[3][NF];
#pragma unroll
    for (int t = 0; t < 4; t++) {
      opaque(e);
      const bool two = t < 3;
      double qa[NF], qb[NF];
      rv_row(e, G, t, qa);
      if (two) rv_row(e, G, 6 - t, qb);
      const unsigned rm = rv_mask(t);  // == rv_mask(6 - t)
#pragma unroll
      for (int m = 0; m < NF; m++)
        if (rm & (1u << m)) {
          Fn[m] += qa[m] * fw[t];
          if (two) h[t][m] = qb[m] * fw[6 - t];
        }
    }
#pragma unroll
    for (int t = 2; t >= 0; t--) {  // waves 4, 5, 6
      const unsigned rm = rv_mask(t);
#pragma unroll
      for (int m = 0; m < NF; m++)
        if (rm & (1u << m)) Fn[m] += h[t][m];
    }
#endif
  } else {
#pragma unroll
    for (int k = 0; k < 7; k++) {
      opaque(e);
      double q[NF];
      rv_row(e, G, k, q);
      const unsigned rm = rv_mask(k);
#pragma unroll
      for (int m = 0; m < NF; m++)
        if (rm & (1u << m)) Fn[m] += q[m] * fw[k];
    }
  }
  // the dummy wave 7 contributes +0 * +0 last in the reference's sums
#pragma unroll
  for (int m = 0; m < NF; m++)
    if (m != 4) Fn[m] = Fn[m] + 0.0;
  if (CHARS) LU[7] = 0.0;
}

// Numerical flux of one interface in the lane's frame: Fn[m], m = 0..7 (Fn[4]
// is the structurally zero component), lam / LU the characteristic outputs.
//
// DENSE = false, the fast form: characteristics 0..6 only, structurally
// zero products skipped.  Skipping a product 0*x changes nothing while every
// x is finite; *nonfinite reports a characteristic flux that is not (the
// reference's 0*inf, 0*NaN would then turn "zero" components into NaN).
// DENSE = true performs every product of the reference's dense 8x8 loops,
// the dummy wave 7 included, and so reproduces its NaN / inf propagation
// exactly; the kernel recomputes flagged interfaces this way.
// MASK (ENO-Roe only): 0 plain; 1 records, per characteristic k, a 4-bit
// code in bits 4k..4k+3 of *mw (bit 0: the ENO- stencil took the left
// pair, bit 1: the ENO+ stencil took the left pair, bits 2-3: upwind choice
// 0 wm, 1 wp, 2 zero); 2 replays the choices stored in *mw instead of
// comparing (the frozen-stencil forward of the adjoint).
template <int SCHEME, bool CHARS, bool DENSE, int MASK = 0>
__device__ __forceinline__ bool interface_flux(const Gas& G, const Lane& L, const double* alpha,
                                               double* Fn, double& smax, int& negp,
                                               double* lam, double* LU, bool& nonfinite,
                                               unsigned* mw = nullptr) {
  double U1[NF], U2[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) {
    U1[k] = L.Q(k, L.l1);
    U2[k] = L.Q(k, L.l2);
  }
  Mid e;
#ifdef MHD_CELL_PRIM
  if (!DENSE) {
    double P1[4], P2[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      P1[k] = L.P(k, L.l1);
      P2[k] = L.P(k, L.l2);
    }
#ifdef MHD_FAST
    if (!midpoint_fast(G, U1, U2, P1, P2, e)) return false;
#else
    if (!midpoint_p(G, U1, U2, P1, P2, e)) return false;
#endif
  } else if (!midpoint(G, U1, U2, e)) {
    return false;
  }
#else
  if (!midpoint(G, U1, U2, e)) return false;
#endif
  negp = e.negp;
  smax = 0.0;
#pragma unroll
  for (int k = 0; k < NF; k++) {
    const double lk = eigenvalue(e, k);
    if (CHARS) lam[k] = lk;
    smax = take_max(smax, fabs(lk));
  }
#pragma unroll
  for (int m = 0; m < NF; m++) Fn[m] = 0.0;

  constexpr int PAIRS = SCHEME == 2 ? MHD_PAIRS_ROE : MHD_PAIRS_LF;
  if constexpr (!DENSE && (MASK == 0 || (MASK == 2 && SCHEME == 2)) && PAIRS >= 0) {
    pair_flux<SCHEME, CHARS, (PAIRS & 1) != 0, (PAIRS & 2) != 0, MASK>(
        e, G, L, U1, alpha, Fn, LU, nonfinite, MASK == 2 ? *mw : 0u);
    return true;
  }

  constexpr int KN = DENSE ? 8 : 7;
#ifndef MHD_K_UNROLL
#define MHD_K_UNROLL 7
#endif
  constexpr int kUnroll = MHD_K_UNROLL;
#pragma unroll kUnroll
  for (int k = 0; k < KN; k++) {
    opaque(e);
    double l[NF];
    if (DENSE) {
#pragma unroll
      for (int m = 0; m < NF; m++) l[m] = 0.0;
    }
    lv_row(e, G, k, l);
    const unsigned lm = DENSE ? 0xFFu : lv_mask(k);
    double fw;
    if constexpr (SCHEME == 2 && MASK == 2 && !DENSE) {
      // frozen replay: only the upwind side's two stencil points are
      // projected (the same sums, in the same order, as the recording's)
      const unsigned c = (*mw >> (4 * k)) & 0xFu;
      const int up = int(c >> 2);
      fw = 0.0;
      if (up != 2) {
        // points pa, pa + 1; pa = 0: -(1/2) wa + (3/2) wb, 1: (1/2) wa + (1/2) wb,
        // 2: (3/2) wa - (1/2) wb
        const int pa = up == 0 ? ((c & 1u) ? 0 : 1) : ((c & 2u) ? 1 : 2);
        double wa = 0.0, wb = 0.0;
#pragma unroll
        for (int m = 0; m < NF; m++) {
          if (!(lm & (1u << m))) continue;
          wa += l[m] * L.F(m, pa);
          wb += l[m] * L.F(m, pa + 1);
        }
        fw = pa == 0 ? (-(1.0 / 2.0) * wa + (3.0 / 2.0) * wb)
           : (pa == 1 ? ((1.0 / 2.0) * wa + (1.0 / 2.0) * wb)
                        : ((3.0 / 2.0) * wa - (1.0 / 2.0) * wb));
      }
    } else if (SCHEME == 2 && MASK == 0 && !DENSE && MHD_ROE_SIDE) {
      fw = roe_side_flux(L, l, lm, eigenvalue(e, k));
    } else if (SCHEME == 2) {  // ENO-Roe: project F and its undivided differences
      // w = lv.F at the 4 points, Vw = lv.(F[p+1] - F[p]) at 3 points; each
      // sum runs over m in ascending order, like the reference's loops
      double w[4] = {0.0, 0.0, 0.0, 0.0}, vw[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int m = 0; m < NF; m++) {
        if (!(lm & (1u << m))) continue;
        const double f0 = L.F(m, 0), f1 = L.F(m, 1), f2 = L.F(m, 2), f3 = L.F(m, 3);
        w[0] += l[m] * f0;
        w[1] += l[m] * f1;
        w[2] += l[m] * f2;
        w[3] += l[m] * f3;
        vw[0] += l[m] * (f1 - f0);
        vw[1] += l[m] * (f2 - f1);
        vw[2] += l[m] * (f3 - f2);
      }
      if constexpr (MASK == 0) {
        const double wm = eno_minus(w[0], w[1], w[2], vw[0], vw[1]);
        const double wp = eno_plus(w[1], w[2], w[3], vw[1], vw[2]);
        const double ak = eigenvalue(e, k);
        fw = (ak >= 0 && wm < 1.0e10) ? wm : ((ak <= 0 && wp < 1.0e10) ? wp : 0.0);
      } else {
        bool em, ep;
        int up;
        if constexpr (MASK == 1) {
          em = fabs(vw[0]) < fabs(vw[1]);
          ep = fabs(vw[1]) < fabs(vw[2]);
        } else {
          const unsigned c = (*mw >> (4 * k)) & 0xFu;
          em = (c & 1u) != 0;
          ep = (c & 2u) != 0;
        }
        const double wm = em ? (-(1.0 / 2.0) * w[0] + (3.0 / 2.0) * w[1])
                             : ((1.0 / 2.0) * w[1] + (1.0 / 2.0) * w[2]);
        const double wp = ep ? ((1.0 / 2.0) * w[1] + (1.0 / 2.0) * w[2])
                             : ((3.0 / 2.0) * w[2] - (1.0 / 2.0) * w[3]);
        if constexpr (MASK == 1) {
          const double ak = eigenvalue(e, k);
          up = (ak >= 0 && wm < 1.0e10) ? 0 : ((ak <= 0 && wp < 1.0e10) ? 1 : 2);
          *mw |= (unsigned(em) | (unsigned(ep) << 1) | (unsigned(up) << 2)) << (4 * k);
        } else {
          up = int((*mw >> (4 * k + 2)) & 3u);
        }
        fw = up == 0 ? wm : (up == 1 ? wp : 0.0);
      }
    } else {  // ENO-LF: split w = (RF +- alpha RU)/2, ENO on each half
      double ru[4], rf[4];
#pragma unroll
      for (int p = 0; p < 4; p++) {
        double a = 0.0, b = 0.0;
#pragma unroll
        for (int m = 0; m < NF; m++)
          if (lm & (1u << m)) {
            a += l[m] * L.Q(m, p);
            b += l[m] * L.F(m, p);
          }
        ru[p] = a;
        rf[p] = b;
      }
      const double al = alpha[k];
      double w[4];
#pragma unroll
      for (int p = 0; p < 4; p++) w[p] = 0.5 * (rf[p] + al * ru[p]);
      const double wm = eno_minus(w[0], w[1], w[2], w[1] - w[0], w[2] - w[1]);
#pragma unroll
      for (int p = 0; p < 4; p++) w[p] = 0.5 * (rf[p] - al * ru[p]);
      const double wp = eno_plus(w[1], w[2], w[3], w[2] - w[1], w[3] - w[2]);
      fw = wm + wp;
      if (CHARS) LU[k] = ru[1];
    }
    if (!DENSE && !isfinite(fw)) nonfinite = true;
    if (CHARS && SCHEME == 2) {
      double acc = 0.0;
#pragma unroll
      for (int m = 0; m < NF; m++)
        if (lm & (1u << m)) acc += l[m] * U1[m];
      LU[k] = acc;
    }
    double q[NF];
    if (DENSE) {
#pragma unroll
      for (int m = 0; m < NF; m++) q[m] = 0.0;
    }
    rv_row(e, G, k, q);
    const unsigned rm = DENSE ? 0xFFu : rv_mask(k);
#pragma unroll
    for (int m = 0; m < NF; m++)
      if (rm & (1u << m)) Fn[m] += q[m] * fw;
  }
  if (!DENSE) {
    // the dummy wave 7 contributes +0 * +0 last in the reference's sums
#pragma unroll
    for (int m = 0; m < NF; m++)
      if (m != 4) Fn[m] = Fn[m] + 0.0;
    if (CHARS) LU[7] = 0.0;
  }
  return true;
}

// One tile of the spatial operator: interior cells i0 = 2 + ti*TI .. +TI,
// j0 = 2 + tj*TJ .. +TJ.  Every thread of the CTA calls it with the same
// (tj, ti); the kernel provides TileGeom::BYTES of dynamic shared memory.  A
// caller that runs several tiles in a row separates them with
// __syncthreads().
template <int SCHEME, bool CHARS, int TI, int TJ, int NW, int MASK = 0>
__device__ __forceinline__ void flux_tile(const Grid& g, const double* __restrict__ U,
                                          double* __restrict__ UL,
                                          const double* __restrict__ alphaF,
                                          const double* __restrict__ alphaG, double inv_dx,
                                          double inv_dy, const Gas& G, Ctl* ctl, const CharOut& co,
                                          int tj, int ti, unsigned* maskX = nullptr,
                                          unsigned* maskY = nullptr) {
#include "mhd_flux_tile.inc"
}

// maskX / maskY: ENO choice words of the x / y interfaces ([NX][NY] by the
// interface's left / lower cell), written (MASK 1) or read (MASK 2).
template <int SCHEME, bool CHARS, int TI, int TJ, int NW, int MASK = 0>
__global__ void __launch_bounds__(NW * 32, NW * 32 > 256 ? 1 : MHD_MINB)
k_flux(Grid g, const double* __restrict__ U, double* __restrict__ UL,
       const double* __restrict__ alphaF, const double* __restrict__ alphaG,
       double inv_dx, double inv_dy, Gas G, Ctl* ctl, CharOut co, unsigned* maskX,
       unsigned* maskY, const __grid_constant__ CUtensorMap tmU, int use_tma, int ti0) {
  if (ctl->skip) return;
  const int tj = blockIdx.x, ti = ti0 + blockIdx.y;  // ti0: first tile row of this launch
#define MHD_TILE_TMA 1
#include "mhd_flux_tile.inc"
#undef MHD_TILE_TMA
}

// ENO-LF dissipation coefficients (spatialmethodenolf.cpp:66-125):
// alphaF[k][j] = max_i |lambda_k(U_ij)|, alphaG[k][i] = max_j |lambda_k(swap U_ij)|
// over i in [1, nx+2), j in [1, ny+2) without the (i < 2 && j < 2) corner.
// The arrays must be zero on entry.  Block = 32 (j) x 8 (i) cells.  Like the
// reference's "if( alphaabs > alpha ) alpha = alphaabs" a NaN eigenvalue
// never enters a maximum: each cell contributes max(0, |lambda|) first.
// One 32 x 8 block of cells (bx, by); all 256 threads call it with the same
// block, col is a shared [8][NF][33] scratch.
__device__ __forceinline__ void lf_alpha_block(const Grid& g, const double* __restrict__ U,
                                               double* alphaF, double* alphaG, Ctl* ctl, int bx,
                                               int by, double (*col)[NF][33]) {
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int j = 1 + bx * 32 + tx, i = 1 + by * 8 + ty;
  double lx[NF], ly[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) { lx[k] = 0.0; ly[k] = 0.0; }
  const bool valid = (i < g.nx + 2) && (j < g.ny + 2) && !(i < 2 && j < 2);
  int negp = 0;
  if (valid) {
    double q[NF], lam[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) q[k] = U[g.at(k, i, j)];
    int np;
    if (!eigenvalues_at(g.gamma, q, lam, np)) {
      atomicExch(&ctl->error, 6);
      atomicAdd(&ctl->negd_count, 1ull);
    } else {
      negp += np;
#pragma unroll
      for (int k = 0; k < NF; k++) lx[k] = take_max(0.0, fabs(lam[k]));
      double s[NF];
#pragma unroll
      for (int k = 0; k < NF; k++) s[k] = q[swap_xy(k)];
      eigenvalues_at(g.gamma, s, lam, np);
      negp += np;
#pragma unroll
      for (int k = 0; k < NF; k++) ly[k] = take_max(0.0, fabs(lam[k]));
    }
  }
  // per-row (alphaG, over j = lanes) maxima
#pragma unroll
  for (int k = 0; k < NF; k++) {
    const double m = warp_max(ly[k]);
    if (tx == 0 && i < g.nx + 2) atomic_max_pos(reinterpret_cast<unsigned long long*>(&alphaG[k * g.NX + i]), m);
  }
  // per-column (alphaF, over i = warps) maxima
#pragma unroll
  for (int k = 0; k < NF; k++) col[ty][k][tx] = lx[k];
  __syncthreads();
  if (ty == 0 && j < g.ny + 2) {
#pragma unroll
    for (int k = 0; k < NF; k++) {
      double m = 0.0;
#pragma unroll
      for (int r = 0; r < 8; r++) m = take_max(m, col[r][k][tx]);
      atomic_max_pos(reinterpret_cast<unsigned long long*>(&alphaF[k * g.NY + j]), m);
    }
  }
  (void)negp;
}

__global__ void __launch_bounds__(256)
k_lf_alpha(Grid g, const double* __restrict__ U, double* alphaF, double* alphaG, Ctl* ctl) {
  if (ctl->skip) return;
  __shared__ double col[8][NF][33];
  lf_alpha_block(g, U, alphaF, alphaG, ctl, blockIdx.x, blockIdx.y, col);
}

}  // namespace MHD_KNS
}  // namespace mhd
