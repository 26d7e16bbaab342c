// Midpoint eigen-system of ideal MHD for the x-direction flux, evaluated one
// characteristic at a time.
//
// Follows SpatialMethodEno::getEigensF (spatialmethodeno.cpp:288-571):
// arithmetic-mean midpoint state (not a sqrt(rho)-weighted Roe average),
// pressure from the mean total pressure clamped at zero, the 8-wave
// right/left eigenvectors with the alpha_f / alpha_s / beta normalisation
// and the sign flips that keep the fast and slow vectors continuous across
// By = 0.  Row 7 (the dummy wave) and column 4 (Bx) are structurally zero
// and never formed; the other rows are produced on demand, so a thread holds
// ~25 midpoint scalars plus one row instead of two dense 8x8 matrices.
//
// Every expression keeps the reference's association order; the parity
// build compiles this with -fmad=false, which makes each entry bit-identical
// to the reference's x86-64 double arithmetic (IEEE division and sqrt on
// both sides).  Products with the sign factors sgn(Bx), cffactor and
// csfactor (exactly +-1) are applied as sign-bit flips, which give the same
// bits as the multiplication and keep the FP64 pipe free.  The y direction
// uses the same code on x/y-swapped inputs, as getEigensG /
// getNumericalFluxG do (spatialmethodeno.cpp:574-598).
#pragma once

#include "mhd_common.cuh"

#ifndef MHD_KNS
#define MHD_KNS exact
#endif

namespace mhd {
namespace MHD_KNS {

// gamma and the gamma-only quantities the formulas use, computed once on
// the host in the same IEEE arithmetic: g1 = gamma - 1, g21 = (gamma - 2) /
// (gamma - 1), rs2 = 1 / sqrt(2).
struct Gas {
  double gm, g1, g21, rs2;
#ifdef MHD_FAST
  double ig1;  // 1 / (gamma - 1)
#endif
};

struct Mid {
  double u, v, w, uu;
  double a2, a, ca2, ca, cs2, cs, cf2, cf;
  double rr, af2, af, as2, as, bty, btz, th1, th2, vb;
#ifdef MHD_FAST
  double irr, icfrr;  // 1 / sqrt(rho), 1 / (c_f sqrt(rho))
#endif
  unsigned sbxm, fcfm, fcsm;  // sign-bit masks of sgn(Bx), cffactor, csfactor
  int negp;                   // midpoint pressure was negative and clamped
};

// x * s for s = +-1 given as a mask of the sign bit of the high word.
__device__ __forceinline__ double flip(double x, unsigned m) {
  return __hiloint2double(__double2hiint(x) ^ (int)m, __double2loint(x));
}

// Products of midpoint().  A translation unit compiled with FMA contraction
// that must still take the uncontracted builds' branches at the midpoint
// (the discrete adjoint's reverse sweep recomputes the recording's midpoint)
// defines MHD_MIDPOINT_UNFUSED: __dmul_rn is never fused into an FMA, so the
// midpoint keeps the parity build's rounding there.  Elsewhere MP_MUL is the
// plain product.
#ifdef MHD_MIDPOINT_UNFUSED
#define MP_MUL(a, b) __dmul_rn((a), (b))
#else
#define MP_MUL(a, b) ((a) * (b))
#endif

// The midpoint state from the averaged density r, velocity (in e.u, e.v,
// e.w), field (bx, by, bz) and total pressure pt.
__device__ __forceinline__ bool midpoint_rest(const Gas& G, double r, double bx, double by,
                                              double bz, double pt, Mid& e);

// One side's total pressure as the midpoint forms it: (gamma - 1)(E -
// |m|^2 / (2 rho) - |B|^2 / 2) + |B|^2 / 2.  The sums of squares are
// frame-independent (the y frame swaps two of the terms of an addition).
__device__ __forceinline__ double side_total_pressure(double gm, const double* q) {
  const double mm = MP_MUL(q[1], q[1]) + MP_MUL(q[2], q[2]) + MP_MUL(q[3], q[3]);
  const double bb = MP_MUL(q[4], q[4]) + MP_MUL(q[5], q[5]) + MP_MUL(q[6], q[6]);
  return MP_MUL(gm - 1.0, q[7] - MP_MUL(0.5, mm) / q[0] - MP_MUL(0.5, bb)) + MP_MUL(0.5, bb);
}

// Returns false on non-positive midpoint density (the reference's
// ErrorNegativeDensity, spatialmethodeno.cpp:307-310).
__device__ __forceinline__ bool midpoint(const Gas& G, const double* U1, const double* U2, Mid& e) {
  const double r = MP_MUL(0.5, U1[0] + U2[0]);
  e.u = MP_MUL(0.5, U1[1] / U1[0] + U2[1] / U2[0]);
  e.v = MP_MUL(0.5, U1[2] / U1[0] + U2[2] / U2[0]);
  e.w = MP_MUL(0.5, U1[3] / U1[0] + U2[3] / U2[0]);
  const double bx = MP_MUL(0.5, U1[4] + U2[4]);
  const double by = MP_MUL(0.5, U1[5] + U2[5]);
  const double bz = MP_MUL(0.5, U1[6] + U2[6]);
  if (r <= 0.0) return false;
  const double pt = MP_MUL(0.5, side_total_pressure(G.gm, U1) + side_total_pressure(G.gm, U2));
  return midpoint_rest(G, r, bx, by, bz, pt, e);
}

// Per-cell part of the midpoint (the cell's velocity components and total
// pressure, P = (u, v, w, pt) in x-frame order) for midpoint_p.
__device__ __forceinline__ void cell_primitives(double gm, const double* q, double* P) {
  P[0] = q[1] / q[0];
  P[1] = q[2] / q[0];
  P[2] = q[3] / q[0];
  P[3] = side_total_pressure(gm, q);
}

// midpoint() from the two sides' cell_primitives (P1, P2 in the interface's
// frame): the same values in the same operations, the per-side divisions
// done once per cell.
__device__ __forceinline__ bool midpoint_p(const Gas& G, const double* U1, const double* U2,
                                           const double* P1, const double* P2, Mid& e) {
  const double r = MP_MUL(0.5, U1[0] + U2[0]);
  e.u = MP_MUL(0.5, P1[0] + P2[0]);
  e.v = MP_MUL(0.5, P1[1] + P2[1]);
  e.w = MP_MUL(0.5, P1[2] + P2[2]);
  const double bx = MP_MUL(0.5, U1[4] + U2[4]);
  const double by = MP_MUL(0.5, U1[5] + U2[5]);
  const double bz = MP_MUL(0.5, U1[6] + U2[6]);
  if (r <= 0.0) return false;
  const double pt = MP_MUL(0.5, P1[3] + P2[3]);
  return midpoint_rest(G, r, bx, by, bz, pt, e);
}

__device__ __forceinline__ bool midpoint_rest(const Gas& G, double r, double bx, double by,
                                              double bz, double pt, Mid& e) {
  const double gm = G.gm;
  const double u = e.u, v = e.v, w = e.w;
  e.uu = MP_MUL(u, u) + MP_MUL(v, v) + MP_MUL(w, w);
  const double bb = MP_MUL(bx, bx) + MP_MUL(by, by) + MP_MUL(bz, bz);
  double p = pt - MP_MUL(0.5, bb);
  e.negp = 0;
  if (p < 0.0) { p = 0.0; e.negp = 1; }

  double a2 = MP_MUL(gm, p) / r;
  if (a2 < 0.0) a2 = 0.0;
  e.a2 = a2;
  e.a = sqrt(a2);
  e.ca2 = MP_MUL(bx, bx) / r;
  e.ca = sqrt(e.ca2);
  const double c2 = MP_MUL(0.5, bb / r + a2);
  double ct = MP_MUL(c2, c2) - MP_MUL(a2, e.ca2);
  if (ct < 0.0) ct = 0.0;
  const double sct = sqrt(ct);
  double cs2 = c2 - sct;
  if (cs2 < 0.0) cs2 = SMALL;
  double cf2 = c2 + sct;
  if (cf2 < 0.0) cf2 = SMALL;
  e.cs2 = cs2; e.cs = sqrt(cs2);
  e.cf2 = cf2; e.cf = sqrt(cf2);

  e.rr = sqrt(r);
  const double bp2 = MP_MUL(by, by) + MP_MUL(bz, bz);
  e.sbxm = (bx < 0.0) ? 0x80000000u : 0u;
  const bool deg = (bp2 < SMALL) && (fabs(e.ca2 - a2) < SMALL);
  double af2 = deg ? 1.0 : (cf2 - e.ca2) / (cf2 - cs2);
  if (af2 < 0.0) af2 = 0.0;
  double as2 = deg ? 1.0 : (cf2 - a2) / (cf2 - cs2);
  if (as2 < 0.0) as2 = 0.0;
  e.af2 = af2; e.af = sqrt(af2);
  e.as2 = as2; e.as = sqrt(as2);
  if (bp2 > SMALL) {
    const double sb = sqrt(bp2);
    e.bty = by / sb;
    e.btz = bz / sb;
  } else {
    e.bty = G.rs2;
    e.btz = G.rs2;
  }
  const double g21 = G.g21;
  e.th1 = 1.0 / (MP_MUL(MP_MUL(af2, a2), cf2 - MP_MUL(g21, a2)) +
                 MP_MUL(MP_MUL(as2, cf2), cs2 - MP_MUL(g21, a2)));
  e.th2 = 1.0 / (flip(MP_MUL(MP_MUL(af2, e.cf), e.a), e.sbxm) +
                 flip(MP_MUL(MP_MUL(as2, e.cs), e.ca), e.sbxm));
  e.vb = MP_MUL(e.bty, v) + MP_MUL(e.btz, w);

  const bool sgnbt_pos = (by > 0.0) || (fabs(by) < SMALL && (bz > 0.0));
  const unsigned bt = sgnbt_pos ? 0u : 0x80000000u;
  e.fcsm = a2 > e.ca2 ? bt : 0u;
  e.fcfm = a2 < e.ca2 ? bt : 0u;
  return true;
}

#ifdef MHD_FAST
// Fast build (MHD_FLAG_FAST_MATH): the same midpoint state, from each
// side's density and magnetic field (U1, U2) and its primitives P = (u, v,
// w, total pressure), which phase 1 of the tile computes once per cell.  The
// reference divides each side's momenta and 0.5*|m|^2 by its density per
// interface and divides by the midpoint density, (c_f^2 - c_s^2), |B_perp|,
// sqrt(rho) and c_f sqrt(rho) several times over; here every distinct
// denominator is inverted once.  Not bit-identical to the reference (the
// parity build is); agrees to the stated FP64 tolerance.
__device__ __forceinline__ bool midpoint_fast(const Gas& G, const double* U1, const double* U2,
                                              const double* P1, const double* P2, Mid& e) {
  const double gm = G.gm;
  const double r = 0.5 * (U1[0] + U2[0]);
  e.u = 0.5 * (P1[0] + P2[0]);
  e.v = 0.5 * (P1[1] + P2[1]);
  e.w = 0.5 * (P1[2] + P2[2]);
  const double bx = 0.5 * (U1[4] + U2[4]);
  const double by = 0.5 * (U1[5] + U2[5]);
  const double bz = 0.5 * (U1[6] + U2[6]);
  if (r <= 0.0) return false;
  const double u = e.u, v = e.v, w = e.w;
  e.uu = u * u + v * v + w * w;
  const double bb = bx * bx + by * by + bz * bz;
  const double pt = 0.5 * (P1[3] + P2[3]);
  double p = pt - 0.5 * bb;
  e.negp = 0;
  if (p < 0.0) { p = 0.0; e.negp = 1; }
  const double ir = 1.0 / r;
  double a2 = gm * p * ir;
  if (a2 < 0.0) a2 = 0.0;
  e.a2 = a2;
  e.a = sqrt(a2);
  e.ca2 = bx * bx * ir;
  e.ca = sqrt(e.ca2);
  const double c2 = 0.5 * (bb * ir + a2);
  double ct = c2 * c2 - a2 * e.ca2;
  if (ct < 0.0) ct = 0.0;
  const double sct = sqrt(ct);
  double cs2 = c2 - sct;
  if (cs2 < 0.0) cs2 = SMALL;
  double cf2 = c2 + sct;
  if (cf2 < 0.0) cf2 = SMALL;
  e.cs2 = cs2; e.cs = sqrt(cs2);
  e.cf2 = cf2; e.cf = sqrt(cf2);
  const double irr = rsqrt(r);
  e.irr = irr;
  e.rr = r * irr;
  const double bp2 = by * by + bz * bz;
  e.sbxm = (bx < 0.0) ? 0x80000000u : 0u;
  const bool deg = (bp2 < SMALL) && (fabs(e.ca2 - a2) < SMALL);
  const double idn = 1.0 / (cf2 - cs2);
  double af2 = deg ? 1.0 : (cf2 - e.ca2) * idn;
  if (af2 < 0.0) af2 = 0.0;
  double as2 = deg ? 1.0 : (cf2 - a2) * idn;
  if (as2 < 0.0) as2 = 0.0;
  e.af2 = af2; e.af = sqrt(af2);
  e.as2 = as2; e.as = sqrt(as2);
  if (bp2 > SMALL) {
    const double isb = rsqrt(bp2);
    e.bty = by * isb;
    e.btz = bz * isb;
  } else {
    e.bty = G.rs2;
    e.btz = G.rs2;
  }
  const double g21 = G.g21;
  e.th1 = 1.0 / (af2 * a2 * (cf2 - g21 * a2) + as2 * cf2 * (cs2 - g21 * a2));
  e.th2 = 1.0 / (flip(af2 * e.cf * e.a, e.sbxm) + flip(as2 * e.cs * e.ca, e.sbxm));
  e.icfrr = irr / e.cf;
  e.vb = e.bty * v + e.btz * w;

  const bool sgnbt_pos = (by > 0.0) || (fabs(by) < SMALL && (bz > 0.0));
  const unsigned bt = sgnbt_pos ? 0u : 0x80000000u;
  e.fcsm = a2 > e.ca2 ? bt : 0u;
  e.fcfm = a2 < e.ca2 ? bt : 0u;
  return true;
}
#endif

// Makes the midpoint scalars opaque to the optimiser at the top of each
// characteristic iteration (an empty asm that "may modify" them, no
// instruction emitted).  Without it the compiler hoists every row's
// coefficient products out of the loop, which needs far more registers
// than one row at a time and ends in local-memory spills.
__device__ __forceinline__ void opaque(Mid& e) {
  asm volatile("" : "+d"(e.u), "+d"(e.v), "+d"(e.w), "+d"(e.uu), "+d"(e.a2), "+d"(e.a),
                    "+d"(e.ca), "+d"(e.cs), "+d"(e.cs2), "+d"(e.cf), "+d"(e.cf2), "+d"(e.rr));
  asm volatile("" : "+d"(e.af), "+d"(e.as), "+d"(e.af2), "+d"(e.as2), "+d"(e.bty), "+d"(e.btz),
                    "+d"(e.th1), "+d"(e.th2), "+d"(e.vb), "+r"(e.sbxm), "+r"(e.fcfm),
                    "+r"(e.fcsm));
#ifdef MHD_FAST
  asm volatile("" : "+d"(e.irr), "+d"(e.icfrr));
#endif
}

__device__ __forceinline__ double eigenvalue(const Mid& e, int k) {
  switch (k) {
    case 0: return e.u - e.cf;
    case 1: return e.u - e.ca;
    case 2: return e.u - e.cs;
    case 3: return e.u;
    case 4: return e.u + e.cs;
    case 5: return e.u + e.ca;
    case 6: return e.u + e.cf;
    default: return 0.0;
  }
}

// Structurally non-zero columns of each left / right row (bit m = column m).
__host__ __device__ constexpr unsigned lv_mask(int k) {
  return (k == 1 || k == 5) ? 0x6Du /* 0,2,3,5,6 */ : (k == 7 ? 0u : 0xEFu /* all but 4 */);
}
__host__ __device__ constexpr unsigned rv_mask(int k) {
  return (k == 1 || k == 5) ? 0xECu /* 2,3,5,6,7 */
       : (k == 3 ? 0x8Fu /* 0,1,2,3,7 */ : (k == 7 ? 0u : 0xEFu));
}

// Left eigenvector row k (spatialmethodeno.cpp:473-552, sign flips 554-568).
__device__ __forceinline__ void lv_row(const Mid& e, const Gas& G, int k, double* l) {
  const double u = e.u, v = e.v, w = e.w, uu = e.uu, a2 = e.a2, a = e.a, ca = e.ca;
  const double cs = e.cs, cs2 = e.cs2, cf = e.cf, cf2 = e.cf2, rr = e.rr;
  const double af = e.af, as = e.as, af2 = e.af2, as2 = e.as2, bty = e.bty, btz = e.btz;
  const double th1 = e.th1, th2 = e.th2, g21 = G.g21, vb = e.vb;
  const unsigned sb = e.sbxm;
  switch (k) {
    case 0:
    case 6: {
      if (k == 0) {
        l[0] = 0.25 * th1 * af * a2 * uu + 0.5 * th2 * (flip(af * a * u, sb) - as * cs * vb);
        l[1] = -0.5 * th1 * af * a2 * u - flip(0.5 * th2 * af * a, sb);
        l[2] = -0.5 * th1 * af * a2 * v + 0.5 * th2 * as * bty * cs;
        l[3] = -0.5 * th1 * af * a2 * w + 0.5 * th2 * as * btz * cs;
      } else {
        l[0] = 0.25 * th1 * af * a2 * uu - 0.5 * th2 * (flip(af * a * u, sb) - as * cs * vb);
        l[1] = -0.5 * th1 * af * a2 * u + flip(0.5 * th2 * af * a, sb);
        l[2] = -0.5 * th1 * af * a2 * v - 0.5 * th2 * as * bty * cs;
        l[3] = -0.5 * th1 * af * a2 * w - 0.5 * th2 * as * btz * cs;
      }
      l[5] = 0.5 * th1 * as * bty * cf * rr * (cs2 - g21 * a2);
      l[6] = 0.5 * th1 * as * btz * cf * rr * (cs2 - g21 * a2);
      l[7] = 0.5 * th1 * af * a2;
      const unsigned f = e.fcfm;
      l[0] = flip(l[0], f); l[1] = flip(l[1], f); l[2] = flip(l[2], f); l[3] = flip(l[3], f);
      l[5] = flip(l[5], f); l[6] = flip(l[6], f); l[7] = flip(l[7], f);
      break;
    }
    case 1:
      l[0] = flip(-0.5 * (btz * v - bty * w), sb);
      l[2] = flip(0.5 * btz, sb);
      l[3] = flip(-0.5 * bty, sb);
      l[5] = 0.5 * btz * rr;
      l[6] = -0.5 * bty * rr;
      break;
    case 2:
    case 4: {
      if (k == 2) {
        l[0] = 0.25 * th1 * as * cf2 * uu + 0.5 * th2 * (flip(as * ca * u, sb) + af * cf * vb);
        l[1] = -0.5 * th1 * as * cf2 * u - flip(0.5 * th2 * as * ca, sb);
        l[2] = -0.5 * th1 * as * cf2 * v - 0.5 * th2 * af * bty * cf;
        l[3] = -0.5 * th1 * as * cf2 * w - 0.5 * th2 * af * btz * cf;
      } else {
        l[0] = 0.25 * th1 * as * cf2 * uu - 0.5 * th2 * (flip(as * ca * u, sb) + af * cf * vb);
        l[1] = -0.5 * th1 * as * cf2 * u + flip(0.5 * th2 * as * ca, sb);
        l[2] = -0.5 * th1 * as * cf2 * v + 0.5 * th2 * af * bty * cf;
        l[3] = -0.5 * th1 * as * cf2 * w + 0.5 * th2 * af * btz * cf;
      }
      l[5] = -0.5 * th1 * af * bty * cf * rr * (cf2 - g21 * a2);
      l[6] = -0.5 * th1 * af * btz * cf * rr * (cf2 - g21 * a2);
      l[7] = 0.5 * th1 * as * cf2;
      const unsigned f = e.fcsm;
      l[0] = flip(l[0], f); l[1] = flip(l[1], f); l[2] = flip(l[2], f); l[3] = flip(l[3], f);
      l[5] = flip(l[5], f); l[6] = flip(l[6], f); l[7] = flip(l[7], f);
      break;
    }
    case 3: {
      l[0] = 1.0 - 0.5 * th1 * uu * (af2 * a2 + as2 * cf2);
      l[1] = th1 * (af2 * a2 + as2 * cf2) * u;
      l[2] = th1 * (af2 * a2 + as2 * cf2) * v;
      l[3] = th1 * (af2 * a2 + as2 * cf2) * w;
      l[5] = th1 * af * as * bty * cf * rr * (cf2 - cs2);
      l[6] = th1 * af * as * btz * cf * rr * (cf2 - cs2);
      l[7] = -th1 * (af2 * a2 + as2 * cf2);
      break;
    }
    case 5:
      l[0] = flip(+0.5 * (btz * v - bty * w), sb);
      l[2] = flip(-0.5 * btz, sb);
      l[3] = flip(0.5 * bty, sb);
      l[5] = 0.5 * btz * rr;
      l[6] = -0.5 * bty * rr;
      break;
    default:
      break;
  }
}

// Right eigenvector row k (spatialmethodeno.cpp:392-471, sign flips 554-568).
// FR (fast build only): divide by sqrt(rho), c_f sqrt(rho) and gamma - 1
// through the midpoint's reciprocals.
template <bool FR = false>
__device__ __forceinline__ void rv_row(const Mid& e, const Gas& G, int k, double* q) {
  const double u = e.u, v = e.v, w = e.w, uu = e.uu, a2 = e.a2, a = e.a, ca = e.ca;
  const double cs = e.cs, cs2 = e.cs2, cf = e.cf, cf2 = e.cf2, rr = e.rr;
  const double af = e.af, as = e.as, bty = e.bty, btz = e.btz, g1 = G.g1, g21 = G.g21;
  const double vb = e.vb;
  const unsigned sb = e.sbxm;
#ifdef MHD_FAST
#define RV_DIV(x, d, inv) (FR ? (x) * (inv) : (x) / (d))
#define DIV_G1(x) (FR ? (x) * G.ig1 : (x) / g1)
#else
#define RV_DIV(x, d, inv) ((x) / (d))
#define DIV_G1(x) ((x) / g1)
#endif
  switch (k) {
    case 0:
    case 6: {
      if (k == 0) {
        q[0] = af;
        q[1] = af * (u - cf);
        q[2] = af * v + flip(as * bty * ca, sb);
        q[3] = af * w + flip(as * btz * ca, sb);
        q[7] = 0.5 * af * uu + DIV_G1(af * cf2) - af * cf * u + flip(as * ca, sb) * vb + g21 * af * (cf2 - a2);
      } else {
        q[0] = af;
        q[1] = af * (u + cf);
        q[2] = af * v - flip(as * bty * ca, sb);
        q[3] = af * w - flip(as * btz * ca, sb);
        q[7] = 0.5 * af * uu + DIV_G1(af * cf2) + af * cf * u - flip(as * ca, sb) * vb + g21 * af * (cf2 - a2);
      }
      q[5] = RV_DIV(as * bty * cf, rr, e.irr);
      q[6] = RV_DIV(as * btz * cf, rr, e.irr);
      const unsigned f = e.fcfm;
      q[0] = flip(q[0], f); q[1] = flip(q[1], f); q[2] = flip(q[2], f); q[3] = flip(q[3], f);
      q[5] = flip(q[5], f); q[6] = flip(q[6], f); q[7] = flip(q[7], f);
      break;
    }
    case 1:
      q[2] = flip(btz, sb);
      q[3] = flip(-bty, sb);
      q[5] = RV_DIV(btz, rr, e.irr);
      q[6] = RV_DIV(-bty, rr, e.irr);
      q[7] = flip(btz * v - bty * w, sb);
      break;
    case 2:
    case 4: {
      if (k == 2) {
        q[0] = as;
        q[1] = as * (u - cs);
        q[2] = as * v - flip(af * bty * a, sb);
        q[3] = as * w - flip(af * btz * a, sb);
        q[7] = 0.5 * as * uu + DIV_G1(as * cs2) - as * cs * u - flip(af * a, sb) * vb + g21 * as * (cs2 - a2);
      } else {
        q[0] = as;
        q[1] = as * (u + cs);
        q[2] = as * v + flip(af * bty * a, sb);
        q[3] = as * w + flip(af * btz * a, sb);
        q[7] = 0.5 * as * uu + DIV_G1(as * cs2) + as * cs * u + flip(af * a, sb) * vb + g21 * as * (cs2 - a2);
      }
      q[5] = RV_DIV(-af * bty * a2, (cf * rr), e.icfrr);
      q[6] = RV_DIV(-af * btz * a2, (cf * rr), e.icfrr);
      const unsigned f = e.fcsm;
      q[0] = flip(q[0], f); q[1] = flip(q[1], f); q[2] = flip(q[2], f); q[3] = flip(q[3], f);
      q[5] = flip(q[5], f); q[6] = flip(q[6], f); q[7] = flip(q[7], f);
      break;
    }
    case 3:
      q[0] = 1.0;
      q[1] = u;
      q[2] = v;
      q[3] = w;
      q[7] = 0.5 * uu;
      break;
    case 5:
      q[2] = flip(-btz, sb);
      q[3] = flip(+bty, sb);
      q[5] = RV_DIV(btz, rr, e.irr);
      q[6] = RV_DIV(-bty, rr, e.irr);
      q[7] = flip(-(btz * v - bty * w), sb);
      break;
    default:
      break;
  }
#undef DIV_G1
#undef RV_DIV
}

// Cell-centred eigenvalues (SpatialMethodEno::getEigenvaluesAt,
// spatialmethodeno.cpp:130-206), used for the ENO-LF dissipation.
// Returns false on non-positive density.
__device__ __forceinline__ bool eigenvalues_at(double gm, const double* U, double* lam, int& negp) {
  const double r = U[0], mx = U[1], u = U[1] / U[0], my = U[2], mz = U[3];
  const double bx = U[4], by = U[5], bz = U[6], en = U[7];
  negp = 0;
  if (r <= 0.0) return false;
  const double mm = mx * mx + my * my + mz * mz;
  const double bb = bx * bx + by * by + bz * bz;
  double p = (gm - 1.0) * (en - 0.5 * mm / r - 0.5 * bb);
  if (p < 0.0) { p = 0.0; negp = 1; }
  double a2 = gm * p / r;
  if (a2 < 0.0) a2 = 0.0;
  const double ca2 = bx * bx / r;
  const double ca = sqrt(ca2);
  const double c2 = 0.5 * (bb / r + a2);
  double ct = c2 * c2 - a2 * ca2;
  if (ct < 0.0) ct = 0.0;
  const double sct = sqrt(ct);
  double cs2 = c2 - sct;
  if (cs2 < 0.0) cs2 = SMALL;
  const double cs = sqrt(cs2);
  double cf2 = c2 + sct;
  if (cf2 < 0.0) cf2 = SMALL;
  const double cf = sqrt(cf2);
  lam[0] = u - cf; lam[1] = u - ca; lam[2] = u - cs; lam[3] = u;
  lam[4] = u + cs; lam[5] = u + ca; lam[6] = u + cf; lam[7] = 0.0;
  return true;
}

}  // namespace MHD_KNS
}  // namespace mhd
