// GENERATED by gen_adjoint.py from the formulas restated there; do not edit.
// Reverse-mode adjoints of the ENO-Roe interface algebra with frozen branches.
#pragma once

#include "mhd_eigen.cuh"

namespace mhd {
namespace MHD_KNS {

// d sqrt(v) / dv, 0 at v = 0 (frozen one-sided branch)
__device__ __forceinline__ double inv2sqrt(double v) {
  return v > 0.0 ? 0.5 * rsqrt(v) : 0.0;
}

// Adjoints of the Mid scalars.
struct MidBar {
  double u, v, w, uu, a2, a, ca2, ca, cs2, cs, cf2, cf, rr, af2, af, as2, as, bty, btz, th1, th2, vb;
};

// Adds the adjoint of rows k and 6 - k of the pair pi (k = 0, 2, 1, 3 for
// pi = 0..3) to mb: LS = lb_k + lb_{6-k}, LD = lb_k - lb_{6-k} (left rows,
// columns 0-3, 5-7 in slots 0-6), and right-row seeds (fS +- fD) * lF.
__device__ __forceinline__ void pair_adjoint(const Mid& e, const Gas& G, int pi,
                                             const double* LS, const double* LD,
                                             double fS, double fD,
                                             const double* lF, MidBar& mb) {
  const double sb = (e.sbxm ? -1.0 : 1.0), fcf = (e.fcfm ? -1.0 : 1.0),
               fcs = (e.fcsm ? -1.0 : 1.0);
  (void)fcf; (void)fcs; (void)sb;
  switch (pi) {
    case 0: {  // rows 0 and 6
      [[maybe_unused]] const double rcp0 = 1.0 / (e.rr);
      [[maybe_unused]] const double rcp1 = 1.0 / (G.g1);
      if (LS[0] != 0.0) {
        mb.th1 = fma(LS[0] * fcf * e.uu * e.a2 * e.af, 0.25, mb.th1);
        mb.af = fma(LS[0] * fcf * e.uu * e.a2, 0.25 * e.th1, mb.af);
        mb.a2 = fma(LS[0] * fcf * e.uu, 0.25 * e.th1 * e.af, mb.a2);
        mb.uu = fma(LS[0] * fcf, 0.25 * e.th1 * e.af * e.a2, mb.uu);
      }
      if (LS[1] != 0.0) {
        mb.th1 = fma(LS[1] * fcf * e.u * e.a2 * e.af, -0.5, mb.th1);
        mb.af = fma(LS[1] * fcf * e.u * e.a2, -0.5 * e.th1, mb.af);
        mb.a2 = fma(LS[1] * fcf * e.u, -0.5 * e.th1 * e.af, mb.a2);
        mb.u = fma(LS[1] * fcf, -0.5 * e.th1 * e.af * e.a2, mb.u);
      }
      if (LS[2] != 0.0) {
        mb.th1 = fma(LS[2] * fcf * e.v * e.a2 * e.af, -0.5, mb.th1);
        mb.af = fma(LS[2] * fcf * e.v * e.a2, -0.5 * e.th1, mb.af);
        mb.a2 = fma(LS[2] * fcf * e.v, -0.5 * e.th1 * e.af, mb.a2);
        mb.v = fma(LS[2] * fcf, -0.5 * e.th1 * e.af * e.a2, mb.v);
      }
      if (LS[3] != 0.0) {
        mb.th1 = fma(LS[3] * fcf * e.w * e.a2 * e.af, -0.5, mb.th1);
        mb.af = fma(LS[3] * fcf * e.w * e.a2, -0.5 * e.th1, mb.af);
        mb.a2 = fma(LS[3] * fcf * e.w, -0.5 * e.th1 * e.af, mb.a2);
        mb.w = fma(LS[3] * fcf, -0.5 * e.th1 * e.af * e.a2, mb.w);
      }
      if (LS[4] != 0.0) {
        mb.th1 += LS[4] * fcf * (e.cs2 - G.g21 * e.a2) * e.rr * e.cf * e.bty * e.as * 0.5;
        mb.as = fma(LS[4] * fcf * (e.cs2 - G.g21 * e.a2) * e.rr * e.cf * e.bty, 0.5 * e.th1, mb.as);
        mb.bty += LS[4] * fcf * (e.cs2 - G.g21 * e.a2) * e.rr * e.cf * (0.5 * e.th1 * e.as);
        mb.cf += LS[4] * fcf * (e.cs2 - G.g21 * e.a2) * e.rr * (0.5 * e.th1 * e.as * e.bty);
        mb.rr += LS[4] * fcf * (e.cs2 - G.g21 * e.a2) * (0.5 * e.th1 * e.as * e.bty * e.cf);
        mb.cs2 += LS[4] * fcf * (0.5 * e.th1 * e.as * e.bty * e.cf * e.rr);
        mb.a2 += -(LS[4] * fcf * (0.5 * e.th1 * e.as * e.bty * e.cf * e.rr)) * G.g21;
      }
      if (LS[5] != 0.0) {
        mb.th1 += LS[5] * fcf * (e.cs2 - G.g21 * e.a2) * e.rr * e.cf * e.btz * e.as * 0.5;
        mb.as = fma(LS[5] * fcf * (e.cs2 - G.g21 * e.a2) * e.rr * e.cf * e.btz, 0.5 * e.th1, mb.as);
        mb.btz += LS[5] * fcf * (e.cs2 - G.g21 * e.a2) * e.rr * e.cf * (0.5 * e.th1 * e.as);
        mb.cf += LS[5] * fcf * (e.cs2 - G.g21 * e.a2) * e.rr * (0.5 * e.th1 * e.as * e.btz);
        mb.rr += LS[5] * fcf * (e.cs2 - G.g21 * e.a2) * (0.5 * e.th1 * e.as * e.btz * e.cf);
        mb.cs2 += LS[5] * fcf * (0.5 * e.th1 * e.as * e.btz * e.cf * e.rr);
        mb.a2 += -(LS[5] * fcf * (0.5 * e.th1 * e.as * e.btz * e.cf * e.rr)) * G.g21;
      }
      if (LS[6] != 0.0) {
        mb.th1 = fma(LS[6] * fcf * e.a2 * e.af, 0.5, mb.th1);
        mb.af = fma(LS[6] * fcf * e.a2, 0.5 * e.th1, mb.af);
        mb.a2 = fma(LS[6] * fcf, 0.5 * e.th1 * e.af, mb.a2);
      }
      if (LD[0] != 0.0) {
        mb.th2 += LD[0] * fcf * (sb * e.af * e.a * e.u - e.as * e.cs * e.vb) * 0.5;
        mb.af = fma(LD[0] * fcf * (0.5 * e.th2) * e.u * e.a, sb, mb.af);
        mb.a = fma(LD[0] * fcf * (0.5 * e.th2) * e.u, sb * e.af, mb.a);
        mb.u = fma(LD[0] * fcf * (0.5 * e.th2), sb * e.af * e.a, mb.u);
        mb.as = fma(-(LD[0] * fcf * (0.5 * e.th2)) * e.vb, e.cs, mb.as);
        mb.cs += -(LD[0] * fcf * (0.5 * e.th2)) * e.vb * e.as;
        mb.vb += -(LD[0] * fcf * (0.5 * e.th2)) * (e.as * e.cs);
      }
      if (LD[1] != 0.0) {
        mb.th2 = fma(-(LD[1] * fcf) * e.a * e.af, sb * 0.5, mb.th2);
        mb.af = fma(-(LD[1] * fcf) * e.a, sb * 0.5 * e.th2, mb.af);
        mb.a = fma(-(LD[1] * fcf), sb * 0.5 * e.th2 * e.af, mb.a);
      }
      if (LD[2] != 0.0) {
        mb.th2 += LD[2] * fcf * e.cs * e.bty * e.as * 0.5;
        mb.as = fma(LD[2] * fcf * e.cs * e.bty, 0.5 * e.th2, mb.as);
        mb.bty += LD[2] * fcf * e.cs * (0.5 * e.th2 * e.as);
        mb.cs += LD[2] * fcf * (0.5 * e.th2 * e.as * e.bty);
      }
      if (LD[3] != 0.0) {
        mb.th2 += LD[3] * fcf * e.cs * e.btz * e.as * 0.5;
        mb.as = fma(LD[3] * fcf * e.cs * e.btz, 0.5 * e.th2, mb.as);
        mb.btz += LD[3] * fcf * e.cs * (0.5 * e.th2 * e.as);
        mb.cs += LD[3] * fcf * (0.5 * e.th2 * e.as * e.btz);
      }
      { const double rs0 = fS * lF[0];
      if (rs0 != 0.0) {
        mb.af = fma(rs0, fcf, mb.af);
      } }
      { const double rs1 = fS * lF[1];
      if (rs1 != 0.0) {
        mb.af = fma(rs1 * fcf, e.u, mb.af);
        mb.u = fma(rs1 * fcf, e.af, mb.u);
      } }
      { const double rs2 = fS * lF[2];
      if (rs2 != 0.0) {
        mb.af = fma(rs2 * fcf, e.v, mb.af);
        mb.v = fma(rs2 * fcf, e.af, mb.v);
      } }
      { const double rs3 = fS * lF[3];
      if (rs3 != 0.0) {
        mb.af = fma(rs3 * fcf, e.w, mb.af);
        mb.w = fma(rs3 * fcf, e.af, mb.w);
      } }
      { const double rs5 = fS * lF[5];
      if (rs5 != 0.0) {
        mb.as = fma(rs5 * fcf * rcp0 * e.cf, e.bty, mb.as);
        mb.bty += rs5 * fcf * rcp0 * e.cf * e.as;
        mb.cf += rs5 * fcf * rcp0 * (e.as * e.bty);
        mb.rr += -(rs5 * fcf) * (e.as * e.bty * e.cf) * rcp0 * rcp0;
      } }
      { const double rs6 = fS * lF[6];
      if (rs6 != 0.0) {
        mb.as = fma(rs6 * fcf * rcp0 * e.cf, e.btz, mb.as);
        mb.btz += rs6 * fcf * rcp0 * e.cf * e.as;
        mb.cf += rs6 * fcf * rcp0 * (e.as * e.btz);
        mb.rr += -(rs6 * fcf) * (e.as * e.btz * e.cf) * rcp0 * rcp0;
      } }
      { const double rs7 = fS * lF[7];
      if (rs7 != 0.0) {
        mb.af = fma(rs7 * fcf * e.uu, 0.5, mb.af);
        mb.uu = fma(rs7 * fcf, 0.5 * e.af, mb.uu);
        mb.af = fma(rs7 * fcf * rcp1, e.cf2, mb.af);
        mb.cf2 = fma(rs7 * fcf * rcp1, e.af, mb.cf2);
        mb.af = fma(rs7 * fcf * (e.cf2 - e.a2), G.g21, mb.af);
        mb.cf2 = fma(rs7 * fcf, G.g21 * e.af, mb.cf2);
        mb.a2 += -(rs7 * fcf * (G.g21 * e.af));
      } }
      { const double rd1 = fD * lF[1];
      if (rd1 != 0.0) {
        mb.af = fma(-(rd1 * fcf), e.cf, mb.af);
        mb.cf = fma(-(rd1 * fcf), e.af, mb.cf);
      } }
      { const double rd2 = fD * lF[2];
      if (rd2 != 0.0) {
        mb.as = fma(rd2 * fcf * e.ca * e.bty, sb, mb.as);
        mb.bty += rd2 * fcf * e.ca * (sb * e.as);
        mb.ca += rd2 * fcf * (sb * e.as * e.bty);
      } }
      { const double rd3 = fD * lF[3];
      if (rd3 != 0.0) {
        mb.as = fma(rd3 * fcf * e.ca * e.btz, sb, mb.as);
        mb.btz += rd3 * fcf * e.ca * (sb * e.as);
        mb.ca += rd3 * fcf * (sb * e.as * e.btz);
      } }
      { const double rd7 = fD * lF[7];
      if (rd7 != 0.0) {
        mb.af = fma(-(rd7 * fcf) * e.u, e.cf, mb.af);
        mb.cf = fma(-(rd7 * fcf) * e.u, e.af, mb.cf);
        mb.u = fma(-(rd7 * fcf), e.af * e.cf, mb.u);
        mb.as = fma(rd7 * fcf * e.vb * e.ca, sb, mb.as);
        mb.ca += rd7 * fcf * e.vb * (sb * e.as);
        mb.vb += rd7 * fcf * (sb * e.as * e.ca);
      } }
      break;
    }
    case 1: {  // rows 2 and 4
      [[maybe_unused]] const double rcp0 = 1.0 / (e.cf * e.rr);
      [[maybe_unused]] const double rcp1 = 1.0 / (G.g1);
      if (LS[0] != 0.0) {
        mb.th1 += LS[0] * fcs * e.uu * e.cf2 * e.as * 0.25;
        mb.as = fma(LS[0] * fcs * e.uu * e.cf2, 0.25 * e.th1, mb.as);
        mb.cf2 += LS[0] * fcs * e.uu * (0.25 * e.th1 * e.as);
        mb.uu += LS[0] * fcs * (0.25 * e.th1 * e.as * e.cf2);
      }
      if (LS[1] != 0.0) {
        mb.th1 += LS[1] * fcs * e.u * e.cf2 * e.as * -0.5;
        mb.as = fma(LS[1] * fcs * e.u * e.cf2, -0.5 * e.th1, mb.as);
        mb.cf2 += LS[1] * fcs * e.u * (-0.5 * e.th1 * e.as);
        mb.u += LS[1] * fcs * (-0.5 * e.th1 * e.as * e.cf2);
      }
      if (LS[2] != 0.0) {
        mb.th1 += LS[2] * fcs * e.v * e.cf2 * e.as * -0.5;
        mb.as = fma(LS[2] * fcs * e.v * e.cf2, -0.5 * e.th1, mb.as);
        mb.cf2 += LS[2] * fcs * e.v * (-0.5 * e.th1 * e.as);
        mb.v += LS[2] * fcs * (-0.5 * e.th1 * e.as * e.cf2);
      }
      if (LS[3] != 0.0) {
        mb.th1 += LS[3] * fcs * e.w * e.cf2 * e.as * -0.5;
        mb.as = fma(LS[3] * fcs * e.w * e.cf2, -0.5 * e.th1, mb.as);
        mb.cf2 += LS[3] * fcs * e.w * (-0.5 * e.th1 * e.as);
        mb.w += LS[3] * fcs * (-0.5 * e.th1 * e.as * e.cf2);
      }
      if (LS[4] != 0.0) {
        mb.th1 = fma(LS[4] * fcs * (e.cf2 - G.g21 * e.a2) * e.rr * e.cf * e.bty * e.af, -0.5, mb.th1);
        mb.af = fma(LS[4] * fcs * (e.cf2 - G.g21 * e.a2) * e.rr * e.cf * e.bty, -0.5 * e.th1, mb.af);
        mb.bty = fma(LS[4] * fcs * (e.cf2 - G.g21 * e.a2) * e.rr * e.cf, -0.5 * e.th1 * e.af, mb.bty);
        mb.cf = fma(LS[4] * fcs * (e.cf2 - G.g21 * e.a2) * e.rr, -0.5 * e.th1 * e.af * e.bty, mb.cf);
        mb.rr = fma(LS[4] * fcs * (e.cf2 - G.g21 * e.a2), -0.5 * e.th1 * e.af * e.bty * e.cf, mb.rr);
        mb.cf2 = fma(LS[4] * fcs, -0.5 * e.th1 * e.af * e.bty * e.cf * e.rr, mb.cf2);
        mb.a2 = fma(-(LS[4] * fcs * (-0.5 * e.th1 * e.af * e.bty * e.cf * e.rr)), G.g21, mb.a2);
      }
      if (LS[5] != 0.0) {
        mb.th1 = fma(LS[5] * fcs * (e.cf2 - G.g21 * e.a2) * e.rr * e.cf * e.btz * e.af, -0.5, mb.th1);
        mb.af = fma(LS[5] * fcs * (e.cf2 - G.g21 * e.a2) * e.rr * e.cf * e.btz, -0.5 * e.th1, mb.af);
        mb.btz = fma(LS[5] * fcs * (e.cf2 - G.g21 * e.a2) * e.rr * e.cf, -0.5 * e.th1 * e.af, mb.btz);
        mb.cf = fma(LS[5] * fcs * (e.cf2 - G.g21 * e.a2) * e.rr, -0.5 * e.th1 * e.af * e.btz, mb.cf);
        mb.rr = fma(LS[5] * fcs * (e.cf2 - G.g21 * e.a2), -0.5 * e.th1 * e.af * e.btz * e.cf, mb.rr);
        mb.cf2 = fma(LS[5] * fcs, -0.5 * e.th1 * e.af * e.btz * e.cf * e.rr, mb.cf2);
        mb.a2 = fma(-(LS[5] * fcs * (-0.5 * e.th1 * e.af * e.btz * e.cf * e.rr)), G.g21, mb.a2);
      }
      if (LS[6] != 0.0) {
        mb.th1 += LS[6] * fcs * e.cf2 * e.as * 0.5;
        mb.as = fma(LS[6] * fcs * e.cf2, 0.5 * e.th1, mb.as);
        mb.cf2 += LS[6] * fcs * (0.5 * e.th1 * e.as);
      }
      if (LD[0] != 0.0) {
        mb.th2 += LD[0] * fcs * (sb * e.as * e.ca * e.u + e.af * e.cf * e.vb) * 0.5;
        mb.as = fma(LD[0] * fcs * (0.5 * e.th2) * e.u * e.ca, sb, mb.as);
        mb.ca += LD[0] * fcs * (0.5 * e.th2) * e.u * (sb * e.as);
        mb.u += LD[0] * fcs * (0.5 * e.th2) * (sb * e.as * e.ca);
        mb.af = fma(LD[0] * fcs * (0.5 * e.th2) * e.vb, e.cf, mb.af);
        mb.cf = fma(LD[0] * fcs * (0.5 * e.th2) * e.vb, e.af, mb.cf);
        mb.vb = fma(LD[0] * fcs * (0.5 * e.th2), e.af * e.cf, mb.vb);
      }
      if (LD[1] != 0.0) {
        mb.th2 += -(LD[1] * fcs) * e.ca * e.as * (sb * 0.5);
        mb.as = fma(-(LD[1] * fcs) * e.ca, sb * 0.5 * e.th2, mb.as);
        mb.ca += -(LD[1] * fcs) * (sb * 0.5 * e.th2 * e.as);
      }
      if (LD[2] != 0.0) {
        mb.th2 = fma(LD[2] * fcs * e.cf * e.bty * e.af, -0.5, mb.th2);
        mb.af = fma(LD[2] * fcs * e.cf * e.bty, -0.5 * e.th2, mb.af);
        mb.bty = fma(LD[2] * fcs * e.cf, -0.5 * e.th2 * e.af, mb.bty);
        mb.cf = fma(LD[2] * fcs, -0.5 * e.th2 * e.af * e.bty, mb.cf);
      }
      if (LD[3] != 0.0) {
        mb.th2 = fma(LD[3] * fcs * e.cf * e.btz * e.af, -0.5, mb.th2);
        mb.af = fma(LD[3] * fcs * e.cf * e.btz, -0.5 * e.th2, mb.af);
        mb.btz = fma(LD[3] * fcs * e.cf, -0.5 * e.th2 * e.af, mb.btz);
        mb.cf = fma(LD[3] * fcs, -0.5 * e.th2 * e.af * e.btz, mb.cf);
      }
      { const double rs0 = fS * lF[0];
      if (rs0 != 0.0) {
        mb.as = fma(rs0, fcs, mb.as);
      } }
      { const double rs1 = fS * lF[1];
      if (rs1 != 0.0) {
        mb.as = fma(rs1 * fcs, e.u, mb.as);
        mb.u += rs1 * fcs * e.as;
      } }
      { const double rs2 = fS * lF[2];
      if (rs2 != 0.0) {
        mb.as = fma(rs2 * fcs, e.v, mb.as);
        mb.v += rs2 * fcs * e.as;
      } }
      { const double rs3 = fS * lF[3];
      if (rs3 != 0.0) {
        mb.as = fma(rs3 * fcs, e.w, mb.as);
        mb.w += rs3 * fcs * e.as;
      } }
      { const double rs5 = fS * lF[5];
      if (rs5 != 0.0) {
        mb.af += -(rs5 * fcs * rcp0 * e.a2 * e.bty);
        mb.bty = fma(rs5 * fcs * rcp0 * e.a2, -e.af, mb.bty);
        mb.a2 = fma(rs5 * fcs * rcp0, -e.af * e.bty, mb.a2);
        mb.cf = fma(-(rs5 * fcs) * (-e.af * e.bty * e.a2) * rcp0 * rcp0, e.rr, mb.cf);
        mb.rr = fma(-(rs5 * fcs) * (-e.af * e.bty * e.a2) * rcp0 * rcp0, e.cf, mb.rr);
      } }
      { const double rs6 = fS * lF[6];
      if (rs6 != 0.0) {
        mb.af += -(rs6 * fcs * rcp0 * e.a2 * e.btz);
        mb.btz = fma(rs6 * fcs * rcp0 * e.a2, -e.af, mb.btz);
        mb.a2 = fma(rs6 * fcs * rcp0, -e.af * e.btz, mb.a2);
        mb.cf = fma(-(rs6 * fcs) * (-e.af * e.btz * e.a2) * rcp0 * rcp0, e.rr, mb.cf);
        mb.rr = fma(-(rs6 * fcs) * (-e.af * e.btz * e.a2) * rcp0 * rcp0, e.cf, mb.rr);
      } }
      { const double rs7 = fS * lF[7];
      if (rs7 != 0.0) {
        mb.as = fma(rs7 * fcs * e.uu, 0.5, mb.as);
        mb.uu += rs7 * fcs * (0.5 * e.as);
        mb.as = fma(rs7 * fcs * rcp1, e.cs2, mb.as);
        mb.cs2 += rs7 * fcs * rcp1 * e.as;
        mb.as = fma(rs7 * fcs * (e.cs2 - e.a2), G.g21, mb.as);
        mb.cs2 += rs7 * fcs * (G.g21 * e.as);
        mb.a2 += -(rs7 * fcs * (G.g21 * e.as));
      } }
      { const double rd1 = fD * lF[1];
      if (rd1 != 0.0) {
        mb.as = fma(-(rd1 * fcs), e.cs, mb.as);
        mb.cs += -(rd1 * fcs) * e.as;
      } }
      { const double rd2 = fD * lF[2];
      if (rd2 != 0.0) {
        mb.af = fma(-(rd2 * fcs) * e.a * e.bty, sb, mb.af);
        mb.bty = fma(-(rd2 * fcs) * e.a, sb * e.af, mb.bty);
        mb.a = fma(-(rd2 * fcs), sb * e.af * e.bty, mb.a);
      } }
      { const double rd3 = fD * lF[3];
      if (rd3 != 0.0) {
        mb.af = fma(-(rd3 * fcs) * e.a * e.btz, sb, mb.af);
        mb.btz = fma(-(rd3 * fcs) * e.a, sb * e.af, mb.btz);
        mb.a = fma(-(rd3 * fcs), sb * e.af * e.btz, mb.a);
      } }
      { const double rd7 = fD * lF[7];
      if (rd7 != 0.0) {
        mb.as = fma(-(rd7 * fcs) * e.u, e.cs, mb.as);
        mb.cs += -(rd7 * fcs) * e.u * e.as;
        mb.u += -(rd7 * fcs) * (e.as * e.cs);
        mb.af = fma(-(rd7 * fcs) * e.vb * e.a, sb, mb.af);
        mb.a = fma(-(rd7 * fcs) * e.vb, sb * e.af, mb.a);
        mb.vb = fma(-(rd7 * fcs), sb * e.af * e.a, mb.vb);
      } }
      break;
    }
    case 2: {  // rows 1 and 5
      [[maybe_unused]] const double rcp0 = 1.0 / (e.rr);
      if (LS[4] != 0.0) {
        mb.btz = fma(LS[4] * e.rr, 0.5, mb.btz);
        mb.rr = fma(LS[4], 0.5 * e.btz, mb.rr);
      }
      if (LS[5] != 0.0) {
        mb.bty = fma(LS[5] * e.rr, -0.5, mb.bty);
        mb.rr = fma(LS[5], -0.5 * e.bty, mb.rr);
      }
      if (LD[0] != 0.0) {
        mb.btz = fma(LD[0] * sb * -0.5, e.v, mb.btz);
        mb.v = fma(LD[0] * sb * -0.5, e.btz, mb.v);
        mb.bty = fma(-(LD[0] * sb * -0.5), e.w, mb.bty);
        mb.w = fma(-(LD[0] * sb * -0.5), e.bty, mb.w);
      }
      if (LD[2] != 0.0) {
        mb.btz = fma(LD[2] * sb, 0.5, mb.btz);
      }
      if (LD[3] != 0.0) {
        mb.bty = fma(LD[3] * sb, -0.5, mb.bty);
      }
      { const double rs5 = fS * lF[5];
      if (rs5 != 0.0) {
        mb.btz = fma(rs5, rcp0, mb.btz);
        mb.rr = fma(-rs5 * e.btz * rcp0, rcp0, mb.rr);
      } }
      { const double rs6 = fS * lF[6];
      if (rs6 != 0.0) {
        mb.bty += -(rs6 * rcp0);
        mb.rr = fma(-rs6 * -e.bty * rcp0, rcp0, mb.rr);
      } }
      { const double rd2 = fD * lF[2];
      if (rd2 != 0.0) {
        mb.btz = fma(rd2, sb, mb.btz);
      } }
      { const double rd3 = fD * lF[3];
      if (rd3 != 0.0) {
        mb.bty = fma(-rd3, sb, mb.bty);
      } }
      { const double rd7 = fD * lF[7];
      if (rd7 != 0.0) {
        mb.btz = fma(rd7 * sb, e.v, mb.btz);
        mb.v = fma(rd7 * sb, e.btz, mb.v);
        mb.bty = fma(-(rd7 * sb), e.w, mb.bty);
        mb.w = fma(-(rd7 * sb), e.bty, mb.w);
      } }
      break;
    }
    case 3: {  // rows 3 and 3
      if (LS[0] != 0.0) {
        mb.th1 = fma(-LS[0] * (e.af2 * e.a2 + e.as2 * e.cf2) * e.uu, 0.5, mb.th1);
        mb.uu = fma(-LS[0] * (e.af2 * e.a2 + e.as2 * e.cf2), 0.5 * e.th1, mb.uu);
        mb.af2 = fma(-LS[0] * (0.5 * e.th1 * e.uu), e.a2, mb.af2);
        mb.a2 = fma(-LS[0] * (0.5 * e.th1 * e.uu), e.af2, mb.a2);
        mb.as2 = fma(-LS[0] * (0.5 * e.th1 * e.uu), e.cf2, mb.as2);
        mb.cf2 = fma(-LS[0] * (0.5 * e.th1 * e.uu), e.as2, mb.cf2);
      }
      if (LS[1] != 0.0) {
        mb.th1 = fma(LS[1] * e.u, e.af2 * e.a2 + e.as2 * e.cf2, mb.th1);
        mb.af2 = fma(LS[1] * e.u * e.th1, e.a2, mb.af2);
        mb.a2 = fma(LS[1] * e.u * e.th1, e.af2, mb.a2);
        mb.as2 = fma(LS[1] * e.u * e.th1, e.cf2, mb.as2);
        mb.cf2 = fma(LS[1] * e.u * e.th1, e.as2, mb.cf2);
        mb.u = fma(LS[1], e.th1 * (e.af2 * e.a2 + e.as2 * e.cf2), mb.u);
      }
      if (LS[2] != 0.0) {
        mb.th1 = fma(LS[2] * e.v, e.af2 * e.a2 + e.as2 * e.cf2, mb.th1);
        mb.af2 = fma(LS[2] * e.v * e.th1, e.a2, mb.af2);
        mb.a2 = fma(LS[2] * e.v * e.th1, e.af2, mb.a2);
        mb.as2 = fma(LS[2] * e.v * e.th1, e.cf2, mb.as2);
        mb.cf2 = fma(LS[2] * e.v * e.th1, e.as2, mb.cf2);
        mb.v = fma(LS[2], e.th1 * (e.af2 * e.a2 + e.as2 * e.cf2), mb.v);
      }
      if (LS[3] != 0.0) {
        mb.th1 = fma(LS[3] * e.w, e.af2 * e.a2 + e.as2 * e.cf2, mb.th1);
        mb.af2 = fma(LS[3] * e.w * e.th1, e.a2, mb.af2);
        mb.a2 = fma(LS[3] * e.w * e.th1, e.af2, mb.a2);
        mb.as2 = fma(LS[3] * e.w * e.th1, e.cf2, mb.as2);
        mb.cf2 = fma(LS[3] * e.w * e.th1, e.as2, mb.cf2);
        mb.w = fma(LS[3], e.th1 * (e.af2 * e.a2 + e.as2 * e.cf2), mb.w);
      }
      if (LS[4] != 0.0) {
        mb.th1 += LS[4] * (e.cf2 - e.cs2) * e.rr * e.cf * e.bty * e.as * e.af;
        mb.af += LS[4] * (e.cf2 - e.cs2) * e.rr * e.cf * e.bty * e.as * e.th1;
        mb.as = fma(LS[4] * (e.cf2 - e.cs2) * e.rr * e.cf * e.bty, e.th1 * e.af, mb.as);
        mb.bty += LS[4] * (e.cf2 - e.cs2) * e.rr * e.cf * (e.th1 * e.af * e.as);
        mb.cf += LS[4] * (e.cf2 - e.cs2) * e.rr * (e.th1 * e.af * e.as * e.bty);
        mb.rr += LS[4] * (e.cf2 - e.cs2) * (e.th1 * e.af * e.as * e.bty * e.cf);
        mb.cf2 += LS[4] * (e.th1 * e.af * e.as * e.bty * e.cf * e.rr);
        mb.cs2 += -(LS[4] * (e.th1 * e.af * e.as * e.bty * e.cf * e.rr));
      }
      if (LS[5] != 0.0) {
        mb.th1 += LS[5] * (e.cf2 - e.cs2) * e.rr * e.cf * e.btz * e.as * e.af;
        mb.af += LS[5] * (e.cf2 - e.cs2) * e.rr * e.cf * e.btz * e.as * e.th1;
        mb.as = fma(LS[5] * (e.cf2 - e.cs2) * e.rr * e.cf * e.btz, e.th1 * e.af, mb.as);
        mb.btz += LS[5] * (e.cf2 - e.cs2) * e.rr * e.cf * (e.th1 * e.af * e.as);
        mb.cf += LS[5] * (e.cf2 - e.cs2) * e.rr * (e.th1 * e.af * e.as * e.btz);
        mb.rr += LS[5] * (e.cf2 - e.cs2) * (e.th1 * e.af * e.as * e.btz * e.cf);
        mb.cf2 += LS[5] * (e.th1 * e.af * e.as * e.btz * e.cf * e.rr);
        mb.cs2 += -(LS[5] * (e.th1 * e.af * e.as * e.btz * e.cf * e.rr));
      }
      if (LS[6] != 0.0) {
        mb.th1 += -(LS[6] * (e.af2 * e.a2 + e.as2 * e.cf2));
        mb.af2 = fma(LS[6] * -e.th1, e.a2, mb.af2);
        mb.a2 = fma(LS[6] * -e.th1, e.af2, mb.a2);
        mb.as2 = fma(LS[6] * -e.th1, e.cf2, mb.as2);
        mb.cf2 = fma(LS[6] * -e.th1, e.as2, mb.cf2);
      }
      { const double rs1 = fS * lF[1];
      if (rs1 != 0.0) {
        mb.u += rs1;
      } }
      { const double rs2 = fS * lF[2];
      if (rs2 != 0.0) {
        mb.v += rs2;
      } }
      { const double rs3 = fS * lF[3];
      if (rs3 != 0.0) {
        mb.w += rs3;
      } }
      { const double rs7 = fS * lF[7];
      if (rs7 != 0.0) {
        mb.uu = fma(rs7, 0.5, mb.uu);
      } }
      break;
    }
    default:
      break;
  }
}

// Adds d(Mid)/d(U1, U2)^T mb to U1b, U2b (midpoint() of mhd_eigen.cuh).
__device__ __forceinline__ void midpoint_adjoint(const Gas& G, const Mid& e, const double* U1, const double* U2, const MidBar& mb, double* U1b, double* U2b) {
  const double a0 = U1[0];
  const double a1 = U1[1];
  const double a2_ = U1[2];
  const double a3 = U1[3];
  const double a4 = U1[4];
  const double a5 = U1[5];
  const double a6 = U1[6];
  const double a7 = U1[7];
  const double b0 = U2[0];
  const double b1 = U2[1];
  const double b2 = U2[2];
  const double b3 = U2[3];
  const double b4 = U2[4];
  const double b5 = U2[5];
  const double b6 = U2[6];
  const double b7 = U2[7];
  const double gm = G.gm, gm1 = gm - 1.0, g21 = G.g21;
  const double sb = (e.sbxm ? -1.0 : 1.0);
  [[maybe_unused]] double r = 0.5 * (a0 + b0);
  [[maybe_unused]] double u = e.u;
  [[maybe_unused]] double v = e.v;
  [[maybe_unused]] double w = e.w;
  [[maybe_unused]] double bx = 0.5 * (a4 + b4);
  [[maybe_unused]] double by = 0.5 * (a5 + b5);
  [[maybe_unused]] double bz = 0.5 * (a6 + b6);
  [[maybe_unused]] double uu = e.uu;
  [[maybe_unused]] double bb = bx * bx + by * by + bz * bz;
  [[maybe_unused]] double mml = a1 * a1 + a2_ * a2_ + a3 * a3;
  [[maybe_unused]] double bbl = a4 * a4 + a5 * a5 + a6 * a6;
  [[maybe_unused]] double mmr = b1 * b1 + b2 * b2 + b3 * b3;
  [[maybe_unused]] double bbr = b4 * b4 + b5 * b5 + b6 * b6;
  [[maybe_unused]] double ptl = gm1 * (a7 - 0.5 * mml / a0 - 0.5 * bbl) + 0.5 * bbl;
  [[maybe_unused]] double ptr = gm1 * (b7 - 0.5 * mmr / b0 - 0.5 * bbr) + 0.5 * bbr;
  [[maybe_unused]] double pt = 0.5 * (ptl + ptr);
  [[maybe_unused]] double p = pt - 0.5 * bb;
  const bool p_fz = p < 0.0;
  if (p_fz) p = 0.0;
  [[maybe_unused]] double a2 = gm * p / r;
  const bool a2_fz = a2 < 0.0;
  if (a2_fz) a2 = 0.0;
  [[maybe_unused]] double a = e.a;
  [[maybe_unused]] double ca2 = e.ca2;
  [[maybe_unused]] double ca = e.ca;
  [[maybe_unused]] double c2 = 0.5 * (bb / r + a2);
  [[maybe_unused]] double ct = c2 * c2 - a2 * ca2;
  const bool ct_fz = ct < 0.0;
  if (ct_fz) ct = 0.0;
  [[maybe_unused]] double sct = sqrt(ct);
  [[maybe_unused]] double cs2 = c2 - sct;
  const bool cs2_fz = cs2 < 0.0;
  if (cs2_fz) cs2 = SMALL;
  [[maybe_unused]] double cf2 = c2 + sct;
  const bool cf2_fz = cf2 < 0.0;
  if (cf2_fz) cf2 = SMALL;
  [[maybe_unused]] double cs = e.cs;
  [[maybe_unused]] double cf = e.cf;
  [[maybe_unused]] double rr = e.rr;
  [[maybe_unused]] double bp2 = by * by + bz * bz;
  const bool deg = (bp2 < SMALL) && (fabs(ca2 - a2) < SMALL);
  [[maybe_unused]] double af2 = (cf2 - ca2) / (cf2 - cs2);
  const bool af2_fz = deg || af2 < 0.0;
  if (af2_fz) af2 = deg ? 1.0 : 0.0;
  [[maybe_unused]] double as2 = (cf2 - a2) / (cf2 - cs2);
  const bool as2_fz = deg || as2 < 0.0;
  if (as2_fz) as2 = deg ? 1.0 : 0.0;
  [[maybe_unused]] double af = e.af;
  [[maybe_unused]] double as_ = e.as;
  [[maybe_unused]] double sbp = sqrt(bp2);
  const bool sbp_fz = !(bp2 > SMALL);
  if (sbp_fz) sbp = 1.0;
  [[maybe_unused]] double bty = e.bty;
  const bool bty_fz = !(bp2 > SMALL);
  [[maybe_unused]] double btz = e.btz;
  const bool btz_fz = !(bp2 > SMALL);
  [[maybe_unused]] double th1 = e.th1;
  [[maybe_unused]] double th2 = e.th2;
  [[maybe_unused]] double vb = e.vb;
  // reverse sweep (one division per distinct denominator)
  [[maybe_unused]] const double rcp2 = 1.0 / (sbp);
  [[maybe_unused]] const double rcp3 = 1.0 / (cf2 - cs2);
  [[maybe_unused]] const double rcp4 = 1.0 / (r);
  [[maybe_unused]] const double rcp5 = 1.0 / (b0);
  [[maybe_unused]] const double rcp6 = 1.0 / (a0);
  double r_b = 0.0;
  double u_b = 0.0;
  double v_b = 0.0;
  double w_b = 0.0;
  double bx_b = 0.0;
  double by_b = 0.0;
  double bz_b = 0.0;
  double uu_b = 0.0;
  double bb_b = 0.0;
  double mml_b = 0.0;
  double bbl_b = 0.0;
  double mmr_b = 0.0;
  double bbr_b = 0.0;
  double ptl_b = 0.0;
  double ptr_b = 0.0;
  double pt_b = 0.0;
  double p_b = 0.0;
  double a2_b = 0.0;
  double a_b = 0.0;
  double ca2_b = 0.0;
  double ca_b = 0.0;
  double c2_b = 0.0;
  double ct_b = 0.0;
  double sct_b = 0.0;
  double cs2_b = 0.0;
  double cf2_b = 0.0;
  double cs_b = 0.0;
  double cf_b = 0.0;
  double rr_b = 0.0;
  double bp2_b = 0.0;
  double af2_b = 0.0;
  double as2_b = 0.0;
  double af_b = 0.0;
  double as__b = 0.0;
  double sbp_b = 0.0;
  double bty_b = 0.0;
  double btz_b = 0.0;
  double th1_b = 0.0;
  double th2_b = 0.0;
  double vb_b = 0.0;
  double a0_b = 0.0;
  double a1_b = 0.0;
  double a2__b = 0.0;
  double a3_b = 0.0;
  double a4_b = 0.0;
  double a5_b = 0.0;
  double a6_b = 0.0;
  double a7_b = 0.0;
  double b0_b = 0.0;
  double b1_b = 0.0;
  double b2_b = 0.0;
  double b3_b = 0.0;
  double b4_b = 0.0;
  double b5_b = 0.0;
  double b6_b = 0.0;
  double b7_b = 0.0;
  u_b += mb.u;
  v_b += mb.v;
  w_b += mb.w;
  uu_b += mb.uu;
  a2_b += mb.a2;
  a_b += mb.a;
  ca2_b += mb.ca2;
  ca_b += mb.ca;
  cs2_b += mb.cs2;
  cs_b += mb.cs;
  cf2_b += mb.cf2;
  cf_b += mb.cf;
  rr_b += mb.rr;
  af2_b += mb.af2;
  af_b += mb.af;
  as2_b += mb.as2;
  as__b += mb.as;
  bty_b += mb.bty;
  btz_b += mb.btz;
  th1_b += mb.th1;
  th2_b += mb.th2;
  vb_b += mb.vb;
  if (vb_b != 0.0) {
    bty_b = fma(vb_b, v, bty_b);
    v_b = fma(vb_b, bty, v_b);
    btz_b = fma(vb_b, w, btz_b);
    w_b = fma(vb_b, btz, w_b);
  }
  if (th2_b != 0.0) {
    af2_b = fma(-th2_b * 1.0 * th2 * th2 * a * cf, sb, af2_b);
    cf_b = fma(-th2_b * 1.0 * th2 * th2 * a, sb * af2, cf_b);
    a_b = fma(-th2_b * 1.0 * th2 * th2, sb * af2 * cf, a_b);
    as2_b = fma(-th2_b * 1.0 * th2 * th2 * ca * cs, sb, as2_b);
    cs_b = fma(-th2_b * 1.0 * th2 * th2 * ca, sb * as2, cs_b);
    ca_b = fma(-th2_b * 1.0 * th2 * th2, sb * as2 * cs, ca_b);
  }
  if (th1_b != 0.0) {
    af2_b = fma(-th1_b * 1.0 * th1 * th1 * (cf2 - g21 * a2), a2, af2_b);
    a2_b = fma(-th1_b * 1.0 * th1 * th1 * (cf2 - g21 * a2), af2, a2_b);
    cf2_b = fma(-th1_b * 1.0 * th1 * th1, af2 * a2, cf2_b);
    a2_b = fma(-(-th1_b * 1.0 * th1 * th1 * (af2 * a2)), g21, a2_b);
    as2_b = fma(-th1_b * 1.0 * th1 * th1 * (cs2 - g21 * a2), cf2, as2_b);
    cf2_b = fma(-th1_b * 1.0 * th1 * th1 * (cs2 - g21 * a2), as2, cf2_b);
    cs2_b = fma(-th1_b * 1.0 * th1 * th1, as2 * cf2, cs2_b);
    a2_b = fma(-(-th1_b * 1.0 * th1 * th1 * (as2 * cf2)), g21, a2_b);
  }
  if (!btz_fz && btz_b != 0.0) {
    bz_b = fma(btz_b, rcp2, bz_b);
    sbp_b = fma(-btz_b * bz * rcp2, rcp2, sbp_b);
  }
  if (!bty_fz && bty_b != 0.0) {
    by_b = fma(bty_b, rcp2, by_b);
    sbp_b = fma(-bty_b * by * rcp2, rcp2, sbp_b);
  }
  if (!sbp_fz && sbp_b != 0.0) {
    bp2_b = fma(sbp_b, inv2sqrt(bp2), bp2_b);
  }
  if (as__b != 0.0) {
    as2_b = fma(as__b, inv2sqrt(as2), as2_b);
  }
  if (af_b != 0.0) {
    af2_b = fma(af_b, inv2sqrt(af2), af2_b);
  }
  if (!as2_fz && as2_b != 0.0) {
    cf2_b = fma(as2_b, rcp3, cf2_b);
    a2_b += -((as2_b) * rcp3);
    cf2_b = fma(-as2_b * (cf2 - a2) * rcp3, rcp3, cf2_b);
    cs2_b += -(-(as2_b) * (cf2 - a2) * rcp3 * rcp3);
  }
  if (!af2_fz && af2_b != 0.0) {
    cf2_b = fma(af2_b, rcp3, cf2_b);
    ca2_b += -((af2_b) * rcp3);
    cf2_b = fma(-af2_b * (cf2 - ca2) * rcp3, rcp3, cf2_b);
    cs2_b += -(-(af2_b) * (cf2 - ca2) * rcp3 * rcp3);
  }
  if (bp2_b != 0.0) {
    by_b = fma(bp2_b, by, by_b);
    by_b = fma(bp2_b, by, by_b);
    bz_b = fma(bp2_b, bz, bz_b);
    bz_b = fma(bp2_b, bz, bz_b);
  }
  if (rr_b != 0.0) {
    r_b = fma(rr_b, inv2sqrt(r), r_b);
  }
  if (cf_b != 0.0) {
    cf2_b = fma(cf_b, inv2sqrt(cf2), cf2_b);
  }
  if (cs_b != 0.0) {
    cs2_b = fma(cs_b, inv2sqrt(cs2), cs2_b);
  }
  if (!cf2_fz && cf2_b != 0.0) {
    c2_b += cf2_b;
    sct_b += cf2_b;
  }
  if (!cs2_fz && cs2_b != 0.0) {
    c2_b += cs2_b;
    sct_b += -(cs2_b);
  }
  if (sct_b != 0.0) {
    ct_b = fma(sct_b, inv2sqrt(ct), ct_b);
  }
  if (!ct_fz && ct_b != 0.0) {
    c2_b = fma(ct_b, c2, c2_b);
    c2_b = fma(ct_b, c2, c2_b);
    a2_b = fma(-ct_b, ca2, a2_b);
    ca2_b = fma(-ct_b, a2, ca2_b);
  }
  if (c2_b != 0.0) {
    bb_b = fma(c2_b * 0.5, rcp4, bb_b);
    r_b = fma(-(c2_b * 0.5) * bb * rcp4, rcp4, r_b);
    a2_b = fma(c2_b, 0.5, a2_b);
  }
  if (ca_b != 0.0) {
    ca2_b = fma(ca_b, inv2sqrt(ca2), ca2_b);
  }
  if (ca2_b != 0.0) {
    bx_b = fma(ca2_b * rcp4, bx, bx_b);
    bx_b = fma(ca2_b * rcp4, bx, bx_b);
    r_b = fma(-ca2_b * (bx * bx) * rcp4, rcp4, r_b);
  }
  if (a_b != 0.0) {
    a2_b = fma(a_b, inv2sqrt(a2), a2_b);
  }
  if (!a2_fz && a2_b != 0.0) {
    p_b = fma(a2_b * rcp4, gm, p_b);
    r_b = fma(-a2_b * (gm * p) * rcp4, rcp4, r_b);
  }
  if (!p_fz && p_b != 0.0) {
    pt_b += p_b;
    bb_b = fma(-p_b, 0.5, bb_b);
  }
  if (pt_b != 0.0) {
    ptl_b = fma(pt_b, 0.5, ptl_b);
    ptr_b = fma(pt_b, 0.5, ptr_b);
  }
  if (ptr_b != 0.0) {
    b7_b = fma(ptr_b, gm1, b7_b);
    mmr_b = fma(-(ptr_b * gm1) * rcp5, 0.5, mmr_b);
    b0_b = fma(- -(ptr_b * gm1) * (0.5 * mmr) * rcp5, rcp5, b0_b);
    bbr_b = fma(-(ptr_b * gm1), 0.5, bbr_b);
    bbr_b = fma(ptr_b, 0.5, bbr_b);
  }
  if (ptl_b != 0.0) {
    a7_b = fma(ptl_b, gm1, a7_b);
    mml_b = fma(-(ptl_b * gm1) * rcp6, 0.5, mml_b);
    a0_b = fma(- -(ptl_b * gm1) * (0.5 * mml) * rcp6, rcp6, a0_b);
    bbl_b = fma(-(ptl_b * gm1), 0.5, bbl_b);
    bbl_b = fma(ptl_b, 0.5, bbl_b);
  }
  if (bbr_b != 0.0) {
    b4_b = fma(bbr_b, b4, b4_b);
    b4_b = fma(bbr_b, b4, b4_b);
    b5_b = fma(bbr_b, b5, b5_b);
    b5_b = fma(bbr_b, b5, b5_b);
    b6_b = fma(bbr_b, b6, b6_b);
    b6_b = fma(bbr_b, b6, b6_b);
  }
  if (mmr_b != 0.0) {
    b1_b = fma(mmr_b, b1, b1_b);
    b1_b = fma(mmr_b, b1, b1_b);
    b2_b = fma(mmr_b, b2, b2_b);
    b2_b = fma(mmr_b, b2, b2_b);
    b3_b = fma(mmr_b, b3, b3_b);
    b3_b = fma(mmr_b, b3, b3_b);
  }
  if (bbl_b != 0.0) {
    a4_b = fma(bbl_b, a4, a4_b);
    a4_b = fma(bbl_b, a4, a4_b);
    a5_b = fma(bbl_b, a5, a5_b);
    a5_b = fma(bbl_b, a5, a5_b);
    a6_b = fma(bbl_b, a6, a6_b);
    a6_b = fma(bbl_b, a6, a6_b);
  }
  if (mml_b != 0.0) {
    a1_b = fma(mml_b, a1, a1_b);
    a1_b = fma(mml_b, a1, a1_b);
    a2__b = fma(mml_b, a2_, a2__b);
    a2__b = fma(mml_b, a2_, a2__b);
    a3_b = fma(mml_b, a3, a3_b);
    a3_b = fma(mml_b, a3, a3_b);
  }
  if (bb_b != 0.0) {
    bx_b = fma(bb_b, bx, bx_b);
    bx_b = fma(bb_b, bx, bx_b);
    by_b = fma(bb_b, by, by_b);
    by_b = fma(bb_b, by, by_b);
    bz_b = fma(bb_b, bz, bz_b);
    bz_b = fma(bb_b, bz, bz_b);
  }
  if (uu_b != 0.0) {
    u_b = fma(uu_b, u, u_b);
    u_b = fma(uu_b, u, u_b);
    v_b = fma(uu_b, v, v_b);
    v_b = fma(uu_b, v, v_b);
    w_b = fma(uu_b, w, w_b);
    w_b = fma(uu_b, w, w_b);
  }
  if (bz_b != 0.0) {
    a6_b = fma(bz_b, 0.5, a6_b);
    b6_b = fma(bz_b, 0.5, b6_b);
  }
  if (by_b != 0.0) {
    a5_b = fma(by_b, 0.5, a5_b);
    b5_b = fma(by_b, 0.5, b5_b);
  }
  if (bx_b != 0.0) {
    a4_b = fma(bx_b, 0.5, a4_b);
    b4_b = fma(bx_b, 0.5, b4_b);
  }
  if (w_b != 0.0) {
    a3_b = fma(w_b * 0.5, rcp6, a3_b);
    a0_b = fma(-(w_b * 0.5) * a3 * rcp6, rcp6, a0_b);
    b3_b = fma(w_b * 0.5, rcp5, b3_b);
    b0_b = fma(-(w_b * 0.5) * b3 * rcp5, rcp5, b0_b);
  }
  if (v_b != 0.0) {
    a2__b = fma(v_b * 0.5, rcp6, a2__b);
    a0_b = fma(-(v_b * 0.5) * a2_ * rcp6, rcp6, a0_b);
    b2_b = fma(v_b * 0.5, rcp5, b2_b);
    b0_b = fma(-(v_b * 0.5) * b2 * rcp5, rcp5, b0_b);
  }
  if (u_b != 0.0) {
    a1_b = fma(u_b * 0.5, rcp6, a1_b);
    a0_b = fma(-(u_b * 0.5) * a1 * rcp6, rcp6, a0_b);
    b1_b = fma(u_b * 0.5, rcp5, b1_b);
    b0_b = fma(-(u_b * 0.5) * b1 * rcp5, rcp5, b0_b);
  }
  if (r_b != 0.0) {
    a0_b = fma(r_b, 0.5, a0_b);
    b0_b = fma(r_b, 0.5, b0_b);
  }
  U1b[0] += a0_b; U1b[1] += a1_b; U1b[2] += a2__b; U1b[3] += a3_b; U1b[4] += a4_b; U1b[5] += a5_b; U1b[6] += a6_b; U1b[7] += a7_b;
  U2b[0] += b0_b; U2b[1] += b1_b; U2b[2] += b2_b; U2b[3] += b3_b; U2b[4] += b4_b; U2b[5] += b5_b; U2b[6] += b6_b; U2b[7] += b7_b;
}

// Adds (dF/dq)^T Fb to qb for the physical x flux F(q) (F[4] = 0).
__device__ __forceinline__ void flux_x_adjoint(double gm, const double* q, const double* Fb, double* qb) {
  const double q0 = q[0];
  const double q1 = q[1];
  const double q2 = q[2];
  const double q3 = q[3];
  const double q4 = q[4];
  const double q5 = q[5];
  const double q6 = q[6];
  const double q7 = q[7];
  const double gm1 = gm - 1.0;
  [[maybe_unused]] double fu = q1 / q0;
  [[maybe_unused]] double fv = q2 / q0;
  [[maybe_unused]] double fw = q3 / q0;
  [[maybe_unused]] double fuu = fu * fu + fv * fv + fw * fw;
  [[maybe_unused]] double fub = fu * q4 + fv * q5 + fw * q6;
  [[maybe_unused]] double fbb = q4 * q4 + q5 * q5 + q6 * q6;
  [[maybe_unused]] double fp = gm1 * (q7 - 0.5 * q0 * fuu - 0.5 * fbb);
  [[maybe_unused]] double fpt = fp + 0.5 * fbb;
  [[maybe_unused]] double fo0 = q1;
  [[maybe_unused]] double fo1 = q1 * fu - q4 * q4 + fpt;
  [[maybe_unused]] double fo2 = q2 * fu - q4 * q5;
  [[maybe_unused]] double fo3 = q3 * fu - q4 * q6;
  [[maybe_unused]] double fo5 = q5 * fu - q4 * fv;
  [[maybe_unused]] double fo6 = q6 * fu - q4 * fw;
  [[maybe_unused]] double fo7 = (q7 + fpt) * fu - q4 * fub;
  // reverse sweep (one division per distinct denominator)
  [[maybe_unused]] const double rcp0 = 1.0 / (q0);
  double fu_b = 0.0;
  double fv_b = 0.0;
  double fw_b = 0.0;
  double fuu_b = 0.0;
  double fub_b = 0.0;
  double fbb_b = 0.0;
  double fp_b = 0.0;
  double fpt_b = 0.0;
  double fo0_b = 0.0;
  double fo1_b = 0.0;
  double fo2_b = 0.0;
  double fo3_b = 0.0;
  double fo5_b = 0.0;
  double fo6_b = 0.0;
  double fo7_b = 0.0;
  double q0_b = 0.0;
  double q1_b = 0.0;
  double q2_b = 0.0;
  double q3_b = 0.0;
  double q4_b = 0.0;
  double q5_b = 0.0;
  double q6_b = 0.0;
  double q7_b = 0.0;
  fo0_b = Fb[0];
  fo1_b = Fb[1];
  fo2_b = Fb[2];
  fo3_b = Fb[3];
  fo5_b = Fb[5];
  fo6_b = Fb[6];
  fo7_b = Fb[7];
  if (fo7_b != 0.0) {
    q7_b = fma(fo7_b, fu, q7_b);
    fpt_b = fma(fo7_b, fu, fpt_b);
    fu_b = fma(fo7_b, q7 + fpt, fu_b);
    q4_b = fma(-fo7_b, fub, q4_b);
    fub_b = fma(-fo7_b, q4, fub_b);
  }
  if (fo6_b != 0.0) {
    q6_b = fma(fo6_b, fu, q6_b);
    fu_b = fma(fo6_b, q6, fu_b);
    q4_b = fma(-fo6_b, fw, q4_b);
    fw_b = fma(-fo6_b, q4, fw_b);
  }
  if (fo5_b != 0.0) {
    q5_b = fma(fo5_b, fu, q5_b);
    fu_b = fma(fo5_b, q5, fu_b);
    q4_b = fma(-fo5_b, fv, q4_b);
    fv_b = fma(-fo5_b, q4, fv_b);
  }
  if (fo3_b != 0.0) {
    q3_b = fma(fo3_b, fu, q3_b);
    fu_b = fma(fo3_b, q3, fu_b);
    q4_b = fma(-fo3_b, q6, q4_b);
    q6_b = fma(-fo3_b, q4, q6_b);
  }
  if (fo2_b != 0.0) {
    q2_b = fma(fo2_b, fu, q2_b);
    fu_b = fma(fo2_b, q2, fu_b);
    q4_b = fma(-fo2_b, q5, q4_b);
    q5_b = fma(-fo2_b, q4, q5_b);
  }
  if (fo1_b != 0.0) {
    q1_b = fma(fo1_b, fu, q1_b);
    fu_b = fma(fo1_b, q1, fu_b);
    q4_b = fma(-fo1_b, q4, q4_b);
    q4_b = fma(-fo1_b, q4, q4_b);
    fpt_b += fo1_b;
  }
  if (fo0_b != 0.0) {
    q1_b += fo0_b;
  }
  if (fpt_b != 0.0) {
    fp_b += fpt_b;
    fbb_b = fma(fpt_b, 0.5, fbb_b);
  }
  if (fp_b != 0.0) {
    q7_b = fma(fp_b, gm1, q7_b);
    q0_b = fma(-(fp_b * gm1) * fuu, 0.5, q0_b);
    fuu_b = fma(-(fp_b * gm1), 0.5 * q0, fuu_b);
    fbb_b = fma(-(fp_b * gm1), 0.5, fbb_b);
  }
  if (fbb_b != 0.0) {
    q4_b = fma(fbb_b, q4, q4_b);
    q4_b = fma(fbb_b, q4, q4_b);
    q5_b = fma(fbb_b, q5, q5_b);
    q5_b = fma(fbb_b, q5, q5_b);
    q6_b = fma(fbb_b, q6, q6_b);
    q6_b = fma(fbb_b, q6, q6_b);
  }
  if (fub_b != 0.0) {
    fu_b = fma(fub_b, q4, fu_b);
    q4_b = fma(fub_b, fu, q4_b);
    fv_b = fma(fub_b, q5, fv_b);
    q5_b = fma(fub_b, fv, q5_b);
    fw_b = fma(fub_b, q6, fw_b);
    q6_b = fma(fub_b, fw, q6_b);
  }
  if (fuu_b != 0.0) {
    fu_b = fma(fuu_b, fu, fu_b);
    fu_b = fma(fuu_b, fu, fu_b);
    fv_b = fma(fuu_b, fv, fv_b);
    fv_b = fma(fuu_b, fv, fv_b);
    fw_b = fma(fuu_b, fw, fw_b);
    fw_b = fma(fuu_b, fw, fw_b);
  }
  if (fw_b != 0.0) {
    q3_b = fma(fw_b, rcp0, q3_b);
    q0_b = fma(-fw_b * q3 * rcp0, rcp0, q0_b);
  }
  if (fv_b != 0.0) {
    q2_b = fma(fv_b, rcp0, q2_b);
    q0_b = fma(-fv_b * q2 * rcp0, rcp0, q0_b);
  }
  if (fu_b != 0.0) {
    q1_b = fma(fu_b, rcp0, q1_b);
    q0_b = fma(-fu_b * q1 * rcp0, rcp0, q0_b);
  }
  qb[0] += q0_b;
  qb[1] += q1_b;
  qb[2] += q2_b;
  qb[3] += q3_b;
  qb[4] += q4_b;
  qb[5] += q5_b;
  qb[6] += q6_b;
  qb[7] += q7_b;
}

}  // namespace MHD_KNS
}  // namespace mhd
