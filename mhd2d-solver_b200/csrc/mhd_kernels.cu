// Kernel instantiations and launchers.  Built twice from this one source:
//   MHD_KSET = kExact  with -fmad=false  (bit-identical to the reference)
//   MHD_KSET = kFast   with -fmad=true   (FMA contraction)
#include <cmath>

#include "mhd_cfd.cuh"
#include "mhd_flux.cuh"
#include "mhd_launch.h"
#include "mhd_misc.cuh"

#ifndef MHD_KSET
#define MHD_KSET kExact
#define MHD_KSET_NAME "exact"
#endif

namespace mhd {
namespace MHD_KNS {

// Tiles of the fused flux kernel, rows x 32 columns and warps per CTA, per
// scheme.  ENO-Roe: 7 x 32, 8 warps: 16 warp tasks per tile = 2 rounds, 90 KB
// of shared memory and at most 128 registers per thread, so 2 CTAs = 16 warps
// per SM (measured best against 8x32/6 warps, 15x32/16 warps (5.43 against
// 5.40 ms at 4096^2), 11x32/12 warps, and smaller tiles at 96 registers).
// ENO-LF: 15 x 32, 16 warps: 32 tasks = 2 rounds, 172 KB, one CTA of 16
// warps per SM, 16/15 x-interface rows per cell row instead of 8/7
// (6.89 against 7.23 ms at 4096^2).
#ifndef MHD_TI
#define MHD_TI 7
#endif
#ifndef MHD_NW
#define MHD_NW 8
#endif
#ifndef MHD_TI_LF
#define MHD_TI_LF 15
#endif
#ifndef MHD_NW_LF
#define MHD_NW_LF 16
#endif
constexpr int TI = MHD_TI, TJ = 32;  // the ENO-Roe tile (Geom: l_smem)
template <int SCHEME>
struct FluxShape {
  static constexpr int TI = MHD_TI, NW = MHD_NW;
};
template <>
struct FluxShape<3> {
  static constexpr int TI = MHD_TI_LF, NW = MHD_NW_LF;
};
using Geom = TileGeom<TI, TJ>;

int grid1d(long long n, int block) {
  long long b = (n + block - 1) / block;
  if (b < 1) b = 1;
  if (b > 148LL * 16) b = 148LL * 16;
  return int(b);
}

void l_bc(const Grid& g, double* U, const double* const snap[4], const Ctl* ctl, cudaStream_t s) {
  Snap d{snap[0], snap[1], snap[2], snap[3]};
  const long long n = 4LL * NF * g.ny + 4LL * NF * g.nx;
  k_bc<<<grid1d(n, 256), 256, 0, s>>>(g, U, d, ctl);
}

void l_snapshot(const Grid& g, const double* U, double* const snap[4], cudaStream_t s) {
  const int m = g.nx > g.ny ? g.nx : g.ny;
  k_snapshot<<<grid1d(NF * m, 256), 256, 0, s>>>(g, U, snap[0], snap[1], snap[2], snap[3]);
}

void l_lf_alpha(const Grid& g, const double* U, double* aF, double* aG, Ctl* ctl, cudaStream_t s) {
  cudaMemsetAsync(aF, 0, sizeof(double) * NF * g.NY, s);
  cudaMemsetAsync(aG, 0, sizeof(double) * NF * g.NX, s);
  dim3 grid((g.ny + 1 + 31) / 32, (g.nx + 1 + 7) / 8);
  k_lf_alpha<<<grid, 256, 0, s>>>(g, U, aF, aG, ctl);
}

// Tile rows [ti0, ti1) of the spatial operator (ti1 < 0: to the last).
template <int SCHEME, bool CHARS>
void flux_t(const Grid& g, const double* U, double* UL, const double* aF, const double* aG,
            Ctl* ctl, double* const ch[4], cudaStream_t s, int ti0 = 0, int ti1 = -1) {
  constexpr int ti = FluxShape<SCHEME>::TI, nw = FluxShape<SCHEME>::NW;
  using Gm = TileGeom<ti, TJ>;
  auto kern = k_flux<SCHEME, CHARS, ti, TJ, nw>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(Gm::TMA_BYTES));
    attr = true;
  }
  const int nti = (g.nx + ti - 1) / ti;
  if (ti1 < 0 || ti1 > nti) ti1 = nti;
  if (ti1 <= ti0) return;
  dim3 grid((g.ny + TJ - 1) / TJ, ti1 - ti0);
  CharOut co{ch ? ch[0] : nullptr, ch ? ch[1] : nullptr, ch ? ch[2] : nullptr,
             ch ? ch[3] : nullptr};
#ifdef MHD_FAST
  const Gas G{g.gamma, g.gamma - 1.0, (g.gamma - 2.0) / (g.gamma - 1.0), 1.0 / std::sqrt(2.0),
              1.0 / (g.gamma - 1.0)};
#else
  const Gas G{g.gamma, g.gamma - 1.0, (g.gamma - 2.0) / (g.gamma - 1.0), 1.0 / std::sqrt(2.0)};
#endif
  CUtensorMap tm{};
  const int use_tma = tile_tma_enabled() && make_box_map(g, U, Gm::CU, Gm::RU, &tm) ? 1 : 0;
  tile_tma_launches() += use_tma;
  kern<<<grid, nw * 32, Gm::TMA_BYTES, s>>>(g, U, UL, aF, aG, 1.0 / g.dx, 1.0 / g.dy, G, ctl, co,
                                          nullptr, nullptr, tm, use_tma, ti0);
}

void l_flux(int scheme, const Grid& g, const double* U, double* UL, const double* aF,
            const double* aG, Ctl* ctl, double* const ch[4], cudaStream_t s) {
  const bool chars = ch && ch[0];
  if (scheme == 1) {  // central FD: checks and maxima, then UL
    dim3 inner((g.ny + CFD_TJ - 1) / CFD_TJ, (g.nx + CFD_TI - 1) / CFD_TI);
    k_cfd_check<<<grid1d((long long)(g.nx + 2) * (g.ny + 2), 256), 256, 0, s>>>(g, U, ctl);
    k_cfd_ul<<<inner, 256, 0, s>>>(g, U, UL, 1.0 / (2.0 * g.dx), 1.0 / (2.0 * g.dy), ctl);
    return;
  }
  if (scheme == 3) {
    if (chars) flux_t<3, true>(g, U, UL, aF, aG, ctl, ch, s);
    else flux_t<3, false>(g, U, UL, aF, aG, ctl, ch, s);
  } else {
    if (chars) flux_t<2, true>(g, U, UL, aF, aG, ctl, ch, s);
    else flux_t<2, false>(g, U, UL, aF, aG, ctl, ch, s);
  }
}

// Tile rows [ti0, ti1) of the ENO spatial operator (schemes 2 and 3; the
// ENO-LF coefficients must be complete).
void l_flux_rows(int scheme, const Grid& g, const double* U, double* UL, const double* aF,
                 const double* aG, Ctl* ctl, double* const ch[4], int ti0, int ti1,
                 cudaStream_t s) {
  const bool chars = ch && ch[0];
  if (scheme == 3) {
    if (chars) flux_t<3, true>(g, U, UL, aF, aG, ctl, ch, s, ti0, ti1);
    else flux_t<3, false>(g, U, UL, aF, aG, ctl, ch, s, ti0, ti1);
  } else {
    if (chars) flux_t<2, true>(g, U, UL, aF, aG, ctl, ch, s, ti0, ti1);
    else flux_t<2, false>(g, U, UL, aF, aG, ctl, ch, s, ti0, ti1);
  }
}

int l_flux_tile_rows(int scheme) {
  return scheme == 3 ? FluxShape<3>::TI : FluxShape<2>::TI;
}

void l_bc_part(const Grid& g, double* U, const double* const snap[4], const Ctl* ctl, int part,
               int i0, int i1, cudaStream_t s) {
  const Snap d{snap[0], snap[1], snap[2], snap[3]};
  const long long n = part == 1 ? 2LL * 2 * NF * g.ny : 2LL * NF * (i1 - i0) * 2;
  if (n <= 0) return;
  k_bc_part<<<grid1d(n, 256), 256, 0, s>>>(g, U, d, ctl, part, i0, i1);
}

void l_combine(const Grid& g, int mode, double* U, double* U1, double* U2, const double* UL,
               const Ctl* ctl, cudaStream_t s) {
  dim3 grid((g.ny + 255) / 256, g.nx, NF);
  k_combine<<<grid, 256, 0, s>>>(g, mode, U, U1, U2, UL, ctl);
}

void l_combine_final_rows(const Grid& g, int i0, int i1, double* U, double* U1, double* U2,
                          const double* UL, const Ctl* ctl, cudaStream_t s) {
  if (i1 <= i0) return;
  dim3 grid((g.NY + 255) / 256, i1 - i0, NF);
  k_combine_final_rows<<<grid, 256, 0, s>>>(g, i0, i1, U, U1, U2, UL, ctl);
}

void l_control(Ctl* ctl, double dx, double dy, double dt_min, double dt_max, double cfl,
               int phase, double arg, cudaStream_t s) {
  StepParams p{dx, dy, dt_min, dt_max, cfl};
  k_control<<<1, 32, 0, s>>>(ctl, p, phase, arg);
}

void l_divb(const Grid& g, double* U, const int range[4], double* partial, int npartial,
            Ctl* ctl, cudaStream_t s) {
  const int m = g.nx > g.ny ? g.nx : g.ny;
  k_divb_wrap<<<grid1d(4LL * m, 256), 256, 0, s>>>(g, U);
  DivRange R{range[0], range[1], range[2], range[3]};
  cudaMemsetAsync(&ctl->divb_max, 0, sizeof(unsigned long long), s);
  const long long n = (long long)(R.x1 - R.x0) * (R.y1 - R.y0);
  int nb = grid1d(n, 256);
  if (nb > npartial) nb = npartial;
  k_divb_reduce<<<nb, 256, 0, s>>>(g, U, R, partial, ctl);
  k_divb_finish<<<1, 32, 0, s>>>(partial, nb, g.dx * g.dy, ctl);
}

void l_sor_rhs(const Grid& g, const double* U, const int range[4], const double coef[6],
               double* xy, cudaStream_t s) {
  DivRange R{range[0], range[1], range[2], range[3]};
  SorCoef c{coef[0], coef[1], coef[2], coef[3], coef[4], coef[5]};
  const long long n = 2LL * (R.x1 - R.x0) * sor_pairs(R);
  k_sor_rhs<<<grid1d(n, 256), 256, 0, s>>>(g, U, R, c, reinterpret_cast<double4*>(xy));
}

template <bool PAIRS>
void sor_sweep_t(const Grid& g, double* phi, const double4* f, const DivRange& R,
                 const SorCoef& c, dim3 grid, int rpb, double rtol, double max_sweeps,
                 double* last_ratio, Ctl* ctl, int fused, cudaStream_t s) {
  const int m = g.nx > g.ny ? g.nx : g.ny;
  if (fused) {
    k_sor_half<true, PAIRS><<<grid, SOR_THREADS, 0, s>>>(g, phi, f, R, c, 0, ctl, rtol,
                                                         max_sweeps, last_ratio, rpb);
    k_sor_half<true, PAIRS><<<grid, SOR_THREADS, 0, s>>>(g, phi, f, R, c, 1, ctl, rtol,
                                                         max_sweeps, last_ratio, rpb);
    return;
  }
  // ghosts are refreshed after each colour: with periodic sides they mirror
  // points of the other colour (see k_sor_half)
  k_sor_half<false, PAIRS><<<grid, SOR_THREADS, 0, s>>>(g, phi, f, R, c, 0, ctl, rtol,
                                                        max_sweeps, last_ratio, rpb);
  k_phi_bc<<<grid1d(2LL * m, 256), 256, 0, s>>>(g, phi, ctl, 0);
  k_sor_half<false, PAIRS><<<grid, SOR_THREADS, 0, s>>>(g, phi, f, R, c, 1, ctl, rtol,
                                                        max_sweeps, last_ratio, rpb);
  k_phi_bc<<<grid1d(2LL * m, 256), 256, 0, s>>>(g, phi, ctl, 0);
  k_sor_check<<<1, 32, 0, s>>>(ctl, rtol, max_sweeps, last_ratio);
}

void l_sor_sweep(const Grid& g, double* phi, const double* xy, const int range[4],
                 const double coef[6], double rtol, double max_sweeps, double* last_ratio,
                 Ctl* ctl, int fused, int rows_mode, cudaStream_t s) {
  DivRange R{range[0], range[1], range[2], range[3]};
  SorCoef c{coef[0], coef[1], coef[2], coef[3], coef[4], coef[5]};
  // rows per block: SOR_ROWS, halved while the grid would have fewer than 4
  // blocks per SM of a B200 (148 SMs)
  const int bx = (sor_pairs(R) + SOR_THREADS - 1) / SOR_THREADS, rows = R.x1 - R.x0;
  int rpb = SOR_ROWS;
  while (rpb > 1 && (long long)bx * ((rows + rpb - 1) / rpb) < 4LL * 148) rpb /= 2;
  dim3 grid(bx, (rows + rpb - 1) / rpb);
  const double4* f = reinterpret_cast<const double4*>(xy);
  // Two rows in flight per thread from 2^19 same-colour pairs per colour
  // (grids of about 2 M cells) up: measured 4-8 % faster per sweep at 2048^2
  // to 4096^2 and ~11 % slower at 512^2 and 1024^2, where reusing loads
  // along one row chain wins.  The same values either way.
  const bool pairs = rows_mode == 0 ? (long long)rows * sor_pairs(R) >= (1LL << 19) : rows_mode == 2;
  if (pairs)
    sor_sweep_t<true>(g, phi, f, R, c, grid, rpb, rtol, max_sweeps, last_ratio, ctl, fused, s);
  else
    sor_sweep_t<false>(g, phi, f, R, c, grid, rpb, rtol, max_sweeps, last_ratio, ctl, fused, s);
}

void l_phi_bc(const Grid& g, double* phi, const Ctl* ctl, cudaStream_t s) {
  const int m = g.nx > g.ny ? g.nx : g.ny;
  k_phi_bc<<<grid1d(2LL * m, 256), 256, 0, s>>>(g, phi, ctl, 1);
}

void l_sor_correct(const Grid& g, double* U, const double* phi, const int range[4], double bxf,
                   double byf, cudaStream_t s) {
  DivRange R{range[0], range[1], range[2], range[3]};
  const long long n = (long long)(R.x1 - R.x0 + 2) * (R.y1 - R.y0 + 2);
  k_sor_correct<<<grid1d(n, 256), 256, 0, s>>>(g, U, phi, R, bxf, byf);
}

int l_totals(const Grid& g, const double* U, double* partial, int max_blocks, cudaStream_t s) {
  int nb = grid1d((long long)g.nx * g.ny, TOT_THREADS);
  if (nb > max_blocks) nb = max_blocks;
  k_totals<<<nb, TOT_THREADS, 0, s>>>(g, U, partial);
  return nb;
}

int l_smem() { return int(Geom::TMA_BYTES); }
int l_launches(int scheme) { return scheme == 2 ? 2 : 3; }  // bc, [alpha], flux; bc, check, UL

}  // namespace MHD_KNS

using namespace MHD_KNS;
extern const KernelSet MHD_KSET = {MHD_KSET_NAME, l_bc, l_snapshot, l_lf_alpha, l_flux,
                                   l_combine, l_control, l_divb, l_sor_rhs, l_sor_sweep,
                                   l_phi_bc, l_sor_correct, l_totals, l_smem, l_launches,
                                   l_bc_part, l_flux_rows, l_flux_tile_rows,
                                   l_combine_final_rows};

}  // namespace mhd
