// Launchers of the discrete adjoint's reverse-sweep kernels (interface
// adjoint, per-cell gather, boundary-fill transpose).  They live in their own
// translation unit, mhd_adjoint_rev.cu, built twice: with FMA contraction
// (the default reverse sweep) and without.  The recording and replay kernels
// of mhd_adjoint.cu stay uncontracted, so the forward trajectory is the
// parity build's either way.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "mhd_common.cuh"

namespace mhd {
namespace adjrev {

// gamma and the gamma-only constants of the eigen-system, as the host
// computes them for the forward kernels.
struct GasConsts {
  double gm, g1, g21, rs2;
};

// The launchers, once per build of mhd_adjoint_rev.cu: `contracted` (FMA
// contraction, the recomputed midpoint kept unfused) and `uncontracted`
// (the parity build's rounding throughout).
#define MHD_ADJREV_LAUNCHERS                                                                   \
  /* Doubles of one direction's cell-record scratch (S of launch_iface). */                   \
  size_t record_doubles(const Grid& g, bool ydir);                                            \
  /* Adjoint of every interface of one direction at stage input X (ENO and upwind choices  */ \
  /* frozen by the recorded words in mask); lB is the adjoint of the stage output, cL the  */ \
  /* coefficient of UL in the stage update.  Writes the direction's cell records to S.     */ \
  void launch_iface(const Grid& g, const GasConsts& G, bool ydir, const double* X,            \
                    const unsigned* mask, const double* lB, double cL, double* S,             \
                    double inv_d, cudaStream_t st);                                           \
  /* Per cell: both directions' records, transposed flux Jacobians, the stage update's     */ \
  /* adjoint (mode), the result added to lU / lU1 / lU2 (in_buf) for interior cells and    */ \
  /* written to T for ghost cells.                                                          */ \
  void launch_gather(const Grid& g, const GasConsts& G, const double* X, const double* SX,    \
                     const double* SY, double* T, int mode, int in_buf, double* lU,           \
                     double* lU1, double* lU2, cudaStream_t st);                              \
  /* Transpose of the boundary fill for the two sides of one direction. */                    \
  void launch_bc(const Grid& g, int ydir, const double* T, double* D, double* lsnap_lo,       \
                 double* lsnap_hi, cudaStream_t st);

namespace contracted {
MHD_ADJREV_LAUNCHERS
}  // namespace contracted
namespace uncontracted {
MHD_ADJREV_LAUNCHERS
}  // namespace uncontracted

}  // namespace adjrev
}  // namespace mhd
