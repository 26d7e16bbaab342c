// Host-side launchers of the device kernels.  The kernel translation unit
// is compiled twice: once with -fmad=false (bit-identical to the reference,
// the default) and once with FMA contraction (MHD_FLAG_FAST_MATH); each
// build exports one KernelSet.
#pragma once

#include <cuda_runtime.h>

#include "mhd_common.cuh"

namespace mhd {

struct CharOut;
struct Snap;
struct StepParams;
struct DivRange;
struct SorCoef;

struct KernelSet {
  const char* name;
  // boundary fill of U in place
  void (*bc)(const Grid& g, double* U, const double* const snap[4], const Ctl* ctl,
             cudaStream_t s);
  void (*snapshot)(const Grid& g, const double* U, double* const snap[4], cudaStream_t s);
  // ENO-LF dissipation (arrays zeroed here)
  void (*lf_alpha)(const Grid& g, const double* U, double* aF, double* aG, Ctl* ctl,
                   cudaStream_t s);
  // fused spatial operator; chars: cx, cy, LUx, LUy or nulls
  void (*flux)(int scheme, const Grid& g, const double* U, double* UL, const double* aF,
               const double* aG, Ctl* ctl, double* const chars[4], cudaStream_t s);
  void (*combine)(const Grid& g, int mode, double* U, double* U1, double* U2, const double* UL,
                  const Ctl* ctl, cudaStream_t s);
  void (*control)(Ctl* ctl, double dx, double dy, double dt_min, double dt_max, double cfl,
                  int phase, double arg, cudaStream_t s);
  // div B: wrap periodic B ghosts, reduce max / sum over [x0,x1) x [y0,y1)
  void (*divb)(const Grid& g, double* U, const int range[4], double* partial, int npartial,
               Ctl* ctl, cudaStream_t s);
  // the fixed source terms of one SOR solve (xy: 4 doubles per same-colour
  // column pair, sor_xy_doubles of them)
  void (*sor_rhs)(const Grid& g, const double* U, const int range[4], const double coef[6],
                  double* xy, cudaStream_t s);
  // one SOR sweep (both colours, potential ghosts, convergence check).
  // fused = 1: two launches that read periodic ghosts at their source and
  // run the convergence check in the second one (sor_fused_ok must hold;
  // the caller refreshes the ghosts with phi_bc before the first and after
  // the last sweep of the solve).  rows_mode: 0 by grid size, 1 one row at a
  // time with reused loads, 2 two rows in flight per thread (same values)
  void (*sor_sweep)(const Grid& g, double* phi, const double* xy, const int range[4],
                    const double coef[6], double rtol, double max_sweeps, double* last_ratio,
                    Ctl* ctl, int fused, int rows_mode, cudaStream_t s);
  // potential ghosts (div_b_fix.cpp:282-364), regardless of the stop flag
  void (*phi_bc)(const Grid& g, double* phi, const Ctl* ctl, cudaStream_t s);
  void (*sor_correct)(const Grid& g, double* U, const double* phi, const int range[4],
                      double bxf, double byf, cudaStream_t s);
  // non-grid output totals: 5 partials per block (entropy, energy, mass,
  // momentum sums, max |u|^2); returns the number of blocks used
  int (*totals)(const Grid& g, const double* U, double* partial, int max_blocks, cudaStream_t s);
  int (*flux_smem_bytes)();
  int (*launches_per_integrate)(int scheme);
  // the boundary fill in parts (the same values as bc): part 1 the left /
  // right sides, part 2 the bottom / top sides of rows [i0, i1) (2 <= i0,
  // i1 <= nx + 2)
  void (*bc_part)(const Grid& g, double* U, const double* const snap[4], const Ctl* ctl,
                  int part, int i0, int i1, cudaStream_t s);
  // tile rows [ti0, ti1) of the ENO spatial operator (flux_tile_rows cell rows each)
  void (*flux_rows)(int scheme, const Grid& g, const double* U, double* UL, const double* aF,
                    const double* aG, Ctl* ctl, double* const chars[4], int ti0, int ti1,
                    cudaStream_t s);
  int (*flux_tile_rows)(int scheme);
  // the last RK3 stage update of rows [i0, i1) (0 <= i0, i1 <= NX) into U1,
  // U's ghost cells copied beside it (mhd_step_host's copy-back overlap)
  void (*combine_final_rows)(const Grid& g, int i0, int i1, double* U, double* U1, double* U2,
                             const double* UL, const Ctl* ctl, cudaStream_t s);
};

extern const KernelSet kExact;
extern const KernelSet kFast;

}  // namespace mhd
