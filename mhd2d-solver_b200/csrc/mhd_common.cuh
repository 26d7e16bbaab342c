// Device-side data layout and small helpers shared by the kernels.
//
// HBM layout of one state block: field-major like the reference
// ([k][i][j], j fastest, vector_utilities.cpp:81-98) but with padded rows:
// row (k, i) starts at k*fstride + i*pitch, and element j of the row lives
// at column off + j.  pitch is a multiple of 16 doubles (128 B) and off = 14,
// so the first interior cell j = 2 of every row sits on a 128-byte line and
// a warp's 32 consecutive interior cells touch exactly two lines.
#pragma once

#include <cstdint>

namespace mhd {

constexpr int NF = 8;           // conserved fields
constexpr int ROW_OFF = 14;     // column of j = 0 inside a padded row
constexpr double SMALL = 1e-20; // EPS of the reference (mhd2d.hpp:76)

enum Bc : int { PERIODIC = 1, DIRICHLET = 2, NEUMANN = 3, OPEN = 4 };
enum Side : int { LEFT = 0, RIGHT = 1, BOTTOM = 2, TOP = 3 };

struct Grid {
  int nx, ny;        // interior cells
  int NX, NY;        // nx+4, ny+4
  int pitch;         // doubles per padded row
  int off;           // ROW_OFF
  long long fstride; // doubles per field plane (NX*pitch)
  double dx, dy, gamma;
  int bc[4];         // left, right, bottom, top
  // bc[side] for a side known only at run time, by selects: indexing the
  // kernel-parameter array with a run-time index copies the Grid to local memory
  __host__ __device__ int bc_of(int side) const {
    return side == 0 ? bc[0] : side == 1 ? bc[1] : side == 2 ? bc[2] : bc[3];
  }
  __host__ __device__ long long at(int k, int i, int j) const {
    return (long long)k * fstride + (long long)i * pitch + off + j;
  }
};

// Fused SOR sweeps: a periodic side's ghost rows / columns are copies of
// interior points (k_phi_bc).  When every periodic side's grid extent is a
// multiple of 4, a copied point lies an odd number of 2-cell blocks away
// from the points that read its ghost, so it has the other colour: during a
// half sweep it does not change, and reading it in place gives the value
// its ghost would hold.  Open sides copy a point that no sweep updates (row / column 2 or
// n+1), so their ghosts need refreshing only once per solve.  A fused sweep
// is then two launches with no ghost refresh in between.
__host__ __device__ inline bool sor_fused_ok(const Grid& g) {
  const bool px = g.bc[LEFT] == PERIODIC || g.bc[RIGHT] == PERIODIC;
  const bool py = g.bc[BOTTOM] == PERIODIC || g.bc[TOP] == PERIODIC;
  return (!px || g.nx % 4 == 0) && (!py || g.ny % 4 == 0);
}

// Device control block of one context: reductions, dt bookkeeping and the
// status words the host reads back once per call.
struct Ctl {
  unsigned long long maxX, maxY;  // bit patterns of max |lambda| (non-negative)
  int skip;        // 1: an earlier kernel asked the rest of the sequence to stand down
  int retry;       // RK3 stage asked for a smaller dt
  int error;       // ReturnStatus of a fatal error, 0 if none
  int neg_last;    // pressure clamped at the last interface of the sweep
  unsigned long long neg_count;  // clamped midpoint pressures
  unsigned long long negd_count; // non-positive densities met
  double dtIdeal;
  double dt1, dt2, dt3, dt;       // RK3: dtFirstStep, dtSecondStep, dtFinalStep, dt
  int upd_status;  // last updateDt result
  int step_done;
  // div B / SOR
  unsigned long long rmax, pmax;  // bit patterns of the sweep maxima
  unsigned long long divb_max;    // bit pattern of max |div B|
  double divb_sum;
  int sor_done, sor_sweeps;
  unsigned sor_ticket;  // blocks of a fused SOR colour launch that have finished
  int pad;
  // central FD (k_cfd_check): kCfdFirstBase - (i*NY + j) of the first
  // non-positive density, 1 + (i*NY + j) of the last non-positive pressure;
  // 0 = none
  unsigned long long cfd_first, cfd_last;
};

constexpr unsigned long long kCfdFirstBase = 1ull << 62;

// Phases of the one-thread time-step controller (k_control).
enum CtlPhase : int {
  PH_RESET_STEP = 0,   // arg: dt_in -> dt1 = dt = dt_in, dt2 = dt3 = dt_max
  PH_RK_FIRST = 1,     // after L(U): updateDt(dt1), dt = min(dt1,dt2,dt3)
  PH_RK_SECOND = 2,    // after L(U1): updateDt(dt2), retry if dt2 < dt
  PH_RK_FINAL = 3,     // after L(U2): updateDt(dt3), retry if dt3 < dt
  PH_RK_RETRY = 4,     // restart of the stage loop
  PH_EULER = 5,        // after L(U): updateDt(dt)
  PH_IDEAL = 6,        // plain integrate: dtIdeal only
  PH_DONE = 7,         // mark the step complete
  PH_RESET_INTEGRATE = 8,
  PH_RESET_CARRY = 9   // as PH_RESET_STEP with dt_in = the previous step's dt (graph step loop)
};

__device__ __forceinline__ void atomic_max_pos(unsigned long long* a, double v) {
  // v is non-negative and not NaN: IEEE order == unsigned order of the bits
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

__device__ __forceinline__ double bits_to_double(unsigned long long b) {
  return __longlong_as_double((long long)b);
}

// NaN-skipping running maximum (a NaN candidate never replaces the value),
// the semantics of "if( x > m ) m = x" used throughout the reference.
__device__ __forceinline__ double take_max(double m, double x) { return x > m ? x : m; }

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = take_max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

}  // namespace mhd
