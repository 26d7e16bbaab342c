// Discrete adjoint of the ENO-Roe RK3-TVD (or Euler) time step
// (include/mhd2d_b200.h, mhd_adj_*).
//
// Forward (recording) run — the reference main loop's stepping
// (TimeIntegrationRK3::step with its retry rule, updateDt) on the device:
//   * every executed spatial operator ("stage") is logged by the controller
//     kernel: which buffer it read (U, U1, U2), the stage update that
//     followed (k_combine mode) and its dt;
//   * the flux kernel records, per interface and characteristic, the ENO-2
//     stencil choices of w- and w+ and the upwind choice as 4-bit codes
//     (one 32-bit word per interface);
//   * U is checkpointed at the start of every K-th step.
// Replay — the same stage sequence with the recorded choices and dt frozen
// (k_flux MASK = 2): bit-identical to the recording on the same initial
// state; on a perturbed one it is the frozen-stencil, frozen-dt map whose
// derivative the adjoint computes (central finite differences use it).
// Backward — for each checkpoint segment, last first: replay the segment
// from its checkpoint keeping every stage input, then walk its stages in
// reverse: adjoint of the stage update (linear), then the adjoint of the
// spatial operator L at the stored stage input (mhd_adjoint_rev.cu, compiled
// with FMA contraction):
//   1. ka_adj_iface: per x / y interface, recompute the midpoint
//      eigen-system and the frozen ENO combination, and form the adjoints
//      of the 4 stencil fluxes and of the two midpoint states
//      (mhd_adjoint_gen.cuh, generated reverse-mode code); it reads the
//      adjoint of UL as a multiple of the stage output's adjoint; each warp
//      takes a tile of interfaces and writes one record per cell its
//      stencils touch (the sums of its interfaces' contributions there);
//   2. ka_adj_gather: per cell, add the one or two records of each
//      direction and apply the transposed flux Jacobians; interior cells
//      also apply the rest of the stage update's adjoint and add the result
//      to the stage input's adjoint, ghost cells go to T;
//   3. ka_adj_bc: transpose of the boundary fill (ghost adjoints in T ->
//      interior; the Dirichlet edges, snapshots of U0, collect their own
//      adjoints).
// The result is dJ/dU0 for J = sum of the kinetic energy |m|^2 / (2 rho)
// dx dy over the final interior.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/mhd2d_b200.h"
#include "mhd_adjoint_rev.h"
#include "mhd_flux.cuh"
#include "mhd_misc.cuh"
#include "mhd_problems.cuh"
#include "mhd_trace.h"

namespace mhd {
namespace MHD_KNS {

constexpr int ATI = 7, ATJ = 32, ANW = 8;  // flux tile of the forward runs
using AGeom = TileGeom<ATI, ATJ>;

struct StageRec {
  int in_buf;  // 0 U, 1 U1, 2 U2
  int mode;    // k_combine mode that followed
  double dt;
};

// The step controller with a log of the executed stages.
__global__ void ka_control(Ctl* c, StepParams p, int phase, double arg, StageRec* log, int* nlog,
                           int cap) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const bool ran = !c->skip && !c->error;  // the stage's flux ran
  control_step(c, p, phase, arg);
  if (!ran || c->error) return;
  int in_buf = -1, mode = -1;
  double dt = c->dt;
  switch (phase) {
    case PH_RK_FIRST: in_buf = 0; mode = 1; break;
    case PH_EULER: in_buf = 0; mode = 0; break;
    case PH_RK_SECOND:
    case PH_RK_FINAL:
      in_buf = phase == PH_RK_SECOND ? 1 : 2;
      if (c->retry) {  // the retry tail starts with U1 = U + dt*UL, dt = min(dt1, dt2, dt3)
        mode = 1;
        dt = min3(c->dt1, c->dt2, c->dt3);
      } else {
        mode = phase == PH_RK_SECOND ? 2 : 3;
      }
      break;
    default: return;
  }
  const int n = *nlog;
  if (n >= cap) {  // the host sized the log; running past it stops the run
    c->error = 10;
    c->skip = 1;
    return;
  }
  log[n] = StageRec{in_buf, mode, dt};
  *nlog = n + 1;
}

// Stage update with an explicit dt (replay).
__global__ void ka_combine(Grid g, int mode, double dt, double* __restrict__ U,
                           double* __restrict__ U1, double* __restrict__ U2,
                           const double* __restrict__ UL) {
  const int j = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = 2 + blockIdx.y;
  const int k = blockIdx.z;
  if (j >= g.ny + 2) return;
  combine_at(mode, dt, g.at(k, i, j), U, U1, U2, UL);
}

// Which buffer a stage update writes (0 U, 1 U1, 2 U2) and the coefficient
// of its UL term.
__host__ __device__ inline int stage_out(int mode) { return mode == 1 ? 1 : (mode == 2 ? 2 : 0); }
__host__ __device__ inline double ul_coef(int mode, double dt) {
  return mode == 2 ? (1.0 / 4.0) * dt : (mode == 3 ? (2.0 / 3.0) * dt : dt);
}

// Transpose of k_snapshot for one side: the edge row / column of U0 gets
// the accumulated adjoint of its snapshot.
__global__ void ka_snap_adj(Grid g, int side, const double* __restrict__ lsnap,
                            double* __restrict__ lU) {
  const bool xs = side == LEFT || side == RIGHT;
  const int nb = xs ? g.ny : g.nx, len = xs ? g.NY : g.NX;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= NF * nb) return;
  const int k = e / nb, c = 2 + e % nb;
  const double v = lsnap[k * len + c];
  if (side == LEFT) lU[g.at(k, 2, c)] += v;
  else if (side == RIGHT) lU[g.at(k, g.nx + 1, c)] += v;
  else if (side == BOTTOM) lU[g.at(k, c, 2)] += v;
  else lU[g.at(k, c, g.ny + 1)] += v;
}

// J = sum over the interior of |m|^2 / (2 rho): per-block partial sums in a
// fixed order (the host adds the partials in block order and scales by dx dy).
__global__ void __launch_bounds__(256) ka_objective(Grid g, const double* __restrict__ U,
                                                   double* partial) {
  __shared__ double sm[256];
  const long long n = (long long)g.nx * g.ny;
  double s = 0.0;
  for (long long e = blockIdx.x * 256LL + threadIdx.x; e < n; e += (long long)gridDim.x * 256) {
    const int i = 2 + int(e / g.ny), j = 2 + int(e % g.ny);
    const double r = U[g.at(0, i, j)], mx = U[g.at(1, i, j)], my = U[g.at(2, i, j)],
                 mz = U[g.at(3, i, j)];
    s += 0.5 * (mx * mx + my * my + mz * mz) / r;
  }
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}

// lU = dJ/dU on the interior.
__global__ void ka_seed(Grid g, const double* __restrict__ U, double* __restrict__ lU,
                        double dxdy) {
  const int j = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = 2 + blockIdx.y;
  if (j >= g.ny + 2) return;
  const double r = U[g.at(0, i, j)], mx = U[g.at(1, i, j)], my = U[g.at(2, i, j)],
               mz = U[g.at(3, i, j)];
  const double mm = mx * mx + my * my + mz * mz;
  lU[g.at(0, i, j)] = -0.5 * mm / (r * r) * dxdy;
  lU[g.at(1, i, j)] = mx / r * dxdy;
  lU[g.at(2, i, j)] = my / r * dxdy;
  lU[g.at(3, i, j)] = mz / r * dxdy;
  for (int k = 4; k < NF; k++) lU[g.at(k, i, j)] = 0.0;
}

// dJ/da_k of the plasma-sheet setup (kb_problem): v = sum_k a_k s_k with
// s_k = sin(k pi y) exp(-x^2/0.04); my = rho v and E = ... + rho v^2 / 2, so
// dU0/da_k = (0, 0, rho s_k, 0, 0, 0, 0, rho v s_k).  Per-block partials.
__global__ void __launch_bounds__(256) ka_sheet_grad(Grid g, const double* __restrict__ U0,
                                                    const double* __restrict__ lU, double x0,
                                                    double y0, int K, double* partial) {
  __shared__ double sm[256];
  const long long n = (long long)g.nx * g.ny;
  for (int kk = 1; kk <= K; kk++) {
    double s = 0.0;
    for (long long e = blockIdx.x * 256LL + threadIdx.x; e < n; e += (long long)gridDim.x * 256) {
      const int ii = int(e / g.ny), jj = int(e % g.ny);
      const int i = 2 + ii, j = 2 + jj;
      const double x = x0 + ii * g.dx, y = y0 + jj * g.dy;
      const double sk = sin(kk * M_PI * y) * exp(-x * x / 0.04);
      const double r = U0[g.at(0, i, j)], v = U0[g.at(2, i, j)] / r;
      s += lU[g.at(2, i, j)] * r * sk + lU[g.at(7, i, j)] * r * v * sk;
    }
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[(kk - 1) * gridDim.x + blockIdx.x] = sm[0];
    __syncthreads();
  }
}

}  // namespace MHD_KNS
}  // namespace mhd

using namespace mhd;
using namespace mhd::MHD_KNS;

namespace {
constexpr int kObjBlocks = 296;
constexpr int kSlotsPerChunk = 64;
}  // namespace

struct mhd_adj {
  int device = 0;
  cudaStream_t stream = nullptr;
  // the y-face interface adjoint runs beside the x-face one on this stream
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  Grid g{};
  Gas G{};
  StepParams sp{};
  int time_method = 2, K = 64;
  bool contract = true;  // reverse sweep with FMA contraction (mhd_adj_set_contract)
  size_t blk = 0;  // doubles per state block
  double *U = nullptr, *U1 = nullptr, *U2 = nullptr, *UL = nullptr;
  double *U0 = nullptr, *Ufinal = nullptr;
  double* snap[4] = {nullptr, nullptr, nullptr, nullptr};   // Dirichlet edges of U0
  double* snapr[4] = {nullptr, nullptr, nullptr, nullptr};  // ... of a replay's own U0
  double* lsnap[4] = {nullptr, nullptr, nullptr, nullptr};  // their adjoints
  double** cur_snap = snap;
  double *aF = nullptr, *aG = nullptr;  // unused by ENO-Roe, passed to the flux kernel
  Ctl *ctl = nullptr, *hctl = nullptr;
  StageRec* dlog = nullptr;
  int* dnlog = nullptr;
  int* hnlog = nullptr;
  int log_cap = 0;
  std::vector<StageRec> log;      // executed stages of the recording
  std::vector<int> step_stage;    // first stage of every step (+ the end)
  std::vector<double*> ckpt;      // U at steps 0, K, 2K, ...
  std::vector<unsigned*> chunks;  // mask slots (2 x NX x NY words per stage)
  size_t slot_words = 0;
  double *lU = nullptr, *lU1 = nullptr, *lU2 = nullptr, *T = nullptr;
  double *SX = nullptr, *SY = nullptr;
  std::vector<double*> seg;  // stage inputs of one replayed segment
  int nseg = 0;              // checkpoint segments of the recording
  // Stage store: the recording keeps the inputs of every stage of segments
  // q >= store_seg0, stage s at store + (s - store_first) * blk while
  // s - store_first < store_slots; the backward skips their replays.
  long long store_limit = -1;  // bytes; -1 automatic, 0 none
  double* store = nullptr;
  size_t store_slots = 0;
  int store_seg0 = 0, store_first = -1;
  int replayed_segments = 0;
  // Masks: keep_masks 1 keeps the ENO codes of every stage (the frozen replay
  // of the whole run needs them); 0 keeps those of stored stages only, the
  // recording writes the others to a scratch slot and the backward's segment
  // replays record them again (bit-identical runs) into seg_masks.
  int keep_masks = 1;
  unsigned* scratch_mask = nullptr;
  unsigned* seg_masks = nullptr;
  int seg_mask_slots = 0;
  int replay_s0 = -1;  // first stage of the segment whose masks are in seg_masks
  double *partial = nullptr, *hpartial = nullptr;
  bool recorded = false, have_grad = false;
  int steps = 0;
  double t = 0.0, dt = 0.0;
  double ms_forward = 0.0, ms_backward = 0.0, ms_replay = 0.0;
  std::string msg;
  bool is_error = false;
  long long launches = 0;
};

namespace {

int aset(mhd_adj* a, int st, bool err, const std::string& m) {
  a->is_error = err;
  a->msg = m;
  return st;
}

int afail(mhd_adj* a, cudaError_t e, const char* where) {
  return aset(a, MHD_ERR_CUDA, true,
              std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e));
}

#define AK(call)                                          \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return afail(a, e_, #call);    \
  } while (0)

int pitch_for(int NY) { return ((NY + ROW_OFF + 15) / 16) * 16; }

cudaError_t alloc_block(mhd_adj* a, double** p) {
  cudaError_t e = cudaMalloc(p, a->blk * sizeof(double));
  if (e == cudaSuccess) e = cudaMemsetAsync(*p, 0, a->blk * sizeof(double), a->stream);
  return e;
}

unsigned* chunk_slot(mhd_adj* a, int i) {
  return a->chunks[i / kSlotsPerChunk] + (size_t)(i % kSlotsPerChunk) * a->slot_words;
}

// Mask slot of stage s (see keep_masks).
unsigned* mask_slot(mhd_adj* a, int s) {
  if (a->replay_s0 >= 0 && s >= a->replay_s0 && s - a->replay_s0 < a->seg_mask_slots)
    return a->seg_masks + (size_t)(s - a->replay_s0) * a->slot_words;
  if (a->keep_masks) return chunk_slot(a, s);
  if (a->store_first >= 0 && s >= a->store_first) return chunk_slot(a, s - a->store_first);
  return a->scratch_mask;
}

// Room for nm kept mask slots.
int ensure_mask_chunks(mhd_adj* a, int nm) {
  while ((int)a->chunks.size() * kSlotsPerChunk < nm) {
    unsigned* p = nullptr;
    AK(cudaMalloc(&p, (size_t)kSlotsPerChunk * a->slot_words * sizeof(unsigned)));
    a->chunks.push_back(p);
  }
  if (!a->scratch_mask) AK(cudaMalloc(&a->scratch_mask, a->slot_words * sizeof(unsigned)));
  return MHD_OK;
}

// Room for stages [0, n): mask slots and the device stage log.
int ensure_slots(mhd_adj* a, int n) {
  int nm = n;  // kept mask slots
  if (!a->keep_masks) nm = a->store_first >= 0 ? std::max(0, n - a->store_first) : 0;
  int st = ensure_mask_chunks(a, nm);
  if (st) return st;
  if (n > a->log_cap) {
    const int cap = std::max(n, 2 * a->log_cap + 64);
    StageRec* d = nullptr;
    AK(cudaMalloc(&d, sizeof(StageRec) * cap));
    if (a->dlog) {
      AK(cudaMemcpyAsync(d, a->dlog, sizeof(StageRec) * a->log_cap, cudaMemcpyDeviceToDevice,
                         a->stream));
      AK(cudaStreamSynchronize(a->stream));
      cudaFree(a->dlog);
    }
    a->dlog = d;
    a->log_cap = cap;
  }
  return MHD_OK;
}

double* buf(mhd_adj* a, int id) { return id == 0 ? a->U : (id == 1 ? a->U1 : a->U2); }

void launch_bc(mhd_adj* a, double* X) {
  double** sn = a->cur_snap;
  const Snap d{sn[0], sn[1], sn[2], sn[3]};
  const long long n = bc_count(a->g);
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_bc<<<int(blocks), 256, 0, a->stream>>>(a->g, X, d, a->ctl);
  a->launches++;
}

template <int MASK>
void launch_flux(mhd_adj* a, const double* X, unsigned* slot) {
  auto kern = k_flux<2, false, ATI, ATJ, ANW, MASK>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(AGeom::TMA_BYTES));
    attr = true;
  }
  const Grid& g = a->g;
  dim3 grid((g.ny + ATJ - 1) / ATJ, (g.nx + ATI - 1) / ATI);
  const CharOut co{nullptr, nullptr, nullptr, nullptr};
  CUtensorMap tm{};
  const int use_tma =
      tile_tma_enabled() && make_box_map(g, X, AGeom::CU, AGeom::RU, &tm) ? 1 : 0;
  tile_tma_launches() += use_tma;
  kern<<<grid, ANW * 32, AGeom::TMA_BYTES, a->stream>>>(g, X, a->UL, a->aF, a->aG, 1.0 / g.dx,
                                                     1.0 / g.dy, a->G, a->ctl, co, slot,
                                                     slot + (size_t)g.NX * g.NY, tm, use_tma, 0);
  a->launches++;
}

void launch_control(mhd_adj* a, int phase, double arg = 0.0) {
  ka_control<<<1, 32, 0, a->stream>>>(a->ctl, a->sp, phase, arg, a->dlog, a->dnlog, a->log_cap);
  a->launches++;
}

void launch_combine_ctl(mhd_adj* a, int mode) {
  const Grid& g = a->g;
  dim3 grid((g.ny + 255) / 256, g.nx, NF);
  k_combine<<<grid, 256, 0, a->stream>>>(g, mode, a->U, a->U1, a->U2, a->UL, a->ctl);
  a->launches++;
}

int read_ctl(mhd_adj* a) {
  AK(cudaMemcpyAsync(a->hctl, a->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, a->stream));
  AK(cudaMemcpyAsync(a->hnlog, a->dnlog, sizeof(int), cudaMemcpyDeviceToHost, a->stream));
  AK(cudaStreamSynchronize(a->stream));
  AK(cudaGetLastError());
  return MHD_OK;
}

// Stage store: keeps the input of stage s (after its boundary fill) when s
// falls into the store.
void keep_input(mhd_adj* a, int s, const double* X) {
  if (a->store_first < 0 || s < a->store_first) return;
  const size_t slot = size_t(s - a->store_first);
  if (slot >= a->store_slots) return;
  cudaMemcpyAsync(a->store + slot * a->blk, X, a->blk * sizeof(double), cudaMemcpyDeviceToDevice,
                  a->stream);
}

// One recorded time step from U (TimeIntegrationRK3::step /
// TimeIntegrationEuler::step, as a context runs it).  The i-th flux launched
// since the last synchronisation, if it runs, is logged as stage base + i,
// so its choices go to that mask slot.  record_issue enqueues the step and
// the read-back of the control block; record_finish waits for it, runs the
// RK3 retry tails (each synchronously) and returns the step's status.

void ctl_readback(mhd_adj* a) {
  cudaMemcpyAsync(a->hctl, a->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, a->stream);
  cudaMemcpyAsync(a->hnlog, a->dnlog, sizeof(int), cudaMemcpyDeviceToHost, a->stream);
}

// The RK3 stages after the first (U1 and U2 fluxes, stage updates, dt control).
void record_rk_tail(mhd_adj* a, int base) {
  launch_combine_ctl(a, 1);
  launch_bc(a, a->U1);
  keep_input(a, base + 1, a->U1);
  launch_flux<1>(a, a->U1, mask_slot(a, base + 1));
  launch_control(a, PH_RK_SECOND);
  launch_combine_ctl(a, 2);
  launch_bc(a, a->U2);
  keep_input(a, base + 2, a->U2);
  launch_flux<1>(a, a->U2, mask_slot(a, base + 2));
  launch_control(a, PH_RK_FINAL);
  launch_combine_ctl(a, 3);
  launch_control(a, PH_DONE);
}

int record_issue(mhd_adj* a, double dt) {
  const int base = *a->hnlog;
  int st;
  if ((st = ensure_slots(a, base + 3))) return st;
  launch_control(a, PH_RESET_STEP, dt);
  launch_bc(a, a->U);
  keep_input(a, base, a->U);
  launch_flux<1>(a, a->U, mask_slot(a, base));
  if (a->time_method == 1) {
    launch_control(a, PH_EULER);
    launch_combine_ctl(a, 0);
    launch_control(a, PH_DONE);
  } else {
    launch_control(a, PH_RK_FIRST);
    record_rk_tail(a, base);
  }
  ctl_readback(a);
  return MHD_OK;
}

int record_finish(mhd_adj* a, double* dt_inout) {
  int st;
  AK(cudaStreamSynchronize(a->stream));
  AK(cudaGetLastError());
  if (a->time_method != 1) {
    // no cap, as in TimeIntegrationRK3::step: every retry lowers dt strictly
    while (a->hctl->retry && !a->hctl->error) {
      const int base = *a->hnlog - 1;  // the retry tail's first flux takes the next slot
      if ((st = ensure_slots(a, base + 3))) return st;
      launch_control(a, PH_RK_RETRY);
      record_rk_tail(a, base);
      if ((st = read_ctl(a))) return st;
    }
  }
  const Ctl& h = *a->hctl;
  if (h.error == 6)
    return aset(a, MHD_ERR_NEGATIVE_DENSITY, true, "negative density encountered\n! getEigens_F");
  if (h.error == 4)
    return aset(a, MHD_ERR_TIME_UNDERFLOW, true, "CFL condition violated!\n! updateDt");
  if (h.error == kErrTileCopyTimeout)
    return aset(a, MHD_ERR_CUDA, true, "flux tile copy did not complete");
  if (h.error)
    return aset(a, MHD_ERR_WRONG_PARAMETER, true, "updateDt: no power-of-two time step fits");
  *dt_inout = h.dt;
  return MHD_OK;
}

// J of a device state (deterministic: fixed grid, partials summed in order).
int objective(mhd_adj* a, const double* U, double* J) {
  ka_objective<<<kObjBlocks, 256, 0, a->stream>>>(a->g, U, a->partial);
  a->launches++;
  AK(cudaMemcpyAsync(a->hpartial, a->partial, kObjBlocks * sizeof(double),
                     cudaMemcpyDeviceToHost, a->stream));
  AK(cudaStreamSynchronize(a->stream));
  double s = 0.0;
  for (int b = 0; b < kObjBlocks; b++) s += a->hpartial[b];
  *J = s * (a->g.dx * a->g.dy);
  return MHD_OK;
}

// Replays stage s on the working buffers; keep (if not null) receives its
// input after the boundary fill.  While replay_s0 is set (masks not kept)
// the stage records its masks again instead of reading them.
void replay_stage(mhd_adj* a, int s, double* keep) {
  const Grid& g = a->g;
  dim3 cgrid((g.ny + 255) / 256, g.nx, NF);
  const StageRec& r = a->log[s];
  double* X = buf(a, r.in_buf);
  launch_bc(a, X);
  if (keep)
    cudaMemcpyAsync(keep, X, a->blk * sizeof(double), cudaMemcpyDeviceToDevice, a->stream);
  if (a->replay_s0 >= 0)
    launch_flux<1>(a, X, mask_slot(a, s));  // the masks again, into seg_masks
  else
    launch_flux<2>(a, X, mask_slot(a, s));
  ka_combine<<<cgrid, 256, 0, a->stream>>>(g, r.mode, r.dt, a->U, a->U1, a->U2, a->UL);
  a->launches++;
}

// Replays stages [s0, s1); with keep, stage s's input goes to a->seg[s - s0].
void replay_stages(mhd_adj* a, int s0, int s1, bool keep) {
  for (int s = s0; s < s1; s++) replay_stage(a, s, keep ? a->seg[s - s0] : nullptr);
}

int reset_ctl(mhd_adj* a) {
  AK(cudaMemsetAsync(a->ctl, 0, sizeof(Ctl), a->stream));
  return MHD_OK;
}

void snapshot_into(mhd_adj* a, const double* U, double* const* dst) {
  const int m = std::max(a->g.nx, a->g.ny);
  k_snapshot<<<(NF * m + 255) / 256, 256, 0, a->stream>>>(a->g, U, dst[0], dst[1], dst[2],
                                                          dst[3]);
  a->launches++;
}

// Adjoint of stage s (its update r.mode, then the spatial operator at its
// stored input X): the adjoint of the stage input, lU / lU1 / lU2 by
// r.in_buf, gets L'(X)^T applied to the adjoint of UL.
void adjoint_stage(mhd_adj* a, int s, const StageRec& r, const double* X) {
  const Grid& g = a->g;
  unsigned* mx = mask_slot(a, s);
  unsigned* my = mx + (size_t)g.NX * g.NY;
  double* lb[3] = {a->lU, a->lU1, a->lU2};
  const double* lB = lb[stage_out(r.mode)];
  const double cL = ul_coef(r.mode, r.dt);
  const adjrev::GasConsts gc{a->G.gm, a->G.g1, a->G.g21, a->G.rs2};
  const auto iface = a->contract ? adjrev::contracted::launch_iface
                                 : adjrev::uncontracted::launch_iface;
  const auto gather = a->contract ? adjrev::contracted::launch_gather
                                  : adjrev::uncontracted::launch_gather;
  const auto bc = a->contract ? adjrev::contracted::launch_bc : adjrev::uncontracted::launch_bc;
  // the two directions read the same inputs and write their own scratch
  // (SX, SY): the y faces run on the side stream, the gather waits for both
  cudaEventRecord(a->fork, a->stream);
  cudaStreamWaitEvent(a->side, a->fork, 0);
  iface(g, gc, false, X, mx, lB, cL, a->SX, 1.0 / g.dx, a->stream);
  iface(g, gc, true, X, my, lB, cL, a->SY, 1.0 / g.dy, a->side);
  cudaEventRecord(a->join, a->side);
  cudaStreamWaitEvent(a->stream, a->join, 0);
  gather(g, gc, X, a->SX, a->SY, a->T, r.mode, r.in_buf, a->lU, a->lU1, a->lU2, a->stream);
  a->launches += 3;
  double* dst = lb[r.in_buf];
  for (int ydir = 0; ydir < 2; ydir++) {
    bc(g, ydir, a->T, dst, a->lsnap[2 * ydir], a->lsnap[2 * ydir + 1], a->stream);
    a->launches++;
  }
}

int check_ready(mhd_adj* a) {
  if (!a->recorded)
    return aset(a, MHD_ERR_WRONG_PARAMETER, true, "no recorded forward run (call mhd_adj_forward)");
  return MHD_OK;
}

int check_replay(mhd_adj* a) {
  int st = check_ready(a);
  if (st) return st;
  if (!a->keep_masks)
    return aset(a, MHD_ERR_WRONG_PARAMETER, true,
                "the recording kept the masks of its stored stages only (mhd_adj_set_masks)");
  return MHD_OK;
}

// Elapsed time between e0 and e1; destroys both events.
int timed_ms(cudaEvent_t e0, cudaEvent_t e1, double* out) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *out = ms;
  return MHD_OK;
}

}  // namespace

// Sizes the stage store for a recording of nsteps steps in nseg segments:
// the last m segments whose stages fit (with room for RK3 retries) in the
// memory left after a reserve for the backward's replay buffers, and in
// budget bytes when budget >= 0.
int plan_store(mhd_adj* a, int nsteps, int nseg, int per_step, long long budget) {
  a->store_seg0 = nseg;
  a->store_first = -1;
  if (a->store_limit == 0) return MHD_OK;
  const size_t mask_b = a->slot_words * sizeof(unsigned);
  // a kept stage holds its input and, without kept masks, its mask slot
  const size_t bb = a->blk * sizeof(double) + (a->keep_masks ? 0 : mask_b);
  auto slots_for = [&](int m) -> size_t {
    const long long kept_steps = (long long)nsteps - (long long)(nseg - m) * a->K;
    return size_t(per_step * kept_steps + 3 * m + 8);
  };
  size_t have = a->store ? a->store_slots * a->blk * sizeof(double) : 0;
  size_t free_b = 0, total_b = 0;
  AK(cudaMemGetInfo(&free_b, &total_b));
  const size_t seg_need = size_t(per_step) * a->K + 2;
  const size_t seg_missing = seg_need > a->seg.size() ? seg_need - a->seg.size() : 0;
  const size_t seg_masks_missing =
      !a->keep_masks && seg_need > size_t(a->seg_mask_slots) ? seg_need - a->seg_mask_slots : 0;
  const size_t reserve =
      seg_missing * a->blk * sizeof(double) + seg_masks_missing * mask_b + (size_t(2) << 30);
  size_t avail = free_b + have > reserve ? free_b + have - reserve : 0;
  if (a->store_limit > 0) avail = std::min(avail, size_t(a->store_limit));
  if (budget >= 0) avail = std::min(avail, size_t(budget));
  int m = nseg;
  while (m > 0 && slots_for(m) * bb > avail) m--;
  if (m == 0) return MHD_OK;
  const size_t want = slots_for(m);
  if (!a->store || a->store_slots < want || a->store_slots > want + want / 4) {
    cudaFree(a->store);
    a->store = nullptr;
    a->store_slots = 0;
    while (m > 0 &&
           cudaMalloc(&a->store, slots_for(m) * a->blk * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      m--;
    }
    if (m == 0) return MHD_OK;
    a->store_slots = slots_for(m);
  }
  a->store_seg0 = nseg - m;
  return MHD_OK;
}

// Recording state between forward_start and forward_end.
struct FwState {
  int nsteps = 0, done = 0, status = MHD_OK;
  double dt = 0.0, t = 0.0;
  bool active = false;
};

// Allocations of a recording of nsteps steps that do not depend on the
// stage store: checkpoints and, with kept masks, every mask slot.
int forward_prepare(mhd_adj* a, int nsteps) {
  AK(cudaSetDevice(a->device));
  a->log.clear();
  a->step_stage.clear();
  a->recorded = false;
  a->have_grad = false;
  a->cur_snap = a->snap;
  a->nseg = (nsteps + a->K - 1) / a->K;
  const int per_step = a->time_method == 2 ? 3 : 1;
  const int chunks_needed =
      a->keep_masks ? (per_step * nsteps + 8 + kSlotsPerChunk - 1) / kSlotsPerChunk : 0;
  if (a->store && ((int)a->ckpt.size() < a->nseg || (int)a->chunks.size() < chunks_needed)) {
    // the store is sized last, from what is left: give its memory back first
    AK(cudaStreamSynchronize(a->stream));
    cudaFree(a->store);
    a->store = nullptr;
    a->store_slots = 0;
  }
  while ((int)a->ckpt.size() < a->nseg) {
    double* c = nullptr;
    AK(cudaMalloc(&c, a->blk * sizeof(double)));
    a->ckpt.push_back(c);
  }
  if (a->keep_masks) return ensure_slots(a, per_step * nsteps + 8);
  return MHD_OK;
}

// The stage store (and, without kept masks, the mask slots of its stages).
int forward_store(mhd_adj* a, int nsteps, long long budget) {
  const int per_step = a->time_method == 2 ? 3 : 1;
  int st = plan_store(a, nsteps, a->nseg, per_step, budget);
  if (st) return st;
  if (!a->keep_masks) {
    if ((st = ensure_mask_chunks(a, int(a->store_slots)))) return st;
    if ((st = ensure_slots(a, per_step * nsteps + 8))) return st;
  }
  return MHD_OK;
}

int forward_start(mhd_adj* a, FwState& f, int nsteps, double dt0) {
  int st;
  if ((st = reset_ctl(a))) return st;
  AK(cudaMemsetAsync(a->dnlog, 0, sizeof(int), a->stream));
  *a->hnlog = 0;
  AK(cudaMemcpyAsync(a->U, a->U0, a->blk * sizeof(double), cudaMemcpyDeviceToDevice, a->stream));
  f = FwState{};
  f.nsteps = nsteps;
  f.dt = dt0;
  f.active = true;
  return MHD_OK;
}

// Enqueues step f.done (its checkpoint first when it starts a segment).
int forward_issue(mhd_adj* a, FwState& f) {
  const int s = f.done;
  if (s % a->K == 0) {
    AK(cudaMemcpyAsync(a->ckpt[s / a->K], a->U, a->blk * sizeof(double),
                       cudaMemcpyDeviceToDevice, a->stream));
    if (s / a->K == a->store_seg0) a->store_first = *a->hnlog;
  }
  a->step_stage.push_back(*a->hnlog);
  return record_issue(a, f.dt);
}

// Completes the issued step; ends the recording on an error or after the
// last step.
void forward_finish(mhd_adj* a, FwState& f) {
  const int st = record_finish(a, &f.dt);
  if (st) {
    f.status = st;
    f.active = false;
    return;
  }
  f.t += f.dt;
  if (++f.done >= f.nsteps) f.active = false;
}

int forward_end(mhd_adj* a, const FwState& f, double* J) {
  int st;
  if (f.status) return f.status;
  a->step_stage.push_back(*a->hnlog);
  a->log.resize(*a->hnlog);
  AK(cudaMemcpy(a->log.data(), a->dlog, sizeof(StageRec) * a->log.size(),
                cudaMemcpyDeviceToHost));
  AK(cudaMemcpyAsync(a->Ufinal, a->U, a->blk * sizeof(double), cudaMemcpyDeviceToDevice,
                     a->stream));
  a->steps = f.done;
  a->t = f.t;
  a->dt = f.dt;
  a->recorded = true;
  if (J && (st = objective(a, a->U, J))) return st;
  return aset(a, MHD_OK, false, "");
}

// Segment q of the recording kept in the stage store (no replay needed).
bool seg_kept(const mhd_adj* a, int q, int s0, int s1) {
  return q >= a->store_seg0 && a->store_first >= 0 && s0 >= a->store_first &&
         size_t(s1 - a->store_first) <= a->store_slots;
}
int seg_first(const mhd_adj* a, int q) { return a->step_stage[q * a->K]; }
int seg_end(const mhd_adj* a, int q) { return a->step_stage[std::min((q + 1) * a->K, a->steps)]; }

// Replay buffers (stage inputs, and masks when not kept) of the largest
// replayed segment.
int backward_prepare(mhd_adj* a) {
  AK(cudaSetDevice(a->device));
  a->cur_snap = a->snap;
  int maxst = 0;
  for (int q = 0; q < a->nseg; q++) {
    const int s0 = seg_first(a, q), s1 = seg_end(a, q);
    if (!seg_kept(a, q, s0, s1)) maxst = std::max(maxst, s1 - s0);
  }
  if (!a->keep_masks && a->seg_mask_slots < maxst) {
    cudaFree(a->seg_masks);
    a->seg_masks = nullptr;
    a->seg_mask_slots = 0;
    AK(cudaMalloc(&a->seg_masks, (size_t)maxst * a->slot_words * sizeof(unsigned)));
    a->seg_mask_slots = maxst;
  }
  while ((int)a->seg.size() < maxst) {
    double* p = nullptr;
    AK(cudaMalloc(&p, a->blk * sizeof(double)));
    a->seg.push_back(p);
  }
  return MHD_OK;
}

// Progress of a reverse sweep: segments last first; in each, a replay of
// its stages (unless kept) and then their adjoints in reverse.
struct BwState {
  enum Phase { SEGMENT, REPLAY, ADJOINT, FINISH, DONE };
  Phase phase = SEGMENT;
  int q = 0, s0 = 0, s1 = 0, s = 0;
  bool kept = false;
};

int backward_start(mhd_adj* a, BwState& b) {
  const Grid& g = a->g;
  for (double* p : {a->lU, a->lU1, a->lU2, a->T})
    AK(cudaMemsetAsync(p, 0, a->blk * sizeof(double), a->stream));
  for (int side = 0; side < 4; side++)
    AK(cudaMemsetAsync(a->lsnap[side], 0, sizeof(double) * NF * std::max(g.NX, g.NY), a->stream));
  dim3 sgrid((g.ny + 255) / 256, g.nx);
  ka_seed<<<sgrid, 256, 0, a->stream>>>(g, a->Ufinal, a->lU, g.dx * g.dy);
  a->launches++;
  a->replayed_segments = 0;
  a->replay_s0 = -1;
  b = BwState{};
  b.q = a->nseg - 1;
  b.phase = b.q >= 0 ? BwState::SEGMENT : BwState::FINISH;
  return MHD_OK;
}

// Enqueues the next unit of the reverse sweep: one replayed stage, one
// stage adjoint, or the closing snapshot adjoints.
int backward_issue(mhd_adj* a, BwState& b) {
  const Grid& g = a->g;
  int st;
  switch (b.phase) {
    case BwState::SEGMENT:
      b.s0 = seg_first(a, b.q);
      b.s1 = seg_end(a, b.q);
      b.kept = seg_kept(a, b.q, b.s0, b.s1);
      if (!b.kept) {
        AK(cudaMemcpyAsync(a->U, a->ckpt[b.q], a->blk * sizeof(double),
                           cudaMemcpyDeviceToDevice, a->stream));
        if ((st = reset_ctl(a))) return st;
        if (!a->keep_masks) a->replay_s0 = b.s0;
        a->replayed_segments++;
        b.s = b.s0;
        b.phase = b.s < b.s1 ? BwState::REPLAY : BwState::ADJOINT;
      } else {
        b.phase = BwState::ADJOINT;
      }
      if (b.phase == BwState::ADJOINT) b.s = b.s1 - 1;
      return MHD_OK;
    case BwState::REPLAY:
      replay_stage(a, b.s, a->seg[b.s - b.s0]);
      if (++b.s == b.s1) {
        b.phase = BwState::ADJOINT;
        b.s = b.s1 - 1;
      }
      return MHD_OK;
    case BwState::ADJOINT:
      if (b.s >= b.s0) {
        const double* X = b.kept ? a->store + size_t(b.s - a->store_first) * a->blk
                                 : a->seg[b.s - b.s0];
        adjoint_stage(a, b.s, a->log[b.s], X);
        b.s--;
      }
      if (b.s < b.s0) {
        a->replay_s0 = -1;
        b.phase = --b.q >= 0 ? BwState::SEGMENT : BwState::FINISH;
      }
      return MHD_OK;
    case BwState::FINISH:
      for (int side = 0; side < 4; side++) {
        if (g.bc[side] != DIRICHLET) continue;
        const int nb = (side < 2) ? g.ny : g.nx;
        ka_snap_adj<<<(NF * nb + 127) / 128, 128, 0, a->stream>>>(g, side, a->lsnap[side],
                                                                  a->lU);
        a->launches++;
      }
      b.phase = BwState::DONE;
      return MHD_OK;
    default:
      return MHD_OK;
  }
}

// Group timing: a stream that waits for every member's work.
struct GroupClock {
  cudaStream_t gs = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::vector<cudaEvent_t> ends;
};

cudaError_t group_begin(GroupClock& c, int n, mhd_adj* const* as) {
  cudaError_t e = cudaStreamCreateWithFlags(&c.gs, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&c.e0);
  if (e == cudaSuccess) e = cudaEventCreate(&c.e1);
  if (e == cudaSuccess) e = cudaEventRecord(c.e0, c.gs);
  for (int i = 0; i < n && e == cudaSuccess; i++) e = cudaStreamWaitEvent(as[i]->stream, c.e0, 0);
  return e;
}

cudaError_t group_end(GroupClock& c, int n, mhd_adj* const* as, double* ms) {
  cudaError_t e = cudaSuccess;
  c.ends.assign(n, nullptr);
  for (int i = 0; i < n && e == cudaSuccess; i++) {
    e = cudaEventCreateWithFlags(&c.ends[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(c.ends[i], as[i]->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c.gs, c.ends[i], 0);
  }
  if (e == cudaSuccess) e = cudaEventRecord(c.e1, c.gs);
  if (e == cudaSuccess) e = cudaEventSynchronize(c.e1);
  float f = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&f, c.e0, c.e1);
  if (ms) *ms = f;
  return e;
}

void group_free(GroupClock& c) {
  for (cudaEvent_t ev : c.ends)
    if (ev) cudaEventDestroy(ev);
  if (c.e0) cudaEventDestroy(c.e0);
  if (c.e1) cudaEventDestroy(c.e1);
  if (c.gs) cudaStreamDestroy(c.gs);
}

int group_check(int n, mhd_adj* const* as) {
  if (n < 1 || !as) return MHD_ERR_WRONG_PARAMETER;
  for (int i = 0; i < n; i++) {
    if (!as[i] || as[i]->device != as[0]->device) return MHD_ERR_WRONG_PARAMETER;
    for (int j = 0; j < i; j++)
      if (as[j] == as[i]) return MHD_ERR_WRONG_PARAMETER;
  }
  return MHD_OK;
}

extern "C" {

int mhd_adj_create(int nx, int ny, double dx, double dy, double gamma, const int bc[4],
                   int time_method, double dt_min, double dt_max, double cfl,
                   int checkpoint_every, int device, mhd_adj** out) {
  if (!out) return MHD_ERR_WRONG_PARAMETER;
  *out = nullptr;
  if (nx < 2 || ny < 2 || !(dx > 0) || !(dy > 0) || !bc || (time_method != 1 && time_method != 2) ||
      checkpoint_every < 1)
    return MHD_ERR_WRONG_PARAMETER;
  for (int s = 0; s < 4; s++)
    if (bc[s] < 1 || bc[s] > 4) return MHD_ERR_WRONG_PARAMETER;
  mhd_adj* a = new (std::nothrow) mhd_adj;
  if (!a) return MHD_ERR_WRONG_PARAMETER;
  *out = a;
  a->device = device;
  a->time_method = time_method;
  a->K = checkpoint_every;
  AK(cudaSetDevice(device));
  AK(cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking));
  AK(cudaStreamCreateWithFlags(&a->side, cudaStreamNonBlocking));
  AK(cudaEventCreateWithFlags(&a->fork, cudaEventDisableTiming));
  AK(cudaEventCreateWithFlags(&a->join, cudaEventDisableTiming));
  Grid& g = a->g;
  g.nx = nx; g.ny = ny; g.NX = nx + 4; g.NY = ny + 4;
  g.pitch = pitch_for(g.NY);
  g.off = ROW_OFF;
  g.fstride = (long long)g.NX * g.pitch;
  g.dx = dx; g.dy = dy; g.gamma = gamma;
  for (int s = 0; s < 4; s++) g.bc[s] = bc[s];
  a->G = Gas{gamma, gamma - 1.0, (gamma - 2.0) / (gamma - 1.0), 1.0 / std::sqrt(2.0)};
  a->sp = StepParams{dx, dy, dt_min, dt_max, cfl};
  a->blk = size_t(NF) * g.fstride + 16;
  a->slot_words = 2 * (size_t)g.NX * g.NY;
  for (double** p : {&a->U, &a->U1, &a->U2, &a->UL, &a->U0, &a->Ufinal, &a->lU, &a->lU1, &a->lU2,
                     &a->T})
    AK(alloc_block(a, p));
  const size_t sn = sizeof(double) * NF * std::max(g.NX, g.NY);
  for (int s = 0; s < 4; s++) {
    for (double** p : {&a->snap[s], &a->snapr[s], &a->lsnap[s]}) {
      AK(cudaMalloc(p, sn));
      AK(cudaMemsetAsync(*p, 0, sn, a->stream));
    }
  }
  AK(cudaMalloc(&a->aF, sizeof(double) * NF * g.NY));
  AK(cudaMalloc(&a->aG, sizeof(double) * NF * g.NX));
  const size_t scx = adjrev::contracted::record_doubles(g, false),
               scy = adjrev::contracted::record_doubles(g, true);
  AK(cudaMalloc(&a->SX, scx * sizeof(double)));
  AK(cudaMalloc(&a->SY, scy * sizeof(double)));
  AK(cudaMemsetAsync(a->SX, 0, scx * sizeof(double), a->stream));
  AK(cudaMemsetAsync(a->SY, 0, scy * sizeof(double), a->stream));
  AK(cudaMalloc(&a->ctl, sizeof(Ctl)));
  AK(cudaMemsetAsync(a->ctl, 0, sizeof(Ctl), a->stream));
  AK(cudaMallocHost(&a->hctl, sizeof(Ctl)));
  AK(cudaMalloc(&a->dnlog, sizeof(int)));
  AK(cudaMallocHost(&a->hnlog, sizeof(int)));
  AK(cudaMalloc(&a->partial, sizeof(double) * kObjBlocks * 40));
  AK(cudaMallocHost(&a->hpartial, sizeof(double) * kObjBlocks * 40));
  AK(cudaStreamSynchronize(a->stream));
  return aset(a, MHD_OK, false, "");
}

int mhd_adj_destroy(mhd_adj* a) {
  if (!a) return MHD_OK;
  cudaSetDevice(a->device);
  if (a->stream) cudaStreamSynchronize(a->stream);
  for (double* p : {a->U, a->U1, a->U2, a->UL, a->U0, a->Ufinal, a->lU, a->lU1, a->lU2, a->T,
                    a->SX, a->SY, a->aF, a->aG, a->partial})
    cudaFree(p);
  for (int s = 0; s < 4; s++) {
    cudaFree(a->snap[s]);
    cudaFree(a->snapr[s]);
    cudaFree(a->lsnap[s]);
  }
  for (double* p : a->ckpt) cudaFree(p);
  cudaFree(a->store);
  for (double* p : a->seg) cudaFree(p);
  for (unsigned* p : a->chunks) cudaFree(p);
  cudaFree(a->scratch_mask);
  cudaFree(a->seg_masks);
  cudaFree(a->dlog);
  cudaFree(a->dnlog);
  cudaFree(a->ctl);
  if (a->hctl) cudaFreeHost(a->hctl);
  if (a->hnlog) cudaFreeHost(a->hnlog);
  if (a->hpartial) cudaFreeHost(a->hpartial);
  if (a->side) {
    cudaStreamSynchronize(a->side);
    cudaStreamDestroy(a->side);
  }
  if (a->fork) cudaEventDestroy(a->fork);
  if (a->join) cudaEventDestroy(a->join);
  if (a->stream) cudaStreamDestroy(a->stream);
  delete a;
  return MHD_OK;
}

int mhd_adj_last_error(mhd_adj* a, char* buf, size_t len, int* is_error) {
  if (!a) return MHD_ERR_WRONG_PARAMETER;
  if (buf && len) {
    std::strncpy(buf, a->msg.c_str(), len - 1);
    buf[len - 1] = 0;
  }
  if (is_error) *is_error = a->is_error ? 1 : 0;
  return MHD_OK;
}

int mhd_adj_upload(mhd_adj* a, const double* U0) {
  if (!a || !U0) return MHD_ERR_WRONG_PARAMETER;
  AK(cudaSetDevice(a->device));
  const Grid& g = a->g;
  AK(cudaMemcpy2DAsync(a->U0 + g.off, g.pitch * sizeof(double), U0, g.NY * sizeof(double),
                       g.NY * sizeof(double), size_t(NF) * g.NX, cudaMemcpyHostToDevice,
                       a->stream));
  snapshot_into(a, a->U0, a->snap);
  AK(cudaStreamSynchronize(a->stream));
  a->recorded = false;
  a->have_grad = false;
  return aset(a, MHD_OK, false, "");
}

int mhd_adj_init_problem(mhd_adj* a, int kind, const double* p, int np) {
  if (!a) return MHD_ERR_WRONG_PARAMETER;
  AK(cudaSetDevice(a->device));
  ProblemArgs pa{};
  std::string err;
  cudaError_t ce = cudaSuccess;
  const int st = problem_args(kind, p, np, a->g.gamma, a->stream, pa, err, ce, &a->g);
  if (ce != cudaSuccess) return afail(a, ce, "problem_args");
  if (st) return aset(a, st, true, err);
  AK(cudaMemsetAsync(a->U0, 0, a->blk * sizeof(double), a->stream));
  enqueue_problem(a->g, a->U0, pa, a->stream);
  AK(release_problem(pa, a->stream));
  snapshot_into(a, a->U0, a->snap);
  a->launches += problem_launches(pa);
  AK(cudaStreamSynchronize(a->stream));
  AK(cudaGetLastError());
  a->recorded = false;
  a->have_grad = false;
  return aset(a, MHD_OK, false, "");
}

int mhd_adj_set_store(mhd_adj* a, long long max_bytes) {
  if (!a || max_bytes < -1) return MHD_ERR_WRONG_PARAMETER;
  a->store_limit = max_bytes;
  if (max_bytes == 0 && a->store) {
    AK(cudaSetDevice(a->device));
    AK(cudaStreamSynchronize(a->stream));
    cudaFree(a->store);
    a->store = nullptr;
    a->store_slots = 0;
  }
  a->store_seg0 = a->nseg;
  a->store_first = -1;
  return aset(a, MHD_OK, false, "");
}

int mhd_adj_set_masks(mhd_adj* a, int keep_all) {
  if (!a || (keep_all != 0 && keep_all != 1)) return MHD_ERR_WRONG_PARAMETER;
  if (a->keep_masks != keep_all) {
    // the mask slots of a recording follow the policy it ran with
    a->keep_masks = keep_all;
    a->recorded = false;
    a->have_grad = false;
  }
  return aset(a, MHD_OK, false, "");
}

int mhd_adj_set_contract(mhd_adj* a, int enable) {
  if (!a || (enable != 0 && enable != 1)) return MHD_ERR_WRONG_PARAMETER;
  a->contract = enable == 1;  // the recording stays valid: only the reverse sweep changes
  a->have_grad = false;
  return aset(a, MHD_OK, false, "");
}

int mhd_adj_forward(mhd_adj* a, int nsteps, double dt0, double* J) {
  MHD_TRACE("mhd_adj_forward");
  if (!a || nsteps < 1) return MHD_ERR_WRONG_PARAMETER;
  // everything the recording needs is allocated before it starts
  int st;
  if ((st = forward_prepare(a, nsteps))) return st;
  if ((st = forward_store(a, nsteps, -1))) return st;
  FwState f;
  if ((st = forward_start(a, f, nsteps, dt0))) return st;
  cudaEvent_t e0, e1;
  AK(cudaEventCreate(&e0));
  AK(cudaEventCreate(&e1));
  AK(cudaEventRecord(e0, a->stream));
  while (f.active) {
    if ((st = forward_issue(a, f))) {
      f.status = st;
      break;
    }
    forward_finish(a, f);
  }
  AK(cudaEventRecord(e1, a->stream));
  AK(cudaEventSynchronize(e1));
  timed_ms(e0, e1, &a->ms_forward);  // destroys e0, e1
  return forward_end(a, f, J);
}

int mhd_adj_forward_group(int n, mhd_adj* const* as, const int* nsteps, const double* dt0,
                          double* J, double* ms) {
  MHD_TRACE("mhd_adj_forward_group");
  int st = group_check(n, as);
  if (st) return st;
  if (!nsteps || !dt0) return MHD_ERR_WRONG_PARAMETER;
  for (int i = 0; i < n; i++)
    if (nsteps[i] < 1) return MHD_ERR_WRONG_PARAMETER;
  if (cudaSetDevice(as[0]->device) != cudaSuccess) return MHD_ERR_CUDA;
  for (int i = 0; i < n; i++)
    if ((st = forward_prepare(as[i], nsteps[i]))) return st;
  // the stage stores share the free memory in proportion to the stage
  // inputs each recording has, after every member's backward reserve
  size_t reserve = size_t(2) << 30, want_total = 0;
  std::vector<size_t> want(n, 0);
  for (int i = 0; i < n; i++) {
    mhd_adj* a = as[i];
    const int per_step = a->time_method == 2 ? 3 : 1;
    const size_t slot_b =
        a->blk * sizeof(double) + (a->keep_masks ? 0 : a->slot_words * sizeof(unsigned));
    const size_t seg_need = size_t(per_step) * a->K + 2;
    if (seg_need > a->seg.size()) reserve += (seg_need - a->seg.size()) * a->blk * sizeof(double);
    if (!a->keep_masks && seg_need > size_t(a->seg_mask_slots))
      reserve += (seg_need - a->seg_mask_slots) * a->slot_words * sizeof(unsigned);
    if (a->store_limit != 0) {
      cudaFree(a->store);
      a->store = nullptr;
      a->store_slots = 0;
      want[i] = size_t(per_step) * nsteps[i] * slot_b;
      want_total += want[i];
    }
  }
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return MHD_ERR_CUDA;
  const double avail = free_b > reserve ? double(free_b - reserve) : 0.0;
  for (int i = 0; i < n; i++) {
    const long long budget =
        want_total ? (long long)(avail * (double(want[i]) / double(want_total))) : 0;
    if ((st = forward_store(as[i], nsteps[i], budget))) return st;
  }
  std::vector<FwState> f(n);
  for (int i = 0; i < n; i++)
    if ((st = forward_start(as[i], f[i], nsteps[i], dt0[i]))) return st;
  GroupClock clk;
  cudaError_t ce = group_begin(clk, n, as);
  std::vector<char> issued(n, 0);
  for (bool any = ce == cudaSuccess; any;) {
    any = false;
    for (int i = 0; i < n; i++) {
      issued[i] = 0;
      if (!f[i].active) continue;
      if ((st = forward_issue(as[i], f[i]))) {
        f[i].status = st;
        f[i].active = false;
        continue;
      }
      issued[i] = 1;
    }
    for (int i = 0; i < n; i++) {
      if (!issued[i]) continue;
      forward_finish(as[i], f[i]);
      any = any || f[i].active;
    }
  }
  if (ce == cudaSuccess) ce = group_end(clk, n, as, ms);
  group_free(clk);
  if (ce != cudaSuccess) return afail(as[0], ce, "mhd_adj_forward_group");
  int first = MHD_OK;
  for (int i = 0; i < n; i++) {
    as[i]->ms_forward = ms ? *ms : 0.0;
    st = forward_end(as[i], f[i], J ? &J[i] : nullptr);
    if (st && first == MHD_OK) first = st;
  }
  return first;
}

int mhd_adj_backward_group(int n, mhd_adj* const* as, double* ms) {
  MHD_TRACE("mhd_adj_backward_group");
  int st = group_check(n, as);
  if (st) return st;
  for (int i = 0; i < n; i++)
    if ((st = check_ready(as[i]))) return st;
  for (int i = 0; i < n; i++)
    if ((st = backward_prepare(as[i]))) return st;
  GroupClock clk;
  cudaError_t ce = group_begin(clk, n, as);
  std::vector<BwState> b(n);
  for (int i = 0; i < n && ce == cudaSuccess; i++)
    if ((st = backward_start(as[i], b[i]))) return st;
  // one unit (a replayed stage or a stage adjoint) per member per round
  for (bool any = ce == cudaSuccess; any;) {
    any = false;
    for (int i = 0; i < n; i++) {
      if (b[i].phase == BwState::DONE) continue;
      if ((st = backward_issue(as[i], b[i]))) return st;
      any = true;
    }
  }
  double gms = 0.0;
  if (ce == cudaSuccess) ce = group_end(clk, n, as, &gms);
  group_free(clk);
  if (ce != cudaSuccess) return afail(as[0], ce, "mhd_adj_backward_group");
  if ((ce = cudaGetLastError()) != cudaSuccess) return afail(as[0], ce, "mhd_adj_backward_group");
  for (int i = 0; i < n; i++) {
    as[i]->ms_backward = gms;
    as[i]->have_grad = true;
    aset(as[i], MHD_OK, false, "");
  }
  if (ms) *ms = gms;
  return MHD_OK;
}

int mhd_adj_replay(mhd_adj* a, const double* U0, double* J) {
  MHD_TRACE("mhd_adj_replay");
  if (!a) return MHD_ERR_WRONG_PARAMETER;
  int st = check_replay(a);
  if (st) return st;
  AK(cudaSetDevice(a->device));
  const Grid& g = a->g;
  if (U0) {
    AK(cudaMemcpy2DAsync(a->U + g.off, g.pitch * sizeof(double), U0, g.NY * sizeof(double),
                         g.NY * sizeof(double), size_t(NF) * g.NX, cudaMemcpyHostToDevice,
                         a->stream));
    // Dirichlet sides take their edges from this initial state, as a run
    // set up from it would
    snapshot_into(a, a->U, a->snapr);
    a->cur_snap = a->snapr;
  } else {
    AK(cudaMemcpyAsync(a->U, a->U0, a->blk * sizeof(double), cudaMemcpyDeviceToDevice,
                       a->stream));
  }
  if ((st = reset_ctl(a))) return st;
  cudaEvent_t e0, e1;
  AK(cudaEventCreate(&e0));
  AK(cudaEventCreate(&e1));
  AK(cudaEventRecord(e0, a->stream));
  replay_stages(a, 0, int(a->log.size()), false);
  a->cur_snap = a->snap;
  AK(cudaEventRecord(e1, a->stream));
  AK(cudaEventSynchronize(e1));
  AK(cudaGetLastError());
  timed_ms(e0, e1, &a->ms_replay);
  if (J && (st = objective(a, a->U, J))) return st;
  return aset(a, MHD_OK, false, "");
}

int mhd_adj_replay_problem(mhd_adj* a, int kind, const double* p, int np, double* J) {
  if (!a) return MHD_ERR_WRONG_PARAMETER;
  int st = check_replay(a);
  if (st) return st;
  AK(cudaSetDevice(a->device));
  ProblemArgs pa{};
  std::string err;
  cudaError_t ce = cudaSuccess;
  st = problem_args(kind, p, np, a->g.gamma, a->stream, pa, err, ce, &a->g);
  if (ce != cudaSuccess) return afail(a, ce, "problem_args");
  if (st) return aset(a, st, true, err);
  AK(cudaMemsetAsync(a->U, 0, a->blk * sizeof(double), a->stream));
  enqueue_problem(a->g, a->U, pa, a->stream);
  AK(release_problem(pa, a->stream));
  a->launches += problem_launches(pa);
  snapshot_into(a, a->U, a->snapr);
  a->cur_snap = a->snapr;
  if ((st = reset_ctl(a))) return st;
  replay_stages(a, 0, int(a->log.size()), false);
  a->cur_snap = a->snap;
  AK(cudaGetLastError());
  if (J && (st = objective(a, a->U, J))) return st;
  return aset(a, MHD_OK, false, "");
}

int mhd_adj_backward(mhd_adj* a) {
  MHD_TRACE("mhd_adj_backward");
  if (!a) return MHD_ERR_WRONG_PARAMETER;
  int st = check_ready(a);
  if (st) return st;
  if ((st = backward_prepare(a))) return st;
  cudaEvent_t e0, e1;
  AK(cudaEventCreate(&e0));
  AK(cudaEventCreate(&e1));
  AK(cudaEventRecord(e0, a->stream));
  BwState b;
  if ((st = backward_start(a, b))) return st;
  while (b.phase != BwState::DONE)
    if ((st = backward_issue(a, b))) return st;
  AK(cudaEventRecord(e1, a->stream));
  AK(cudaEventSynchronize(e1));
  AK(cudaGetLastError());
  timed_ms(e0, e1, &a->ms_backward);  // destroys e0, e1
  a->have_grad = true;
  return aset(a, MHD_OK, false, "");
}

int mhd_adj_gradient(mhd_adj* a, double* dJdU0) {
  if (!a || !dJdU0) return MHD_ERR_WRONG_PARAMETER;
  if (!a->have_grad)
    return aset(a, MHD_ERR_WRONG_PARAMETER, true, "no adjoint (call mhd_adj_backward)");
  AK(cudaSetDevice(a->device));
  const Grid& g = a->g;
  AK(cudaMemcpy2DAsync(dJdU0, g.NY * sizeof(double), a->lU + g.off, g.pitch * sizeof(double),
                       g.NY * sizeof(double), size_t(NF) * g.NX, cudaMemcpyDeviceToHost,
                       a->stream));
  AK(cudaStreamSynchronize(a->stream));
  return MHD_OK;
}

int mhd_adj_sheet_gradient(mhd_adj* a, double x0, double y0, int K, double* dJda) {
  if (!a || !dJda || K < 1 || K > 40) return MHD_ERR_WRONG_PARAMETER;
  if (!a->have_grad)
    return aset(a, MHD_ERR_WRONG_PARAMETER, true, "no adjoint (call mhd_adj_backward)");
  AK(cudaSetDevice(a->device));
  ka_sheet_grad<<<kObjBlocks, 256, 0, a->stream>>>(a->g, a->U0, a->lU, x0, y0, K, a->partial);
  a->launches++;
  AK(cudaMemcpyAsync(a->hpartial, a->partial, sizeof(double) * kObjBlocks * K,
                     cudaMemcpyDeviceToHost, a->stream));
  AK(cudaStreamSynchronize(a->stream));
  AK(cudaGetLastError());
  for (int k = 0; k < K; k++) {
    double s = 0.0;
    for (int b = 0; b < kObjBlocks; b++) s += a->hpartial[k * kObjBlocks + b];
    dJda[k] = s;
  }
  return MHD_OK;
}

int mhd_adj_download(mhd_adj* a, int which, double* U) {
  if (!a || !U || which < 0 || which > 2) return MHD_ERR_WRONG_PARAMETER;
  AK(cudaSetDevice(a->device));
  const Grid& g = a->g;
  const double* src = which == 0 ? a->U0 : (which == 1 ? a->Ufinal : a->U);
  AK(cudaMemcpy2DAsync(U, g.NY * sizeof(double), src + g.off, g.pitch * sizeof(double),
                       g.NY * sizeof(double), size_t(NF) * g.NX, cudaMemcpyDeviceToHost,
                       a->stream));
  AK(cudaStreamSynchronize(a->stream));
  return MHD_OK;
}

int mhd_adj_info(mhd_adj* a, mhd_adj_stats* out) {
  if (!a || !out) return MHD_ERR_WRONG_PARAMETER;
  out->steps = a->steps;
  out->stages = int(a->log.size());
  out->checkpoints = a->nseg;
  int retries = 0;
  for (size_t s = 0; s < a->log.size(); s++)
    if (a->log[s].mode == 1 && a->log[s].in_buf != 0) retries++;
  out->retries = retries;
  out->t = a->t;
  out->dt = a->dt;
  out->ms_forward = a->ms_forward;
  out->ms_backward = a->ms_backward;
  out->ms_replay = a->ms_replay;
  out->launches = a->launches;
  out->stored_stages = 0;
  if (a->store_first >= 0 && a->log.size() > size_t(a->store_first))
    out->stored_stages =
        int(std::min(a->log.size() - size_t(a->store_first), a->store_slots));
  out->replayed_segments = a->replayed_segments;
  return MHD_OK;
}

}  // extern "C"
