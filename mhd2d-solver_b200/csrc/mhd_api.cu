// C ABI of the device hot path (include/mhd2d_b200.h): context, memory,
// and the host-side orchestration of one integrate / step / SOR solve.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>
#include <string>
#include <vector>

#include "../../include/mhd2d_b200.h"
#include "mhd_launch.h"
#include "mhd_output.h"
#include "mhd_tma.cuh"
#include "mhd_trace.h"

using namespace mhd;

namespace {
// Counters of a graph step loop (mhd_ctx::gcnt).
enum : int { G_STEPS = 0, G_RETRIES = 1, G_WANTED = 2, G_STEP_RETRIES = 3, G_NEG = 4, G_COUNT = 5 };
// RK3 passes of one step the device loop allows: every retry restarts from
// min(dt1, dt2, dt3), strictly below the dt it replaces, and a step retries a
// few times in practice; a step that has not settled after this many passes
// ends the loop with MHD_ERR_NOT_CONVERGED (the host loop has no bound)
constexpr long long kGraphRetryBound = 4096;

// SOR sweeps per pass of the device solve loop (mhd_set_sor_graph).
constexpr int kSorChunk = 16;

// After each pass of the SOR graph: go on while the solve has not met its
// stop rule (the sweeps turn into no-ops once it has: r_max/phi_max <= rmax
// or the sweep cap), at most `bound` passes.
__global__ void k_sor_again(const Ctl* c, long long* cnt, long long bound,
                            cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const long long n = *cnt + 1;
  *cnt = n;
  cudaGraphSetConditional(h, (!c->sor_done && n < bound) ? 1u : 0u);
}

// Before the retry loop and at the end of each retry pass: run another pass
// while the controller asks for one.
__global__ void k_graph_retry(const Ctl* c, long long* cnt, cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const bool again = c->retry && !c->error && cnt[G_STEP_RETRIES] < kGraphRetryBound;
  if (again) {
    cnt[G_STEP_RETRIES] += 1;
    cnt[G_RETRIES] += 1;
  }
  cudaGraphSetConditional(h, again ? 1u : 0u);
}

// End of one step of the device loop: count it, keep its dt, and go on while
// steps are wanted and the step completed.
__global__ void k_graph_step_end(const Ctl* c, long long* cnt, double* dts,
                                 cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const bool done = !c->error && c->step_done;
  cnt[G_NEG] += (long long)c->neg_count;
  cnt[G_STEP_RETRIES] = 0;
  if (done) {
    dts[cnt[G_STEPS]] = c->dt;  // G_STEPS < G_WANTED <= capacity (the loop stops at G_WANTED)
    cnt[G_STEPS] += 1;
  }
  cudaGraphSetConditional(h, (done && cnt[G_STEPS] < cnt[G_WANTED]) ? 1u : 0u);
}

__global__ void k_graph_arm(long long* cnt, long long wanted) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int q = 0; q < G_COUNT; q++) cnt[q] = 0;
  cnt[G_WANTED] = wanted;
}

// FP64 FMA throughput probe: 8 independent chains per thread.
__global__ void __launch_bounds__(256) k_fma_peak(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int q = 0; q < 8; q++) x[q] = threadIdx.x * 1e-3 + q;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int q = 0; q < 8; q++) x[q] = __fma_rn(x[q], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 8; q++) s += x[q];
  if (s == 12345.678) out[0] = s;  // keeps the chains live; never true in practice
}
}  // namespace

struct mhd_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  Grid g{};
  int scheme = 2, time_method = 2, flags = 0;
  double dt_min = 0, dt_max = 0, cfl = 0;
  bool dirichlet_needed = false, dirichlet_ready = false;
  const KernelSet* ks = &kExact;
  size_t block_elems = 0;  // doubles per state block
  double *U = nullptr, *U1 = nullptr, *U2 = nullptr, *UL = nullptr;
  // input of the last spatial integration (0 U, 1 U1, 2 U2) while it is
  // unchanged, else -1: the characteristics of that integration can be
  // recomputed on request (mhd_get_characteristics without the flag)
  int chars_buf = -1;
  double *ch[4] = {nullptr, nullptr, nullptr, nullptr};  // cx, cy, LUx, LUy
  double *aF = nullptr, *aG = nullptr;
  double *snap[4] = {nullptr, nullptr, nullptr, nullptr};  // left, right, bottom, top
  double *phi = nullptr, *partial = nullptr, *ratio = nullptr;
  double* sor_xy = nullptr;  // source terms of the current SOR solve (allocated on first use)
  int sor_fused = 1;         // fused SOR sweeps where the grid allows them (mhd_set_sor_fused)
  int sor_rows = 0;          // rows per SOR thread step (mhd_set_sor_rows; 0: by grid size)
  int npartial = 0;
  Ctl* ctl = nullptr;
  Ctl* hctl = nullptr;  // pinned mirror
  double* hnan = nullptr;  // pinned: U[0][2][2] for the run loop's NaN stop
  std::string msg;
  bool is_error = false;
  long long launches = 0, neg_pressure = 0;
  // mhd_steps as one CUDA graph: a while node over steps, a nested while node
  // over the RK3 retries (see build_step_graph)
  int use_step_graph = 1;
  cudaGraphExec_t step_graph = nullptr;
  bool step_graph_chars = false;
  int step_graph_tma = -1;
  long long step_graph_launches[2] = {0, 0};  // kernels per step body / per retry pass
  long long* gcnt = nullptr;   // device: G_* counters of a graph step loop
  long long* hgcnt = nullptr;  // pinned mirror
  double* gdts = nullptr;      // device: dt of every completed step
  int gdts_cap = 0;
  void* grid_buf = nullptr;    // device: packed grid-dump records (mhd_grid_pack)
  size_t grid_buf_bytes = 0;
  // an SOR solve's sweep loop as one CUDA graph (a while node over passes of
  // kSorChunk sweeps); rebuilt when the solve parameters it bakes in change
  int use_sor_graph = 1;
  cudaGraphExec_t sor_graph = nullptr;
  double sor_graph_key[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // rmax, sweep cap, omega, fused, rows
  long long* sor_cnt = nullptr;  // device: passes the SOR graph ran
  long long sor_graph_launches = 0;  // kernels per pass
  // mhd_step_host: the host state is copied in row bands on copy_stream
  int use_banded_h2d = 1;  // mhd_set_step_host_banded
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t band_ev[9] = {};  // [0]: the main stream's work before the copy; [1..8]: bands
};

namespace {

int set_status(mhd_ctx* c, int st, bool err, const std::string& m) {
  c->is_error = err;
  c->msg = m;
  return st;
}

int cuda_fail(mhd_ctx* c, cudaError_t e, const char* where) {
  std::string m = std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e);
  if (c) return set_status(c, MHD_ERR_CUDA, true, m);
  std::fprintf(stderr, "mhd2d_b200: %s\n", m.c_str());
  return MHD_ERR_CUDA;
}

#define CK(call)                                             \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, #call);   \
  } while (0)

int pitch_for(int NY) { return ((NY + ROW_OFF + 15) / 16) * 16; }

cudaError_t alloc_block(mhd_ctx* c, double** p) {
  cudaError_t e = cudaMalloc(p, c->block_elems * sizeof(double));
  if (e == cudaSuccess) e = cudaMemsetAsync(*p, 0, c->block_elems * sizeof(double), c->stream);
  return e;
}

// copy a host [8][NX][NY] block into / out of the pitched device block
cudaError_t h2d(mhd_ctx* c, double* dst, const double* src) {
  const Grid& g = c->g;
  if (dst == c->U && c->chars_buf == 0) c->chars_buf = -1;  // new interior for U
  return cudaMemcpy2DAsync(dst + g.off, g.pitch * sizeof(double), src, g.NY * sizeof(double),
                           g.NY * sizeof(double), size_t(NF) * g.NX, cudaMemcpyHostToDevice,
                           c->stream);
}
cudaError_t d2h(mhd_ctx* c, double* dst, const double* src) {
  const Grid& g = c->g;
  return cudaMemcpy2DAsync(dst, g.NY * sizeof(double), src + g.off, g.pitch * sizeof(double),
                           g.NY * sizeof(double), size_t(NF) * g.NX, cudaMemcpyDeviceToHost,
                           c->stream);
}

int read_ctl(mhd_ctx* c) {
  CK(cudaMemcpyAsync(c->hctl, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  return MHD_OK;
}

int check_bc_ready(mhd_ctx* c) {
  if (c->dirichlet_needed && !c->dirichlet_ready)
    return set_status(c, MHD_ERR_WRONG_PARAMETER, true,
                      "SpatialIntegrationMethod::applyBoundaryConditions: boundary not initialized.");
  return MHD_OK;
}

// Enqueue one spatial integration of state X into UL.
void enqueue_integrate(mhd_ctx* c, double* X, bool chars) {
  MHD_TRACE(X == c->U ? "L(U)" : (X == c->U1 ? "L(U1)" : "L(U2)"));
  const Grid& g = c->g;
  c->ks->bc(g, X, c->snap, c->ctl, c->stream);
  if (c->scheme == 3) c->ks->lf_alpha(g, X, c->aF, c->aG, c->ctl, c->stream);
  c->ks->flux(c->scheme, g, X, c->UL, c->aF, c->aG, c->ctl, chars ? c->ch : nullptr, c->stream);
  c->launches += c->ks->launches_per_integrate(c->scheme);
  c->chars_buf = X == c->U ? 0 : (X == c->U1 ? 1 : (X == c->U2 ? 2 : -1));
}

// Row bands of mhd_step_host's copy of the host state.
constexpr int kStepHostBands = 8;

// The first spatial operator of a step whose state arrives from host memory:
// the state is copied in kStepHostBands row bands on copy_stream, and on the
// main stream each band is followed by the bottom / top ghost fill of the
// rows it completes and the flux tile rows whose cells (ghosts included)
// are then all in place.  After the last band: the left / right ghost fill
// and the remaining tile rows (the first, which reads the left ghost rows,
// and the last ones).  Every tile and every ghost value is computed as in
// enqueue_integrate (the same kernels on the same inputs), so the results are
// bit-identical; the copy of the later bands overlaps the earlier tiles.
// ENO-Roe only: ENO-LF needs its dissipation coefficients from the whole grid
// first.
int enqueue_integrate_from_host(mhd_ctx* c, const double* Uh, bool chars) {
  MHD_TRACE("L(U) from host");
  const Grid& g = c->g;
  if (!c->copy_stream) {
    CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    for (cudaEvent_t& e : c->band_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  if (c->chars_buf == 0) c->chars_buf = -1;  // new interior for U
  // the copy overwrites U: after the main stream's work on it so far
  CK(cudaEventRecord(c->band_ev[0], c->stream));
  CK(cudaStreamWaitEvent(c->copy_stream, c->band_ev[0], 0));
  const int tr = c->ks->flux_tile_rows(c->scheme);
  const int nti = (g.nx + tr - 1) / tr;
  double* const* ch = chars ? c->ch : nullptr;
  int ydone = 2;  // bottom / top ghosts filled for rows [2, ydone)
  int tdone = 1;  // tile rows [1, tdone) launched
  for (int b = 0; b < kStepHostBands; b++) {
    const int r0 = int((long long)b * g.NX / kStepHostBands);
    const int r1 = int((long long)(b + 1) * g.NX / kStepHostBands);
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < NF && e == cudaSuccess; k++)
      e = cudaMemcpy2DAsync(c->U + k * g.fstride + (long long)r0 * g.pitch + g.off,
                            g.pitch * sizeof(double), Uh + ((long long)k * g.NX + r0) * g.NY,
                            g.NY * sizeof(double), g.NY * sizeof(double), size_t(r1 - r0),
                            cudaMemcpyHostToDevice, c->copy_stream);
    if (e == cudaSuccess) e = cudaEventRecord(c->band_ev[1 + b], c->copy_stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->band_ev[1 + b], 0);
    if (e != cudaSuccess) {
      cudaStreamSynchronize(c->copy_stream);  // no copy into U outlives the call
      return cuda_fail(c, e, "mhd_step_host: banded copy");
    }
    // rows [0, r1) are on the device; a row's bottom / top ghosts read its
    // neighbour rows too (Neumann div B terms)
    const int yhi = std::min(r1 - 1, g.nx + 2);
    if (yhi > ydone) {
      c->ks->bc_part(g, c->U, c->snap, c->ctl, 2, ydone, yhi, c->stream);
      c->launches += 1;
      ydone = yhi;
    }
    // tile row t reads cell rows [t*tr, t*tr + tr + 4): all filled, none a right ghost row
    const int ready = std::min(ydone, g.nx + 2);
    const int thi = ready >= tr + 4 ? (ready - tr - 4) / tr + 1 : 0;
    if (thi > tdone) {
      c->ks->flux_rows(c->scheme, g, c->U, c->UL, c->aF, c->aG, c->ctl, ch, tdone, thi,
                       c->stream);
      c->launches += 1;
      tdone = thi;
    }
  }
  c->ks->bc_part(g, c->U, c->snap, c->ctl, 1, 0, 0, c->stream);
  c->launches += 1;
  if (ydone < g.nx + 2) {
    c->ks->bc_part(g, c->U, c->snap, c->ctl, 2, ydone, g.nx + 2, c->stream);
    c->launches += 1;
  }
  c->ks->flux_rows(c->scheme, g, c->U, c->UL, c->aF, c->aG, c->ctl, ch, 0, 1, c->stream);
  c->launches += 1;
  if (tdone < nti) {
    c->ks->flux_rows(c->scheme, g, c->U, c->UL, c->aF, c->aG, c->ctl, ch, tdone, nti,
                     c->stream);
    c->launches += 1;
  }
  c->chars_buf = 0;
  return MHD_OK;
}

// The interior of buffer b (0 U, 1 U1, 2 U2) is about to change.
void touch_buf(mhd_ctx* c, int b) {
  if (c->chars_buf == b) c->chars_buf = -1;
}

void enqueue_control(mhd_ctx* c, int phase, double arg = 0.0) {
  c->ks->control(c->ctl, c->g.dx, c->g.dy, c->dt_min, c->dt_max, c->cfl, phase, arg, c->stream);
  c->launches += 1;
}

void enqueue_combine(mhd_ctx* c, int mode) {
  touch_buf(c, mode == 1 ? 1 : (mode == 2 ? 2 : 0));
  c->ks->combine(c->g, mode, c->U, c->U1, c->U2, c->UL, c->ctl, c->stream);
  c->launches += 1;
}

// The stage loop of TimeIntegrationRK3::step from U1 = U + dt*UL onwards.
void enqueue_rk3_tail(mhd_ctx* c, bool chars) {
  enqueue_combine(c, 1);
  enqueue_integrate(c, c->U1, false);
  enqueue_control(c, PH_RK_SECOND);
  enqueue_combine(c, 2);
  enqueue_integrate(c, c->U2, chars);
  enqueue_control(c, PH_RK_FINAL);
  enqueue_combine(c, 3);
  enqueue_control(c, PH_DONE);
}

// The RK3 stages after the first operator for a step whose result goes to
// host memory (mhd_step_host): the first two stage updates and L(U1) as in
// enqueue_rk3_tail, then L(U2) in kStepHostBands bands of flux tile rows.
// After each band, its rows' last stage update goes to U1
// (combine_final_rows: the values the in-place update gives U, with U's
// ghost cells beside them) and copy_stream copies those rows to Uh while the
// next bands are computed.  The last stage's retry decision needs every
// band's wave-speed maxima, so it follows the last band: do_step keeps the
// copied rows only when no retry and no error followed (and then copies U1
// to U on the device), otherwise it waits for the copies, runs the step as
// enqueue_rk3_tail would and the caller copies U again.  The tiles, stage
// updates and maxima are the same kernels on the same inputs: bit-identical.
int enqueue_rk3_tail_to_host(mhd_ctx* c, bool chars, double* Uh) {
  MHD_TRACE("RK3 tail to host");
  const Grid& g = c->g;
  if (!c->copy_stream) {
    CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    for (cudaEvent_t& e : c->band_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  enqueue_combine(c, 1);
  enqueue_integrate(c, c->U1, false);
  enqueue_control(c, PH_RK_SECOND);
  enqueue_combine(c, 2);
  MHD_TRACE("L(U2) in bands");
  c->ks->bc(g, c->U2, c->snap, c->ctl, c->stream);
  if (c->scheme == 3) c->ks->lf_alpha(g, c->U2, c->aF, c->aG, c->ctl, c->stream);
  c->launches += c->scheme == 3 ? 2 : 1;
  const int tr = c->ks->flux_tile_rows(c->scheme);
  const int nti = (g.nx + tr - 1) / tr;
  double* const* ch = chars ? c->ch : nullptr;
  for (int b = 0; b < kStepHostBands; b++) {
    const int t0 = int((long long)b * nti / kStepHostBands);
    const int t1 = int((long long)(b + 1) * nti / kStepHostBands);
    // tile row t updates cell rows [2 + t*tr, 2 + (t+1)*tr); the first band
    // also takes ghost rows 0, 1 and the last one the rows from its tiles to NX
    const int r0 = b == 0 ? 0 : 2 + t0 * tr;
    const int r1 = b == kStepHostBands - 1 ? g.NX : 2 + t1 * tr;
    if (t1 > t0) {
      c->ks->flux_rows(c->scheme, g, c->U2, c->UL, c->aF, c->aG, c->ctl, ch, t0, t1, c->stream);
      c->launches += 1;
    }
    c->ks->combine_final_rows(g, r0, r1, c->U, c->U1, c->U2, c->UL, c->ctl, c->stream);
    c->launches += 1;
    cudaError_t e = cudaEventRecord(c->band_ev[1 + b], c->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->copy_stream, c->band_ev[1 + b], 0);
    for (int k = 0; k < NF && e == cudaSuccess && r1 > r0; k++)
      e = cudaMemcpy2DAsync(Uh + ((long long)k * g.NX + r0) * g.NY, g.NY * sizeof(double),
                            c->U1 + k * g.fstride + (long long)r0 * g.pitch + g.off,
                            g.pitch * sizeof(double), g.NY * sizeof(double), size_t(r1 - r0),
                            cudaMemcpyDeviceToHost, c->copy_stream);
    if (e != cudaSuccess) {
      cudaStreamSynchronize(c->copy_stream);  // no copy into Uh outlives the call
      return cuda_fail(c, e, "mhd_step_host: banded copy back");
    }
  }
  c->chars_buf = 2;
  enqueue_control(c, PH_RK_FINAL);
  enqueue_control(c, PH_DONE);
  return MHD_OK;
}

// Fatal statuses of the central-FD integration, with the reference's
// message (spatialmethodcentralfd2.cpp:71-77, 151-156) and a caller suffix.
int cfd_status(mhd_ctx* c, const char* where) {
  const Ctl& h = *c->hctl;
  const bool dens = h.error == 6;
  const unsigned long long lin = dens ? kCfdFirstBase - h.cfd_first : h.cfd_last - 1;
  const int i = int(lin / c->g.NY) - 2, j = int(lin % c->g.NY) - 2;
  char buf[256];
  std::snprintf(buf, sizeof buf,
                "Negative %s encountered at i = %d, j = %d\n! SpatialMethodCentralFD2::integrate%s",
                dens ? "density" : "pressure", i, j, where);
  return set_status(c, dens ? MHD_ERR_NEGATIVE_DENSITY : MHD_ERR_NEGATIVE_PRESSURE, true, buf);
}

int step_status(mhd_ctx* c) {
  const Ctl& h = *c->hctl;
  c->neg_pressure += (long long)h.neg_count;
  if (c->scheme == 1 && (h.error == 6 || h.error == 7))
    return cfd_status(c, "\n! mhd_step: spatial integration");
  if (h.error == 6)
    return set_status(c, MHD_ERR_NEGATIVE_DENSITY, true,
                      "negative density encountered\n! getEigens_F\n! mhd_step: spatial integration");
  if (h.error == 4) {
    char buf[256];
    std::snprintf(buf, sizeof buf,
                  "CFL condition violated!\nMinimum time step = %f\n! updateDt\n! mhd_step: update time step",
                  c->dt_min);
    return set_status(c, MHD_ERR_TIME_UNDERFLOW, true, buf);
  }
  if (h.error == 10)
    return set_status(c, MHD_ERR_WRONG_PARAMETER, true,
                      "updateDt: no power-of-two time step satisfies the CFL window\n! mhd_step");
  if (h.error == kErrTileCopyTimeout)
    return set_status(c, MHD_ERR_CUDA, true, "flux tile copy did not complete\n! mhd_step");
  return MHD_OK;
}

// One time step on the device state; dt in/out.  Uh (optional): the state
// comes from host memory, copied in row bands that the first spatial
// operator follows (enqueue_integrate_from_host).  Uo (optional, RK3): the
// result goes to host memory in row bands that follow the last spatial
// operator (enqueue_rk3_tail_to_host); *copied tells whether Uo got it.
int do_step(mhd_ctx* c, double* dt_inout, const double* Uh = nullptr, double* Uo = nullptr,
            bool* copied = nullptr) {
  if (copied) *copied = false;
  MHD_TRACE("step");
  int st = check_bc_ready(c);
  if (st) return st;
  const bool chars = (c->flags & MHD_FLAG_CHARACTERISTICS) != 0;
  enqueue_control(c, PH_RESET_STEP, *dt_inout);
  if (Uh) {
    if ((st = enqueue_integrate_from_host(c, Uh, c->time_method == 1 && chars))) return st;
  } else {
    enqueue_integrate(c, c->U, c->time_method == 1 && chars);
  }
  if (c->time_method == 1) {
    enqueue_control(c, PH_EULER);
    enqueue_combine(c, 0);
    enqueue_control(c, PH_DONE);
    if ((st = read_ctl(c))) return st;
  } else {
    enqueue_control(c, PH_RK_FIRST);
    if (Uo) {
      if ((st = enqueue_rk3_tail_to_host(c, chars, Uo))) return st;
      st = read_ctl(c);
      const bool keep = !st && !c->hctl->retry && !c->hctl->error;
      cudaError_t e = cudaSuccess;
      // the step's result, now in U1, becomes the device state (overlapping
      // the copies still in flight, which read U1)
      if (keep)
        e = cudaMemcpyAsync(c->U, c->U1, size_t(NF) * c->g.fstride * sizeof(double),
                            cudaMemcpyDeviceToDevice, c->stream);
      const cudaError_t e2 = cudaStreamSynchronize(c->copy_stream);
      if (st) return st;
      if (e == cudaSuccess) e = e2;
      if (e != cudaSuccess) return cuda_fail(c, e, "mhd_step_host: copy back");
      if (copied) *copied = keep;
    } else {
      enqueue_rk3_tail(c, chars);
      if ((st = read_ctl(c))) return st;
    }
    // Like TimeIntegrationRK3::step (timeintegrationrk3.cpp:81-148) the
    // retries have no cap: each one restarts from min(dt1, dt2, dt3), which
    // is strictly below the dt it replaces, so the ladder runs out in
    // underflow (ErrorTimeUnderflow) or in update_dt's bounded loops.
    while (c->hctl->retry && !c->hctl->error) {
      enqueue_control(c, PH_RK_RETRY);
      enqueue_rk3_tail(c, chars);
      if ((st = read_ctl(c))) return st;
    }
  }
  if ((st = step_status(c))) return st;
  *dt_inout = c->hctl->dt;
  return set_status(c, MHD_OK, false, "");
}

void free_step_graph(mhd_ctx* c) {
  if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
  c->step_graph = nullptr;
}

// Adds a while node to the graph being captured on c->stream, after what
// was captured so far; returns its body graph.
cudaError_t capture_while(mhd_ctx* c, cudaGraphConditionalHandle h, cudaGraph_t* body) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(c->stream, &cs, nullptr, &cg, &deps, &nd);
  if (e != cudaSuccess) return e;
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  if ((e = cudaGraphAddNode(&node, cg, deps, nd, &p)) != cudaSuccess) return e;
  *body = p.conditional.phGraph_out[0];
  return cudaStreamUpdateCaptureDependencies(c->stream, &node, 1,
                                             cudaStreamSetCaptureDependencies);
}

// mhd_steps as one graph: while (steps wanted) { one step: the same launches
// as do_step, with the RK3 retry loop as a nested while node whose condition
// the controller's retry flag sets }.  Nothing is read on the host between
// steps; the dt of every step lands in gdts.
int build_step_graph(mhd_ctx* c, bool chars) {
  free_step_graph(c);
  const long long l0 = c->launches;
  const bool rk3 = c->time_method != 1;
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle hs{}, hr{};
  cudaGraph_t body = nullptr, rbody = nullptr;
  cudaError_t e = cudaGraphConditionalHandleCreate(&hs, g, 1, cudaGraphCondAssignDefault);
  if (e == cudaSuccess) {
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = hs;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g, nullptr, 0, &p);
    if (e == cudaSuccess) body = p.conditional.phGraph_out[0];
  }
  if (e == cudaSuccess && rk3) e = cudaGraphConditionalHandleCreate(&hr, body, 0, 0);
  if (e == cudaSuccess)
    e = cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    enqueue_control(c, PH_RESET_CARRY);
    enqueue_integrate(c, c->U, !rk3 && chars);
    if (!rk3) {
      enqueue_control(c, PH_EULER);
      enqueue_combine(c, 0);
      enqueue_control(c, PH_DONE);
    } else {
      enqueue_control(c, PH_RK_FIRST);
      enqueue_rk3_tail(c, chars);
      k_graph_retry<<<1, 32, 0, c->stream>>>(c->ctl, c->gcnt, hr);
      e = capture_while(c, hr, &rbody);
    }
    k_graph_step_end<<<1, 32, 0, c->stream>>>(c->ctl, c->gcnt, c->gdts, hs);
    cudaGraph_t out = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(c->stream, &out);
    if (e == cudaSuccess) e = e2;
  }
  c->step_graph_launches[0] = c->launches - l0 + (rk3 ? 2 : 1);
  if (e == cudaSuccess && rk3) {
    const long long l1 = c->launches;
    e = cudaStreamBeginCaptureToGraph(c->stream, rbody, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      enqueue_control(c, PH_RK_RETRY);
      enqueue_rk3_tail(c, chars);
      k_graph_retry<<<1, 32, 0, c->stream>>>(c->ctl, c->gcnt, hr);
      cudaGraph_t out = nullptr;
      e = cudaStreamEndCapture(c->stream, &out);
    }
    c->step_graph_launches[1] = c->launches - l1 + 1;
  }
  c->launches = l0;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&c->step_graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    c->step_graph = nullptr;
    cudaGetLastError();
    return cuda_fail(c, e, "build_step_graph");
  }
  c->step_graph_chars = chars;
  c->step_graph_tma = tile_tma_enabled() ? 1 : 0;
  return MHD_OK;
}

// nsteps steps through the step graph; the same results and statuses as
// nsteps calls of do_step.
int graph_steps(mhd_ctx* c, int nsteps, double* dt_inout, double* dts) {
  int st = check_bc_ready(c);
  if (st) return st;
  const bool chars = (c->flags & MHD_FLAG_CHARACTERISTICS) != 0;
  if (!c->gcnt) {
    CK(cudaMalloc(&c->gcnt, G_COUNT * sizeof(long long)));
    CK(cudaMallocHost(&c->hgcnt, G_COUNT * sizeof(long long)));
  }
  if (c->gdts_cap < nsteps) {  // the graph holds the buffer's address
    free_step_graph(c);
    if (c->gdts) CK(cudaFree(c->gdts));
    c->gdts = nullptr;
    CK(cudaMalloc(&c->gdts, size_t(nsteps) * sizeof(double)));
    c->gdts_cap = nsteps;
  }
  if (!c->step_graph || c->step_graph_chars != chars ||
      c->step_graph_tma != (tile_tma_enabled() ? 1 : 0))
    if ((st = build_step_graph(c, chars))) return st;
  k_graph_arm<<<1, 32, 0, c->stream>>>(c->gcnt, nsteps);
  enqueue_control(c, PH_RESET_STEP, *dt_inout);  // the first step's dt_in
  CK(cudaGraphLaunch(c->step_graph, c->stream));
  CK(cudaMemcpyAsync(c->hgcnt, c->gcnt, G_COUNT * sizeof(long long), cudaMemcpyDeviceToHost,
                     c->stream));
  if ((st = read_ctl(c))) return st;
  const long long done = c->hgcnt[G_STEPS];
  c->launches += 1 + done * c->step_graph_launches[0] +
                 c->hgcnt[G_RETRIES] * c->step_graph_launches[1] + (done < nsteps ? 1 : 0);
  c->neg_pressure += c->hgcnt[G_NEG] - (long long)c->hctl->neg_count;  // step_status adds the last
  if (done > 0) {
    std::vector<double> h(done);
    CK(cudaMemcpy(h.data(), c->gdts, done * sizeof(double), cudaMemcpyDeviceToHost));
    if (dts) std::memcpy(dts, h.data(), done * sizeof(double));
    *dt_inout = h[done - 1];
  }
  if (done == nsteps) {
    c->neg_pressure += (long long)c->hctl->neg_count;
    return set_status(c, MHD_OK, false, "");
  }
  if ((st = step_status(c))) return st;  // the failing step's status, as do_step reports it
  return set_status(c, MHD_ERR_NOT_CONVERGED, true,
                    "RK3 retry loop of the device step loop passed its bound\n! mhd_steps");
}

void divb_range(const mhd_ctx* c, int r[4]) {
  const Grid& g = c->g;
  r[0] = g.bc[LEFT] == PERIODIC ? 2 : 3;
  r[1] = g.bc[RIGHT] == PERIODIC ? g.nx + 2 : g.nx + 1;
  r[2] = g.bc[BOTTOM] == PERIODIC ? 2 : 3;
  r[3] = g.bc[TOP] == PERIODIC ? g.ny + 2 : g.ny + 1;
}

int do_divb_calc(mhd_ctx* c, double* mx, double* tot) {
  MHD_TRACE("divBCalculation");
  int r[4];
  divb_range(c, r);
  c->ks->divb(c->g, c->U, r, c->partial, c->npartial, c->ctl, c->stream);
  c->launches += 3;
  int st = read_ctl(c);
  if (st) return st;
  const unsigned long long b = c->hctl->divb_max;
  double m;
  std::memcpy(&m, &b, sizeof m);
  *mx = m;
  *tot = c->hctl->divb_sum;
  return MHD_OK;
}

// The sweep loop of one SOR solve on the device: a graph with a while node
// whose body is kSorChunk sweeps and k_sor_again.  It replaces the host loop's
// passes of kSorChunk sweeps and its read of the stop flag after each; the
// sweeps, their order and their values are the same.
int sor_graph_solve(mhd_ctx* c, const int r[4], const double coef[6], double rmax,
                    double max_sweeps, int fused) {
  const double key[5] = {rmax, max_sweeps, coef[5], double(fused), double(c->sor_rows)};
  if (c->sor_graph && std::memcmp(key, c->sor_graph_key, sizeof key) != 0) {
    cudaGraphExecDestroy(c->sor_graph);
    c->sor_graph = nullptr;
  }
  if (!c->sor_cnt) CK(cudaMalloc(&c->sor_cnt, sizeof(long long)));
  if (!c->sor_graph) {
    const double passes = std::ceil(max_sweeps / kSorChunk) + 1.0;
    const long long bound = passes < 9.0e18 ? (long long)passes : (long long)9.0e18;
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h{};
    cudaGraph_t body = nullptr;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
      cudaGraphNodeParams np{};
      np.type = cudaGraphNodeTypeConditional;
      np.conditional.handle = h;
      np.conditional.type = cudaGraphCondTypeWhile;
      np.conditional.size = 1;
      cudaGraphNode_t node;
      e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
      if (e == cudaSuccess) body = np.conditional.phGraph_out[0];
    }
    const long long l0 = c->launches;
    if (e == cudaSuccess)
      e = cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      for (int s = 0; s < kSorChunk; s++)
        c->ks->sor_sweep(c->g, c->phi, c->sor_xy, r, coef, rmax, max_sweeps, c->ratio, c->ctl,
                         fused, c->sor_rows, c->stream);
      k_sor_again<<<1, 32, 0, c->stream>>>(c->ctl, c->sor_cnt, bound, h);
      cudaGraph_t out = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(c->stream, &out);
      if (e == cudaSuccess) e = e2;
    }
    c->sor_graph_launches = (long long)kSorChunk * (fused ? 2 : 5) + 1;
    c->launches = l0;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&c->sor_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      c->sor_graph = nullptr;
      cudaGetLastError();
      return cuda_fail(c, e, "sor_graph_solve");
    }
    std::memcpy(c->sor_graph_key, key, sizeof key);
  }
  CK(cudaMemsetAsync(c->sor_cnt, 0, sizeof(long long), c->stream));
  CK(cudaGraphLaunch(c->sor_graph, c->stream));
  long long passes = 0;
  CK(cudaMemcpyAsync(&passes, c->sor_cnt, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
  const int st = read_ctl(c);  // synchronizes the stream
  c->launches += 1 + passes * c->sor_graph_launches;
  return st;
}

int do_sor(mhd_ctx* c, const mhd_sor_params* p, int* sweeps) {
  MHD_TRACE("divBCorrectionSOR");
  touch_buf(c, 0);  // the B correction changes U's interior
  int r[4];
  divb_range(c, r);
  const Grid& g = c->g;
  // periodic wrap of the B ghosts, as divBCorrectionSOR starts with (div_b_fix.cpp:161-245)
  c->ks->divb(g, c->U, r, c->partial, c->npartial, c->ctl, c->stream);
  const double pxf = 1.0 / (g.dx * g.dx), pyf = 1.0 / (g.dy * g.dy);
  double omega;
  if (p->omega_use_static) {
    omega = p->omega;
  } else {
    const double t = std::cos(g.dx) + std::cos(g.dy);
    omega = (8.0 - std::sqrt(64.0 - 16.0 * t * t)) / (t * t);
  }
  const double coef[6] = {pxf, pyf, 4.0 / (2.0 * g.dx), 4.0 / (2.0 * g.dy),
                          1.0 / (2 * (pxf + pyf)), omega};
  double nan_ratio = std::numeric_limits<double>::quiet_NaN();  // no sweep: 0/0, "converged"
  if (!c->sor_xy) {  // 2 colours x rows x pairs x 4 doubles covers every range of this grid
    const size_t n = 2ull * g.nx * ((g.ny + 2 + 3) / 4 + 1) * 4;
    CK(cudaMalloc(&c->sor_xy, n * sizeof(double)));
  }
  c->ks->sor_rhs(g, c->U, r, coef, c->sor_xy, c->stream);
  c->launches += 1;
  CK(cudaMemsetAsync(&c->ctl->rmax, 0, 2 * sizeof(unsigned long long), c->stream));
  CK(cudaMemsetAsync(&c->ctl->sor_done, 0, 3 * sizeof(int), c->stream));  // + sor_ticket
  CK(cudaMemcpyAsync(c->ratio, &nan_ratio, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  long long issued = 0;
  const int chunk = kSorChunk;
  // fused sweeps: 2 launches per sweep instead of 5 (same arithmetic, same
  // values; see sor_fused_ok), with the ghosts refreshed around the solve
  const int fused = sor_fused_ok(g) && c->sor_fused ? 1 : 0;
  if (p->sor_rsteps > 0) {
    if (fused) {
      c->ks->phi_bc(g, c->phi, c->ctl, c->stream);
      c->launches += 1;
    }
    if (c->use_sor_graph) {
      const int st = sor_graph_solve(c, r, coef, p->sor_rmax, p->sor_rsteps, fused);
      if (st) return st;
    } else {
      for (;;) {
        for (int s = 0; s < chunk; s++) {
          c->ks->sor_sweep(g, c->phi, c->sor_xy, r, coef, p->sor_rmax, p->sor_rsteps, c->ratio,
                           c->ctl, fused, c->sor_rows, c->stream);
          c->launches += fused ? 2 : 5;
        }
        issued += chunk;
        int st = read_ctl(c);
        if (st) return st;
        if (c->hctl->sor_done) break;
      }
    }
    if (fused) {
      c->ks->phi_bc(g, c->phi, c->ctl, c->stream);
      c->launches += 1;
    }
  }
  double last = 0.0;
  CK(cudaMemcpyAsync(&last, c->ratio, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *sweeps = c->hctl->sor_sweeps;
  if (last > p->sor_rmax)  // div_b_fix.cpp:387: NaN counts as converged
    return set_status(c, MHD_ERR_NOT_CONVERGED, true, "SOR divergence cleaning failed to converge");
  c->ks->sor_correct(g, c->U, c->phi, r, 1.0 / (2.0 * g.dx), 1.0 / (2.0 * g.dy), c->stream);
  c->launches += 1;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  (void)issued;
  return set_status(c, MHD_OK, false, "");
}

}  // namespace

int do_nongrid(mhd_ctx* c, double out[7]) {
  double mx = 0.0, tot = 0.0;
  int st = do_divb_calc(c, &mx, &tot);
  if (st) return st;
  const int nb = c->ks->totals(c->g, c->U, c->partial, c->npartial / 5, c->stream);
  c->launches++;
  std::vector<double> h(5 * (size_t)nb);
  CK(cudaMemcpyAsync(h.data(), c->partial, h.size() * sizeof(double), cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  double ent = 0.0, en = 0.0, mass = 0.0, mom = 0.0, uumax = 0.0;
  for (int b = 0; b < nb; b++) {
    ent += h[5 * b];
    en += h[5 * b + 1];
    mass += h[5 * b + 2];
    mom += h[5 * b + 3];
    if (h[5 * b + 4] > uumax) uumax = h[5 * b + 4];
  }
  const double dxdy = c->g.dx * c->g.dy;
  // the columns u_max .. total_entropy of the record line (file_access.cpp:1713-1733)
  out[0] = std::sqrt(uumax);
  out[1] = mx;
  out[2] = tot;
  out[3] = mass * dxdy;
  out[4] = mom * dxdy;
  out[5] = en * dxdy;
  out[6] = ent * dxdy;
  return MHD_OK;
}

extern "C" {

int mhd_ctx_create(int nx, int ny, int halo, double dx, double dy, double gamma, const int bc[4],
                   int scheme, int time_method, double dt_min, double dt_max, double cfl, int flags,
                   int device, mhd_ctx** out) {
  if (!out) return MHD_ERR_WRONG_PARAMETER;
  *out = nullptr;
  if (halo != 2 || nx < 2 || ny < 2 || !(dx > 0) || !(dy > 0) || scheme < 1 || scheme > 3 ||
      (time_method != 1 && time_method != 2) || !bc)
    return MHD_ERR_WRONG_PARAMETER;
  for (int s = 0; s < 4; s++)
    if (bc[s] < PERIODIC || bc[s] > OPEN) return MHD_ERR_WRONG_PARAMETER;
  mhd_ctx* c = new (std::nothrow) mhd_ctx();
  if (!c) return MHD_ERR_CUDA;
  c->device = device;
  c->scheme = scheme;
  c->time_method = time_method;
  c->flags = flags;
  c->dt_min = dt_min;
  c->dt_max = dt_max;
  c->cfl = cfl;
  c->ks = (flags & MHD_FLAG_FAST_MATH) ? &kFast : &kExact;
  Grid& g = c->g;
  g.nx = nx; g.ny = ny; g.NX = nx + 4; g.NY = ny + 4;
  g.pitch = pitch_for(g.NY);
  g.off = ROW_OFF;
  g.fstride = (long long)g.NX * g.pitch;
  g.dx = dx; g.dy = dy; g.gamma = gamma;
  for (int s = 0; s < 4; s++) g.bc[s] = bc[s];
  c->dirichlet_needed = bc[0] == DIRICHLET || bc[1] == DIRICHLET || bc[2] == DIRICHLET ||
                        bc[3] == DIRICHLET;
  c->block_elems = size_t(NF) * g.fstride;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = alloc_block(c, &c->U);
  if (e == cudaSuccess) e = alloc_block(c, &c->UL);
  if (e == cudaSuccess && time_method == 2) e = alloc_block(c, &c->U1);
  if (e == cudaSuccess && time_method == 2) e = alloc_block(c, &c->U2);
  if (e == cudaSuccess && (flags & MHD_FLAG_CHARACTERISTICS))
    for (int q = 0; q < 4 && e == cudaSuccess; q++) e = alloc_block(c, &c->ch[q]);
  const size_t edge = size_t(NF) * std::max(g.NX, g.NY);
  for (int q = 0; q < 4 && e == cudaSuccess; q++) {
    e = cudaMalloc(&c->snap[q], edge * sizeof(double));
    if (e == cudaSuccess) e = cudaMemsetAsync(c->snap[q], 0, edge * sizeof(double), c->stream);
  }
  if (e == cudaSuccess) e = cudaMalloc(&c->aF, sizeof(double) * NF * g.NY);
  if (e == cudaSuccess) e = cudaMalloc(&c->aG, sizeof(double) * NF * g.NX);
  if (e == cudaSuccess) e = cudaMalloc(&c->phi, sizeof(double) * g.fstride);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->phi, 0, sizeof(double) * g.fstride, c->stream);
  c->npartial = 148 * 16;
  if (e == cudaSuccess) e = cudaMalloc(&c->partial, sizeof(double) * c->npartial);
  if (e == cudaSuccess) e = cudaMalloc(&c->ratio, sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&c->ctl, sizeof(Ctl));
  if (e == cudaSuccess) e = cudaMemsetAsync(c->ctl, 0, sizeof(Ctl), c->stream);
  if (e == cudaSuccess) e = cudaMallocHost(&c->hctl, sizeof(Ctl));
  if (e == cudaSuccess) e = cudaMallocHost(&c->hnan, sizeof(double));
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    cuda_fail(nullptr, e, "mhd_ctx_create");
    mhd_ctx_destroy(c);
    return MHD_ERR_CUDA;
  }
  std::memset(c->hctl, 0, sizeof(Ctl));
  *out = c;
  return MHD_OK;
}

int mhd_ctx_destroy(mhd_ctx* c) {
  if (!c) return MHD_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  double* bufs[] = {c->U, c->U1, c->U2, c->UL, c->ch[0], c->ch[1], c->ch[2], c->ch[3], c->aF,
                    c->aG, c->snap[0], c->snap[1], c->snap[2], c->snap[3], c->phi, c->partial,
                    c->ratio, c->sor_xy};
  for (double* b : bufs)
    if (b) cudaFree(b);
  free_step_graph(c);
  if (c->gcnt) cudaFree(c->gcnt);
  if (c->hgcnt) cudaFreeHost(c->hgcnt);
  if (c->gdts) cudaFree(c->gdts);
  if (c->ctl) cudaFree(c->ctl);
  if (c->hctl) cudaFreeHost(c->hctl);
  if (c->hnan) cudaFreeHost(c->hnan);
  if (c->grid_buf) cudaFree(c->grid_buf);
  if (c->sor_graph) cudaGraphExecDestroy(c->sor_graph);
  if (c->sor_cnt) cudaFree(c->sor_cnt);
  for (cudaEvent_t& e : c->band_ev)
    if (e) cudaEventDestroy(e);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return MHD_OK;
}

int mhd_set_stepper(mhd_ctx* c, int time_method, double dt_min, double dt_max, double cfl) {
  if (!c || (time_method != 1 && time_method != 2)) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  if (time_method == 2) {
    if (!c->U1) CK(alloc_block(c, &c->U1));
    if (!c->U2) CK(alloc_block(c, &c->U2));
    CK(cudaStreamSynchronize(c->stream));
  }
  c->time_method = time_method;
  c->dt_min = dt_min;
  c->dt_max = dt_max;
  c->cfl = cfl;
  free_step_graph(c);  // its controller launches carry the old limits
  return set_status(c, MHD_OK, false, "");
}

int mhd_set_step_graph(mhd_ctx* c, int enable) {
  if (!c) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  c->use_step_graph = enable ? 1 : 0;
  if (!enable) free_step_graph(c);
  return MHD_OK;
}

int mhd_last_error(const mhd_ctx* c, char* msg, size_t len, int* is_error) {
  if (!c) return MHD_ERR_WRONG_PARAMETER;
  if (msg && len) {
    std::strncpy(msg, c->msg.c_str(), len - 1);
    msg[len - 1] = '\0';
  }
  if (is_error) *is_error = c->is_error ? 1 : 0;
  return MHD_OK;
}

int mhd_upload(mhd_ctx* c, const double* U) {
  if (!c || !U) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  CK(h2d(c, c->U, U));
  CK(cudaStreamSynchronize(c->stream));
  return set_status(c, MHD_OK, false, "");
}

int mhd_download(mhd_ctx* c, double* U) {
  if (!c || !U) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  CK(d2h(c, U, c->U));
  CK(cudaStreamSynchronize(c->stream));
  return MHD_OK;
}

int mhd_download_ul(mhd_ctx* c, double* UL) {
  if (!c || !UL) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  CK(d2h(c, UL, c->UL));
  CK(cudaStreamSynchronize(c->stream));
  return MHD_OK;
}

int mhd_init_dirichlet(mhd_ctx* c) {
  if (!c) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  c->ks->snapshot(c->g, c->U, c->snap, c->stream);
  c->chars_buf = -1;  // another Dirichlet snapshot, other boundary values
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  c->dirichlet_ready = true;
  return set_status(c, MHD_OK, false, "");
}

int mhd_set_dirichlet(mhd_ctx* c, const double* left, const double* right, const double* bottom,
                      const double* top) {
  if (!c || !left || !right || !bottom || !top) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  const size_t ny = size_t(NF) * c->g.NY * sizeof(double), nx = size_t(NF) * c->g.NX * sizeof(double);
  CK(cudaMemcpyAsync(c->snap[0], left, ny, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->snap[1], right, ny, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->snap[2], bottom, nx, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->snap[3], top, nx, cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->dirichlet_ready = true;
  c->chars_buf = -1;  // other boundary values
  return set_status(c, MHD_OK, false, "");
}

int mhd_integrate(mhd_ctx* c, double* dtIdeal) {
  MHD_TRACE("mhd_integrate");
  if (!c) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  int st = check_bc_ready(c);
  if (st) return st;
  enqueue_control(c, PH_RESET_INTEGRATE);
  enqueue_integrate(c, c->U, (c->flags & MHD_FLAG_CHARACTERISTICS) != 0);
  enqueue_control(c, PH_IDEAL);
  if ((st = read_ctl(c))) return st;
  const Ctl& h = *c->hctl;
  c->neg_pressure += (long long)h.neg_count;
  if (c->scheme == 1 && (h.error == 6 || h.error == 7)) {
    if (h.error == 7 && dtIdeal) *dtIdeal = h.dtIdeal;  // formed before the status
    return cfd_status(c, "\n! mhd_integrate");
  }
  if (h.error == 6)
    return set_status(c, MHD_ERR_NEGATIVE_DENSITY, true,
                      "negative density encountered\n! getEigens_F\n! mhd_integrate");
  if (dtIdeal) *dtIdeal = h.dtIdeal;
  if (h.neg_last)  // status of the last interface, as the reference reports it
    return set_status(c, MHD_ERR_NEGATIVE_PRESSURE, false,
                      "negative pressure encountered\n! getEigens_F\n! mhd_integrate");
  return set_status(c, MHD_OK, false, "");
}

int mhd_integrate_host(mhd_ctx* c, double* U, double* UL, double* dtIdeal) {
  MHD_TRACE("mhd_integrate_host");
  if (!c || !U) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  CK(h2d(c, c->U, U));
  int st = mhd_integrate(c, dtIdeal);
  if (c->is_error) return st;
  CK(d2h(c, U, c->U));
  if (UL) CK(d2h(c, UL, c->UL));
  CK(cudaStreamSynchronize(c->stream));
  return st;
}

int mhd_step(mhd_ctx* c, double* dt_inout) {
  if (!c || !dt_inout) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  return do_step(c, dt_inout);
}

int mhd_step_host(mhd_ctx* c, double* U, double* dt_inout) {
  MHD_TRACE("mhd_step_host");
  if (!c || !U || !dt_inout) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  int st;
  // ENO-Roe on grids of many tile rows: the copy of the state overlaps the
  // first spatial operator (bit-identical; see enqueue_integrate_from_host)
  const int tr = c->ks->flux_tile_rows(c->scheme);
  const bool bands = c->use_banded_h2d && c->g.nx >= 4 * kStepHostBands * tr;
  // RK3 with an ENO scheme: the copy back follows the last spatial
  // operator's row bands (see enqueue_rk3_tail_to_host)
  double* Uo = bands && c->time_method != 1 && (c->scheme == 2 || c->scheme == 3) ? U : nullptr;
  bool copied = false;
  if (c->scheme == 2 && bands) {
    st = do_step(c, dt_inout, U, Uo, &copied);
  } else {
    CK(h2d(c, c->U, U));
    st = do_step(c, dt_inout, nullptr, Uo, &copied);
  }
  if (!copied) CK(d2h(c, U, c->U));
  CK(cudaStreamSynchronize(c->stream));
  return st;
}

int mhd_steps(mhd_ctx* c, int nsteps, double* dt_inout, double* dts) {
  MHD_TRACE("mhd_steps");
  if (!c || !dt_inout || nsteps < 0) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  if (c->use_step_graph && nsteps > 0) return graph_steps(c, nsteps, dt_inout, dts);
  for (int n = 0; n < nsteps; n++) {
    int st = do_step(c, dt_inout);
    if (st) return st;
    if (dts) dts[n] = *dt_inout;
  }
  return MHD_OK;
}

int mhd_get_characteristics(mhd_ctx* c, double* cx, double* cy, double* LUx, double* LUy) {
  if (!c) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  // central FD keeps no characteristics: the base class's getCharacteristicsX/Y
  // return false and leave the arrays (spatialintegrationmethod.cpp:69-82)
  if (c->scheme == 1) return set_status(c, MHD_NO_CHANGE, false, "no characteristics (central FD)");
  if (!(c->flags & MHD_FLAG_CHARACTERISTICS)) {
    // on request: the last spatial integration again, on its unchanged input,
    // with the characteristics kernel (the same values the flag would keep)
    if (c->chars_buf < 0)
      return set_status(c, MHD_ERR_WRONG_PARAMETER, true,
                        "characteristics not available: the input of the last spatial "
                        "integration has changed since (or none ran); create the context with "
                        "MHD_FLAG_CHARACTERISTICS to keep them every time");
    for (int q = 0; q < 4; q++)
      if (!c->ch[q]) CK(alloc_block(c, &c->ch[q]));
    double* X = c->chars_buf == 0 ? c->U : (c->chars_buf == 1 ? c->U1 : c->U2);
    enqueue_control(c, PH_RESET_INTEGRATE);
    enqueue_integrate(c, X, true);
    int st = read_ctl(c);
    if (st) return st;
  }
  double* dst[4] = {cx, cy, LUx, LUy};
  for (int q = 0; q < 4; q++)
    if (dst[q]) CK(d2h(c, dst[q], c->ch[q]));
  CK(cudaStreamSynchronize(c->stream));
  return MHD_OK;
}

int mhd_divb_calc(mhd_ctx* c, double* maxdivb, double* totdivb) {
  if (!c || !maxdivb || !totdivb) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  return do_divb_calc(c, maxdivb, totdivb);
}

int mhd_nongrid_data(mhd_ctx* c, double out[7]) {
  if (!c || !out) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  int st = do_nongrid(c, out);
  if (st) return st;
  return set_status(c, MHD_OK, false, "");
}

int mhd_run(mhd_ctx* c, const mhd_run_params* p, mhd_nongrid_record* records, int max_records,
            mhd_run_result* res) {
  MHD_TRACE("mhd_run");
  if (!c || !p || !res || (p->time_mode != 1 && p->time_mode != 2) ||
      (p->time_mode == 1 && p->steps < 1) || (p->nongrid_mode == 1 && p->nongrid_steps < 1) ||
      (p->nongrid_mode == 2 && !(p->nongrid_t > 0.0)) ||
      (p->sor.sor_steps > 0 && p->sor.divb_skip_steps < 1))
    return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  *res = mhd_run_result{};
  int st = MHD_OK, step = 1, nrec = 0;
  double t = 0.0, dt = p->dt0, next_t = p->nongrid_t;
  auto record = [&](int s) -> int {
    if (records && nrec < max_records) {
      mhd_nongrid_record& r = records[nrec];
      r.step = s;
      r.t = t;
      r.dt = dt;
      const int e = do_nongrid(c, r.values);
      if (e) return e;
    }
    nrec++;
    return MHD_OK;
  };
  if (p->nongrid_mode && (st = record(0))) return st;
  for (bool done = false; !done;) {
    st = do_step(c, &dt);
    res->status = st;
    res->is_error = c->is_error ? 1 : 0;
    if (st == MHD_ERR_TIME_UNDERFLOW || c->is_error) break;
    if (p->sor.sor_steps > 0 && step % p->sor.divb_skip_steps == 0) {  // main.cpp:207-242
      double mx = 0.0, tot = 0.0;
      for (int it = 0; it < p->sor.sor_steps; it++) {
        int e = do_divb_calc(c, &mx, &tot);
        if (e) return e;
        if (mx < p->sor.sor_divbmax) break;
        int sw = 0;
        e = do_sor(c, &p->sor, &sw);
        res->sor_sweeps += sw;
        if (e == MHD_ERR_NOT_CONVERGED) break;
        if (e) return e;
      }
      int e = do_divb_calc(c, &mx, &tot);
      if (e) return e;
    }
    t += dt;
    done = p->time_mode == 1 ? step == p->steps : t >= p->t_max;
    bool out = false;
    if (p->nongrid_mode == 1) {
      out = step % p->nongrid_steps == 0;
    } else if (p->nongrid_mode == 2) {
      out = t >= next_t;
      while (out && next_t <= t) next_t += p->nongrid_t;
    }
    if (out && (st = record(step))) return st;
    double u00 = 0.0;  // the NaN stop of main.cpp:335-341
    CK(cudaMemcpyAsync(c->hnan, c->U + c->g.at(0, 2, 2), sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    u00 = *c->hnan;
    if (std::isnan(u00)) {
      res->nan_stop = 1;
      done = true;
    }
    res->steps = step;
    step++;
  }
  res->t = t;
  res->dt = dt;
  res->records = nrec;
  return res->status;
}

int mhd_divb_sor(mhd_ctx* c, const mhd_sor_params* p, int* sweeps) {
  if (!c || !p) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  int sw = 0;
  int st = do_sor(c, p, &sw);
  if (sweeps) *sweeps = sw;
  return st;
}

int mhd_divb_clean(mhd_ctx* c, const mhd_sor_params* p, double* maxdivb, int* total_sweeps) {
  MHD_TRACE("mhd_divb_clean");
  if (!c || !p) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  double mx = -1.0, tot = 0.0;
  int total = 0, st = MHD_OK;
  if (p->sor_steps > 0) {
    for (int it = 0; it < p->sor_steps; it++) {
      if ((st = do_divb_calc(c, &mx, &tot))) return st;
      if (mx < p->sor_divbmax) break;
      int sw = 0;
      st = do_sor(c, p, &sw);
      total += sw;
      if (st == MHD_ERR_NOT_CONVERGED) break;
      if (st) return st;
    }
    int st2 = do_divb_calc(c, &mx, &tot);
    if (st2) return st2;
  }
  if (maxdivb) *maxdivb = mx;
  if (total_sweeps) *total_sweeps = total;
  return st;
}

int mhd_get_counters(mhd_ctx* c, long long* neg_pressure, long long* launches) {
  if (!c) return MHD_ERR_WRONG_PARAMETER;
  if (neg_pressure) *neg_pressure = c->neg_pressure;
  if (launches) *launches = c->launches;
  return MHD_OK;
}

int mhd_set_step_host_banded(mhd_ctx* c, int enable) {
  if (!c || (enable != 0 && enable != 1)) return MHD_ERR_WRONG_PARAMETER;
  c->use_banded_h2d = enable;
  return set_status(c, MHD_OK, false, "");
}

int mhd_set_sor_graph(mhd_ctx* c, int enable) {
  if (!c || (enable != 0 && enable != 1)) return MHD_ERR_WRONG_PARAMETER;
  c->use_sor_graph = enable;
  return set_status(c, MHD_OK, false, "");
}

int mhd_grid_pack(mhd_ctx* c, const mhd_grid_pack_params* p, void* out, size_t out_bytes,
                  size_t* bytes) {
  MHD_TRACE("mhd_grid_pack");
  if (!c || !p) return MHD_ERR_WRONG_PARAMETER;
  const auto flag = [](int v) { return v == 0 || v == 1; };
  if (!flag(p->natural) || !flag(p->conservation) || !flag(p->single))
    return set_status(c, MHD_ERR_WRONG_PARAMETER, true, "mhd_grid_pack: flags must be 0 or 1");
  const size_t need = size_t(output::grid_fields(p->natural, p->conservation)) * size_t(c->g.nx) *
                      size_t(c->g.ny) * (p->single ? sizeof(float) : sizeof(double));
  if (bytes) *bytes = need;
  if (!out) return set_status(c, MHD_OK, false, "");  // size query
  if (out_bytes < need)
    return set_status(c, MHD_ERR_WRONG_PARAMETER, true, "mhd_grid_pack: output buffer too small");
  CK(cudaSetDevice(c->device));
  if (c->grid_buf_bytes < need) {
    if (c->grid_buf) CK(cudaFree(c->grid_buf));
    c->grid_buf = nullptr;
    c->grid_buf_bytes = 0;
    CK(cudaMalloc(&c->grid_buf, need));
    c->grid_buf_bytes = need;
  }
  output::launch_grid_pack(c->g, c->U, p->natural != 0, p->conservation != 0, p->single != 0,
                           p->start_x, p->start_y, c->grid_buf, c->stream);
  CK(cudaPeekAtLastError());
  c->launches++;
  CK(cudaMemcpyAsync(out, c->grid_buf, need, cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return set_status(c, MHD_OK, false, "");
}

int mhd_layout(const mhd_ctx* c, int* pitch, int* row_offset) {
  if (!c) return MHD_ERR_WRONG_PARAMETER;
  if (pitch) *pitch = c->g.pitch;
  if (row_offset) *row_offset = c->g.off;
  return MHD_OK;
}

int mhd_fp64_peak(int device, double* tflops) {
  mhd_ctx* c = nullptr;
  if (!tflops) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(device));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  double* out = nullptr;
  CK(cudaMalloc(&out, sizeof(double)));
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  const int blocks = sms * 8, threads = 256, iters = 8192;
  k_fma_peak<<<blocks, threads>>>(out, 64, 0.999999, 1e-9);  // warm-up
  CK(cudaEventRecord(a));
  k_fma_peak<<<blocks, threads>>>(out, iters, 0.999999, 1e-9);
  CK(cudaEventRecord(b));
  CK(cudaEventSynchronize(b));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  CK(cudaGetLastError());
  *tflops = 2.0 * 8.0 * double(iters) * blocks * threads / (double(ms) * 1e-3) / 1e12;
  return MHD_OK;
}

int mhd_set_tile_tma(int enable, long long* tma_launches) {
  if (enable != 0 && enable != 1 && enable != -1) return MHD_ERR_WRONG_PARAMETER;
  if (enable >= 0) tile_tma_flag() = enable != 0;
  if (tma_launches) *tma_launches = tile_tma_launches();
  return MHD_OK;
}

int mhd_set_sor_rows(mhd_ctx* c, int mode) {
  if (!c || mode < 0 || mode > 2) return MHD_ERR_WRONG_PARAMETER;
  c->sor_rows = mode;
  return MHD_OK;
}

int mhd_set_sor_fused(mhd_ctx* c, int enable) {
  if (!c || (enable != 0 && enable != 1)) return MHD_ERR_WRONG_PARAMETER;
  c->sor_fused = enable;
  return MHD_OK;
}

int mhd_stream(const mhd_ctx* c, void** stream) {
  if (!c || !stream) return MHD_ERR_WRONG_PARAMETER;
  *stream = (void*)c->stream;
  return MHD_OK;
}

int mhd_time_integrate(mhd_ctx* c, int n, double* avg_ms) {
  if (!c || n < 1 || !avg_ms) return MHD_ERR_WRONG_PARAMETER;
  CK(cudaSetDevice(c->device));
  int st = check_bc_ready(c);
  if (st) return st;
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  enqueue_control(c, PH_RESET_INTEGRATE);
  CK(cudaEventRecord(a, c->stream));
  for (int q = 0; q < n; q++) enqueue_integrate(c, c->U, false);
  CK(cudaEventRecord(b, c->stream));
  CK(cudaEventSynchronize(b));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  CK(cudaGetLastError());
  *avg_ms = double(ms) / n;
  return MHD_OK;
}

}  // extern "C"
