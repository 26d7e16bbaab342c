// Batched runs (include/mhd2d_b200.h, mhd_batch_*): many independent
// problems of uneven sizes, schemes, boundary conditions and end times on
// one GPU, advanced together.
//
// Device data:
//   * one pooled allocation holds every run's U, U1, U2, UL blocks (padded
//     rows like a context's), its ENO-LF alpha arrays and Dirichlet edges;
//   * BInst[n]  — per-run constants (grid, buffers, dt limits, end time);
//   * BState[n] — per-run progress: the controller block (CFL maxima, dt1,
//     dt2, dt3, dt, error word), t, steps, the RK3 phase, the stage update
//     the controller chose, active flag and final status;
//   * a flux-tile table (run, tile) over the active runs and an alpha-block
//     table over the active ENO-LF runs, rebuilt when runs finish.
// One stage = kb_bc -> kb_alpha -> kb_flux (persistent: a fixed grid of
// CTAs pulls tiles from an atomic counter) -> kb_control -> kb_combine ->
// kb_finish.  Every kernel acts on each run according to that run's own
// phase, so runs whose RK3 step restarted (a dt retry) simply take more
// stages while the others go on; nothing waits on the host.  A sequence of
// stages is captured once as a CUDA graph and replayed.
//
// The arithmetic of a run is the context path's (same device functions,
// same -fmad=false build), so a run in a batch is bit-identical to the same
// problem run alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mhd2d_b200.h"
#include "mhd_flux.cuh"
#include "mhd_misc.cuh"
#include "mhd_problems.cuh"
#include "mhd_trace.h"

namespace mhd {
namespace MHD_KNS {

struct BInst {
  Grid g;
  double *U, *U1, *U2, *UL;
  double *aF, *aG;
  const double* snap[4];
  StepParams sp;
  Gas G;
  double inv_dx, inv_dy;
  double t_end;
  int scheme, time_method, max_steps, pad;
};

struct BState {
  Ctl c;
  double t;
  long long retries;
  int phase;     // 0: next operator on U, 1: on U1, 2: on U2
  int mode;      // stage update chosen by the controller (k_combine modes), -1: none
  int active;
  int status;
  int steps;
  int step_end;  // the stage update completes a time step
};

__device__ __forceinline__ double* stage_buf(const BInst& in, int phase) {
  return phase == 0 ? in.U : (phase == 1 ? in.U1 : in.U2);
}

// Ghost fill of each active run's current stage buffer; zeroes the ENO-LF
// alpha arrays, and resets the two flux tile counters next[0..1].
__global__ void __launch_bounds__(256) kb_bc(const BInst* __restrict__ I, BState* S, int* next) {
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x < 2) next[threadIdx.x] = 0;
  const int b = blockIdx.y;
  if (!S[b].active) return;
  const BInst& in = I[b];
  double* X = stage_buf(in, S[b].phase);
  const Snap d{in.snap[0], in.snap[1], in.snap[2], in.snap[3]};
  const long long n = bc_count(in.g);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (long long e = t0; e < n; e += stride) bc_elem(in.g, X, d, e);
  if (in.scheme == 3) {
    const long long na = (long long)NF * (in.g.NX + in.g.NY);
    for (long long e = t0; e < na; e += stride) {
      if (e < (long long)NF * in.g.NY) in.aF[e] = 0.0;
      else in.aG[e - (long long)NF * in.g.NY] = 0.0;
    }
  }
}

// ENO-LF dissipation coefficients over the alpha-block table.
__global__ void __launch_bounds__(256) kb_alpha(const BInst* __restrict__ I, BState* S,
                                                const int2* __restrict__ tab,
                                                const int* __restrict__ count) {
  __shared__ double col[8][NF][33];
  const int n = *count;
  for (int t = blockIdx.x; t < n; t += gridDim.x) {
    const int2 e = tab[t];
    const int b = e.x;
    if (!S[b].active) continue;  // uniform over the block
    const BInst& in = I[b];
    const int nbx = (in.g.ny + 1 + 31) / 32;
    const int by = e.y / nbx, bx = e.y - by * nbx;
    lf_alpha_block(in.g, stage_buf(in, S[b].phase), in.aF, in.aG, &S[b].c, bx, by, col);
    __syncthreads();
  }
}

// The persistent flux launch of one scheme: a fixed grid of CTAs pulls
// (run, tile) items [first, first + count) of the table through an atomic
// counter until they are exhausted.  The ENO-Roe and ENO-LF launches of a
// stage run side by side on two streams.
template <int SCHEME, int TI, int NW, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB)
kb_flux(const BInst* __restrict__ I, BState* S, const int2* __restrict__ tab,
        const int* __restrict__ range, int* next) {
  __shared__ BInst s_in;
  __shared__ int s_t, s_phase;
  const int first = range[0], n = range[1];
  for (;;) {
    __syncthreads();  // the previous tile is done with shared memory
    if (threadIdx.x == 0) {
      const int t = atomicAdd(next, 1);
      s_t = t;
      if (t < n) {
        const int b = tab[first + t].x;
        s_phase = S[b].active ? S[b].phase : -1;
      }
    }
    __syncthreads();
    const int t = s_t;
    if (t >= n) break;
    if (s_phase < 0) continue;
    const int2 e = tab[first + t];
    {  // the run's descriptor, staged once per tile
      const int* src = reinterpret_cast<const int*>(&I[e.x]);
      int* dst = reinterpret_cast<int*>(&s_in);
      for (int q = threadIdx.x; q < int(sizeof(BInst) / sizeof(int)); q += NW * 32) dst[q] = src[q];
    }
    __syncthreads();
    const int ntj = (s_in.g.ny + 31) / 32;
    const int ti = e.y / ntj, tj = e.y - ti * ntj;
    const double* X = stage_buf(s_in, s_phase);
    const CharOut co{nullptr, nullptr, nullptr, nullptr};
    flux_tile<SCHEME, false, TI, 32, NW>(s_in.g, X, s_in.UL, s_in.aF, s_in.aG, s_in.inv_dx,
                                         s_in.inv_dy, s_in.G, &S[e.x].c, co, tj, ti);
  }
}

// Per-run time-step controller: dtIdeal from the run's CFL maxima, updateDt
// on the stage's dt slot, the RK3 restart rule, and the stage update that
// follows (timeintegrationrk3.cpp:48-156, timeintegrationeuler.cpp:26-64).
__device__ __forceinline__ void stop_run(BState& s, int status, int* n_active) {
  s.active = 0;
  s.status = status;
  s.mode = -1;
  atomicSub(n_active, 1);
}

__global__ void kb_control(const BInst* __restrict__ I, BState* S, int n, int* n_active) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  BState& s = S[b];
  s.mode = -1;
  if (!s.active) return;
  const BInst& in = I[b];
  Ctl& c = s.c;
  const double ax = in.sp.dx / bits_to_double(c.maxX), ay = in.sp.dy / bits_to_double(c.maxY);
  const double ideal = (ay < ax) ? ay : ax;  // std::min(a, b)
  c.dtIdeal = ideal;
  c.maxX = 0ull;
  c.maxY = 0ull;
  if (c.error) { stop_run(s, c.error, n_active); return; }
  int st;
  if (in.time_method == 1) {
    st = update_dt(in.sp, c.dt, ideal);
    if (st == 4 || st == 10) { stop_run(s, st, n_active); return; }
    s.mode = 0;
    s.step_end = 1;
    return;
  }
  switch (s.phase) {
    case 0:
      st = update_dt(in.sp, c.dt1, ideal);
      if (st == 4 || st == 10) { stop_run(s, st, n_active); return; }
      c.dt = min3(c.dt1, c.dt2, c.dt3);
      s.mode = 1;
      s.phase = 1;
      break;
    case 1:
      st = update_dt(in.sp, c.dt2, ideal);
      if (st == 4 || st == 10) { stop_run(s, st, n_active); return; }
      if (c.dt2 < c.dt) {  // restart the stage loop with the smaller dt and the current UL
        s.retries += 1;
        c.dt = min3(c.dt1, c.dt2, c.dt3);
        s.mode = 1;
      } else {
        s.mode = 2;
        s.phase = 2;
      }
      break;
    default:
      st = update_dt(in.sp, c.dt3, ideal);
      if (st == 4 || st == 10) { stop_run(s, st, n_active); return; }
      if (c.dt3 < c.dt) {
        s.retries += 1;
        c.dt = min3(c.dt1, c.dt2, c.dt3);
        s.mode = 1;
        s.phase = 1;
      } else {
        s.mode = 3;
        s.step_end = 1;
      }
      break;
  }
}

// Stage updates over the flux-tile table (TI x 32 cells x 8 fields per item).
__global__ void __launch_bounds__(256) kb_combine(const BInst* __restrict__ I,
                                                  const BState* __restrict__ S,
                                                  const int2* __restrict__ tab,
                                                  const int* __restrict__ count, int TI) {
  const int n = *count;
  for (int t = blockIdx.x; t < n; t += gridDim.x) {
    const int2 e = tab[t];
    const int mode = S[e.x].mode;
    if (mode < 0) continue;
    const BInst& in = I[e.x];
    const Grid& g = in.g;
    const double dt = S[e.x].c.dt;
    const int ntj = (g.ny + 31) / 32;
    const int ti = e.y / ntj, tj = e.y - ti * ntj;
    const int cells = TI * 32;
    for (int q = threadIdx.x; q < NF * cells; q += blockDim.x) {
      const int k = q / cells, r = (q - k * cells) >> 5, cj = q & 31;
      const int i = 2 + ti * TI + r, j = 2 + tj * 32 + cj;
      if (i < g.nx + 2 && j < g.ny + 2) combine_at(mode, dt, g.at(k, i, j), in.U, in.U1, in.U2, in.UL);
    }
  }
}

// End of a time step: t += dt, the main loop's stop rules, next step's dt slots.
__global__ void kb_finish(const BInst* __restrict__ I, BState* S, int n, int* n_active) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  BState& s = S[b];
  if (!s.active || !s.step_end) return;
  const BInst& in = I[b];
  s.step_end = 0;
  s.t += s.c.dt;
  s.steps += 1;
  bool done = s.t >= in.t_end;
  if (in.max_steps > 0 && s.steps >= in.max_steps) done = true;
  if (isnan(in.U[in.g.at(0, 2, 2)])) done = true;  // main.cpp: NaN check at U[0][2][2]
  if (done) {
    s.active = 0;
    s.status = 0;
    atomicSub(n_active, 1);
    return;
  }
  s.c.dt1 = s.c.dt;
  s.c.dt2 = in.sp.dt_max;
  s.c.dt3 = in.sp.dt_max;
  s.phase = 0;
}

// Re-arm one run (after an upload or a device-side initial state).
__global__ void kb_arm(const BInst* __restrict__ I, BState* S, int b, double dt0, int* n_active) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  BState& s = S[b];
  const bool was = s.active != 0;
  memset(&s, 0, sizeof(BState));
  s.c.dt1 = dt0;
  s.c.dt = dt0;
  s.c.dt2 = I[b].sp.dt_max;
  s.c.dt3 = I[b].sp.dt_max;
  s.mode = -1;
  s.active = 1;
  if (!was) atomicAdd(n_active, 1);
}

}  // namespace MHD_KNS
}  // namespace mhd

using namespace mhd;
using namespace mhd::MHD_KNS;

// ---------------------------------------------------------------------------
// Host side.
namespace {

struct TileShape {
  int TI, NW;
  const void* kern[2];  // ENO-Roe, ENO-LF
  int smem;
};

template <int TI, int NW, int MINB>
TileShape shape() {
  return TileShape{TI,
                   NW,
                   {reinterpret_cast<const void*>(&kb_flux<2, TI, NW, MINB>),
                    reinterpret_cast<const void*>(&kb_flux<3, TI, NW, MINB>)},
                   int(TileGeom<TI, 32>::BYTES)};
}

// Device control words (dints) of a batch.
enum : int {
  W_ROE_FIRST = 0, W_ROE_COUNT = 1,  // ENO-Roe items of the flux table
  W_LF_FIRST = 2, W_LF_COUNT = 3,    // ENO-LF items
  W_ITEMS = 4,                       // all flux items (stage updates)
  W_ALPHA = 5,                       // alpha-block items
  W_NEXT_ROE = 6, W_NEXT_LF = 7,     // tile counters of the two flux launches
  W_ACTIVE = 8,                      // active runs
  W_COUNT = 16
};

const TileShape& tile_shape(int code) {
  static const TileShape s[MHD_BATCH_TILE_COUNT] = {shape<7, 8, 2>(), shape<3, 4, 4>()};
  return s[code];
}

constexpr int kMaxStagesPerGraph = 24;

}  // namespace

struct mhd_batch {
  int device = 0, n = 0;
  cudaStream_t stream = nullptr, side = nullptr;  // side: the ENO-LF flux launch
  cudaEvent_t fork = nullptr, join = nullptr;
  std::vector<mhd_batch_desc> desc;
  std::vector<BInst> hinst;
  BInst* dinst = nullptr;
  BState* dstate = nullptr;
  BState* hstate = nullptr;  // pinned mirror
  double* pool = nullptr;
  int2 *dftab = nullptr, *datab = nullptr;
  int* dints = nullptr;  // W_* control words
  int* hints = nullptr;  // pinned mirror
  int alpha_items = 0;   // ENO-LF dissipation blocks of the item table
  size_t ftab_cap = 0, atab_cap = 0;
  int tile = MHD_BATCH_TILE_7x32, ctas_per_sm = 0, nsm = 148;
  int grid_flux[2] = {0, 0};
  bool any_roe = false, any_lf = false;
  std::vector<char> in_table;  // run belongs in the work tables
  bool tables_dirty = true;
  cudaGraphExec_t graph = nullptr;
  int graph_stages = 0;
  std::string msg;
  bool is_error = false;
  long long launches = 0;
};

namespace {

int bset(mhd_batch* b, int st, bool err, const std::string& m) {
  b->is_error = err;
  b->msg = m;
  return st;
}

int bfail(mhd_batch* b, cudaError_t e, const char* where) {
  std::string m = std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e);
  if (b) return bset(b, MHD_ERR_CUDA, true, m);
  std::fprintf(stderr, "mhd2d_b200: %s\n", m.c_str());
  return MHD_ERR_CUDA;
}

#define BK(call)                                           \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return bfail(b, e_, #call);     \
  } while (0)

int pitch_for(int NY) { return ((NY + ROW_OFF + 15) / 16) * 16; }

void free_graph(mhd_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  b->graph_stages = 0;
}

int flux_tiles_of(const mhd_batch_desc& d, int TI) {
  return ((d.ny + 31) / 32) * ((d.nx + TI - 1) / TI);
}
int alpha_blocks_of(const mhd_batch_desc& d) {
  return ((d.ny + 1 + 31) / 32) * ((d.nx + 1 + 7) / 8);
}

// (Re)build the work tables over the runs flagged in b->in_table.
int build_tables(mhd_batch* b) {
  const int TI = tile_shape(b->tile).TI;
  std::vector<int2> ft, at;
  // large runs first: their tiles start while the small ones fill the tail
  std::vector<int> order;
  for (int r = 0; r < b->n; r++)
    if (b->in_table[r]) order.push_back(r);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return (long long)b->desc[x].nx * b->desc[x].ny > (long long)b->desc[y].nx * b->desc[y].ny;
  });
  int nroe = 0;
  for (int pass = 0; pass < 2; pass++)  // ENO-Roe items, then ENO-LF items
    for (int r : order) {
      if ((b->desc[r].scheme == 3) != (pass == 1)) continue;
      const int nt = flux_tiles_of(b->desc[r], TI);
      for (int t = 0; t < nt; t++) ft.push_back(make_int2(r, t));
      if (pass == 0) nroe += nt;
      if (pass == 1) {
        const int na = alpha_blocks_of(b->desc[r]);
        for (int t = 0; t < na; t++) at.push_back(make_int2(r, t));
      }
    }
  if (ft.size() > b->ftab_cap || at.size() > b->atab_cap) {
    free_graph(b);
    if (ft.size() > b->ftab_cap) {
      if (b->dftab) cudaFree(b->dftab);
      b->dftab = nullptr;
      b->ftab_cap = std::max<size_t>(ft.size(), 1);
      BK(cudaMalloc(&b->dftab, b->ftab_cap * sizeof(int2)));
    }
    if (at.size() > b->atab_cap) {
      if (b->datab) cudaFree(b->datab);
      b->datab = nullptr;
      b->atab_cap = std::max<size_t>(at.size(), 1);
      BK(cudaMalloc(&b->datab, b->atab_cap * sizeof(int2)));
    }
  }
  if (!ft.empty())
    BK(cudaMemcpyAsync(b->dftab, ft.data(), ft.size() * sizeof(int2), cudaMemcpyHostToDevice,
                       b->stream));
  if (!at.empty())
    BK(cudaMemcpyAsync(b->datab, at.data(), at.size() * sizeof(int2), cudaMemcpyHostToDevice,
                       b->stream));
  b->hints[W_ROE_FIRST] = 0;
  b->hints[W_ROE_COUNT] = nroe;
  b->hints[W_LF_FIRST] = nroe;
  b->hints[W_LF_COUNT] = int(ft.size()) - nroe;
  b->hints[W_ITEMS] = int(ft.size());
  b->hints[W_ALPHA] = int(at.size());
  b->alpha_items = int(at.size());
  BK(cudaMemcpyAsync(b->dints, b->hints, (W_ALPHA + 1) * sizeof(int), cudaMemcpyHostToDevice,
                     b->stream));
  BK(cudaStreamSynchronize(b->stream));  // the pinned staging words are reused
  const bool roe = nroe > 0, lf = !at.empty();
  if (b->any_lf != lf || b->any_roe != roe) free_graph(b);  // the stage's launches change
  b->any_lf = lf;
  b->any_roe = roe;
  b->tables_dirty = false;
  return MHD_OK;
}

int refresh_tables(mhd_batch* b) { return b->tables_dirty ? build_tables(b) : MHD_OK; }

int choose_grid(mhd_batch* b) {
  const TileShape& s = tile_shape(b->tile);
  for (int q = 0; q < 2; q++) {
    BK(cudaFuncSetAttribute(s.kern[q], cudaFuncAttributeMaxDynamicSharedMemorySize, s.smem));
    int occ = 0;
    BK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, s.kern[q], s.NW * 32, s.smem));
    if (occ < 1) occ = 1;
    const int per = (b->ctas_per_sm > 0 && b->ctas_per_sm < occ) ? b->ctas_per_sm : occ;
    b->grid_flux[q] = b->nsm * per;
  }
  return MHD_OK;
}

// One CTA per ENO-LF dissipation block (32 x 8 cells of one run): the blocks
// are independent.
int alpha_blocks(const mhd_batch* b) { return b->alpha_items > 0 ? b->alpha_items : 1; }

// The two persistent flux launches of a stage: ENO-Roe on the main stream,
// ENO-LF on the side stream, joined before the controller.
void enqueue_flux(mhd_batch* b, const TileShape& s) {
  int* d = b->dints;
  if (b->any_lf && b->any_roe) {
    cudaEventRecord(b->fork, b->stream);
    cudaStreamWaitEvent(b->side, b->fork, 0);
  }
  for (int q = 0; q < 2; q++) {
    if (q == 0 ? !b->any_roe : !b->any_lf) continue;
    int* range = d + (q == 0 ? W_ROE_FIRST : W_LF_FIRST);
    int* next = d + (q == 0 ? W_NEXT_ROE : W_NEXT_LF);
    void* kargs[] = {&b->dinst, &b->dstate, &b->dftab, &range, &next};
    cudaStream_t st = (q == 1 && b->any_roe) ? b->side : b->stream;
    cudaLaunchKernel(s.kern[q], dim3(b->grid_flux[q]), dim3(s.NW * 32), kargs, size_t(s.smem), st);
    b->launches += 1;
  }
  if (b->any_lf && b->any_roe) {
    cudaEventRecord(b->join, b->side);
    cudaStreamWaitEvent(b->stream, b->join, 0);
  }
}

// Enqueue one stage for every active run.
void enqueue_stage(mhd_batch* b) {
  MHD_TRACE("batch stage");
  const TileShape& s = tile_shape(b->tile);
  int* d = b->dints;
  kb_bc<<<dim3(16, b->n), 256, 0, b->stream>>>(b->dinst, b->dstate, d + W_NEXT_ROE);
  if (b->any_lf) {
    kb_alpha<<<alpha_blocks(b), 256, 0, b->stream>>>(b->dinst, b->dstate, b->datab, d + W_ALPHA);
    b->launches += 1;
  }
  enqueue_flux(b, s);
  kb_control<<<(b->n + 127) / 128, 128, 0, b->stream>>>(b->dinst, b->dstate, b->n, d + W_ACTIVE);
  kb_combine<<<b->nsm * 8, 256, 0, b->stream>>>(b->dinst, b->dstate, b->dftab, d + W_ITEMS, s.TI);
  kb_finish<<<(b->n + 127) / 128, 128, 0, b->stream>>>(b->dinst, b->dstate, b->n, d + W_ACTIVE);
  b->launches += 4;
}

int launches_per_stage(const mhd_batch* b) {
  return 4 + (b->any_lf ? 2 : 0) + (b->any_roe ? 1 : 0);
}

int capture_graph(mhd_batch* b, int stages) {
  free_graph(b);
  cudaGraph_t g = nullptr;
  BK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  const long long l0 = b->launches;
  for (int q = 0; q < stages; q++) enqueue_stage(b);
  b->launches = l0;
  cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (e != cudaSuccess) return bfail(b, e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return bfail(b, e, "cudaGraphInstantiate");
  b->graph_stages = stages;
  return MHD_OK;
}

int read_states(mhd_batch* b) {
  BK(cudaMemcpyAsync(b->hstate, b->dstate, sizeof(BState) * b->n, cudaMemcpyDeviceToHost,
                     b->stream));
  BK(cudaMemcpyAsync(b->hints + W_ACTIVE, b->dints + W_ACTIVE, sizeof(int), cudaMemcpyDeviceToHost,
                     b->stream));
  BK(cudaStreamSynchronize(b->stream));
  BK(cudaGetLastError());
  return MHD_OK;
}

int check_idx(mhd_batch* b, int idx) {
  if (!b || idx < 0 || idx >= b->n) return MHD_ERR_WRONG_PARAMETER;
  return MHD_OK;
}

// After a run was (re)armed: it belongs in the work tables (rebuilt lazily).
void ensure_in_table(mhd_batch* b, int idx) {
  if (b->in_table[idx]) return;
  b->in_table[idx] = 1;
  b->tables_dirty = true;
}

int arm(mhd_batch* b, int idx) {
  kb_arm<<<1, 32, 0, b->stream>>>(b->dinst, b->dstate, idx, b->desc[idx].dt0, b->dints + W_ACTIVE);
  b->launches += 1;
  const mhd_batch_desc& d = b->desc[idx];
  bool dir = false;
  for (int s = 0; s < 4; s++) dir = dir || d.bc[s] == DIRICHLET;
  if (dir) {
    const BInst& in = b->hinst[idx];
    const int m = d.nx > d.ny ? d.nx : d.ny;
    k_snapshot<<<(NF * m + 255) / 256, 256, 0, b->stream>>>(
        in.g, in.U, const_cast<double*>(in.snap[0]), const_cast<double*>(in.snap[1]),
        const_cast<double*>(in.snap[2]), const_cast<double*>(in.snap[3]));
    b->launches += 1;
  }
  BK(cudaGetLastError());
  ensure_in_table(b, idx);
  BK(cudaStreamSynchronize(b->stream));
  return bset(b, MHD_OK, false, "");
}

}  // namespace

extern "C" {

int mhd_batch_create(int n, const mhd_batch_desc* runs, int device, mhd_batch** out) {
  if (!out) return MHD_ERR_WRONG_PARAMETER;
  *out = nullptr;
  if (n < 1 || !runs) return MHD_ERR_WRONG_PARAMETER;
  for (int r = 0; r < n; r++) {
    const mhd_batch_desc& d = runs[r];
    if (d.nx < 2 || d.ny < 2 || !(d.dx > 0) || !(d.dy > 0) || (d.scheme != 2 && d.scheme != 3) ||
        (d.time_method != 1 && d.time_method != 2))
      return MHD_ERR_WRONG_PARAMETER;
    for (int s = 0; s < 4; s++)
      if (d.bc[s] < 1 || d.bc[s] > 4) return MHD_ERR_WRONG_PARAMETER;
  }
  mhd_batch* b = new (std::nothrow) mhd_batch;
  if (!b) return MHD_ERR_WRONG_PARAMETER;
  b->device = device;
  b->n = n;
  b->desc.assign(runs, runs + n);
  b->in_table.assign(n, 0);
  *out = b;
  BK(cudaSetDevice(device));
  BK(cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, device));
  BK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  BK(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking));
  BK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
  BK(cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming));
  // pool layout per run: U, U1, U2, UL blocks, then aF, aG and the four edges
  std::vector<size_t> off(n);
  size_t total = 0;
  b->hinst.resize(n);
  for (int r = 0; r < n; r++) {
    const mhd_batch_desc& d = runs[r];
    Grid g{};
    g.nx = d.nx; g.ny = d.ny; g.NX = d.nx + 4; g.NY = d.ny + 4;
    g.pitch = pitch_for(g.NY);
    g.off = ROW_OFF;
    g.fstride = (long long)g.NX * g.pitch;
    g.dx = d.dx; g.dy = d.dy; g.gamma = d.gamma;
    for (int s = 0; s < 4; s++) g.bc[s] = d.bc[s];
    b->hinst[r].g = g;
    off[r] = total;
    const size_t blk = size_t(NF) * g.fstride + 16;
    const size_t aux = size_t(NF) * (g.NX + g.NY) * 3;  // alpha + edges
    total += ((4 * blk + aux + 31) / 32) * 32;
  }
  BK(cudaMalloc(&b->pool, total * sizeof(double)));
  BK(cudaMemsetAsync(b->pool, 0, total * sizeof(double), b->stream));
  for (int r = 0; r < n; r++) {
    const mhd_batch_desc& d = runs[r];
    BInst& in = b->hinst[r];
    const Grid& g = in.g;
    const size_t blk = size_t(NF) * g.fstride + 16;
    double* base = b->pool + off[r];
    in.U = base;
    in.U1 = base + blk;
    in.U2 = base + 2 * blk;
    in.UL = base + 3 * blk;
    double* aux = base + 4 * blk;
    in.aF = aux;
    in.aG = aux + size_t(NF) * g.NY;
    double* edges = aux + size_t(NF) * (g.NX + g.NY);
    in.snap[0] = edges;                               // left  [8][NY]
    in.snap[1] = edges + size_t(NF) * g.NY;           // right [8][NY]
    in.snap[2] = edges + size_t(NF) * 2 * g.NY;       // bottom [8][NX]
    in.snap[3] = edges + size_t(NF) * (2 * g.NY + g.NX);  // top [8][NX]
    in.sp = StepParams{d.dx, d.dy, d.dt_min, d.dt_max, d.cfl};
    in.G = Gas{d.gamma, d.gamma - 1.0, (d.gamma - 2.0) / (d.gamma - 1.0), 1.0 / std::sqrt(2.0)};
    in.inv_dx = 1.0 / d.dx;
    in.inv_dy = 1.0 / d.dy;
    in.t_end = d.t_end;
    in.scheme = d.scheme;
    in.time_method = d.time_method;
    in.max_steps = d.max_steps;
  }
  BK(cudaMalloc(&b->dinst, sizeof(BInst) * n));
  BK(cudaMemcpyAsync(b->dinst, b->hinst.data(), sizeof(BInst) * n, cudaMemcpyHostToDevice,
                     b->stream));
  BK(cudaMalloc(&b->dstate, sizeof(BState) * n));
  BK(cudaMemsetAsync(b->dstate, 0, sizeof(BState) * n, b->stream));
  BK(cudaMallocHost(&b->hstate, sizeof(BState) * n));
  std::memset(b->hstate, 0, sizeof(BState) * n);
  BK(cudaMalloc(&b->dints, W_COUNT * sizeof(int)));
  BK(cudaMemsetAsync(b->dints, 0, W_COUNT * sizeof(int), b->stream));
  BK(cudaMallocHost(&b->hints, W_COUNT * sizeof(int)));
  std::memset(b->hints, 0, W_COUNT * sizeof(int));
  int st = choose_grid(b);
  if (st) return st;
  BK(cudaStreamSynchronize(b->stream));
  return bset(b, MHD_OK, false, "");
}

int mhd_batch_destroy(mhd_batch* b) {
  if (!b) return MHD_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  free_graph(b);
  cudaFree(b->pool);
  cudaFree(b->dinst);
  cudaFree(b->dstate);
  cudaFree(b->dftab);
  cudaFree(b->datab);
  cudaFree(b->dints);
  if (b->hstate) cudaFreeHost(b->hstate);
  if (b->hints) cudaFreeHost(b->hints);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->join) cudaEventDestroy(b->join);
  if (b->side) cudaStreamDestroy(b->side);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return MHD_OK;
}

int mhd_batch_last_error(mhd_batch* b, char* buf, size_t len, int* is_error) {
  if (!b) return MHD_ERR_WRONG_PARAMETER;
  if (buf && len) {
    std::strncpy(buf, b->msg.c_str(), len - 1);
    buf[len - 1] = 0;
  }
  if (is_error) *is_error = b->is_error ? 1 : 0;
  return MHD_OK;
}

int mhd_batch_upload(mhd_batch* b, int idx, const double* U) {
  if (check_idx(b, idx) || !U) return MHD_ERR_WRONG_PARAMETER;
  BK(cudaSetDevice(b->device));
  const Grid& g = b->hinst[idx].g;
  BK(cudaMemcpy2DAsync(b->hinst[idx].U + g.off, g.pitch * sizeof(double), U, g.NY * sizeof(double),
                       g.NY * sizeof(double), size_t(NF) * g.NX, cudaMemcpyHostToDevice,
                       b->stream));
  return arm(b, idx);
}

int mhd_batch_download(mhd_batch* b, int idx, double* U) {
  if (check_idx(b, idx) || !U) return MHD_ERR_WRONG_PARAMETER;
  BK(cudaSetDevice(b->device));
  const Grid& g = b->hinst[idx].g;
  BK(cudaMemcpy2DAsync(U, g.NY * sizeof(double), b->hinst[idx].U + g.off, g.pitch * sizeof(double),
                       g.NY * sizeof(double), size_t(NF) * g.NX, cudaMemcpyDeviceToHost,
                       b->stream));
  BK(cudaStreamSynchronize(b->stream));
  return MHD_OK;
}

int mhd_batch_init_problem(mhd_batch* b, int idx, int kind, const double* p, int np) {
  if (check_idx(b, idx)) return MHD_ERR_WRONG_PARAMETER;
  BK(cudaSetDevice(b->device));
  ProblemArgs a{};
  std::string err;
  cudaError_t ce = cudaSuccess;
  const int st = problem_args(kind, p, np, b->desc[idx].gamma, b->stream, a, err, ce,
                              &b->hinst[idx].g);
  if (ce != cudaSuccess) return bfail(b, ce, "problem_args");
  if (st) return bset(b, st, true, err);
  if (kind == MHD_PROBLEM_WAVE) b->launches += 1;
  enqueue_problem(b->hinst[idx].g, b->hinst[idx].U, a, b->stream);
  b->launches += problem_launches(a);
  BK(cudaGetLastError());
  BK(release_problem(a, b->stream));
  return arm(b, idx);
}

int mhd_batch_advance(mhd_batch* b, int stages, int check_every, int* n_active) {
  MHD_TRACE("mhd_batch_advance");
  if (!b || stages < 0) return MHD_ERR_WRONG_PARAMETER;
  BK(cudaSetDevice(b->device));
  int st = refresh_tables(b);
  if (st) return st;
  if ((st = read_states(b))) return st;
  int left = stages;
  const int chunk = check_every > 0 ? check_every : stages;
  while (left > 0 && b->hints[W_ACTIVE] > 0) {
    int todo = std::min(left, chunk);
    left -= todo;
    // whole graph replays first, the remainder as plain launches
    const int gs = std::min(todo, kMaxStagesPerGraph);
    if (todo >= gs && gs > 1) {
      if (b->graph_stages != gs) {
        if ((st = capture_graph(b, gs))) return st;
      }
      while (todo >= gs) {
        BK(cudaGraphLaunch(b->graph, b->stream));
        b->launches += (long long)gs * launches_per_stage(b);
        todo -= gs;
      }
    }
    for (; todo > 0; todo--) enqueue_stage(b);
    BK(cudaGetLastError());
    if ((st = read_states(b))) return st;
    // runs that stopped leave the work tables
    bool changed = false;
    for (int r = 0; r < b->n; r++)
      if (b->in_table[r] && !b->hstate[r].active) {
        b->in_table[r] = 0;
        changed = true;
      }
    if (changed && (st = build_tables(b))) return st;
  }
  if (n_active) *n_active = b->hints[W_ACTIVE];
  return bset(b, MHD_OK, false, "");
}

int mhd_batch_get_state(mhd_batch* b, int idx, mhd_batch_state* out) {
  if (check_idx(b, idx) || !out) return MHD_ERR_WRONG_PARAMETER;
  const BState& s = b->hstate[idx];
  out->t = s.t;
  out->dt = s.c.dt;
  out->steps = s.steps;
  out->active = s.active;
  out->status = s.status;
  out->phase = s.phase;
  out->retries = s.retries;
  out->neg_pressure = (long long)s.c.neg_count;
  return MHD_OK;
}

int mhd_batch_set_tile(mhd_batch* b, int tile, int ctas_per_sm) {
  if (!b || tile < 0 || tile >= MHD_BATCH_TILE_COUNT) return MHD_ERR_WRONG_PARAMETER;
  BK(cudaSetDevice(b->device));
  free_graph(b);
  b->tile = tile;
  b->ctas_per_sm = ctas_per_sm;
  b->tables_dirty = true;  // the tile table depends on the tile rows
  return choose_grid(b);
}

int mhd_batch_tune(mhd_batch* b, int reps, int* tile, int* ctas_per_sm, double* best_ms) {
  if (!b) return MHD_ERR_WRONG_PARAMETER;
  if (reps < 1) reps = 1;
  BK(cudaSetDevice(b->device));
  BK(cudaStreamSynchronize(b->stream));
  // A candidate is timed on the boundary fill, alpha pass and both flux
  // launches of a stage.  These only rewrite ghosts, UL, the alpha arrays
  // and the controller maxima / counters; the controller blocks are saved
  // here and restored afterwards, so the runs continue exactly as before.
  BState* saved = nullptr;
  BK(cudaMalloc(&saved, sizeof(BState) * b->n));
  BK(cudaMemcpyAsync(saved, b->dstate, sizeof(BState) * b->n, cudaMemcpyDeviceToDevice, b->stream));
  cudaEvent_t e0, e1;
  BK(cudaEventCreate(&e0));
  BK(cudaEventCreate(&e1));
  double best = 1e300;
  int best_tile = b->tile, best_per = b->ctas_per_sm;
  int st = MHD_OK;
  for (int t = 0; t < MHD_BATCH_TILE_COUNT && !st; t++) {
    for (int per = 0; per < 2 && !st; per++) {
      b->tile = t;
      b->ctas_per_sm = per;  // 0: occupancy limit, 1: one CTA per SM
      st = choose_grid(b);
      if (!st) st = build_tables(b);
      if (st) break;
      const TileShape& s = tile_shape(t);
      int* d = b->dints;
      for (int r = 0; r <= reps; r++) {  // r = 0 warms up
        if (r == 1) cudaEventRecord(e0, b->stream);
        kb_bc<<<dim3(16, b->n), 256, 0, b->stream>>>(b->dinst, b->dstate, d + W_NEXT_ROE);
        if (b->any_lf)
          kb_alpha<<<alpha_blocks(b), 256, 0, b->stream>>>(b->dinst, b->dstate, b->datab, d + W_ALPHA);
        enqueue_flux(b, s);
        b->launches += b->any_lf ? 2 : 1;
      }
      cudaEventRecord(e1, b->stream);
      cudaError_t e = cudaEventSynchronize(e1);
      if (e == cudaSuccess) e = cudaGetLastError();
      if (e != cudaSuccess) { st = bfail(b, e, "mhd_batch_tune"); break; }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      const double per_stage = double(ms) / reps;
      if (per_stage < best) {
        best = per_stage;
        best_tile = t;
        best_per = per;
      }
      if (per == 0 && b->grid_flux[0] <= b->nsm && b->grid_flux[1] <= b->nsm) break;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaMemcpyAsync(b->dstate, saved, sizeof(BState) * b->n, cudaMemcpyDeviceToDevice, b->stream);
  cudaError_t e = cudaStreamSynchronize(b->stream);
  cudaFree(saved);
  if (st) return st;
  if (e != cudaSuccess) return bfail(b, e, "mhd_batch_tune");
  if ((st = mhd_batch_set_tile(b, best_tile, best_per))) return st;
  if ((st = refresh_tables(b))) return st;
  if (tile) *tile = best_tile;
  if (ctas_per_sm) *ctas_per_sm = b->grid_flux[0] / b->nsm;
  if (best_ms) *best_ms = best;
  return bset(b, MHD_OK, false, "");
}

int mhd_batch_stream(mhd_batch* b, void** stream) {
  if (!b || !stream) return MHD_ERR_WRONG_PARAMETER;
  *stream = b->stream;
  return MHD_OK;
}

int mhd_batch_launches(mhd_batch* b, long long* launches) {
  if (!b || !launches) return MHD_ERR_WRONG_PARAMETER;
  *launches = b->launches;
  return MHD_OK;
}

}  // extern "C"
