// mhd_divb_calc_noalloc: the div B diagnostic (divBCalculation,
// div_b_fix.cpp:4-126) for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: plug-ins living inside a host
// application that owns all device memory through its own pool, and
// runtimes that forbid allocation once they are running (cudaMalloc can
// synchronise the device and stall every other stream, which a solver
// stepping in a time-critical loop cannot afford).  This entry point works on buffers the caller already
// owns (the state and a 2-double result) and keeps its own scratch - one
// partial maximum and one partial sum per grid row - in the file-scope
// device array below, which every GPU that loads the library holds until
// the process exits.
//
// Limits and sharing: at most MHD_NOALLOC_MAX_ROWS interior rows (nx);
// larger grids are rejected.  All calls share the array, so calls whose
// work overlaps on the GPU (other streams, other threads) race; serialise
// them.  Nothing in the array has to start at zero: every call writes each
// row slot it later reads.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/mhd2d_b200.h"

#define MHD_NOALLOC_MAX_ROWS 16384
#define MHD_NOALLOC_MAX_DEVICES 64

namespace {

// [0, MAX_ROWS): per-row max |div B|; [MAX_ROWS, 2*MAX_ROWS): per-row sums.
static __device__ __align__(256) double g_divb_scratch[2 * MHD_NOALLOC_MAX_ROWS];

double* g_scratch_addr[MHD_NOALLOC_MAX_DEVICES] = {};
std::mutex g_scratch_mu;

struct Layout {
  long long fstride;  // NX * pitch
  int pitch, off;
  __device__ long long at(int k, int i, int j) const {
    return (long long)k * fstride + (long long)i * pitch + off + j;
  }
};

// Periodic wrap of the Bx, By ghost layers (div_b_fix.cpp:19-101).
__global__ void k_na_wrap(double* __restrict__ U, Layout L, int nx, int ny, int4 bc) {
  const int m = nx > ny ? nx : ny;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 4 * m; e += gridDim.x * blockDim.x) {
    const int k = 4 + (e / m) % 2, which = e / (2 * m), p = 2 + e % m;
    if (which == 0 && p < ny + 2) {
      if (bc.x == 1) {
        U[L.at(k, 0, p)] = U[L.at(k, nx, p)];
        U[L.at(k, 1, p)] = U[L.at(k, nx + 1, p)];
      }
      if (bc.y == 1) {
        U[L.at(k, nx + 2, p)] = U[L.at(k, 2, p)];
        U[L.at(k, nx + 3, p)] = U[L.at(k, 3, p)];
      }
    }
    if (which == 1 && p < nx + 2) {
      if (bc.z == 1) {
        U[L.at(k, p, 0)] = U[L.at(k, p, ny)];
        U[L.at(k, p, 1)] = U[L.at(k, p, ny + 1)];
      }
      if (bc.w == 1) {
        U[L.at(k, p, ny + 2)] = U[L.at(k, p, 2)];
        U[L.at(k, p, ny + 3)] = U[L.at(k, p, 3)];
      }
    }
  }
}

__device__ __forceinline__ double na_max(double m, double x) { return x > m ? x : m; }

// One block per row i of [x0, x1): row maximum and row sum of |div B| over
// [y0, y1) into the scratch array.
__global__ void __launch_bounds__(256) k_na_rows(const double* __restrict__ U, Layout L, int x0,
                                                 int y0, int y1, double d2x, double d2y,
                                                 double* scratch) {
  const int i = x0 + blockIdx.x;
  double mx = 0.0, sum = 0.0;
  for (int j = y0 + threadIdx.x; j < y1; j += blockDim.x) {
    const double d = fabs((U[L.at(4, i + 1, j)] - U[L.at(4, i - 1, j)]) / d2x +
                          (U[L.at(5, i, j + 1)] - U[L.at(5, i, j - 1)]) / d2y);
    mx = na_max(mx, d);
    sum += d;
  }
  __shared__ double s_max[8], s_sum[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = na_max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
  }
  if ((threadIdx.x & 31) == 0) {
    s_max[threadIdx.x >> 5] = mx;
    s_sum[threadIdx.x >> 5] = sum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0, s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      m = na_max(m, s_max[w]);
      s += s_sum[w];
    }
    scratch[blockIdx.x] = m;
    scratch[MHD_NOALLOC_MAX_ROWS + blockIdx.x] = s;
  }
}

// Rows combined in row order; result[0] = max, result[1] = sum * dx * dy.
__global__ void k_na_finish(const double* scratch, int rows, double dxdy, double* result) {
  __shared__ double s_max[256], s_sum[256];
  double m = 0.0, s = 0.0;
  // contiguous chunk per thread, chunks summed in thread order below
  const int per = (rows + blockDim.x - 1) / blockDim.x;
  const int r0 = threadIdx.x * per, r1 = min(rows, r0 + per);
  for (int r = r0; r < r1; r++) {
    m = na_max(m, scratch[r]);
    s += scratch[MHD_NOALLOC_MAX_ROWS + r];
  }
  s_max[threadIdx.x] = m;
  s_sum[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = 0.0, ss = 0.0;
    for (int t = 0; t < (int)blockDim.x; t++) {
      mm = na_max(mm, s_max[t]);
      ss += s_sum[t];
    }
    result[0] = mm;
    result[1] = ss * dxdy;
  }
}

// Device address of the scratch array for `device` (the current device).
// Host code must not pass g_divb_scratch itself to a kernel: on the host it
// names a stand-in, not device memory.
cudaError_t scratch_address(int device, double** out) {
  if (device < 0 || device >= MHD_NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_divb_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

}  // namespace

extern "C" int mhd_divb_calc_noalloc(double* U, int nx, int ny, int pitch, int row_offset,
                                     double dx, double dy, const int bc[4], double* result,
                                     void* stream) {
  if (!U || !result || !bc || nx < 2 || ny < 2 || pitch < ny + 4 + row_offset || row_offset < 0 ||
      !(dx > 0) || !(dy > 0))
    return MHD_ERR_WRONG_PARAMETER;
  if (nx > MHD_NOALLOC_MAX_ROWS) return MHD_ERR_WRONG_PARAMETER;  // scratch holds one slot per row
  for (int s = 0; s < 4; s++)
    if (bc[s] < 1 || bc[s] > 4) return MHD_ERR_WRONG_PARAMETER;
  // An error left pending by the caller's earlier work is not ours to
  // report or to clear: leave it in place and launch nothing.
  if (cudaPeekAtLastError() != cudaSuccess) return MHD_ERR_CUDA;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return MHD_ERR_CUDA;
  double* scratch = nullptr;
  if (scratch_address(device, &scratch) != cudaSuccess) return MHD_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Layout L{(long long)(nx + 4) * pitch, pitch, row_offset};
  const int4 b = make_int4(bc[0], bc[1], bc[2], bc[3]);
  const int m = nx > ny ? nx : ny;
  k_na_wrap<<<(4 * m + 255) / 256, 256, 0, s>>>(U, L, nx, ny, b);
  // one cell in from every non-periodic side (div_b_fix.cpp:17-101)
  const int x0 = bc[0] == 1 ? 2 : 3, x1 = bc[1] == 1 ? nx + 2 : nx + 1;
  const int y0 = bc[2] == 1 ? 2 : 3, y1 = bc[3] == 1 ? ny + 2 : ny + 1;
  // nx = 2 with both x sides non-periodic leaves no row: max and sum are 0
  // (k_na_finish reads no slot then), as divBCalculation's empty loops give
  const int rows = x1 > x0 ? x1 - x0 : 0;
  if (rows > 0) k_na_rows<<<rows, 256, 0, s>>>(U, L, x0, y0, y1, 2.0 * dx, 2.0 * dy, scratch);
  k_na_finish<<<1, 256, 0, s>>>(scratch, rows, dx * dy, result);
  // nothing was pending on entry, so an error here is one of these launches
  return cudaGetLastError() == cudaSuccess ? MHD_OK : MHD_ERR_CUDA;
}
