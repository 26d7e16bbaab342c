// Tensor-memory-accelerator (TMA) staging of a flux tile's state box.
//
// The box of a TI x TJ tile is the (TI+4) x (TJ+4) x 8 block of the pitched
// state around it (rows i0-2 .., columns j0-2 .., all 8 fields).  A 3-D
// tensor map describes the state block: x = row offset + j (contiguous),
// y = i (stride pitch), z = field (stride fstride).  One thread issues the
// box copy (cp.async.bulk.tensor, no multicast) against an mbarrier; every
// thread waits on the barrier with an iteration limit.  Elements past the
// grid (x >= off + NY or y >= NX) arrive as zeros, as the cp.async staging
// writes them.
//
// Alignment: the box's first x is off + j0 - 2 = 14 + TJ * tj, a multiple of
// 2 doubles (16 bytes); its width (TJ+4) * 8 bytes and both strides are
// multiples of 16 bytes; the shared destination is rounded up to a 128-byte
// boundary inside the kernel's dynamic shared memory.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include "mhd_common.cuh"

namespace mhd {

// Ctl::error code of a tile copy that did not complete within the limit.
constexpr int kErrTileCopyTimeout = 11;
// try_wait rounds before a tile copy is given up (each round may suspend the
// thread for a hardware-defined interval; this is seconds, far beyond a copy)
constexpr unsigned kTmaWaitLimit = 1u << 24;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// true once the barrier's phase `parity` has completed
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for phase `parity`; false if the limit was reached.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  for (unsigned it = 0; it < kTmaWaitLimit; it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// One 3-D box copy global -> shared, completing `bar` with its byte count.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y,
                                            int z, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z),
      "r"(smem_addr(bar))
      : "memory");
}

// Host: whether flux tiles are staged by TMA (process-wide; mhd_set_tile_tma).
inline bool& tile_tma_flag() {
  static bool on = true;
  return on;
}
inline bool tile_tma_enabled() { return tile_tma_flag(); }
// Host: flux launches whose tiles were staged by TMA (process-wide count).
inline long long& tile_tma_launches() {
  static long long n = 0;
  return n;
}

// Host: the tensor map of state block U for boxes of cu x ru x 8 doubles.
// Returns false if the driver entry point or the encoding is unavailable.
inline bool make_box_map(const Grid& g, const double* U, int cu, int ru, CUtensorMap* out) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  static bool looked = false;
  if (!looked) {
    looked = true;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    else
      cudaGetLastError();
  }
  if (!encode) return false;
  const cuuint64_t dims[3] = {cuuint64_t(g.off + g.NY), cuuint64_t(g.NX), cuuint64_t(NF)};
  const cuuint64_t strides[2] = {cuuint64_t(g.pitch) * sizeof(double),
                                 cuuint64_t(g.fstride) * sizeof(double)};
  const cuuint32_t box[3] = {cuuint32_t(cu), cuuint32_t(ru), cuuint32_t(NF)};
  const cuuint32_t estr[3] = {1, 1, 1};
  return encode(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(U), dims, strides,
                box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace mhd
