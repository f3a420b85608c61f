// Tensor-memory-accelerator (TMA) tile loads for the stencil kernels: 2D
// tensor maps over this GPU's own field planes, one elected thread issuing
// cp.async.bulk.tensor loads that complete on a shared-memory mbarrier, and
// a time-bounded wait on that barrier.  No multicast: every CTA loads its
// own tile.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include "internal.cuh"

namespace cup2d {

// A 2D tensor map over a row-major ny x nx plane of doubles, copied in
// boxes of boxY rows x boxX columns (boxX * 8 a multiple of 16 bytes);
// out-of-range elements of a box read as zero.
inline cudaError_t make_tmap_f64(CUtensorMap* map, const double* base, int nx, int ny, int boxX, int boxY) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)ny};
  const cuuint64_t strides[1] = {(cuuint64_t)nx * sizeof(double)};
  const cuuint32_t box[2] = {(cuuint32_t)boxX, (cuuint32_t)boxY};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dims, strides,
                            box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one arrival that also announces `bytes` of asynchronous transactions
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// box of the tensor map starting at column x (x * 8 a multiple of 16 bytes),
// row y (any value: rows outside the plane read as zero) into dst
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      :: "r"(smem_u32(dst)), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y),
         "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long timer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the barrier's phase `parity` to complete, for at most limitNs
// nanoseconds of %globaltimer; false if it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned long long limitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = timer_ns();
  while (!mbar_try_wait(bar, parity))
    if (timer_ns() - t0 > limitNs) return false;
  return true;
}

// The wait limit of the pipeline's TMA loads: a tile arrives in
// microseconds; a second means the copy will not complete.
constexpr unsigned long long TMA_WAIT_NS = 1000000000ull;

// advDiff's staged tile: the 32x32 block with a two-cell halo each side (the
// fused divergence needs the new velocity one cell beyond the block, whose
// stencil reaches one further); its left edge, column 32 bx - 2, starts on
// a 16-byte boundary
constexpr int ADV_HT = BS + 4;

} // namespace cup2d
