// bhr_device.cuh -- device helpers shared by the kernel translation units:
// the reference's constants, PTX wrappers (mbarrier, TMA, bulk groups,
// programmatic dependent launch), the 6th-order stencils, the
// Newton-refined reciprocal and square root, and the work-item lookup of
// batch launch groups.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <utility>

#include "bhr_internal.h"

namespace bhr {
namespace {

constexpr double kThird = 0.33333333333333333;   // HighOrder/kern.cu:46
constexpr double kPie = 3.141592653589793;       // HighOrder/kern.cu:1188
constexpr long long kMaxWaitIters = 1LL << 22;   // bounded mbarrier wait

// ---- PTX helpers ---------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t phase) {
  for (long long i = 0; i < kMaxWaitIters; i++)
    if (mbar_try_wait(bar, phase)) return true;
  return false;
}
// Programmatic dependent launch: wait for the kernels this one depends on
// (their writes become visible), and let the next kernel start launching.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// 3D tiled TMA load, no multicast.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// 3D tiled prefetch of a box into L2 (no shared-memory destination, no completion).
__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap *map, int x, int y, int z) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(z)
               : "memory");
}

// 3D tiled TMA store from shared memory, tracked by this thread's bulk group.
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *src, int x, int y, int z) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// The bulk stores of this thread have finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// The bulk stores of this thread are complete.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void named_barrier_sync(int id, int threads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// ---- stencils (HighOrder/kern.cu:192-261) ---------------------------------
__device__ __forceinline__ double d1c(const double *v, int c) {
  return 45.0 * (v[c + 1] - v[c - 1]) - 9.0 * (v[c + 2] - v[c - 2]) + (v[c + 3] - v[c - 3]);
}
__device__ __forceinline__ double ko8c(const double *v, int c) {
  return (v[c + 4] + v[c - 4]) - 8.0 * (v[c + 3] + v[c - 3]) + 28.0 * (v[c + 2] + v[c - 2]) -
         56.0 * (v[c + 1] + v[c - 1]) + 70.0 * v[c];
}

// Reciprocal by Newton-Raphson iteration y <- y (2 - x y) from the hardware
// approximation (two steps take its ~2^-22 relative error below 1 ulp).
__device__ __forceinline__ double rcp_nr(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// Square root of x >= 0: Newton-Raphson for 1/sqrt(x), y <- y (3/2 - x y^2 / 2),
// from the hardware approximation, then one correction of s = x y by the
// residual x - s^2.
__device__ __forceinline__ double sqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  y = y * fma(-0.5 * x * y, y, 1.5);
  y = y * fma(-0.5 * x * y, y, 1.5);
  double s = x * y;
  s = fma(fma(-s, s, x), 0.5 * y, s);
  return x > 0.0 ? s : 0.0;
}

// 1/bir = 1/(B0 + B1 sin^2 theta) (HighOrder/kern.cu:132-149).
__device__ __forceinline__ double inv_bir(double b0, double b1, double s2) { return rcp_nr(fma(b1, s2, b0)); }

// Work item t of a launch group: the index of its solve in the group and
// the tile corner (tiles of `rows` rows).  Every value read comes from the
// kernel's parameter space and depends on t alone, so all of a block's
// threads compute the same result.
template <class Args>
__device__ __forceinline__ int group_item(const WorkGroup<Args> &G, const int t, const int rows, int &c0, int &b0) {
  int lo = 0, hi = G.nsolves - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (G.first[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  const int k = t - G.first[lo], nx = G.tiles_x[lo];
  c0 = (k % nx) * TC;
  b0 = (k / nx) * rows;
  return lo;
}

// Launch with programmatic stream serialisation allowed (pdl): the kernel
// may begin while its predecessor on the stream drains, and holds every
// read of the predecessor's results behind grid_dependency_wait().  Without
// it the launch waits for the predecessor to complete, as a plain launch.
template <class... KArgs, class... Args>
static cudaError_t launch_ex(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                             cudaStream_t st, Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}
template <class... KArgs, class... Args>
static cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args &&...args) {
  return launch_ex(true, kernel, grid, block, smem, st, std::forward<Args>(args)...);
}

}  // namespace
}  // namespace bhr
