// tma_ring.cuh -- TMA plane staging for k-marching stencil kernels on sm_100a.
//
// A block owns a (TX x TY) tile of (i,j) columns and marches along k.  For each
// k it needs planes k-1, k, k+1 of every input field (with a one-cell halo in
// i and j); one elected thread streams whole halo planes of all fields into a
// ring of shared-memory slots with cp.async.bulk.tensor (3-D tiled TMA) a few
// planes ahead of use, each slot completing on its own mbarrier.  Every wait is
// bounded: on expiry the kernel records an error word and returns.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace tma {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// true when the phase with the given parity has completed
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait: returns false after `limit` unsuccessful polls
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit = (1u << 24)) {
  for (uint32_t it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 3-D tiled bulk tensor load of one box into shared memory, completing on bar
__device__ __forceinline__ void load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace tma

// Host: encode a 3-D tiled tensor map over an (nx,ny,nz) Fortran array of
// `esize`-byte elements with a (bx,by,1) box.  Returns 0 on success.
int make_tensor_map_3d(CUtensorMap *map, const void *base, int nx, int ny, int nz, int bx, int by, int esize);
