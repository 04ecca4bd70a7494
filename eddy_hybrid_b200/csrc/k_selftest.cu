// k_selftest.cu -- check, on the GPU, that a barrier wait which can never
// complete ends: one thread waits on an mbarrier that expects one arrival
// nobody makes, through the same bounded wait every kernel of the library
// uses, and reports whether the wait gave up and after how long (global
// timer).  No counterpart in the reference.
#include <cstdint>

#include "eddy_internal.h"
#include "umma.cuh"

namespace {

__global__ void k_wait_nobody(unsigned long long *out) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    umma::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    unsigned long long t0, t1;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    const bool done = umma::mbar_wait(&bar, 0);
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
    out[0] = done ? 0ull : 1ull;
    out[1] = t1 - t0;
  }
}

}  // namespace

extern "C" int eddy_selftest_wait_bound(int device, int *gave_up, double *seconds) {
  if (!gave_up || !seconds) return EDDY_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return EDDY_ECUDA;
  unsigned long long *d = nullptr, h[2] = {0, 0};
  if (cudaMalloc(&d, sizeof(h)) != cudaSuccess) return EDDY_ECUDA;
  k_wait_nobody<<<1, 32>>>(d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return EDDY_ECUDA;
  *gave_up = (int)h[0];
  *seconds = 1e-9 * (double)h[1];
  return EDDY_OK;
}
