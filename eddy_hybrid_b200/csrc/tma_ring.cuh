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

// bounded wait: returns false after `limit` unsuccessful polls or 2 s of
// wall time (the global timer, read every 256 polls), whichever comes first,
// so a wait that cannot complete ends in bounded time whatever the length of
// one suspended poll
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit = (1u << 24)) {
  if (mbar_try_wait(bar, parity)) return true;
  uint64_t t0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (uint32_t it = 1; it < limit; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 0) {
      uint64_t t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      if (t - t0 > 2000000000ull) return false;
    }
  }
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
// `esize`-byte elements with row pitch `pitch` elements and a (bx,by,1) box.
// Returns 0 on success.
int make_tensor_map_3d(CUtensorMap *map, const void *base, int nx, int ny, int nz, int bx, int by, int esize,
                       int pitch = 0);
// 2-D FP32 (w, h) row-major array (row stride w elements) with a (bx, by)
// box; swizzle32: 32-byte swizzle (bx * 4 must then be 32)
int make_tensor_map_2d(CUtensorMap *map, const void *base, long long w, long long h, int bx, int by,
                       int swizzle32 = 0);

// ---------------------------------------------------------------------------
// Generic k-marching driver over a 4-slot ring of halo planes of NF fields.
// Block = TX x TY threads, tile = TX x TY (i,j) columns starting at the
// interior origin (ix1, jy1) + block offset; k runs over a chunk of KC planes.
// body(i, j, k, active, acc) is called once per plane per thread after planes
// k-1, k, k+1 are resident; acc.at(f, di, dj, dk) reads field f at the offset.
template <int NF>
struct alignas(64) TmaMaps {
  CUtensorMap m[NF];
};

template <int TX, int TY, class T = double>
struct RingGeom {
  // box rows must span a multiple of 16 bytes: TX + 2 halo columns rounded up
  static constexpr int PX = (((TX + 2) * (int)sizeof(T) + 15) / 16) * 16 / (int)sizeof(T), PY = TY + 2;
  static constexpr int EPL = 128 / (int)sizeof(T);                 // elements per 128 bytes
  static constexpr int PLANE = ((PX * PY + EPL - 1) / EPL) * EPL;  // elements, 128-byte multiple
  static constexpr unsigned BOX_BYTES = PX * PY * sizeof(T);
};

template <int TX, int TY, int NF, class T = double>
struct RingAcc {
  using G = RingGeom<TX, TY, T>;
  const T *sm;
  int s0, s1, s2, c;
  __device__ __forceinline__ T at(int f, int di, int dj, int dk) const {
    int so = dk < 0 ? s0 : (dk == 0 ? s1 : s2);
    return sm[so + f * G::PLANE + c + dj * G::PX + di];
  }
};

template <int NF, int TX, int TY, class T = double>
constexpr size_t ring_smem_bytes() {
  return (size_t)4 * NF * RingGeom<TX, TY, T>::PLANE * sizeof(T) + 128;
}

template <int NF, int TX, int TY, int KC, class T = double, class Body>
__device__ __forceinline__ void tma_march(int ix1, int ix2, int jy1, int jy2, int kz1, int kz2,
                                          const TmaMaps<NF> &maps, int *err, Body &&body) {
  using G = RingGeom<TX, TY, T>;
  constexpr int NSLOT = 4, SLOT = NF * G::PLANE;
  extern __shared__ unsigned char smraw_[];
  __shared__ __align__(8) uint64_t bar[NSLOT];
  // 128-byte aligned ring start, as an offset into the shared array (pointer
  // arithmetic on it keeps the shared address space visible to the compiler)
  const unsigned align_off = (128u - (unsigned)(reinterpret_cast<uintptr_t>(smraw_) & 127u)) & 127u;
  T *sm = reinterpret_cast<T *>(smraw_ + align_off);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = ix1 + blockIdx.x * TX, j0 = jy1 + blockIdx.y * TY;
  const int k0 = kz1 + blockIdx.z * KC;
  const int k1 = min(k0 + KC, kz2 + 1);
  const int pfirst = k0 - 1, plast = k1;
  const int bx = i0 - 2, by = j0 - 2;
  if (tid == 0) {
    for (int q = 0; q < NSLOT; q++) tma::mbar_init(&bar[q], 1);
    tma::fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int p) {
    int u = p - pfirst, sl = u & (NSLOT - 1);
    tma::mbar_expect_tx(&bar[sl], NF * G::BOX_BYTES);
    for (int f = 0; f < NF; f++) tma::load_3d(sm + sl * SLOT + f * G::PLANE, &maps.m[f], bx, by, p - 1, &bar[sl]);
  };
  if (tid == 0)
    for (int p = pfirst; p <= min(pfirst + NSLOT - 1, plast); p++) issue(p);
  const int i = i0 + tx, j = j0 + ty;
  const bool active = (i <= ix2 && j <= jy2);
  const int c = (ty + 1) * G::PX + (tx + 1);
  for (int k = k0; k < k1; k++) {
    // planes k-1 and k were waited for in earlier iterations
    bool ok = true;
    for (int p = k == k0 ? k - 1 : k + 1; p <= k + 1; p++) {
      int u = p - pfirst;
      ok = ok && tma::mbar_wait(&bar[u & (NSLOT - 1)], (u >> 2) & 1);
    }
    if (ok) {
      RingAcc<TX, TY, NF, T> S{sm, ((k - 1 - pfirst) & 3) * SLOT, ((k - pfirst) & 3) * SLOT,
                               ((k + 1 - pfirst) & 3) * SLOT, c};
      body(i, j, k, active, S);
    }
    int failed = __syncthreads_or(ok ? 0 : 1);
    if (failed) {
      if (tid == 0) {
        atomicExch(err, 1);
        for (int p = k + 2; p <= min(k + NSLOT - 1, plast); p++) {
          int u = p - pfirst;
          tma::mbar_wait(&bar[u & (NSLOT - 1)], (u >> 2) & 1, 1u << 20);
        }
      }
      return;
    }
    if (tid == 0 && k + NSLOT - 1 <= plast) {
      tma::fence_proxy_async();
      issue(k + NSLOT - 1);
    }
  }
}
