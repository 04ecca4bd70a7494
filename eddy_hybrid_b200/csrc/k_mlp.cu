// k_mlp.cu -- learned eddy-viscosity closure on the 5th-generation tensor
// cores: a per-cell MLP 12 -> 64 -> 64 -> 64 -> 2 (SiLU, softplus outputs),
// BF16 operands, FP32 accumulation in TMEM (tcgen05.mma kind::f16).
//
//  * k_umma_gemm      : D[M x N] (+)= A[M x K] * B[N x K]^T, BF16 in, FP32 out;
//                       the training GEMMs (forward, input gradient, weight
//                       gradient) all map onto it.
//  * k_mlp_infer      : fused per-cell inference: features of a 128-cell tile
//                       -> four MMA layers with bias/SiLU epilogues from TMEM
//                       -> nu_t, kappa_t.
// The closure stands in for the dynamic procedure's test filtering and
// coefficient averaging (src/vt.f:172-431).
#include <cuda_bf16.h>

#include <cmath>
#include <vector>

#include "eddy_internal.h"
#include "umma.cuh"

namespace {

constexpr int GT = 128;  // threads per GEMM CTA (4 warps, one TMEM lane quadrant each)
constexpr int GKC = 64;  // K chunk per smem stage

// D[M x N] = A[M x K] B[N x K]^T (+ D if acc).  A, B row-major bf16 with K
// contiguous; D row-major f32.  M multiple of 128, N multiple of 16 (<= 256),
// K multiple of 16.  Rows of A beyond M read as zero.
__global__ void __launch_bounds__(GT)
    k_umma_gemm(int M, int N, int K, const __nv_bfloat16 *__restrict__ A, const __nv_bfloat16 *__restrict__ B,
                float *__restrict__ D, int acc, int *err) {
  extern __shared__ __align__(1024) unsigned char sm_[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  unsigned char *sa = sm_;                       // 128 x GKC bf16 = 16 KB
  unsigned char *sb = sm_ + 128 * GKC * 2;       // N x GKC bf16
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.x * 128;
  uint32_t ncols = 32;
  while ((int)ncols < N) ncols <<= 1;
  if (warp == 0) {
    umma::tmem_alloc(&tmem_base, ncols);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    umma::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tm = tmem_base;
  const uint32_t idesc = umma::make_idesc_bf16(128, N);
  bool ok = true;
  int phase = 0;
  for (int k0 = 0; k0 < K; k0 += GKC) {
    int kc = min(GKC, K - k0);
    // stage A (128 x kc) and B (N x kc) into the canonical K-major layout
    for (int e = tid; e < 128 * (kc / 8); e += GT) {
      int r = e / (kc / 8), c8 = (e % (kc / 8)) * 8;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (m0 + r < M) v = *reinterpret_cast<const uint4 *>(A + (size_t)(m0 + r) * K + k0 + c8);
      *reinterpret_cast<uint4 *>(sa + umma::kmajor_offset(r, c8, kc)) = v;
    }
    for (int e = tid; e < N * (kc / 8); e += GT) {
      int r = e / (kc / 8), c8 = (e % (kc / 8)) * 8;
      uint4 v = *reinterpret_cast<const uint4 *>(B + (size_t)r * K + k0 + c8);
      *reinterpret_cast<uint4 *>(sb + umma::kmajor_offset(r, c8, kc)) = v;
    }
    umma::fence_smem_to_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (tid == 0) {
      for (int ks = 0; ks < kc; ks += 16) {
        // K step of 16 = two core matrices along K: byte offset 2 * LBO
        uint64_t ad = umma::make_desc(sa + (ks / 8) * 128, 128, 128 * (kc / 8));
        uint64_t bd = umma::make_desc(sb + (ks / 8) * 128, 128, 128 * (kc / 8));
        umma::mma_bf16(tm, ad, bd, idesc, (k0 > 0 || ks > 0) ? 1u : 0u);
      }
      umma::commit(&bar);
    }
    ok = ok && umma::mbar_wait(&bar, phase);
    phase ^= 1;
    umma::fence_after_sync();
    __syncthreads();
  }
  if (!ok && tid == 0) atomicExch(err, 1);
  // epilogue: warp w owns rows 32w..32w+31 (TMEM lanes), 16 columns per load
  int row = m0 + warp * 32 + (tid & 31);
  for (int c0 = 0; c0 < N; c0 += 16) {
    float v[16];
    umma::tmem_ld16(tm + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
    if (ok && row < M) {
      float *dst = D + (size_t)row * N + c0;
#pragma unroll
      for (int q = 0; q < 16; q++) dst[q] = acc ? dst[q] + v[q] : v[q];
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tm, ncols);
}

}  // namespace

// host launcher for the generic GEMM; A, B, D device pointers
int launch_umma_gemm(eddy_ctx *ctx, int M, int N, int K, const void *A, const void *B, float *D, int acc) {
  if (M % 128 || N % 16 || N < 16 || N > 256 || K % 16 || K < 16) {
    ctx->err = "umma gemm: M%128, N%16 (16..256), K%16 required";
    return EDDY_EINVAL;
  }
  size_t smem = (size_t)(128 + N) * GKC * 2 + 1024;
  EDDY_CUDA(cudaFuncSetAttribute(k_umma_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_umma_gemm<<<M / 128, GT, smem, ctx->stream>>>(M, N, K, static_cast<const __nv_bfloat16 *>(A),
                                                  static_cast<const __nv_bfloat16 *>(B), D, acc, ctx->err_flag);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

extern "C" int eddy_umma_gemm_bf16(eddy_ctx *ctx, int M, int N, int K, const uint16_t *A, const uint16_t *B,
                                   float *D, int acc) {
  if (!ctx || !A || !B || !D) return EDDY_EINVAL;
  size_t ba = sizeof(uint16_t) * (size_t)M * K, bb = sizeof(uint16_t) * (size_t)N * K,
         bd = sizeof(float) * (size_t)M * N;
  void *dA = nullptr, *dB = nullptr;
  float *dD = nullptr;
  EDDY_CUDA(cudaMalloc(&dA, ba));
  EDDY_CUDA(cudaMalloc(&dB, bb));
  EDDY_CUDA(cudaMalloc(&dD, bd));
  EDDY_CUDA(cudaMemcpyAsync(dA, A, ba, cudaMemcpyHostToDevice, ctx->stream));
  EDDY_CUDA(cudaMemcpyAsync(dB, B, bb, cudaMemcpyHostToDevice, ctx->stream));
  EDDY_CUDA(cudaMemcpyAsync(dD, D, bd, cudaMemcpyHostToDevice, ctx->stream));
  int rc = launch_umma_gemm(ctx, M, N, K, dA, dB, dD, acc);
  if (rc == EDDY_OK) {
    EDDY_CUDA(cudaMemcpyAsync(D, dD, bd, cudaMemcpyDeviceToHost, ctx->stream));
    EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dD);
  return rc;
}
