// k_mlp.cu -- learned eddy-viscosity closure on the 5th-generation tensor
// cores: a per-cell MLP 12 -> 64 -> 64 -> 64 -> 2 (hard-swish hidden
// activations, softplus outputs),
// BF16 operands, FP32 accumulation in TMEM (tcgen05.mma kind::f16).
//
//  * k_umma_gemm      : D[M x N] (+)= A[M x K] * B[N x K]^T, BF16 in, FP32 out;
//                       the training GEMMs (forward, input gradient, weight
//                       gradient) all map onto it.
//  * k_mlp_infer      : fused per-cell inference: features of a 128-cell tile
//                       -> three MMA layers with bias/activation epilogues from TMEM
//                       -> the 64 -> 2 output layer on the CUDA cores
//                       -> coefficients C_nu, C_kappa -> nu_t = C_nu Delta^2 |S|,
//                       kappa_t = C_kappa Delta^2 |S|.
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
                float *__restrict__ D, int acc, int kper, int *err) {
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
  const int kbeg = blockIdx.y * kper, kend = min(K, kbeg + kper);
  for (int k0 = kbeg; k0 < kend; k0 += GKC) {
    int kc = min(GKC, kend - k0);
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
        umma::mma_bf16(tm, ad, bd, idesc, (k0 > kbeg || ks > 0) ? 1u : 0u);
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
      if (gridDim.y > 1) {
#pragma unroll
        for (int q = 0; q < 16; q++) atomicAdd(dst + q, v[q]);
      } else {
#pragma unroll
        for (int q = 0; q < 16; q++) dst[q] = acc ? dst[q] + v[q] : v[q];
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tm, ncols);
}

}  // namespace

// host launcher for the generic GEMM; A, B, D device pointers
// splitk > 1: K is split over that many CTAs whose partial products are
// atomically added into D (which then always accumulates).
int launch_umma_gemm(eddy_ctx *ctx, int M, int N, int K, const void *A, const void *B, float *D, int acc,
                     int splitk = 1) {
  if (M < 1 || N % 16 || N < 16 || N > 256 || K % 16 || K < 16 || splitk < 1) {
    ctx->err = "umma gemm: N%16 (16..256), K%16 required";
    return EDDY_EINVAL;
  }
  int kper = ((K + splitk - 1) / splitk + GKC - 1) / GKC * GKC;
  int ns = (K + kper - 1) / kper;
  size_t smem = (size_t)(128 + N) * GKC * 2 + 1024;
  EDDY_CUDA(cudaFuncSetAttribute(k_umma_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_umma_gemm<<<dim3((M + 127) / 128, ns), GT, smem, ctx->stream>>>(
      M, N, K, static_cast<const __nv_bfloat16 *>(A), static_cast<const __nv_bfloat16 *>(B), D, acc, kper,
      ctx->err_flag);
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

// ===========================================================================
// Closure network: parameters, features, fused inference, training.
// theta layout (FP32): W1[64][16] b1[64] W2[64][64] b2[64] W3[64][64] b3[64]
// W4[16][64] b4[16]; W[n][k] is output n, input k (K-major rows).  Inputs 12..15
// of layer 1 and outputs 2..15 of layer 4 are padding (zero weights).
// meta (FP32): feat_mean[12] feat_istd[12] env_lo[12] env_hi[12] s_nu s_kappa.
// ===========================================================================
namespace {

constexpr int NFEAT = 12, KIN = 16, HID = 64, NOUT = 16;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + HID * KIN, OFF_W2 = OFF_B1 + HID, OFF_B2 = OFF_W2 + HID * HID,
              OFF_W3 = OFF_B2 + HID, OFF_B3 = OFF_W3 + HID * HID, OFF_W4 = OFF_B3 + HID,
              OFF_B4 = OFF_W4 + NOUT * HID, NTHETA = OFF_B4 + NOUT;
constexpr int NMETA = 4 * NFEAT + 2;

struct MlpMeta {
  float mean[NFEAT], istd[NFEAT], lo[NFEAT], hi[NFEAT], s_nu, s_kappa;
};

// hidden activation: hard-swish x * sat(x/6 + 1/2) (SiLU-shaped, FMA-pipe only)
__device__ __forceinline__ float hswish(float x) { return x * __saturatef(fmaf(x, 1.f / 6.f, 0.5f)); }
__device__ __forceinline__ float hswish_grad(float x) {
  return x <= -3.f ? 0.f : (x >= 3.f ? 1.f : fmaf(x, 1.f / 3.f, 0.5f));
}
__device__ __forceinline__ float sigm(float x) { return 1.f / (1.f + __expf(-x)); }
__device__ __forceinline__ float softplus(float x) { return x > 20.f ? x : log1pf(__expf(x)); }

// raw features of interior cell (i,j,k) and its filter width Delta
// (9 velocity-gradient components * Delta, |grad rho| * Delta, N^2 = -g drho/dx,
// distance to the nearest x wall)
// cube roots of the cell widths along x, y, z: Delta = cx[i] cy[j] cz[k]
struct CellGeom {
  const double *cx, *cy, *cz;
};

// T: storage of the fields (FP64 arrays of pitch NX, or the mixed form's
// FP32 copies of pitch px); A: arithmetic of the gradients
template <class T, class A>
__device__ __forceinline__ void cell_features(const Dims &d, const DevMetrics &m, const CellGeom &cg, double grav,
                                              double xwall_lo, double xwall_hi, int pitch, const T *__restrict__ uo,
                                              const T *__restrict__ vo, const T *__restrict__ wo,
                                              const T *__restrict__ dens, const double *__restrict__ xc, int i, int j,
                                              int k, float *f, float &delta) {
  const long long q = pidx(d, pitch, i, j, k);
  const long long sy = pitch, sz = (long long)pitch * d.ny;
  const A h = (A)0.5;
  auto U = [&](long long o) { return (A)uo[q + o]; };
  auto V = [&](long long o) { return (A)vo[q + o]; };
  auto W = [&](long long o) { return (A)wo[q + o]; };
  auto R = [&](long long o) { return (A)dens[q + o]; };
  auto UC = [&](long long o) { return h * (U(o - 1) + U(o)); };
  auto VC = [&](long long o) { return h * (V(o - sy) + V(o)); };
  auto WC = [&](long long o) { return h * (W(o - sz) + W(o)); };
  const A api = (A)m.ap[i], aui = (A)m.au[i], aum = (A)m.au[i - 1];
  const A bpj = (A)m.bp[j], bvj = (A)m.bv[j], bvm = (A)m.bv[j - 1];
  const A cpk = (A)m.cp[k], cwk = (A)m.cw[k], cwm = (A)m.cw[k - 1];
  A dudx = api * (U(0) - U(-1));
  A dudy = h * (bvj * (UC(sy) - UC(0)) + bvm * (UC(0) - UC(-sy)));
  A dudz = h * (cwk * (UC(sz) - UC(0)) + cwm * (UC(0) - UC(-sz)));
  A dvdx = h * (aui * (VC(1) - VC(0)) + aum * (VC(0) - VC(-1)));
  A dvdy = bpj * (V(0) - V(-sy));
  A dvdz = h * (cwk * (VC(sz) - VC(0)) + cwm * (VC(0) - VC(-sz)));
  A dwdx = h * (aui * (WC(1) - WC(0)) + aum * (WC(0) - WC(-1)));
  A dwdy = h * (bvj * (WC(sy) - WC(0)) + bvm * (WC(0) - WC(-sy)));
  A dwdz = cpk * (W(0) - W(-sz));
  A drx = h * (aui * (R(1) - R(0)) + aum * (R(0) - R(-1)));
  A dry = h * (bvj * (R(sy) - R(0)) + bvm * (R(0) - R(-sy)));
  A drz = h * (cwk * (R(sz) - R(0)) + cwm * (R(0) - R(-sz)));
  A del = (A)(cg.cx[i] * cg.cy[j] * cg.cz[k]);
  delta = (float)del;
  f[0] = (float)(del * dudx); f[1] = (float)(del * dudy); f[2] = (float)(del * dudz);
  f[3] = (float)(del * dvdx); f[4] = (float)(del * dvdy); f[5] = (float)(del * dvdz);
  f[6] = (float)(del * dwdx); f[7] = (float)(del * dwdy); f[8] = (float)(del * dwdz);
  f[9] = (float)(del * sqrt(drx * drx + dry * dry + drz * drz));
  f[10] = (float)(-(A)grav * drx);
  double x = xc[i];
  f[11] = (float)fmin(x - xwall_lo, xwall_hi - x);
}

// interior cell number t (x fastest) -> (i,j,k); the interior has fewer
// than 2^32 cells (checked at launch)
__device__ __forceinline__ void interior_ijk(const Dims &d, unsigned t, int &i, int &j, int &k) {
  unsigned mi = d.ix2 - d.ix1 + 1, mj = d.jy2 - d.jy1 + 1;
  unsigned r = t / mi;
  i = d.ix1 + (int)(t - r * mi);
  unsigned kk = r / mj;
  j = d.jy1 + (int)(r - kk * mj);
  k = d.kz1 + (int)kk;
}

// raw features (n x 12) and dynamic-model targets nu_t/Delta for a list of
// interior cell indices
__global__ void k_harvest(Dims d, DevMetrics m, CellGeom cg, double grav, double xlo, double xhi, const double *uo,
                          const double *vo, const double *wo, const double *dens, const double *xc, const double *tv,
                          const long long *cells, int n, float *X, float *T) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int i, j, k;
  interior_ijk(d, (unsigned)cells[s], i, j, k);
  float f[NFEAT], del;
  cell_features<double, double>(d, m, cg, grav, xlo, xhi, d.nx, uo, vo, wo, dens, xc, i, j, k, f, del);
  for (int c = 0; c < NFEAT; c++) X[(size_t)s * NFEAT + c] = f[c];
  T[s] = (float)(tv[fidx(d, i, j, k)] / del);
}

// ---- fused inference ------------------------------------------------------
// One CTA of 128 threads runs two 128-cell tiles at a time (thread t owns
// cell t of each), with separate activation buffers and TMEM accumulators
// (columns 0..63 and 64..127): while the tensor core runs one tile's layer,
// the threads run the other tile's epilogue.
constexpr int IT = 128;
struct InferSmem {
  unsigned char w1[HID * KIN * 2], w2[HID * HID * 2], w3[HID * HID * 2];
  // h[g]: layer input of tile g; the normalised features (layer 1's input,
  // 128 x KIN) occupy its first 4 KB until layer 1's MMA has read them
  unsigned char h[2][128 * HID * 2];
  float b1[HID], b2[HID], b3[HID], b4[NOUT];
  // output layer rows 0 and 1 in FP32: computed on the CUDA cores from the
  // layer-3 activations in registers (no fourth MMA round trip)
  __align__(16) float w4f[2][HID];
  MlpMeta meta;
  uint64_t bar[2];
  uint32_t tmem;
  int nout;
};

__device__ __forceinline__ void stage_weights(unsigned char *dst, const __nv_bfloat16 *src, int rows, int K) {
  for (int e = threadIdx.x; e < rows * K / 8; e += blockDim.x) {
    int r = e / (K / 8), c8 = (e % (K / 8)) * 8;
    *reinterpret_cast<uint4 *>(dst + umma::kmajor_offset(r, c8, K)) =
        *reinterpret_cast<const uint4 *>(src + (size_t)r * K + c8);
  }
}

__device__ __forceinline__ void mma_layer(uint32_t tm, const unsigned char *a, const unsigned char *b, int N, int K) {
  uint32_t idesc = umma::make_idesc_bf16(128, N);
  for (int ks = 0; ks < K; ks += 16) {
    uint64_t ad = umma::make_desc(a + (ks / 8) * 128, 128, 128 * (K / 8));
    uint64_t bd = umma::make_desc(b + (ks / 8) * 128, 128, 128 * (K / 8));
    umma::mma_bf16(tm, ad, bd, idesc, ks > 0 ? 1u : 0u);
  }
}

// two activations packed to BF16x2 (round to nearest)
__device__ __forceinline__ uint32_t act2_bf16(float x0, float x1) {
  __nv_bfloat162 hb = __floats2bfloat162_rn(hswish(x0), hswish(x1));
  return *reinterpret_cast<uint32_t *>(&hb);
}

// hidden epilogue: TMEM (64 cols of this thread's row) + bias -> hard-swish
// -> bf16 row of the next layer's A operand
__device__ __forceinline__ void hidden_epilogue(uint32_t tm, int warp, int row, const float *bias,
                                                unsigned char *h) {
  uint32_t r[HID];
  umma::tmem_ld64(tm + ((uint32_t)(warp * 32) << 16), r);
  auto x = [&](int c) { return __uint_as_float(r[c]) + bias[c]; };
#pragma unroll
  for (int c0 = 0; c0 < HID; c0 += 8) {
    uint4 o;
    o.x = act2_bf16(x(c0 + 0), x(c0 + 1));
    o.y = act2_bf16(x(c0 + 2), x(c0 + 3));
    o.z = act2_bf16(x(c0 + 4), x(c0 + 5));
    o.w = act2_bf16(x(c0 + 6), x(c0 + 7));
    *reinterpret_cast<uint4 *>(h + umma::kmajor_offset(row, c0, HID)) = o;
  }
}

// last hidden layer (TMEM + bias -> hard-swish, FP32) and the output layer's
// two rows: v[n] = b4[n] + sum_c w4[n][c] act[c]
__device__ __forceinline__ void output_layer(uint32_t tm, int warp, const float *bias, const float (*w4)[HID],
                                             const float *b4, float *v) {
  uint32_t r[HID];
  umma::tmem_ld64(tm + ((uint32_t)(warp * 32) << 16), r);
  float o0 = b4[0], o1 = b4[1];
#pragma unroll
  for (int c = 0; c < HID; c += 4) {
    const float4 p = *reinterpret_cast<const float4 *>(w4[0] + c), q = *reinterpret_cast<const float4 *>(w4[1] + c);
    const float a0 = hswish(__uint_as_float(r[c]) + bias[c]), a1 = hswish(__uint_as_float(r[c + 1]) + bias[c + 1]);
    const float a2 = hswish(__uint_as_float(r[c + 2]) + bias[c + 2]);
    const float a3 = hswish(__uint_as_float(r[c + 3]) + bias[c + 3]);
    o0 = fmaf(p.x, a0, fmaf(p.y, a1, fmaf(p.z, a2, fmaf(p.w, a3, o0))));
    o1 = fmaf(q.x, a0, fmaf(q.y, a1, fmaf(q.z, a2, fmaf(q.w, a3, o1))));
  }
  v[0] = o0;
  v[1] = o1;
}

// one thread waits on the MMA barrier, the block meets at a barrier (the
// other warps sleep there instead of polling the mbarrier)
__device__ __forceinline__ bool sync_and_wait(uint64_t *bar, int &phase) {
  int ok = 1;
  if (threadIdx.x == 0) ok = umma::mbar_wait(bar, phase) ? 1 : 0;
  phase ^= 1;
  ok = __syncthreads_and(ok);
  umma::fence_after_sync();
  return ok != 0;
}

__device__ __forceinline__ void publish_smem() {
  umma::fence_smem_to_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
}

// one cell of a tile: where it is and what the output needs
struct CellIn {
  bool valid, outside;
  int i, j, k;
  float del, dsr;
};

// nu_t -> tv, kappa_t -> kappa for every interior cell; cells whose
// normalised features leave [lo, hi] take the fallback (last dynamic-model
// value).  counts[0] += out-of-envelope cells.  T: storage of the input
// fields (pitch `pitch`); tv32/kv32 (pitch px32, may be null): FP32 copies
// of the outputs for the mixed form's stencils.
template <class T>
__global__ void __launch_bounds__(IT)
    k_mlp_infer(Dims d, DevMetrics m, CellGeom cg, double grav, double xlo, double xhi, int pitch,
                const T *__restrict__ uo, const T *__restrict__ vo, const T *__restrict__ wo,
                const T *__restrict__ dens, const double *__restrict__ xc, const __nv_bfloat16 *__restrict__ wbf,
                const float *__restrict__ theta, const float *__restrict__ meta, const double *__restrict__ fallback,
                double *__restrict__ tv, double *__restrict__ kappa, float *__restrict__ tv32,
                float *__restrict__ kv32, int px32, unsigned long long *counts, int *err) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  InferSmem &S = *reinterpret_cast<InferSmem *>(smraw);
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    umma::tmem_alloc(&S.tmem, 128);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    umma::mbar_init(&S.bar[0], 1);
    umma::mbar_init(&S.bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    S.nout = 0;
  }
  stage_weights(S.w1, wbf + OFF_W1, HID, KIN);
  stage_weights(S.w2, wbf + OFF_W2, HID, HID);
  stage_weights(S.w3, wbf + OFF_W3, HID, HID);
  for (int e = tid; e < HID; e += IT) {
    S.b1[e] = theta[OFF_B1 + e];
    S.b2[e] = theta[OFF_B2 + e];
    S.b3[e] = theta[OFF_B3 + e];
  }
  if (tid < NOUT) S.b4[tid] = theta[OFF_B4 + tid];
  for (int e = tid; e < 2 * HID; e += IT) S.w4f[e / HID][e % HID] = theta[OFF_W4 + e];
  for (int e = tid; e < NMETA; e += IT) reinterpret_cast<float *>(&S.meta)[e] = meta[e];
  publish_smem();
  const uint32_t tm = S.tmem;
  const unsigned ninner = (unsigned)(d.ix2 - d.ix1 + 1) * (d.jy2 - d.jy1 + 1) * (d.kz2 - d.kz1 + 1);
  const unsigned ntiles = (ninner + 127) / 128, npairs = (ntiles + 1) / 2;
  const unsigned char *wl[2] = {S.w2, S.w3};
  const float *bl[3] = {S.b1, S.b2, S.b3};
  int phase[2] = {0, 0};
  bool ok = true;
  int nout = 0;
  for (unsigned pair = blockIdx.x; pair < npairs && ok; pair += gridDim.x) {
    CellIn c[2];
#pragma unroll
    for (int g = 0; g < 2; g++) {
      const unsigned t = (2 * pair + g) * 128 + tid;
      CellIn &C = c[g];
      C.valid = t < ninner;
      C.outside = false;
      C.i = d.ix1; C.j = d.jy1; C.k = d.kz1;
      C.del = 1.f; C.dsr = 0.f;
      float f[NFEAT];
      if (C.valid) {
        interior_ijk(d, t, C.i, C.j, C.k);
        cell_features<T, T>(d, m, cg, grav, xlo, xhi, pitch, uo, vo, wo, dens, xc, C.i, C.j, C.k, f, C.del);
        // Delta |S| = Delta sqrt(2 S_ij S_ij) from the raw gradient features
        const float s01 = 0.5f * (f[1] + f[3]), s02 = 0.5f * (f[2] + f[6]), s12 = 0.5f * (f[5] + f[7]);
        C.dsr = sqrtf(2.f * (f[0] * f[0] + f[4] * f[4] + f[8] * f[8] + 2.f * (s01 * s01 + s02 * s02 + s12 * s12)));
        for (int q = 0; q < NFEAT; q++) {
          f[q] = (f[q] - S.meta.mean[q]) * S.meta.istd[q];
          C.outside = C.outside || !(f[q] >= S.meta.lo[q] && f[q] <= S.meta.hi[q]);
        }
      } else {
        for (int q = 0; q < NFEAT; q++) f[q] = 0.f;
      }
      __align__(16) __nv_bfloat16 o[16];
      for (int q = 0; q < 16; q++) o[q] = __float2bfloat16_rn(q < NFEAT ? f[q] : 0.f);
      *reinterpret_cast<uint4 *>(S.h[g] + umma::kmajor_offset(tid, 0, KIN)) = *reinterpret_cast<uint4 *>(o);
      *reinterpret_cast<uint4 *>(S.h[g] + umma::kmajor_offset(tid, 8, KIN)) = *reinterpret_cast<uint4 *>(o + 8);
    }
    publish_smem();
    if (tid == 0) {
      mma_layer(tm, S.h[0], S.w1, HID, KIN);
      umma::commit(&S.bar[0]);
      mma_layer(tm + 64, S.h[1], S.w1, HID, KIN);
      umma::commit(&S.bar[1]);
    }
    // layers 2..3: epilogue of layer L of one tile while the other tile's
    // layer runs on the tensor core
#pragma unroll
    for (int L = 0; L < 2; L++) {
#pragma unroll
      for (int g = 0; g < 2; g++) {
        ok = sync_and_wait(&S.bar[g], phase[g]) && ok;
        hidden_epilogue(tm + 64 * g, warp, tid, bl[L], S.h[g]);
        publish_smem();
        if (tid == 0) {
          mma_layer(tm + 64 * g, S.h[g], wl[L], HID, HID);
          umma::commit(&S.bar[g]);
        }
      }
    }
    // layer 3's activations and the 64 -> 2 output layer in registers
#pragma unroll
    for (int g = 0; g < 2; g++) {
      ok = sync_and_wait(&S.bar[g], phase[g]) && ok;
      float v[2];
      output_layer(tm + 64 * g, warp, S.b3, S.w4f, S.b4, v);
      const CellIn &C = c[g];
      if (C.valid && ok) {
        long long q = fidx(d, C.i, C.j, C.k);
        double nu, ka;
        if (C.outside) {
          nu = fallback[q];
          ka = fallback[q];
          nout++;
        } else {
          // nu_t = C_nu Delta^2 |S|, kappa_t = C_kappa Delta^2 |S|
          nu = (double)C.del * (double)C.dsr * S.meta.s_nu * softplus(v[0]);
          ka = (double)C.del * (double)C.dsr * S.meta.s_kappa * softplus(v[1]);
        }
        tv[q] = nu;
        kappa[q] = ka;
        if (tv32) {
          const long long p = pidx(d, px32, C.i, C.j, C.k);
          tv32[p] = (float)nu;
          kv32[p] = (float)ka;
        }
      }
    }
    umma::fence_before_sync();
    ok = __syncthreads_and(ok ? 1 : 0) != 0;  // block-uniform loop exit
    umma::fence_after_sync();
  }
  if (!ok && tid == 0) atomicExch(err, 1);
  atomicAdd(&S.nout, nout);
  umma::fence_before_sync();
  __syncthreads();
  if (tid == 0 && S.nout) atomicAdd(counts, (unsigned long long)S.nout);
  if (warp == 0) umma::tmem_dealloc(tm, 128);
}

// ---- training -------------------------------------------------------------
// Z (B x n, f32, pre-bias) += bias; A = bf16(hswish(Z)) in both B x n and n x B
__global__ void k_fwd_act(int B, int n, float *Z, const float *bias, __nv_bfloat16 *A, __nv_bfloat16 *AT) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)B * n) return;
  int b = (int)(t / n), c = (int)(t % n);
  float z = Z[t] + bias[c];
  Z[t] = z;
  __nv_bfloat16 a = __float2bfloat16_rn(hswish(z));
  A[t] = a;
  AT[(size_t)c * B + b] = a;
}

// output layer: P = softplus(Z4 + b4) on columns 0,1; loss and dZ4
__global__ void k_out_grad(int B, float *Z4, const float *b4, const float *Y, __nv_bfloat16 *dZ, __nv_bfloat16 *dZT,
                           float *db, double *loss) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  __shared__ float sdb[2];
  __shared__ double sl;
  if (threadIdx.x < 2) sdb[threadIdx.x] = 0.f;
  if (threadIdx.x == 0) sl = 0.;
  __syncthreads();
  if (b < B) {
    for (int c = 0; c < NOUT; c++) {
      float g = 0.f;
      if (c < 2) {
        float z = Z4[(size_t)b * NOUT + c] + b4[c];
        float p = softplus(z), r = p - Y[(size_t)b * 2 + c];
        atomicAdd(&sl, (double)(r * r) / B);
        g = 2.f * r * sigm(z) / B;
        atomicAdd(&sdb[c], g);
      }
      __nv_bfloat16 gb = __float2bfloat16_rn(g);
      dZ[(size_t)b * NOUT + c] = gb;
      dZT[(size_t)c * B + b] = gb;
    }
  }
  __syncthreads();
  if (threadIdx.x < 2) atomicAdd(&db[threadIdx.x], sdb[threadIdx.x]);
  if (threadIdx.x == 0) atomicAdd(loss, sl);
}

// hidden backward: dZ = dA * act'(Z) (bf16, both layouts), db += column sums
__global__ void k_bwd_act(int B, int n, const float *dA, const float *Z, __nv_bfloat16 *dZ, __nv_bfloat16 *dZT,
                          float *db) {
  __shared__ float sdb[HID];
  for (int c = threadIdx.x; c < n; c += blockDim.x) sdb[c] = 0.f;
  __syncthreads();
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < (long long)B * n) {
    int b = (int)(t / n), c = (int)(t % n);
    float g = dA[t] * hswish_grad(Z[t]);
    __nv_bfloat16 gb = __float2bfloat16_rn(g);
    dZ[t] = gb;
    dZT[(size_t)c * B + b] = gb;
    atomicAdd(&sdb[c], g);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += blockDim.x) atomicAdd(&db[c], sdb[c]);
}

// gather a batch: X (bf16 n x 16 normalised features), Y (f32 n x 2)
__global__ void k_gather(int B, const long long *perm, long long off, const __nv_bfloat16 *X, const float *Y,
                         __nv_bfloat16 *Xb, __nv_bfloat16 *XbT, float *Yb) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  long long s = perm[off + b];
  for (int c = 0; c < KIN; c++) {
    __nv_bfloat16 v = X[s * KIN + c];
    Xb[(size_t)b * KIN + c] = v;
    XbT[(size_t)c * B + b] = v;
  }
  Yb[2 * b] = Y[2 * s];
  Yb[2 * b + 1] = Y[2 * s + 1];
}

// Adam on theta, then refresh the bf16 weights (W and W^T)
__global__ void k_adam(int n, float *theta, const float *grad, float *m1, float *m2, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  float g = grad[t];
  float a = b1 * m1[t] + (1.f - b1) * g, v = b2 * m2[t] + (1.f - b2) * g * g;
  m1[t] = a;
  m2[t] = v;
  theta[t] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
}

__global__ void k_weights_bf16(const float *theta, __nv_bfloat16 *w, __nv_bfloat16 *wt) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NTHETA) return;
  w[t] = __float2bfloat16_rn(theta[t]);
  // transposed copies of the four weight matrices at the same offsets
  int off = 0, rows = 0, cols = 0;
  if (t < OFF_B1) { off = OFF_W1; rows = HID; cols = KIN; }
  else if (t >= OFF_W2 && t < OFF_B2) { off = OFF_W2; rows = HID; cols = HID; }
  else if (t >= OFF_W3 && t < OFF_B3) { off = OFF_W3; rows = HID; cols = HID; }
  else if (t >= OFF_W4 && t < OFF_B4) { off = OFF_W4; rows = NOUT; cols = HID; }
  else return;
  int r = (t - off) / cols, c = (t - off) % cols;
  wt[off + c * rows + r] = __float2bfloat16_rn(theta[t]);
}

__global__ void k_normalise(long long n, const float *raw, const float *meta, __nv_bfloat16 *X) {
  long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  for (int c = 0; c < KIN; c++)
    X[s * KIN + c] = __float2bfloat16_rn(c < NFEAT ? (raw[s * NFEAT + c] - meta[c]) * meta[NFEAT + c] : 0.f);
}

}  // namespace

// ---- host side ---------------------------------------------------------------
struct MlpTrainBuffers {
  int B = 0;
  __nv_bfloat16 *Xb = nullptr, *XbT = nullptr, *A1 = nullptr, *A1T = nullptr, *A2 = nullptr, *A2T = nullptr,
                *A3 = nullptr, *A3T = nullptr, *dZ4 = nullptr, *dZ4T = nullptr, *dZ = nullptr, *dZT = nullptr;
  float *Yb = nullptr, *Z1 = nullptr, *Z2 = nullptr, *Z3 = nullptr, *Z4 = nullptr, *dA = nullptr;
  void release() {
    void *p[] = {Xb, XbT, A1, A1T, A2, A2T, A3, A3T, dZ4, dZ4T, dZ, dZT, Yb, Z1, Z2, Z3, Z4, dA};
    for (void *q : p) if (q) cudaFree(q);
    *this = MlpTrainBuffers{};
  }
};

struct MlpState {
  float *theta = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr, *meta = nullptr;
  __nv_bfloat16 *w = nullptr, *wt = nullptr;
  double *loss = nullptr;
  unsigned long long *counts = nullptr;
  double *fallback = nullptr;  // last dynamic-model nu_t
  double *cbw = nullptr;       // cube roots of the cell widths (x, y, z blocks)
  int adam_t = 0;
  bool ready = false;
  MlpTrainBuffers tb;
};

static MlpState *mlp_state(eddy_ctx *ctx) {
  if (!ctx->mlp) {
    MlpState *s = new MlpState();
    ctx->mlp = s;
  }
  return static_cast<MlpState *>(ctx->mlp);
}

void mlp_release(eddy_ctx *ctx) {
  MlpState *s = static_cast<MlpState *>(ctx->mlp);
  if (!s) return;
  void *p[] = {s->theta, s->grad, s->m1, s->m2, s->meta, s->w, s->wt, s->loss, s->counts, s->fallback, s->cbw};
  for (void *q : p) if (q) cudaFree(q);
  s->tb.release();
  delete s;
  ctx->mlp = nullptr;
}

// Delta = (cell volume)^(1/3) as a product of per-axis cube roots
static int mlp_geom(eddy_ctx *ctx, MlpState *s, CellGeom &cg) {
  const Dims &d = ctx->d;
  size_t nx = d.nx + 2, ny = d.ny + 2, nz = d.nz + 2;
  if (!s->cbw) {
    std::vector<double> h(nx + ny + nz, 0.0);
    const std::vector<double> &ap = ctx->h[2], &bp = ctx->h[8], &cp = ctx->h[14];
    for (size_t i = 0; i < nx && i < ap.size(); i++) h[i] = ap[i] > 0 ? std::cbrt(1.0 / ap[i]) : 0.0;
    for (size_t j = 0; j < ny && j < bp.size(); j++) h[nx + j] = bp[j] > 0 ? std::cbrt(1.0 / bp[j]) : 0.0;
    for (size_t k = 0; k < nz && k < cp.size(); k++) h[nx + ny + k] = cp[k] > 0 ? std::cbrt(1.0 / cp[k]) : 0.0;
    EDDY_CUDA(cudaMalloc(&s->cbw, sizeof(double) * h.size()));
    EDDY_CUDA(cudaMemcpy(s->cbw, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
  }
  cg.cx = s->cbw;
  cg.cy = s->cbw + nx;
  cg.cz = s->cbw + nx + ny;
  return EDDY_OK;
}

static int mlp_alloc(eddy_ctx *ctx, MlpState *s) {
  if (s->theta) return EDDY_OK;
  EDDY_CUDA(cudaMalloc(&s->theta, sizeof(float) * NTHETA));
  EDDY_CUDA(cudaMalloc(&s->grad, sizeof(float) * NTHETA));
  EDDY_CUDA(cudaMalloc(&s->m1, sizeof(float) * NTHETA));
  EDDY_CUDA(cudaMalloc(&s->m2, sizeof(float) * NTHETA));
  EDDY_CUDA(cudaMalloc(&s->meta, sizeof(float) * NMETA));
  EDDY_CUDA(cudaMalloc(&s->w, sizeof(__nv_bfloat16) * NTHETA));
  EDDY_CUDA(cudaMalloc(&s->wt, sizeof(__nv_bfloat16) * NTHETA));
  EDDY_CUDA(cudaMalloc(&s->loss, sizeof(double)));
  EDDY_CUDA(cudaMalloc(&s->counts, sizeof(unsigned long long)));
  EDDY_CUDA(cudaMemset(s->m1, 0, sizeof(float) * NTHETA));
  EDDY_CUDA(cudaMemset(s->m2, 0, sizeof(float) * NTHETA));
  EDDY_CUDA(cudaMemset(s->wt, 0, sizeof(__nv_bfloat16) * NTHETA));
  return EDDY_OK;
}

static int tb_alloc(eddy_ctx *ctx, MlpTrainBuffers &t, int B) {
  if (t.B == B) return EDDY_OK;
  t.release();
  t.B = B;
  auto bf = [&](__nv_bfloat16 **p, size_t n) { return cudaMalloc(p, n * sizeof(__nv_bfloat16)); };
  auto fl = [&](float **p, size_t n) { return cudaMalloc(p, n * sizeof(float)); };
  size_t b = (size_t)B;
  if (bf(&t.Xb, b * KIN) || bf(&t.XbT, b * KIN) || bf(&t.A1, b * HID) || bf(&t.A1T, b * HID) ||
      bf(&t.A2, b * HID) || bf(&t.A2T, b * HID) || bf(&t.A3, b * HID) || bf(&t.A3T, b * HID) ||
      bf(&t.dZ4, b * NOUT) || bf(&t.dZ4T, b * NOUT) || bf(&t.dZ, b * HID) || bf(&t.dZT, b * HID) ||
      fl(&t.Yb, b * 2) || fl(&t.Z1, b * HID) || fl(&t.Z2, b * HID) || fl(&t.Z3, b * HID) || fl(&t.Z4, b * NOUT) ||
      fl(&t.dA, b * HID)) {
    ctx->err = "closure training buffers: allocation failed";
    return EDDY_ENOMEM;
  }
  return EDDY_OK;
}

int launch_umma_gemm(eddy_ctx *ctx, int M, int N, int K, const void *A, const void *B, float *D, int acc,
                     int splitk);

// one forward + backward pass over the batch staged in tb (Xb, XbT, Yb);
// gradients into s->grad, loss into s->loss (added)
static int fwd_bwd(eddy_ctx *ctx, MlpState *s) {
  MlpTrainBuffers &t = s->tb;
  const int B = t.B;
  cudaStream_t st = ctx->stream;
  int rc;
  const int nt = 256;
  auto blocks = [&](long long n) { return (unsigned)((n + nt - 1) / nt); };
  const __nv_bfloat16 *w = s->w, *wt = s->wt;
  float *th = s->theta, *g = s->grad;
  int splitk = B >= 4096 ? B / 1024 : 1;
  // forward
  if ((rc = launch_umma_gemm(ctx, B, HID, KIN, t.Xb, w + OFF_W1, t.Z1, 0, 1))) return rc;
  k_fwd_act<<<blocks((long long)B * HID), nt, 0, st>>>(B, HID, t.Z1, th + OFF_B1, t.A1, t.A1T);
  EDDY_LAUNCHED(ctx);
  if ((rc = launch_umma_gemm(ctx, B, HID, HID, t.A1, w + OFF_W2, t.Z2, 0, 1))) return rc;
  k_fwd_act<<<blocks((long long)B * HID), nt, 0, st>>>(B, HID, t.Z2, th + OFF_B2, t.A2, t.A2T);
  EDDY_LAUNCHED(ctx);
  if ((rc = launch_umma_gemm(ctx, B, HID, HID, t.A2, w + OFF_W3, t.Z3, 0, 1))) return rc;
  k_fwd_act<<<blocks((long long)B * HID), nt, 0, st>>>(B, HID, t.Z3, th + OFF_B3, t.A3, t.A3T);
  EDDY_LAUNCHED(ctx);
  if ((rc = launch_umma_gemm(ctx, B, NOUT, HID, t.A3, w + OFF_W4, t.Z4, 0, 1))) return rc;
  // backward
  EDDY_CUDA(cudaMemsetAsync(g, 0, sizeof(float) * NTHETA, st));
  k_out_grad<<<blocks(B), nt, 0, st>>>(B, t.Z4, th + OFF_B4, t.Yb, t.dZ4, t.dZ4T, g + OFF_B4, s->loss);
  EDDY_LAUNCHED(ctx);
  // layer 4: dW4 = dZ4^T A3 ; dA3 = dZ4 W4
  if ((rc = launch_umma_gemm(ctx, NOUT, HID, B, t.dZ4T, t.A3T, g + OFF_W4, 1, splitk))) return rc;
  if ((rc = launch_umma_gemm(ctx, B, HID, NOUT, t.dZ4, wt + OFF_W4, t.dA, 0, 1))) return rc;
  k_bwd_act<<<blocks((long long)B * HID), nt, 0, st>>>(B, HID, t.dA, t.Z3, t.dZ, t.dZT, g + OFF_B3);
  EDDY_LAUNCHED(ctx);
  // layer 3
  if ((rc = launch_umma_gemm(ctx, HID, HID, B, t.dZT, t.A2T, g + OFF_W3, 1, splitk))) return rc;
  if ((rc = launch_umma_gemm(ctx, B, HID, HID, t.dZ, wt + OFF_W3, t.dA, 0, 1))) return rc;
  k_bwd_act<<<blocks((long long)B * HID), nt, 0, st>>>(B, HID, t.dA, t.Z2, t.dZ, t.dZT, g + OFF_B2);
  EDDY_LAUNCHED(ctx);
  // layer 2
  if ((rc = launch_umma_gemm(ctx, HID, HID, B, t.dZT, t.A1T, g + OFF_W2, 1, splitk))) return rc;
  if ((rc = launch_umma_gemm(ctx, B, HID, HID, t.dZ, wt + OFF_W2, t.dA, 0, 1))) return rc;
  k_bwd_act<<<blocks((long long)B * HID), nt, 0, st>>>(B, HID, t.dA, t.Z1, t.dZ, t.dZT, g + OFF_B1);
  EDDY_LAUNCHED(ctx);
  // layer 1
  if ((rc = launch_umma_gemm(ctx, HID, KIN, B, t.dZT, t.XbT, g + OFF_W1, 1, splitk))) return rc;
  return EDDY_OK;
}

static int refresh_bf16(eddy_ctx *ctx, MlpState *s) {
  k_weights_bf16<<<(NTHETA + 255) / 256, 256, 0, ctx->stream>>>(s->theta, s->w, s->wt);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

extern "C" {

int eddy_closure_set(eddy_ctx *ctx, const float *meta, const float *theta) {
  if (!ctx || !meta || !theta) return EDDY_EINVAL;
  MlpState *s = mlp_state(ctx);
  int rc = mlp_alloc(ctx, s);
  if (rc) return rc;
  EDDY_CUDA(cudaMemcpyAsync(s->meta, meta, sizeof(float) * NMETA, cudaMemcpyHostToDevice, ctx->stream));
  EDDY_CUDA(cudaMemcpyAsync(s->theta, theta, sizeof(float) * NTHETA, cudaMemcpyHostToDevice, ctx->stream));
  EDDY_CUDA(cudaMemsetAsync(s->m1, 0, sizeof(float) * NTHETA, ctx->stream));
  EDDY_CUDA(cudaMemsetAsync(s->m2, 0, sizeof(float) * NTHETA, ctx->stream));
  s->adam_t = 0;
  if ((rc = refresh_bf16(ctx, s))) return rc;
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  s->ready = true;
  return EDDY_OK;
}

int eddy_closure_get(eddy_ctx *ctx, float *meta, float *theta) {
  if (!ctx || !ctx->mlp) return EDDY_EINVAL;
  MlpState *s = mlp_state(ctx);
  if (meta) EDDY_CUDA(cudaMemcpy(meta, s->meta, sizeof(float) * NMETA, cudaMemcpyDeviceToHost));
  if (theta) EDDY_CUDA(cudaMemcpy(theta, s->theta, sizeof(float) * NTHETA, cudaMemcpyDeviceToHost));
  return EDDY_OK;
}

// features (raw) and targets nu_t/Delta of the given interior cells from the
// current fields (TV holds the dynamic model's viscosity)
int eddy_closure_harvest(eddy_ctx *ctx, const long long *cells, int n, float *X, float *T) {
  if (!ctx || !cells || !X || !T || n <= 0) return EDDY_EINVAL;
  CellGeom cg;
  int rc = mlp_geom(ctx, mlp_state(ctx), cg);
  if (rc) return rc;
  long long *dc = nullptr;
  float *dX = nullptr, *dT = nullptr;
  EDDY_CUDA(cudaMalloc(&dc, sizeof(long long) * n));
  EDDY_CUDA(cudaMalloc(&dX, sizeof(float) * (size_t)n * NFEAT));
  EDDY_CUDA(cudaMalloc(&dT, sizeof(float) * n));
  EDDY_CUDA(cudaMemcpyAsync(dc, cells, sizeof(long long) * n, cudaMemcpyHostToDevice, ctx->stream));
  const std::vector<double> &xu = ctx->h[0];
  k_harvest<<<(n + 255) / 256, 256, 0, ctx->stream>>>(ctx->d, ctx->m, cg, ctx->sc.grav, xu[1], xu[ctx->d.ix2],
                                                      ctx->f[EDDY_UO], ctx->f[EDDY_VO], ctx->f[EDDY_WO],
                                                      ctx->f[EDDY_DENS], ctx->xc_dev, ctx->f[EDDY_TV], dc, n, dX, dT);
  EDDY_LAUNCHED(ctx);
  EDDY_CUDA(cudaMemcpyAsync(X, dX, sizeof(float) * (size_t)n * NFEAT, cudaMemcpyDeviceToHost, ctx->stream));
  EDDY_CUDA(cudaMemcpyAsync(T, dT, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream));
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  cudaFree(dc);
  cudaFree(dX);
  cudaFree(dT);
  return EDDY_OK;
}

// gradients of the mean-squared loss over one batch (n multiple of 128) of
// raw features X (n x 12) and targets Y (n x 2), at the current parameters
int eddy_closure_grad(eddy_ctx *ctx, const float *X, const float *Y, int n, float *grad, double *loss) {
  if (!ctx || !ctx->mlp || !X || !Y || !grad || n <= 0 || n % 128) return EDDY_EINVAL;
  MlpState *s = mlp_state(ctx);
  int rc = tb_alloc(ctx, s->tb, n);
  if (rc) return rc;
  float *draw = nullptr, *dY = nullptr;
  __nv_bfloat16 *dXn = nullptr;
  long long *perm = nullptr;
  EDDY_CUDA(cudaMalloc(&draw, sizeof(float) * (size_t)n * NFEAT));
  EDDY_CUDA(cudaMalloc(&dY, sizeof(float) * (size_t)n * 2));
  EDDY_CUDA(cudaMalloc(&dXn, sizeof(__nv_bfloat16) * (size_t)n * KIN));
  EDDY_CUDA(cudaMalloc(&perm, sizeof(long long) * n));
  std::vector<long long> id(n);
  for (int q = 0; q < n; q++) id[q] = q;
  EDDY_CUDA(cudaMemcpyAsync(perm, id.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, ctx->stream));
  EDDY_CUDA(cudaMemcpyAsync(draw, X, sizeof(float) * (size_t)n * NFEAT, cudaMemcpyHostToDevice, ctx->stream));
  EDDY_CUDA(cudaMemcpyAsync(dY, Y, sizeof(float) * (size_t)n * 2, cudaMemcpyHostToDevice, ctx->stream));
  k_normalise<<<(n + 255) / 256, 256, 0, ctx->stream>>>(n, draw, s->meta, dXn);
  EDDY_LAUNCHED(ctx);
  k_gather<<<(n + 255) / 256, 256, 0, ctx->stream>>>(n, perm, 0, dXn, dY, s->tb.Xb, s->tb.XbT, s->tb.Yb);
  EDDY_LAUNCHED(ctx);
  EDDY_CUDA(cudaMemsetAsync(s->loss, 0, sizeof(double), ctx->stream));
  rc = fwd_bwd(ctx, s);
  if (rc == EDDY_OK) {
    EDDY_CUDA(cudaMemcpyAsync(grad, s->grad, sizeof(float) * NTHETA, cudaMemcpyDeviceToHost, ctx->stream));
    if (loss) EDDY_CUDA(cudaMemcpyAsync(loss, s->loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  cudaFree(draw);
  cudaFree(dY);
  cudaFree(dXn);
  cudaFree(perm);
  return rc;
}

// Adam training on the GPU: raw features X (n x 12), targets Y (n x 2),
// minibatches of `batch` (multiple of 128) drawn from a seeded permutation
// per epoch; loss_hist[e] = mean batch loss of epoch e.
int eddy_closure_train(eddy_ctx *ctx, const float *X, const float *Y, long long n, int epochs, int batch, float lr,
                       unsigned long long seed, double *loss_hist) {
  if (!ctx || !ctx->mlp || !X || !Y || n < batch || batch <= 0 || batch % 128 || epochs < 1) return EDDY_EINVAL;
  MlpState *s = mlp_state(ctx);
  int rc = tb_alloc(ctx, s->tb, batch);
  if (rc) return rc;
  float *draw = nullptr, *dY = nullptr;
  __nv_bfloat16 *dXn = nullptr;
  long long *perm = nullptr;
  EDDY_CUDA(cudaMalloc(&draw, sizeof(float) * (size_t)n * NFEAT));
  EDDY_CUDA(cudaMalloc(&dY, sizeof(float) * (size_t)n * 2));
  EDDY_CUDA(cudaMalloc(&dXn, sizeof(__nv_bfloat16) * (size_t)n * KIN));
  EDDY_CUDA(cudaMalloc(&perm, sizeof(long long) * n));
  EDDY_CUDA(cudaMemcpyAsync(draw, X, sizeof(float) * (size_t)n * NFEAT, cudaMemcpyHostToDevice, ctx->stream));
  EDDY_CUDA(cudaMemcpyAsync(dY, Y, sizeof(float) * (size_t)n * 2, cudaMemcpyHostToDevice, ctx->stream));
  k_normalise<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(n, draw, s->meta, dXn);
  EDDY_LAUNCHED(ctx);
  std::vector<long long> p((size_t)n);
  uint64_t state = seed ^ 0x9E3779B97F4A7C15ull;
  auto rnd = [&]() {
    state += 0x9E3779B97F4A7C15ull;
    uint64_t z = state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  long long nb = n / batch;
  for (int e = 0; e < epochs && rc == EDDY_OK; e++) {
    for (long long q = 0; q < n; q++) p[(size_t)q] = q;
    for (long long q = n - 1; q > 0; q--) std::swap(p[(size_t)q], p[(size_t)(rnd() % (uint64_t)(q + 1))]);
    EDDY_CUDA(cudaMemcpyAsync(perm, p.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, ctx->stream));
    EDDY_CUDA(cudaMemsetAsync(s->loss, 0, sizeof(double), ctx->stream));
    for (long long b = 0; b < nb && rc == EDDY_OK; b++) {
      k_gather<<<(batch + 255) / 256, 256, 0, ctx->stream>>>(batch, perm, b * batch, dXn, dY, s->tb.Xb, s->tb.XbT,
                                                             s->tb.Yb);
      EDDY_LAUNCHED(ctx);
      rc = fwd_bwd(ctx, s);
      if (rc) break;
      s->adam_t++;
      const float b1 = 0.9f, b2 = 0.999f;
      float c1 = 1.f - powf(b1, (float)s->adam_t), c2 = 1.f - powf(b2, (float)s->adam_t);
      k_adam<<<(NTHETA + 255) / 256, 256, 0, ctx->stream>>>(NTHETA, s->theta, s->grad, s->m1, s->m2, lr, b1, b2,
                                                            1e-8f, c1, c2);
      EDDY_LAUNCHED(ctx);
      rc = refresh_bf16(ctx, s);
    }
    double l = 0.;
    EDDY_CUDA(cudaMemcpyAsync(&l, s->loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
    if (loss_hist) loss_hist[e] = l / (double)nb;
  }
  cudaFree(draw);
  cudaFree(dY);
  cudaFree(dXn);
  cudaFree(perm);
  return rc;
}

}  // extern "C"

// nu_t, kappa_t over the whole field from the fused tensor-core kernel;
// cells out of the training envelope take `fallback` (the last dynamic
// nu_t).  out_of_envelope receives the count.
int launch_closure(eddy_ctx *ctx, const double *fallback, double *kappa, unsigned long long *out_of_envelope) {
  MlpState *s = static_cast<MlpState *>(ctx->mlp);
  if (!s || !s->ready) {
    ctx->err = "learned closure requested but no network is loaded";
    return EDDY_EINVAL;
  }
  const Dims &d = ctx->d;
  const std::vector<double> &xu = ctx->h[0];
  CellGeom cg;
  int rc = mlp_geom(ctx, s, cg);
  if (rc) return rc;
  if ((long long)(d.ix2 - d.ix1 + 1) * (d.jy2 - d.jy1 + 1) * (d.kz2 - d.kz1 + 1) >= (1LL << 32) - 256) {
    ctx->err = "learned closure: interior larger than 2^32 cells";
    return EDDY_EINVAL;
  }
  EDDY_CUDA(cudaMemsetAsync(s->counts, 0, sizeof(unsigned long long), ctx->stream));
  size_t smem = sizeof(InferSmem) + 1024;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
  long long ninner = (long long)(d.ix2 - d.ix1 + 1) * (d.jy2 - d.jy1 + 1) * (d.kz2 - d.kz1 + 1);
  long long npairs = ((ninner + 127) / 128 + 1) / 2;
  int grid = (int)std::min<long long>(npairs, (long long)nsm * 4);
  MixedViews mv;
  if (ctx->mixed && mixed_views(ctx, &mv) == EDDY_OK) {
    // the mixed form: features from the FP32 copies, FP32 outputs alongside
    EDDY_CUDA(cudaFuncSetAttribute(k_mlp_infer<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_mlp_infer<float><<<grid, IT, smem, ctx->stream>>>(d, ctx->m, cg, ctx->sc.grav, xu[1], xu[d.ix2], mv.px, mv.uo,
                                                        mv.vo, mv.wo, mv.dens, ctx->xc_dev, s->w, s->theta, s->meta,
                                                        fallback, ctx->f[EDDY_TV], kappa, mv.tv, mv.kv, mv.px,
                                                        s->counts, ctx->err_flag);
  } else {
    EDDY_CUDA(cudaFuncSetAttribute(k_mlp_infer<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_mlp_infer<double><<<grid, IT, smem, ctx->stream>>>(d, ctx->m, cg, ctx->sc.grav, xu[1], xu[d.ix2], d.nx,
                                                         ctx->f[EDDY_UO], ctx->f[EDDY_VO], ctx->f[EDDY_WO],
                                                         ctx->f[EDDY_DENS], ctx->xc_dev, s->w, s->theta, s->meta,
                                                         fallback, ctx->f[EDDY_TV], kappa, nullptr, nullptr, 0,
                                                         s->counts, ctx->err_flag);
  }
  EDDY_LAUNCHED(ctx);
  if (out_of_envelope)
    EDDY_CUDA(cudaMemcpyAsync(out_of_envelope, s->counts, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                              ctx->stream));
  return EDDY_OK;
}
