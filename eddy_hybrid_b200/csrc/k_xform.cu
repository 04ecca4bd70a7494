// k_xform.cu -- the x eigen-transforms of the mixed-precision Poisson solve on
// the 5th-generation tensor cores.
//
// Out[p][n] = sum_k In[p][k] B[n][k] for all P = L*N spectral lines p (the
// (J,k) lines of the solve, x index contiguous), K = N = M = NX-2.  Storage is
// FP32; products use the 3xTF32 split (a = a_hi + a_lo with a_hi the TF32
// truncation): A_hi B_hi + A_hi B_lo + A_lo B_hi, accumulated in FP32 in TMEM by
// tcgen05.mma kind::tf32, which keeps the transform at FP32 accuracy (the
// refinement sweeps then see the same convergence as with an FP32 GEMM).
//
// One CTA per 128-line tile, all M outputs (TMEM columns 0..M-1, M <= 512).
// K is streamed in chunks of 16 through a 3-stage shared-memory pipeline:
// the A chunk arrives by four 2-D TMA boxes (16 bytes x 128 lines each) so
// shared memory holds it in the canonical no-swizzle K-major layout
// [k/4][line][4]; the B chunks (prepared on the host in that layout, hi and
// lo) arrive by 1-D bulk copies.  The CTA splits A into hi/lo in shared
// memory, one thread issues the MMAs and commits them to the stage's "empty"
// barrier; the epilogue reads TMEM (lane = line) and stores rows.
#include <cstring>
#include <vector>

#include "eddy_internal.h"
#include "tma_ring.cuh"
#include "umma.cuh"

namespace {

constexpr int XT = 128;  // threads per CTA
constexpr int KC = 16;   // K per pipeline stage

__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          tma::smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(tma::smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(tma::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(tma::smem_u32(bar))
      : "memory");
}

// kind::tf32 instruction descriptor: D f32, A/B tf32, both K-major
__device__ __forceinline__ uint32_t idesc_tf32(int M, int N) {
  uint32_t d = 0;
  d |= 1u << 4;                   // D format f32
  d |= 2u << 7;                   // A format tf32
  d |= 2u << 10;                  // B format tf32
  d |= (uint32_t)(N >> 3) << 17;  // N / 8
  d |= (uint32_t)(M >> 4) << 24;  // M / 16
  return d;
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

struct StageGeom {
  int nn;             // outputs (= M)
  uint32_t a_bytes;   // 128 x KC floats
  uint32_t b_bytes;   // nn x KC floats (one of hi / lo)
  uint32_t stage;     // bytes per stage: A, A_lo, B_hi, B_lo
};

__host__ __device__ inline StageGeom stage_geom(int nn) {
  StageGeom g;
  g.nn = nn;
  g.a_bytes = 128u * KC * 4u;
  g.b_bytes = (uint32_t)nn * KC * 4u;
  g.stage = 2u * g.a_bytes + 2u * g.b_bytes;
  return g;
}

__global__ void __launch_bounds__(XT, 1)
    k_xform_tf32(const __grid_constant__ CUtensorMap amap, const float *__restrict__ bhi,
                 const float *__restrict__ blo, float *__restrict__ out, long long P, int M, int nst, int *err) {
  extern __shared__ __align__(1024) unsigned char xsm[];
  __shared__ __align__(8) uint64_t full[4], empty[4];
  __shared__ uint32_t tmem_base;
  unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(xsm) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5;
  const StageGeom G = stage_geom(M);
  const int nch = M / KC;
  const long long p0 = (long long)blockIdx.x * 128;
  const int part0 = M < 256 ? M : 256, part1 = M - part0;
  uint32_t ncols = 64;
  while ((int)ncols < M) ncols <<= 1;
  if (warp == 0) {
    umma::tmem_alloc(&tmem_base, ncols);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    for (int s = 0; s < nst; s++) {
      umma::mbar_init(&full[s], 1);
      umma::mbar_init(&empty[s], 1);
    }
    tma::fence_mbar_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tm = tmem_base;
  auto st_a = [&](int s) { return base + (size_t)s * G.stage; };
  auto st_alo = [&](int s) { return base + (size_t)s * G.stage + G.a_bytes; };
  auto st_bhi = [&](int s) { return base + (size_t)s * G.stage + 2 * G.a_bytes; };
  auto st_blo = [&](int s) { return base + (size_t)s * G.stage + 2 * G.a_bytes + G.b_bytes; };
  auto issue = [&](int c) {
    const int s = c % nst;
    tma::mbar_expect_tx(&full[s], G.a_bytes + 2 * G.b_bytes);
    for (int q = 0; q < KC / 4; q++)
      load_2d(st_a(s) + q * 128 * 16, &amap, c * KC + 4 * q, (int)p0, &full[s]);
    const size_t boff = (size_t)c * (KC / 4) * M * 4;  // floats
    bulk_load(st_bhi(s), bhi + boff, G.b_bytes, &full[s]);
    bulk_load(st_blo(s), blo + boff, G.b_bytes, &full[s]);
  };
  if (tid == 0)
    for (int c = 0; c < nst && c < nch; c++) issue(c);
  const uint32_t id0 = idesc_tf32(128, part0), id1 = part1 ? idesc_tf32(128, part1) : 0u;
  const uint32_t lbo_a = 128 * 16, lbo_b = (uint32_t)M * 16;
  bool ok = true;
  int c = 0;
  for (; c < nch; c++) {
    const int s = c % nst;
    ok = tma::mbar_wait(&full[s], (c / nst) & 1);
    if (__syncthreads_or(ok ? 0 : 1)) { ok = false; break; }
    // split A into TF32 hi (in place) and lo
    float4 *a4 = reinterpret_cast<float4 *>(st_a(s));
    float4 *l4 = reinterpret_cast<float4 *>(st_alo(s));
    for (int e = tid; e < 128 * KC / 4; e += XT) {
      float4 v = a4[e], h, l;
      h.x = __uint_as_float(__float_as_uint(v.x) & 0xFFFFE000u); l.x = v.x - h.x;
      h.y = __uint_as_float(__float_as_uint(v.y) & 0xFFFFE000u); l.y = v.y - h.y;
      h.z = __uint_as_float(__float_as_uint(v.z) & 0xFFFFE000u); l.z = v.z - h.z;
      h.w = __uint_as_float(__float_as_uint(v.w) & 0xFFFFE000u); l.w = v.w - h.w;
      a4[e] = h;
      l4[e] = l;
    }
    umma::fence_smem_to_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (tid == 0) {
      for (int ks = 0; ks < KC / 8; ks++) {
        const uint32_t ko = ks * 2;  // two k-groups of 4 per MMA
        uint64_t ah = umma::make_desc(st_a(s) + ko * lbo_a, lbo_a, 128);
        uint64_t al = umma::make_desc(st_alo(s) + ko * lbo_a, lbo_a, 128);
        const uint32_t first = (c == 0 && ks == 0) ? 0u : 1u;
        for (int part = 0; part < (part1 ? 2 : 1); part++) {
          const uint32_t boff = ko * lbo_b + (part ? part0 * 16 : 0);
          uint64_t bh = umma::make_desc(st_bhi(s) + boff, lbo_b, 128);
          uint64_t bl = umma::make_desc(st_blo(s) + boff, lbo_b, 128);
          const uint32_t d = tm + (part ? (uint32_t)part0 : 0u);
          const uint32_t id = part ? id1 : id0;
          mma_tf32(d, ah, bh, id, first);
          mma_tf32(d, ah, bl, id, 1u);
          mma_tf32(d, al, bh, id, 1u);
        }
      }
      umma::commit(&empty[s]);
      // refill the stage the previous chunk used, once its MMAs are done
      if (c >= 1 && c - 1 + nst < nch) {
        const int sp = (c - 1) % nst;
        if (!umma::mbar_wait(&empty[sp], ((c - 1) / nst) & 1)) {
          atomicExch(err, 1);
        } else {
          issue(c - 1 + nst);
        }
      }
    }
  }
  // all MMAs complete: the last chunk's commit covers every earlier MMA
  bool done = false;
  if (ok && c == nch) done = umma::mbar_wait(&empty[(nch - 1) % nst], ((nch - 1) / nst) & 1);
  if (!done && tid == 0) {
    atomicExch(err, 1);
    // bounded waits for the copies and MMAs that may still be in flight
    const int cf = c < nch ? c : nch - 1;
    for (int q = cf; q < nch && q <= cf + nst - 2; q++) tma::mbar_wait(&full[q % nst], (q / nst) & 1, 1u << 20);
    if (cf >= 1) umma::mbar_wait(&empty[(cf - 1) % nst], ((cf - 1) / nst) & 1, 1u << 20);
  }
  done = __syncthreads_and(done ? 1 : 0) != 0;
  umma::fence_after_sync();
  if (done) {
    const long long row = p0 + warp * 32 + (tid & 31);
    for (int c0 = 0; c0 < M; c0 += 64) {
      uint32_t r[64];
      umma::tmem_ld64(tm + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
      if (row < P) {
        float4 *dst = reinterpret_cast<float4 *>(out + row * M + c0);
        const int nv = (M - c0 < 64 ? M - c0 : 64) / 4;
#pragma unroll
        for (int q = 0; q < 16; q++)
          if (q < nv)
            dst[q] = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                                 __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tm, ncols);
}

}  // namespace

// Device B matrices (hi, lo) in the [k/4][n][4] layout from a column-major
// M x M FP64 matrix T with B[n][k] = T(n, k).
int xform_prepare(eddy_ctx *ctx, const double *T_dev, float **bhi, float **blo) {
  const int M = ctx->pp.M;
  std::vector<double> T((size_t)M * M);
  EDDY_CUDA(cudaMemcpy(T.data(), T_dev, sizeof(double) * T.size(), cudaMemcpyDeviceToHost));
  std::vector<float> hi((size_t)M * M), lo((size_t)M * M);
  for (int n = 0; n < M; n++)
    for (int k = 0; k < M; k++) {
      double x = T[(size_t)n + (size_t)M * k];
      float f = (float)x;
      uint32_t u;
      std::memcpy(&u, &f, 4);
      u &= 0xFFFFE000u;
      float h;
      std::memcpy(&h, &u, 4);
      float l = (float)(x - (double)h);
      size_t o = ((size_t)(k / 4) * M + n) * 4 + (k % 4);
      hi[o] = h;
      lo[o] = l;
    }
  EDDY_CUDA(cudaMalloc(bhi, sizeof(float) * hi.size()));
  EDDY_CUDA(cudaMalloc(blo, sizeof(float) * lo.size()));
  EDDY_CUDA(cudaMemcpy(*bhi, hi.data(), sizeof(float) * hi.size(), cudaMemcpyHostToDevice));
  EDDY_CUDA(cudaMemcpy(*blo, lo.data(), sizeof(float) * lo.size(), cudaMemcpyHostToDevice));
  return EDDY_OK;
}

bool xform_supported(int M) { return M >= 16 && M <= 512 && M % 16 == 0; }

static int xform_stages(int M) {
  size_t st = stage_geom(M).stage;
  return (3 * st + 2048 <= 227 * 1024) ? 3 : 2;
}

// out (P x M) = in (P x M) * B^T on the tensor cores
int launch_xform(eddy_ctx *ctx, const float *in, float *out, const float *bhi, const float *blo) {
  const int M = ctx->pp.M;
  const long long P = (long long)ctx->pp.L * ctx->pp.N;
  const CUtensorMap *mp = nullptr;
  for (TmaEntry &e : ctx->tmaps)
    if (e.ptr == in && e.bx == 4 && e.by == -128) mp = &e.map;
  if (!mp) {
    TmaEntry e;
    e.ptr = in;
    e.bx = 4;
    e.by = -128;  // key: 2-D (M, P) view with a 4 x 128 box
    int r = make_tensor_map_2d(&e.map, in, M, P, 4, 128);
    if (r != 0) {
      ctx->err = "cuTensorMapEncodeTiled (transform) failed (" + std::to_string(r) + ")";
      return EDDY_ECUDA;
    }
    ctx->tmaps.push_back(e);
    mp = &ctx->tmaps.back().map;
  }
  const int nst = xform_stages(M);
  const size_t smem = (size_t)nst * stage_geom(M).stage + 1024;
  EDDY_CUDA(cudaFuncSetAttribute(k_xform_tf32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const unsigned grid = (unsigned)((P + 127) / 128);
  k_xform_tf32<<<grid, XT, smem, ctx->stream>>>(*mp, bhi, blo, out, P, M, nst, ctx->err_flag);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}
