// k_xform64.cu -- the x eigen-transforms of the Poisson solve (the dense part
// of the per-wavenumber solve that replaces BLKTRI, src/direct.f:788-870) on
// the FP64 tensor cores (mma.sync m8n8k4 .f64), with FP64 accumulation.
//
// Every spectral line (one (J,k) pair, M contiguous values) is multiplied by
// the same M x M matrix: forward Af (x values -> mode coefficients), backward
// Ab (modes -> x values).  When the x operator is mirror-symmetric (a grid
// symmetric about its centre with the same boundary type at both ends; found
// at plan time to 1e-9) every eigenvector is even or odd, so with the modes
// ordered even then odd each transform is two H x H products (H = M/2):
//   forward  C_even = E^T (S_top + flip S_bot),  C_odd = O^T (S_top - flip S_bot)
//   backward X_top = E Y_even + O Y_odd,         X_bot = flip(E Y_even - O Y_odd)
// which halves the multiply-adds.  Otherwise one M x M product.
//
// A CTA takes 32 lines and, one parity after the other, stages them (mirrored
// into sums or differences for the forward transform) in shared memory, then
// streams that parity's matrix through a double-buffered cp.async ring in
// chunks of 8 along the reduction index (84 KB of shared memory at M = 384:
// two CTAs per SM).  Warp w owns m-tiles w, w+8, ... of both parities, so the
// backward transform forms E+O and E-O in registers.  Input and output may be
// FP64 (the plain form) or FP32 (the mixed form's correction solves on grids
// its TF32 tensor-core transform does not take); arithmetic is FP64.
#include <cmath>
#include <vector>

#include "eddy_internal.h"

namespace {

constexpr int NL = 32;    // lines per CTA
constexpr int KC = 8;     // reduction-index chunk
constexpr int AS = 12;    // shared row stride of a matrix chunk (96 B: conflict-free fragment loads)
constexpr int NT = 256;   // threads (8 warps)

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// D = A (8x4, row) * B (4x8, col) + C; lane l holds A[l/4][l%4], B[l%4][l/4],
// C/D[l/4][2(l%4)], [l/4][2(l%4)+1]
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// NP = 2: split form (Hp = padded H, K = H); NP = 1: one product (Hp = padded
// M, K = M).  The parities run one after the other through the same shared
// buffers (half the footprint: two CTAs per SM); the backward transform keeps
// the even part in registers until the odd one is done.
template <int NP, int MT, int DIR, class TI, class TO>
__global__ void __launch_bounds__(NT, NP * MT >= 7 ? 1 : 2)
    k_xform64(int M, int Hp, long long nlines, const double *__restrict__ A, const TI *__restrict__ in,
              TO *__restrict__ out) {
  extern __shared__ __align__(16) double smx[];
  const int KS = Hp + 4;               // B row stride (Hp is a multiple of 8)
  double *Bs = smx;                    // [NL][KS]
  double *Asm = smx + (size_t)NL * KS; // [2][Hp][AS]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, t4 = lane & 3;
  const long long l0 = (long long)blockIdx.x * NL;
  const int H = NP == 2 ? M / 2 : M;   // valid rows / reduction length
  const int nch = Hp / KC;
  const size_t chunk = (size_t)Hp * KC; // doubles per matrix chunk in global

  double acc[NP][MT][4][2];
#pragma unroll
  for (int p = 0; p < NP; p++)
#pragma unroll
    for (int j = 0; j < MT; j++)
#pragma unroll
      for (int n = 0; n < 4; n++) acc[p][j][n][0] = acc[p][j][n][1] = 0.;

#pragma unroll
  for (int p = 0; p < NP; p++) {
    const double *Ap = A + (size_t)p * nch * chunk;
    auto issue = [&](int c) {
      if (c < nch) {
        double *dst = Asm + (size_t)(c & 1) * Hp * AS;
        const double *src = Ap + (size_t)c * chunk;
        for (int e = threadIdx.x; e < Hp * (KC / 2); e += NT) {
          const int r = e / (KC / 2), q = e % (KC / 2);
          cp_async16(dst + (size_t)r * AS + 2 * q, src + (size_t)r * KC + 2 * q);
        }
      }
      cp_commit();
    };
    if (p > 0) __syncthreads();  // the previous parity's readers are done with both buffers
    issue(0);
    // the 32 lines of this parity (forward split: sums for the even part,
    // differences for the odd one); each thread issues a batch of loads
    // before its first shared store
    constexpr int UB = 8;
    for (int e0 = threadIdx.x; e0 < NL * Hp; e0 += NT * UB) {
      double v0[UB], v1[UB];
#pragma unroll
      for (int u = 0; u < UB; u++) {
        const int e = e0 + u * NT;
        const int l = e / Hp, k = e % Hp;
        const long long line = l0 + l;
        v0[u] = 0.;
        v1[u] = 0.;
        if (e < NL * Hp && line < nlines && k < H) {
          const TI *src = in + line * (long long)M;
          if (NP == 2 && DIR == 0) {
            v0[u] = (double)src[k];
            v1[u] = (double)src[M - 1 - k];
          } else {
            v0[u] = (double)src[p * H + k];
          }
        }
      }
#pragma unroll
      for (int u = 0; u < UB; u++) {
        const int e = e0 + u * NT;
        if (e >= NL * Hp) break;
        const int l = e / Hp, k = e % Hp;
        Bs[(size_t)l * KS + k] = (NP == 2 && DIR == 0) ? (p == 0 ? v0[u] + v1[u] : v0[u] - v1[u]) : v0[u];
      }
    }
    issue(1);
    for (int c = 0; c < nch; c++) {
      cp_wait<1>();
      __syncthreads();
      const double *As = Asm + (size_t)(c & 1) * Hp * AS;
#pragma unroll
      for (int kk = 0; kk < KC; kk += 4) {
        double a[MT], b[4];
#pragma unroll
        for (int j = 0; j < MT; j++) {
          const int mt = w + 8 * j;
          a[j] = mt * 8 < Hp ? As[(size_t)(mt * 8 + g) * AS + kk + t4] : 0.;
        }
#pragma unroll
        for (int n = 0; n < 4; n++) b[n] = Bs[(size_t)(n * 8 + g) * KS + c * KC + kk + t4];
#pragma unroll
        for (int j = 0; j < MT; j++)
          if ((w + 8 * j) * 8 < Hp) {
#pragma unroll
            for (int n = 0; n < 4; n++) dmma(acc[p][j][n][0], acc[p][j][n][1], a[j], b[n]);
          }
      }
      __syncthreads();  // every warp is done with this buffer
      issue(c + 2);
    }
    cp_wait<0>();
    // lane: row g of each m-tile, lines 2*t4 and 2*t4+1 of each line tile.
    // Modes (forward, or the unsplit product) are stored per parity; the
    // split backward transform combines both parities after the last one.
    if (DIR == 0 || NP == 1 || p == NP - 1) {
#pragma unroll
      for (int j = 0; j < MT; j++) {
        const int m = (w + 8 * j) * 8 + g;
        if (m >= H) continue;
#pragma unroll
        for (int n = 0; n < 4; n++)
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const long long line = l0 + n * 8 + 2 * t4 + e;
            if (line >= nlines) continue;
            TO *dst = out + line * (long long)M;
            if (DIR == 0 || NP == 1) {
              dst[p * H + m] = (TO)acc[p][j][n][e];
            } else {
              const double E = acc[0][j][n][e], O = acc[NP - 1][j][n][e];
              dst[m] = (TO)(E + O);
              dst[M - 1 - m] = (TO)(E - O);
            }
          }
      }
    }
  }
}

size_t xform64_smem(int hp) { return sizeof(double) * ((size_t)NL * (hp + 4) + (size_t)2 * hp * AS); }

template <int NP, int MT, int DIR, class TI, class TO>
int launch_t(eddy_ctx *ctx, const double *A, const TI *in, TO *out) {
  const PoissonPlan &pp = ctx->pp;
  const long long nlines = (long long)pp.L * pp.N;
  const size_t smem = xform64_smem(pp.dHp);
  EDDY_CUDA(cudaFuncSetAttribute(k_xform64<NP, MT, DIR, TI, TO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  const unsigned grid = (unsigned)((nlines + NL - 1) / NL);
  k_xform64<NP, MT, DIR, TI, TO><<<grid, NT, smem, ctx->stream>>>(pp.M, pp.dHp, nlines, A, in, out);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

template <int DIR, class TI, class TO>
int dispatch(eddy_ctx *ctx, const TI *in, TO *out) {
  const PoissonPlan &pp = ctx->pp;
  const double *A = pp.dA[DIR];
  const int mt = (pp.dHp / 8 + 7) / 8;
  if (pp.dsym) {
    switch (mt) {
      case 1: return launch_t<2, 1, DIR>(ctx, A, in, out);
      case 2: return launch_t<2, 2, DIR>(ctx, A, in, out);
      case 3: return launch_t<2, 3, DIR>(ctx, A, in, out);
      case 4: return launch_t<2, 4, DIR>(ctx, A, in, out);
    }
  } else {
    switch (mt) {
      case 1: return launch_t<1, 1, DIR>(ctx, A, in, out);
      case 2: return launch_t<1, 2, DIR>(ctx, A, in, out);
      case 3: return launch_t<1, 3, DIR>(ctx, A, in, out);
      case 4: return launch_t<1, 4, DIR>(ctx, A, in, out);
      case 5: return launch_t<1, 5, DIR>(ctx, A, in, out);
      case 6: return launch_t<1, 6, DIR>(ctx, A, in, out);
      case 7: return launch_t<1, 7, DIR>(ctx, A, in, out);
    }
  }
  ctx->err = "x transform: unsupported size";
  return EDDY_EINVAL;
}

}  // namespace

// Split (or plain) transform matrices in [parity][chunk][row][KC] order,
// rows zero-padded to Hp, the reduction index zero-padded to Hp; the
// eigenvalues and the null mode in the transforms' mode order.
int xform64_prepare(eddy_ctx *ctx, const std::vector<double> &Af, const std::vector<double> &Ab,
                    const std::vector<double> &lam) {
  PoissonPlan &pp = ctx->pp;
  const int M = pp.M, H = M / 2;
  auto af = [&](int n, int x) { return Af[(size_t)n + (size_t)M * x]; };  // Af(n, x)
  auto ab = [&](int x, int n) { return Ab[(size_t)x + (size_t)M * n]; };  // Ab(x, n)
  std::vector<int> even, odd;
  bool sym = M % 2 == 0;
  for (int n = 0; n < M && sym; n++) {
    double dot = 0., mf = 0., mb = 0.;
    for (int x = 0; x < M; x++) {
      dot += af(n, x) * af(n, M - 1 - x);
      mf = std::fmax(mf, std::fabs(af(n, x)));
      mb = std::fmax(mb, std::fabs(ab(x, n)));
    }
    const double sg = dot >= 0. ? 1. : -1.;
    for (int x = 0; x < M && sym; x++) {
      if (std::fabs(af(n, x) - sg * af(n, M - 1 - x)) > 1e-9 * mf) sym = false;
      if (std::fabs(ab(x, n) - sg * ab(M - 1 - x, n)) > 1e-9 * mb) sym = false;
    }
    (sg > 0. ? even : odd).push_back(n);
  }
  if (sym && ((int)even.size() != H || (int)odd.size() != H)) sym = false;
  const int np = sym ? 2 : 1, K = sym ? H : M;
  const int hp = (K + 7) / 8 * 8;
  if ((sym && hp > 256) || (!sym && hp > 448)) {
    ctx->err = "x transform: NX-2 too large for the tensor-core transform (split form up to 512, else 448)";
    return EDDY_EINVAL;
  }
  std::vector<int> perm(M);
  for (int m = 0; m < M; m++) perm[m] = m;
  if (sym) {
    for (int m = 0; m < H; m++) { perm[m] = even[m]; perm[H + m] = odd[m]; }
  }
  const int nch = hp / KC;
  std::vector<double> F((size_t)np * nch * hp * KC, 0.), B(F.size(), 0.);
  for (int p = 0; p < np; p++)
    for (int r = 0; r < K; r++)
      for (int k = 0; k < K; k++) {
        const size_t o = (((size_t)p * nch + (size_t)(k / KC)) * hp + (size_t)r) * KC + k % KC;
        if (sym) {
          F[o] = af(perm[p * H + r], k);  // row: mode r of parity p, column: x
          B[o] = ab(r, perm[p * H + k]);  // row: x, column: mode k of parity p
        } else {
          F[o] = af(r, k);
          B[o] = ab(r, k);
        }
      }
  std::vector<double> lp(M);
  int m0 = pp.m0;
  for (int m = 0; m < M; m++) {
    lp[m] = lam[perm[m]];
    if (perm[m] == pp.m0) m0 = m;
  }
  pp.dsym = sym ? 1 : 0;
  pp.dHp = hp;
  pp.dm0 = m0;
  const size_t bytes = sizeof(double) * F.size();
  EDDY_CUDA(cudaMalloc(&pp.dA[0], bytes));
  EDDY_CUDA(cudaMalloc(&pp.dA[1], bytes));
  EDDY_CUDA(cudaMalloc(&pp.dlam, sizeof(double) * M));
  EDDY_CUDA(cudaMemcpy(pp.dA[0], F.data(), bytes, cudaMemcpyHostToDevice));
  EDDY_CUDA(cudaMemcpy(pp.dA[1], B.data(), bytes, cudaMemcpyHostToDevice));
  EDDY_CUDA(cudaMemcpy(pp.dlam, lp.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
  return EDDY_OK;
}

int launch_xform64(eddy_ctx *ctx, int dir, const double *in, double *out) {
  return dir == 0 ? dispatch<0>(ctx, in, out) : dispatch<1>(ctx, in, out);
}

int launch_xform64_f32(eddy_ctx *ctx, int dir, const float *in, float *out) {
  return dir == 0 ? dispatch<0>(ctx, in, out) : dispatch<1>(ctx, in, out);
}
