// k_poisson.cu -- pressure Poisson solve DIRECT (src/direct.f:2-1118) on one
// GPU, replacing the z-slab MPI transposes (direct.f:651,989) by layout:
//
//   1. divergence/alfxdt fused with the forward real FFT along y (packed
//      FFTPACK order, src/fftpack.f RFFTF) -> spectral array S[k][J][i]
//   2. eigen-transform of the stretched x operator over all (J,k) lines,
//      G = Af * S  (Af = Q^T D^-1/2, D = diag(ap)), on the FP64 tensor cores
//      (k_xform64.cu; even/odd split for a mirror-symmetric operator)
//   3. per (m,J) line a tridiagonal (Thomas) solve along stretched z with
//      diagonal bn(k) + lambda_m - AK(J); the Neumann null mode (J=0, m=m0)
//      is pinned by dropping its first z equation
//   4. back-transform X = Ab * Y (Ab = D^1/2 Q), zero-mean J=0 plane
//      (direct.f:895-898)
//   5. /L and backward real FFT (direct.f:1036, RFFTB) -> DP interior, DIRECT's
//      ghost convention (direct.f:1090-1106).
// The FFT is a radix-2 decimation-in-time in shared memory; lengths must be
// powers of two.
#include <cmath>
#include <vector>

#include "eddy_internal.h"

namespace {

constexpr int TI = 16;     // lines (consecutive i) per FFT block
constexpr int FT = 256;    // threads per FFT block

#include "fft_lines.cuh"

// Step 1.  mode 0: f = divergence(us,vs,ws)/alfxdt (src/timeindeg.f:941-949,
// src/Eddy6.f:2715); mode 1: f = rhs interior.
__global__ void __launch_bounds__(FT, 3)
    k_div_fft_fwd(Dims d, DevMetrics m, const double *__restrict__ us, const double *__restrict__ vs,
                  const double *__restrict__ ws, const double *__restrict__ rhs, int mode, double alfxdt,
                  int code, const double *__restrict__ twr, const double *__restrict__ twi,
                  double *__restrict__ spec) {
  extern __shared__ double sm[];
  const int L = fft_len(code), M = d.nx - 2;
  double *re = sm, *im = sm + L * TI;
  double *tsr = sm + 2 * L * TI, *tsi = tsr + L / 2;
  load_twiddles(tsr, tsi, twr, twi, L / 2);
  int i0 = d.ix1 + blockIdx.x * TI;
  int k = d.kz1 + blockIdx.y;
  // gathers batched U per thread (loads issued before the shared stores)
  constexpr int U = 8;
  const int NT = L * TI;
  for (int t0 = threadIdx.x; t0 < NT; t0 += FT * U) {
    double v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * FT;
      const int ii = t % TI, jj = t / TI;
      const int i = i0 + ii, j = d.jy1 + jj;
      v[u] = 0.;
      if (t < NT && i <= d.ix2) {
        if (mode == 0) {
          double x = (m.ap[i] * (us[fidx(d, i, j, k)] - us[fidx(d, i - 1, j, k)]) +
                      m.bp[j] * (vs[fidx(d, i, j, k)] - vs[fidx(d, i, j - 1, k)]) +
                      m.cp[k] * (ws[fidx(d, i, j, k)] - ws[fidx(d, i, j, k - 1)]));
          v[u] = x / alfxdt;
        } else {
          v[u] = rhs[fidx(d, i, j, k)];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * FT;
      if (t < NT) {
        const int ii = t % TI, r = fft_slot(t / TI, code);
        re[r * TI + ii] = v[u];
        im[r * TI + ii] = 0.;
      }
    }
  }
  __syncthreads();
  fft_lines_any<double, TI>(re, im, code, tsr, tsi);
  // packed order [a0, a1, b1, ..., a_{L/2}]
  long long lineK = (long long)(k - d.kz1) * L;
  for (int t = threadIdx.x; t < L * TI; t += blockDim.x) {
    int ii = t % TI, J = t / TI;
    int i = i0 + ii;
    if (i > d.ix2) continue;
    double v;
    if (J == 0) v = re[0 * TI + ii];
    else if (J == L - 1) v = re[(L / 2) * TI + ii];
    else {
      int qq = (J + 1) / 2;
      v = (J & 1) ? re[qq * TI + ii] : im[qq * TI + ii];
    }
    spec[(long long)(i - d.ix1) + (long long)M * (J + lineK)] = v;
  }
}

// Step 5: (S - dpm[J==0]) / L, Hermitian extension, inverse DIT, real part.
__global__ void __launch_bounds__(FT, 3)
    k_fft_bwd(Dims d, const double *__restrict__ spec, const double *__restrict__ dpm, int code,
              const double *__restrict__ twr, const double *__restrict__ twi, double *__restrict__ dp) {
  extern __shared__ double sm[];
  const int L = fft_len(code), M = d.nx - 2;
  double *re = sm, *im = sm + L * TI;
  double *tsr = sm + 2 * L * TI, *tsi = tsr + L / 2;
  load_twiddles(tsr, tsi, twr, twi, L / 2);
  int i0 = d.ix1 + blockIdx.x * TI;
  int k = d.kz1 + blockIdx.y;
  long long lineK = (long long)(k - d.kz1) * L;
  double mean = dpm[0];
  constexpr int U = 8;
  const int NT = L * TI;
  for (int t0 = threadIdx.x; t0 < NT; t0 += FT * U) {
    double xr[U], xi[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * FT;
      const int ii = t % TI, q = t / TI;  // q: complex index 0..L-1
      const int i = i0 + ii;
      xr[u] = 0.;
      xi[u] = 0.;
      if (t < NT && i <= d.ix2) {
        const double *S = spec + (long long)(i - d.ix1);
        auto get = [&](int J) {
          double v = S[(long long)M * (J + lineK)];
          if (J == 0) v = v - mean;
          return v / (double)L;
        };
        if (q == 0) xr[u] = get(0);
        else if (q == L / 2) xr[u] = get(L - 1);
        else if (q < L / 2) { xr[u] = get(2 * q - 1); xi[u] = get(2 * q); }
        else { const int qq = L - q; xr[u] = get(2 * qq - 1); xi[u] = -get(2 * qq); }
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * FT;
      if (t < NT) {
        const int ii = t % TI, r = fft_slot(t / TI, code);
        re[r * TI + ii] = xr[u];
        im[r * TI + ii] = xi[u];
      }
    }
  }
  __syncthreads();
  fft_lines_any<double, TI>(re, im, code, tsr, tsi);
  for (int t = threadIdx.x; t < L * TI; t += blockDim.x) {
    int ii = t % TI, jj = t / TI;
    int i = i0 + ii;
    if (i > d.ix2) continue;
    dp[fidx(d, i, d.jy1 + jj, k)] = re[jj * TI + ii];
  }
}

// Step 3: Thomas along z for each (m,J) line; S laid out [k][J][m].
#include "tridiag_z.cuh"

// Step 4b: mean of the J = 0 plane (M*N values), deterministic two-stage.
__global__ void k_plane_sum_partial(int M, int L, int N, const double *__restrict__ s, double *part) {
  __shared__ double sh[256];
  double acc = 0.;
  long long n = (long long)M * N;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    long long k = t / M, i = t % M;
    acc += s[i + (long long)M * L * k];
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_plane_sum_final(int nparts, long long count, const double *part, double *out) {
  if (threadIdx.x != 0) return;
  double s = 0.;
  for (int b = 0; b < nparts; b++) s += part[b];
  out[0] = s / (double)count;
}

// DIRECT's ghosts: z planes zero, x Neumann copies, y periodic copies.
__global__ void k_dp_ghost(Dims d, double *dp) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long sxy = (long long)d.nx * d.ny, sxz = (long long)d.nx * d.nz, syz = (long long)d.ny * d.nz;
  int i, j, k;
  if (t < 2 * sxy) {
    long long r = t % sxy;
    i = 1 + (int)(r % d.nx); j = 1 + (int)(r / d.nx); k = (t / sxy) ? d.nz : 1;
    dp[fidx(d, i, j, k)] = 0.;
    return;
  } else if (t < 2 * sxy + 2 * sxz) {
    long long u = t - 2 * sxy, r = u % sxz;
    i = 1 + (int)(r % d.nx); k = 1 + (int)(r / d.nx); j = (u / sxz) ? d.ny : 1;
  } else if (t < 2 * sxy + 2 * sxz + 2 * syz) {
    long long u = t - 2 * sxy - 2 * sxz, r = u % syz;
    j = 1 + (int)(r % d.ny); k = 1 + (int)(r / d.ny); i = (u / syz) ? d.nx : 1;
  } else {
    return;
  }
  if (k == 1 || k == d.nz) return;
  int si = (i == 1) ? 2 : (i == d.nx ? d.nx - 1 : i);
  int sj = (j == 1) ? d.ny - 1 : (j == d.ny ? 2 : j);
  dp[fidx(d, i, j, k)] = dp[fidx(d, si, sj, k)];
}

// max |div| over the interior, two-stage
__global__ void k_maxdiv_partial(Dims d, DevMetrics m, const double *u, const double *v, const double *w,
                                 double *part) {
  __shared__ double sh[256];
  double mx = 0.;
  long long mi = d.ix2 - d.ix1 + 1, mj = d.jy2 - d.jy1 + 1, mk = d.kz2 - d.kz1 + 1;
  long long n = mi * mj * mk;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    int i = d.ix1 + (int)(t % mi), j = d.jy1 + (int)((t / mi) % mj), k = d.kz1 + (int)(t / (mi * mj));
    double dv = (m.ap[i] * (u[fidx(d, i, j, k)] - u[fidx(d, i - 1, j, k)]) +
                 m.bp[j] * (v[fidx(d, i, j, k)] - v[fidx(d, i, j - 1, k)]) +
                 m.cp[k] * (w[fidx(d, i, j, k)] - w[fidx(d, i, j, k - 1)]));
    mx = fmax(mx, fabs(dv));
  }
  sh[threadIdx.x] = mx;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_max_final(int nparts, const double *part, double *out) {
  if (threadIdx.x != 0) return;
  double mx = 0.;
  for (int b = 0; b < nparts; b++) mx = fmax(mx, part[b]);
  out[0] = mx;
}

constexpr int NPART = 296;

int solve_from_spec(eddy_ctx *ctx, double *dp) {
  PoissonPlan &pp = ctx->pp;
  const Dims &d = ctx->d;
  int M = pp.M, L = pp.L, N = pp.N;
  int rc;
  {
    ProfScope ps(ctx, PROF_GEMM_FWD);
    if ((rc = launch_xform64(ctx, 0, pp.spec, pp.spec2))) return rc;
  }
  long long nl = (long long)M * L;
  {
    ProfScope ps(ctx, PROF_TRIDIAG);
    // modes in the transforms' order (even then odd when split)
    k_line_mean<double><<<1, 256, 0, ctx->stream>>>(M, L, N, pp.dm0, pp.wz, pp.spec2, ctx->scal + 5);
    EDDY_LAUNCHED(ctx);
    // the eliminated right-hand side overwrites the spectrum in place
    k_tridiag_lines<double, double, 8, false><<<(unsigned)((nl + 127) / 128), 128, 0, ctx->stream>>>(
        M, L, N, pp.dm0, pp.dlam, pp.ak, pp.an, pp.bn, pp.cn, ctx->scal + 5, pp.spec2, pp.cprime, pp.spec2);
    EDDY_LAUNCHED(ctx);
  }
  {
    ProfScope ps(ctx, PROF_GEMM_BWD);
    if ((rc = launch_xform64(ctx, 1, pp.spec2, pp.spec))) return rc;
  }
  ProfScope psb(ctx, PROF_FFT_BWD);
  k_plane_sum_partial<<<NPART, 256, 0, ctx->stream>>>(M, L, N, pp.spec, pp.red);
  EDDY_LAUNCHED(ctx);
  k_plane_sum_final<<<1, 32, 0, ctx->stream>>>(NPART, (long long)M * N, pp.red, ctx->scal + 3);
  EDDY_LAUNCHED(ctx);
  const int code = fft_code(L);
  size_t smem = sizeof(double) * (2 * L * TI + L);
  dim3 g((M + TI - 1) / TI, N);
  k_fft_bwd<<<g, FT, smem, ctx->stream>>>(d, pp.spec, ctx->scal + 3, code, pp.twr + L / 2, pp.twi + L / 2, dp);
  EDDY_LAUNCHED(ctx);
  long long ng = 2LL * d.nx * d.ny + 2LL * d.nx * d.nz + 2LL * d.ny * d.nz;
  k_dp_ghost<<<(unsigned)((ng + 255) / 256), 256, 0, ctx->stream>>>(d, dp);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

}  // namespace

int poisson_plan_create(eddy_ctx *ctx) {
  PoissonPlan &pp = ctx->pp;
  const Dims &d = ctx->d;
  int M = d.nx - 2, L = d.ny - 2, N = d.nz - 2;
  pp.M = M; pp.L = L; pp.N = N;
  if (d.mp != 1 || d.np != 1 || d.lp != 0) {
    ctx->err = "DIRECT on the device needs Neumann x and z and periodic y";
    return EDDY_EINVAL;
  }
  if (fft_code(L) < 0) {
    ctx->err = "the periodic (FFT) extent NY-2 must be 2^m or 3 x 2^m (m >= 1)";
    return EDDY_EINVAL;
  }
  if (M < 3 || N < 3) { ctx->err = "grid too small"; return EDDY_EINVAL; }
  const std::vector<double> &ap = ctx->h[2], &au = ctx->h[3], &cp = ctx->h[14], &cw = ctx->h[17];
  // coefficients of direct.f:337-379 (interior numbering)
  std::vector<double> am(M), bm(M), cm(M), an(N), bn(N), cn(N);
  for (int i = 0; i < M; i++) { am[i] = ap[i + 2] * au[i + 1]; cm[i] = ap[i + 2] * au[i + 2]; }
  am[0] = 0.; cm[M - 1] = 0.;
  for (int i = 0; i < M; i++) bm[i] = -am[i] - cm[i];
  for (int k = 0; k < N; k++) { an[k] = cp[k + 2] * cw[k + 1]; cn[k] = cp[k + 2] * cw[k + 2]; }
  an[0] = 0.; cn[N - 1] = 0.;
  for (int k = 0; k < N; k++) bn[k] = -an[k] - cn[k];
  // symmetrised x operator S = D^1/2 T D^1/2, tridiagonal
  std::vector<double> sq(M), dd(M), ee(M > 1 ? M - 1 : 1), Q;
  for (int i = 0; i < M; i++) sq[i] = std::sqrt(ap[i + 2]);
  for (int i = 0; i < M; i++) dd[i] = bm[i];
  for (int i = 0; i < M - 1; i++) ee[i] = sq[i] * sq[i + 1] * au[i + 2];
  // A mirror-symmetric operator (the same entries read from either end, bit
  // for bit) has even and odd eigenvectors [u; flip u] / sqrt 2 and
  // [u; -flip u] / sqrt 2, u the eigenvectors of the upper half with the
  // coupling across the middle added to / subtracted from its last diagonal
  // entry.  Solving the two half-size problems makes the symmetry exact, which
  // the transforms' even/odd split relies on.
  bool mirror = M % 2 == 0 && M >= 4;
  for (int i = 0; i < M && mirror; i++) mirror = dd[i] == dd[M - 1 - i] && sq[i] == sq[M - 1 - i];
  for (int i = 0; i < M - 1 && mirror; i++) mirror = ee[i] == ee[M - 2 - i];
  if (mirror) {
    const int H = M / 2;
    Q.assign((size_t)M * M, 0.);
    std::vector<double> lamv(M);
    for (int par = 0; par < 2; par++) {
      std::vector<double> dh(dd.begin(), dd.begin() + H), eh(ee.begin(), ee.begin() + (H > 1 ? H - 1 : 1)), Qh;
      dh[H - 1] = par == 0 ? dh[H - 1] + ee[H - 1] : dh[H - 1] - ee[H - 1];
      if (tridiag_eigen(H, dh, eh, Qh) != 0) {
        ctx->err = "x-operator eigensolver did not converge";
        return EDDY_ESINGULAR;
      }
      const double r2 = 1.0 / std::sqrt(2.0);
      for (int m = 0; m < H; m++) {
        lamv[par * H + m] = dh[m];
        for (int i = 0; i < H; i++) {
          const double v = Qh[(size_t)i * H + m] * r2;
          Q[(size_t)i * M + par * H + m] = v;
          Q[(size_t)(M - 1 - i) * M + par * H + m] = par == 0 ? v : -v;
        }
      }
    }
    dd = lamv;
  } else if (tridiag_eigen(M, dd, ee, Q) != 0) {
    ctx->err = "x-operator eigensolver did not converge";
    return EDDY_ESINGULAR;
  }
  // the null mode (constant pressure along x): exact eigenvalue 0 and the
  // exact normalised vector D^-1/2 1 (even, so it stays in the even set)
  int m0 = 0;
  for (int mm = 1; mm < M; mm++) if (std::fabs(dd[mm]) < std::fabs(dd[m0])) m0 = mm;
  dd[m0] = 0.;
  double nrm = 0.;
  for (int i = 0; i < M; i++) nrm += 1. / ap[i + 2];
  nrm = std::sqrt(nrm);
  double sgn = Q[(size_t)0 * M + m0] >= 0 ? 1. : -1.;
  for (int i = 0; i < M; i++) Q[(size_t)i * M + m0] = sgn / (sq[i] * nrm);
  pp.m0 = m0;
  std::vector<double> Af((size_t)M * M), Ab((size_t)M * M);
  for (int i = 0; i < M; i++)
    for (int mm = 0; mm < M; mm++) {
      double q = Q[(size_t)i * M + mm];
      Af[(size_t)mm + (size_t)M * i] = q / sq[i];  // Af(m,i), column-major
      Ab[(size_t)i + (size_t)M * mm] = sq[i] * q;  // Ab(i,m)
    }
  // modified wavenumbers (direct.f:321-331) per packed index J (0-based)
  std::vector<double> akv(L);
  for (int J = 0; J < L; J++) {
    int kk = (J + 1) / 2;  // packed index J+1 (1-based) -> wavenumber (J+1)/2
    double a = (kk < L / 2) ? 2. * M_PI * kk : -2. * M_PI * (L - kk);
    akv[J] = 2. * (1. - std::cos(a / (double)L)) / ctx->delysq;
  }
  // twiddles, same expressions as the oracle's DIT (fwd then bwd tables)
  std::vector<double> twr(L), twi(L);
  for (int r = 0; r < L / 2; r++) {
    double angf = -2.0 * M_PI * (double)r / (double)L;
    double angb = 2.0 * M_PI * (double)r / (double)L;
    twr[r] = std::cos(angf); twi[r] = std::sin(angf);
    twr[L / 2 + r] = std::cos(angb); twi[L / 2 + r] = std::sin(angb);
  }
  size_t bytesM2 = sizeof(double) * (size_t)M * M, vol = sizeof(double) * (size_t)M * L * N;
  EDDY_CUDA(cudaMalloc(&pp.Af, bytesM2));
  EDDY_CUDA(cudaMalloc(&pp.Ab, bytesM2));
  EDDY_CUDA(cudaMalloc(&pp.lam, sizeof(double) * M));
  EDDY_CUDA(cudaMalloc(&pp.ak, sizeof(double) * L));
  EDDY_CUDA(cudaMalloc(&pp.an, sizeof(double) * N));
  EDDY_CUDA(cudaMalloc(&pp.bn, sizeof(double) * N));
  EDDY_CUDA(cudaMalloc(&pp.cn, sizeof(double) * N));
  EDDY_CUDA(cudaMalloc(&pp.wz, sizeof(double) * N));
  EDDY_CUDA(cudaMalloc(&pp.twr, sizeof(double) * L));
  EDDY_CUDA(cudaMalloc(&pp.twi, sizeof(double) * L));
  EDDY_CUDA(cudaMalloc(&pp.spec, vol));
  EDDY_CUDA(cudaMalloc(&pp.spec2, vol));
  EDDY_CUDA(cudaMalloc(&pp.cprime, vol));
  EDDY_CUDA(cudaMalloc(&pp.red, sizeof(double) * NPART));
  EDDY_CUDA(cudaMemcpy(pp.Af, Af.data(), bytesM2, cudaMemcpyHostToDevice));
  EDDY_CUDA(cudaMemcpy(pp.Ab, Ab.data(), bytesM2, cudaMemcpyHostToDevice));
  EDDY_CUDA(cudaMemcpy(pp.lam, dd.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
  EDDY_CUDA(cudaMemcpy(pp.ak, akv.data(), sizeof(double) * L, cudaMemcpyHostToDevice));
  EDDY_CUDA(cudaMemcpy(pp.an, an.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  EDDY_CUDA(cudaMemcpy(pp.bn, bn.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  EDDY_CUDA(cudaMemcpy(pp.cn, cn.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  std::vector<double> wz(N);
  for (int k = 0; k < N; k++) wz[k] = 1.0 / cp[k + 2];
  EDDY_CUDA(cudaMemcpy(pp.wz, wz.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  EDDY_CUDA(cudaMemcpy(pp.twr, twr.data(), sizeof(double) * L, cudaMemcpyHostToDevice));
  EDDY_CUDA(cudaMemcpy(pp.twi, twi.data(), sizeof(double) * L, cudaMemcpyHostToDevice));
  int rc = xform64_prepare(ctx, Af, Ab, dd);
  if (rc) return rc;
  size_t smem = sizeof(double) * (2 * L * TI + L);
  if (smem > 48 * 1024) {
    EDDY_CUDA(cudaFuncSetAttribute(k_div_fft_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    EDDY_CUDA(cudaFuncSetAttribute(k_fft_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  return EDDY_OK;
}

int poisson_plan_destroy(eddy_ctx *ctx) {
  PoissonPlan &pp = ctx->pp;
  void *ptrs[] = {pp.Af, pp.Ab, pp.dA[0], pp.dA[1], pp.dlam, pp.lam, pp.ak, pp.an, pp.bn, pp.cn, pp.wz,
                  pp.twr, pp.twi, pp.spec, pp.spec2, pp.cprime, pp.red};
  for (void *p : ptrs) if (p) cudaFree(p);
  pp = PoissonPlan{};
  return EDDY_OK;
}

static int fwd(eddy_ctx *ctx, const double *us, const double *vs, const double *ws, const double *rhs, int mode,
               double alfxdt) {
  PoissonPlan &pp = ctx->pp;
  const Dims &d = ctx->d;
  const int code = fft_code(pp.L);
  size_t smem = sizeof(double) * (2 * pp.L * TI + pp.L);
  dim3 g((pp.M + TI - 1) / TI, pp.N);
  ProfScope ps(ctx, PROF_DIV_FFT);
  k_div_fft_fwd<<<g, FT, smem, ctx->stream>>>(d, ctx->m, us, vs, ws, rhs, mode, alfxdt, code, pp.twr, pp.twi,
                                              pp.spec);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

int launch_direct(eddy_ctx *ctx, const double *us, const double *vs, const double *ws, double alfxdt) {
  int rc = fwd(ctx, us, vs, ws, nullptr, 0, alfxdt);
  if (rc) return rc;
  return solve_from_spec(ctx, ctx->f[EDDY_DP]);
}

int launch_poisson_rhs(eddy_ctx *ctx, const double *rhs, double *dp) {
  int rc = fwd(ctx, nullptr, nullptr, nullptr, rhs, 1, 1.0);
  if (rc) return rc;
  return solve_from_spec(ctx, dp);
}

int launch_dp_ghost(eddy_ctx *ctx, double *dp) {
  const Dims &d = ctx->d;
  long long ng = 2LL * d.nx * d.ny + 2LL * d.nx * d.nz + 2LL * d.ny * d.nz;
  k_dp_ghost<<<(unsigned)((ng + 255) / 256), 256, 0, ctx->stream>>>(d, dp);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

int launch_max_divergence(eddy_ctx *ctx, double *out_host) {
  const Dims &d = ctx->d;
  k_maxdiv_partial<<<NPART, 256, 0, ctx->stream>>>(d, ctx->m, ctx->f[EDDY_UO], ctx->f[EDDY_VO], ctx->f[EDDY_WO],
                                                   ctx->pp.red);
  EDDY_LAUNCHED(ctx);
  k_max_final<<<1, 32, 0, ctx->stream>>>(NPART, ctx->pp.red, ctx->scal + 4);
  EDDY_LAUNCHED(ctx);
  EDDY_CUDA(cudaMemcpyAsync(out_host, ctx->scal + 4, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  return EDDY_OK;
}
