/*
 * eo_poisson.c -- oracle restatement of the pressure Poisson solve DIRECT
 * (src/direct.f:2-1118) and of the real FFT it uses (src/fftpack.f RFFTF
 * :2561, RFFTB :2151, packed half-complex order).  TEST INFRASTRUCTURE ONLY.
 *
 * The reference solves, per packed y-wavenumber J, the separable system
 *   AM(i)X(i-1,k)+CM(i)X(i+1,k)+(BML(i)+BN(k))X(i,k)+AN(k)X(i,k-1)+CN(k)X(i,k+1)=F
 * with BLKTRI (direct.f:337-379 coefficients, :534-537 BML, :792-794 solve),
 * subtracts the plane mean for J=1 (:895-898), and divides by L before the
 * backward FFT (:1036).  BLKTRI exists only as a prebuilt object, so the oracle
 * solves the same linear system two independent ways:
 *   method 0: eigen-decomposition of the symmetrised x operator (cyclic Jacobi),
 *             tridiagonal (Thomas) solves along z per eigenmode;
 *   method 1: block-tridiagonal Gaussian elimination along z with dense x
 *             blocks (small sizes only).
 * The singular Neumann mode (J=1, constant in x and z) is pinned by dropping
 * the first z equation of the constant x-eigenmode (method 0) or the (1,1)
 * equation (method 1); both give the same zero-mean answer for a compatible
 * right-hand side.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "eddy_oracle.h"

#define NX (g->nx)
#define NY (g->ny)
#define NZ (g->nz)
#define IX(i, j, k) ((size_t)((i) - 1) + (size_t)NX * ((size_t)((j) - 1) + (size_t)NY * (size_t)((k) - 1)))
#define A(a, i, j, k) (a)[IX(i, j, k)]

/* ---------------- FFT ---------------- */
static void dft_full(int n, const double *x, double *re, double *im) {
  /* X_k = sum_j x_j exp(-2 pi i jk/n), k = 0..n/2; exact index reduction */
  int pow2 = n > 0 && (n & (n - 1)) == 0;
  if (pow2) {
    double *cr = (double *)malloc(sizeof(double) * n), *ci = (double *)malloc(sizeof(double) * n);
    for (int j = 0; j < n; j++) {
      int r = 0;
      for (int b = 1, t = j; b < n; b <<= 1, t >>= 1) r = (r << 1) | (t & 1);
      cr[r] = x[j];
      ci[r] = 0.;
    }
    for (int len = 2; len <= n; len <<= 1) {
      int h = len / 2;
      for (int s = 0; s < n; s += len)
        for (int q = 0; q < h; q++) {
          double ang = -2.0 * M_PI * (double)(q * (n / len)) / (double)n;
          double wr = cos(ang), wi = sin(ang);
          double tr = wr * cr[s + q + h] - wi * ci[s + q + h];
          double ti = wr * ci[s + q + h] + wi * cr[s + q + h];
          cr[s + q + h] = cr[s + q] - tr;
          ci[s + q + h] = ci[s + q] - ti;
          cr[s + q] += tr;
          ci[s + q] += ti;
        }
    }
    for (int k = 0; k <= n / 2; k++) { re[k] = cr[k]; im[k] = ci[k]; }
    free(cr); free(ci);
  } else {
    for (int k = 0; k <= n / 2; k++) {
      double sr = 0., si = 0.;
      for (int j = 0; j < n; j++) {
        long m = ((long)j * k) % n;
        double ang = -2.0 * M_PI * (double)m / (double)n;
        sr += x[j] * cos(ang);
        si += x[j] * sin(ang);
      }
      re[k] = sr; im[k] = si;
    }
  }
}

void eo_rfftf(int n, double *r) {
  double *re = (double *)malloc(sizeof(double) * (n / 2 + 1));
  double *im = (double *)malloc(sizeof(double) * (n / 2 + 1));
  dft_full(n, r, re, im);
  r[0] = re[0];
  for (int k = 1; k <= (n - 1) / 2; k++) { r[2 * k - 1] = re[k]; r[2 * k] = im[k]; }
  if (n % 2 == 0) r[n - 1] = re[n / 2];
  free(re); free(im);
}

void eo_rfftb(int n, double *r) {
  /* x_j = r0 + 2 sum_k (Re_k cos - Im_k sin)(2 pi jk/n) + (-1)^j r_{n-1} */
  double *x = (double *)malloc(sizeof(double) * n);
  /* evaluate as a forward transform of the Hermitian extension */
  double *cr = (double *)calloc(n, sizeof(double)), *ci = (double *)calloc(n, sizeof(double));
  cr[0] = r[0];
  for (int k = 1; k <= (n - 1) / 2; k++) {
    cr[k] = r[2 * k - 1]; ci[k] = r[2 * k];
    cr[n - k] = r[2 * k - 1]; ci[n - k] = -r[2 * k];
  }
  if (n % 2 == 0) cr[n / 2] = r[n - 1];
  int pow2 = n > 0 && (n & (n - 1)) == 0;
  if (pow2) {
    double *ar = (double *)malloc(sizeof(double) * n), *ai = (double *)malloc(sizeof(double) * n);
    for (int j = 0; j < n; j++) {
      int rv = 0;
      for (int b = 1, t = j; b < n; b <<= 1, t >>= 1) rv = (rv << 1) | (t & 1);
      ar[rv] = cr[j]; ai[rv] = ci[j];
    }
    for (int len = 2; len <= n; len <<= 1) {
      int h = len / 2;
      for (int s = 0; s < n; s += len)
        for (int q = 0; q < h; q++) {
          double ang = 2.0 * M_PI * (double)(q * (n / len)) / (double)n;
          double wr = cos(ang), wi = sin(ang);
          double tr = wr * ar[s + q + h] - wi * ai[s + q + h];
          double ti = wr * ai[s + q + h] + wi * ar[s + q + h];
          ar[s + q + h] = ar[s + q] - tr;
          ai[s + q + h] = ai[s + q] - ti;
          ar[s + q] += tr;
          ai[s + q] += ti;
        }
    }
    for (int j = 0; j < n; j++) x[j] = ar[j];
    free(ar); free(ai);
  } else {
    for (int j = 0; j < n; j++) {
      double sr = 0.;
      for (int k = 0; k < n; k++) {
        long m = ((long)j * k) % n;
        double ang = 2.0 * M_PI * (double)m / (double)n;
        sr += cr[k] * cos(ang) - ci[k] * sin(ang);
      }
      x[j] = sr;
    }
  }
  memcpy(r, x, sizeof(double) * n);
  free(x); free(cr); free(ci);
}

/* ---------------- symmetric eigensolver (cyclic Jacobi) ---------------- */
/* a: n x n symmetric (row-major), destroyed; v: eigenvectors in columns
 * (v[i*n+m] = component i of vector m); w: eigenvalues. */
static void jacobi_eig(int n, double *a, double *v, double *w) {
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) v[i * n + j] = (i == j) ? 1. : 0.;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0., diag = 0.;
    for (int i = 0; i < n; i++) {
      diag += a[i * n + i] * a[i * n + i];
      for (int j = i + 1; j < n; j++) off += a[i * n + j] * a[i * n + j];
    }
    if (off <= 1e-34 * diag || off == 0.) break;
    for (int pp = 0; pp < n - 1; pp++)
      for (int q = pp + 1; q < n; q++) {
        double apq = a[pp * n + q];
        if (apq == 0.) continue;
        double app = a[pp * n + pp], aqq = a[q * n + q];
        double theta = (aqq - app) / (2. * apq);
        double t = (theta >= 0. ? 1. : -1.) / (fabs(theta) + sqrt(theta * theta + 1.));
        double c = 1. / sqrt(t * t + 1.), s = t * c;
        for (int k = 0; k < n; k++) {
          double akp = a[k * n + pp], akq = a[k * n + q];
          a[k * n + pp] = c * akp - s * akq;
          a[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {
          double apk = a[pp * n + k], aqk = a[q * n + k];
          a[pp * n + k] = c * apk - s * aqk;
          a[q * n + k] = s * apk + c * aqk;
        }
        a[pp * n + q] = 0.; a[q * n + pp] = 0.;
        for (int k = 0; k < n; k++) {
          double vkp = v[k * n + pp], vkq = v[k * n + q];
          v[k * n + pp] = c * vkp - s * vkq;
          v[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < n; i++) w[i] = a[i * n + i];
}

/* coefficient arrays of direct.f:337-379, interior numbering 0..M-1 / 0..N-1 */
static void direct_coeffs(const eo_grid *g, double *am, double *bm, double *cm,
                          double *an, double *bn, double *cn) {
  int M = NX - 2, N = NZ - 2;
  for (int i = 0; i < M; i++) {
    int I = i + 2;
    am[i] = g->ap[I] * g->au[I - 1];
    cm[i] = g->ap[I] * g->au[I];
  }
  am[0] = 0.; cm[M - 1] = 0.;          /* MP = 1 */
  for (int i = 0; i < M; i++) bm[i] = -am[i] - cm[i];
  for (int k = 0; k < N; k++) {
    int K = k + 2;
    an[k] = g->cp[K] * g->cw[K - 1];
    cn[k] = g->cp[K] * g->cw[K];
  }
  an[0] = 0.; cn[N - 1] = 0.;          /* NP = 1 */
  for (int k = 0; k < N; k++) bn[k] = -an[k] - cn[k];
}

static double ak_of(const eo_grid *g, int Jp) {
  /* direct.f:321-331, packed index Jp (1-based) -> AK(Jp/2+1) */
  int L = NY - 2, kk = Jp / 2;
  double a = (kk <= L / 2 - 1 || kk == 0) ? 2. * M_PI * kk : -2. * M_PI * (L - kk);
  if (kk >= L / 2) a = -2. * M_PI * (L - kk);
  return 2. * (1. - cos(a / (double)L)) / g->delysq;
}

/* Thomas algorithm; pin = 1 drops the first equation and sets x0 = 0 */
static void thomas(int n, const double *a, const double *b, const double *c,
                   const double *f, double *x, int pin) {
  double *cp = (double *)malloc(sizeof(double) * n), *dp = (double *)malloc(sizeof(double) * n);
  int s0 = 0;
  if (pin) { x[0] = 0.; s0 = 1; }
  double prev_c = 0., prev_d = 0.;
  for (int k = s0; k < n; k++) {
    double ak = (k == s0) ? 0. : a[k];
    double rhs = f[k];
    if (pin && k == 1) rhs = f[k] - a[k] * 0.;
    double den = b[k] - ak * prev_c;
    cp[k] = c[k] / den;
    dp[k] = (rhs - ak * prev_d) / den;
    prev_c = cp[k]; prev_d = dp[k];
  }
  x[n - 1] = dp[n - 1];
  for (int k = n - 2; k >= s0; k--) x[k] = dp[k] - cp[k] * x[k + 1];
  free(cp); free(dp);
}

/* dense solve with partial pivoting: A (n x n, destroyed), B (n x m) -> X in B */
static int gauss_solve(int n, int m, double *Am, double *B) {
  for (int c = 0; c < n; c++) {
    int piv = c;
    for (int r = c + 1; r < n; r++) if (fabs(Am[r * n + c]) > fabs(Am[piv * n + c])) piv = r;
    if (Am[piv * n + c] == 0.) return -1;
    if (piv != c) {
      for (int q = 0; q < n; q++) { double t = Am[c * n + q]; Am[c * n + q] = Am[piv * n + q]; Am[piv * n + q] = t; }
      for (int q = 0; q < m; q++) { double t = B[c * m + q]; B[c * m + q] = B[piv * m + q]; B[piv * m + q] = t; }
    }
    for (int r = c + 1; r < n; r++) {
      double f = Am[r * n + c] / Am[c * n + c];
      if (f == 0.) continue;
      for (int q = c; q < n; q++) Am[r * n + q] -= f * Am[c * n + q];
      for (int q = 0; q < m; q++) B[r * m + q] -= f * B[c * m + q];
    }
  }
  for (int c = n - 1; c >= 0; c--) {
    for (int q = 0; q < m; q++) {
      double sacc = B[c * m + q];
      for (int r = c + 1; r < n; r++) sacc -= Am[c * n + r] * B[r * m + q];
      B[c * m + q] = sacc / Am[c * n + c];
    }
  }
  return 0;
}

/* Solve one wavenumber by block elimination; F (M x N, i fastest) in/out */
static int solve_block(int M, int N, const double *am, const double *bml,
                       const double *cm, const double *an, const double *bn,
                       const double *cn, double *F, int pin) {
  /* blocks along k of size M: B_k = Lx + bn(k) I, lower an(k) I, upper cn(k) I */
  double *Bp = (double *)malloc(sizeof(double) * (size_t)M * M * N);  /* B'_k^{-1} C_k stored as G_k */
  double *Fp = (double *)malloc(sizeof(double) * (size_t)M * N);
  double *Bk = (double *)malloc(sizeof(double) * (size_t)M * M);
  double *rhs = (double *)malloc(sizeof(double) * (size_t)M * (M + 1));
  int rc = 0;
  for (int k = 0; k < N && rc == 0; k++) {
    /* B_k - an(k) * G_{k-1} */
    for (int i = 0; i < M * M; i++) Bk[i] = 0.;
    for (int i = 0; i < M; i++) {
      Bk[i * M + i] = bml[i] + bn[k];
      if (i > 0) Bk[i * M + i - 1] = am[i];
      if (i < M - 1) Bk[i * M + i + 1] = cm[i];
    }
    double ck = cn[k];
    /* right-hand sides: [C_k | F'_k] */
    for (int i = 0; i < M; i++) {
      for (int q = 0; q < M; q++) rhs[i * (M + 1) + q] = (i == q) ? ck : 0.;
      rhs[i * (M + 1) + M] = F[(size_t)k * M + i];
    }
    if (pin && k == 0) {
      for (int q = 0; q < M; q++) Bk[q] = (q == 0) ? 1. : 0.;
      for (int q = 0; q <= M; q++) rhs[q] = 0.;
    }
    if (k > 0) {
      double a = an[k];
      const double *Gm = Bp + (size_t)(k - 1) * M * M;
      for (int i = 0; i < M * M; i++) Bk[i] -= a * Gm[i];
      for (int i = 0; i < M; i++) rhs[i * (M + 1) + M] -= a * Fp[(size_t)(k - 1) * M + i];
    }
    rc = gauss_solve(M, M + 1, Bk, rhs);
    double *Gk = Bp + (size_t)k * M * M;
    for (int i = 0; i < M; i++) {
      for (int q = 0; q < M; q++) Gk[i * M + q] = rhs[i * (M + 1) + q];
      Fp[(size_t)k * M + i] = rhs[i * (M + 1) + M];
    }
  }
  if (rc == 0) {
    for (int i = 0; i < M; i++) F[(size_t)(N - 1) * M + i] = Fp[(size_t)(N - 1) * M + i];
    for (int k = N - 2; k >= 0; k--) {
      const double *Gk = Bp + (size_t)k * M * M;
      for (int i = 0; i < M; i++) {
        double sacc = Fp[(size_t)k * M + i];
        for (int q = 0; q < M; q++) sacc -= Gk[i * M + q] * F[(size_t)(k + 1) * M + q];
        F[(size_t)k * M + i] = sacc;
      }
    }
  }
  free(Bp); free(Fp); free(Bk); free(rhs);
  return rc;
}

int eo_direct(eo_state *s, int method) {
  const eo_grid *g = s->g;
  if (g->mp != 1 || g->np != 1 || g->lp != 0) return -3;
  int M = NX - 2, L = NY - 2, N = NZ - 2;
  double *dp = s->dp;
  /* forward FFT along y into spectral buffer spec[J][k][i] */
  double *spec = (double *)malloc(sizeof(double) * (size_t)M * L * N);
#pragma omp parallel
  {
    double *line = (double *)malloc(sizeof(double) * L);
#pragma omp for schedule(static)
    for (int k = 0; k < N; k++)
      for (int i = 0; i < M; i++) {
        for (int j = 0; j < L; j++) line[j] = A(dp, i + 2, j + 2, k + 2);
        eo_rfftf(L, line);
        for (int j = 0; j < L; j++) spec[(size_t)j * M * N + (size_t)k * M + i] = line[j];
      }
    free(line);
  }
  double *am = (double *)malloc(sizeof(double) * M), *bm = (double *)malloc(sizeof(double) * M);
  double *cm = (double *)malloc(sizeof(double) * M), *an = (double *)malloc(sizeof(double) * N);
  double *bn = (double *)malloc(sizeof(double) * N), *cn = (double *)malloc(sizeof(double) * N);
  direct_coeffs(g, am, bm, cm, an, bn, cn);
  int rc = 0;
  double *Q = NULL, *lam = NULL, *sq = NULL;
  int m0 = -1;
  if (method == 0) {
    /* S = D^1/2 T D^1/2 with Lx = D T, D = diag(ap) */
    double *S = (double *)calloc((size_t)M * M, sizeof(double));
    Q = (double *)malloc(sizeof(double) * (size_t)M * M);
    lam = (double *)malloc(sizeof(double) * M);
    sq = (double *)malloc(sizeof(double) * M);
    for (int i = 0; i < M; i++) sq[i] = sqrt(g->ap[i + 2]);
    for (int i = 0; i < M; i++) {
      S[i * M + i] = bm[i];
      if (i > 0) S[i * M + i - 1] = am[i] / sq[i] * sq[i - 1];
      if (i < M - 1) S[i * M + i + 1] = cm[i] / sq[i] * sq[i + 1];
    }
    /* symmetrise exactly: off-diagonal = sqrt(ap_i ap_{i+1}) au_I */
    for (int i = 0; i < M - 1; i++) {
      double o = sq[i] * sq[i + 1] * g->au[i + 2];
      S[i * M + i + 1] = o; S[(i + 1) * M + i] = o;
    }
    jacobi_eig(M, S, Q, lam);
    double best = 1e300;
    for (int m = 0; m < M; m++) if (fabs(lam[m]) < best) { best = fabs(lam[m]); m0 = m; }
    lam[m0] = 0.;
    /* exact null vector q0 ~ 1/sqrt(ap) */
    double nrm = 0.;
    for (int i = 0; i < M; i++) nrm += 1. / g->ap[i + 2];
    nrm = sqrt(nrm);
    double sgn = Q[0 * M + m0] >= 0 ? 1. : -1.;
    for (int i = 0; i < M; i++) Q[i * M + m0] = sgn / (sq[i] * nrm);
    free(S);
  }
#pragma omp parallel
  {
    double *bml = (double *)malloc(sizeof(double) * M);
    double *G = (double *)malloc(sizeof(double) * (size_t)M * N);
    double *fz = (double *)malloc(sizeof(double) * N), *xz = (double *)malloc(sizeof(double) * N);
    double *bz = (double *)malloc(sizeof(double) * N);
#pragma omp for schedule(dynamic)
    for (int Jp = 1; Jp <= L; Jp++) {
      double ak = ak_of(g, Jp);
      double *F = spec + (size_t)(Jp - 1) * M * N;
      for (int i = 0; i < M; i++) bml[i] = bm[i] - ak;
      if (Jp == 1) {
        /* compatibility: remove the volume-weighted mean of the k=0 right-hand
         * side (the component outside the range of the Neumann operator) */
        double sv = 0., vv = 0.;
        for (int k = 0; k < N; k++)
          for (int i = 0; i < M; i++) {
            double v = 1.0 / (g->ap[i + 2] * g->cp[k + 2]);
            sv += F[(size_t)k * M + i] * v;
            vv += v;
          }
        double cmean = sv / vv;
        for (long q = 0; q < (long)M * N; q++) F[q] = F[q] - cmean;
      }
      if (method == 1) {
        int r = solve_block(M, N, am, bml, cm, an, bn, cn, F, Jp == 1);
        if (r) rc = r;
      } else {
        /* forward transform G = Q^T D^-1/2 F (per k) */
        for (int k = 0; k < N; k++)
          for (int m = 0; m < M; m++) {
            double acc = 0.;
            for (int i = 0; i < M; i++) acc += Q[i * M + m] * (F[(size_t)k * M + i] / sq[i]);
            G[(size_t)k * M + m] = acc;
          }
        for (int m = 0; m < M; m++) {
          for (int k = 0; k < N; k++) { fz[k] = G[(size_t)k * M + m]; bz[k] = bn[k] + lam[m] - ak; }
          thomas(N, an, bz, cn, fz, xz, Jp == 1 && m == m0);
          for (int k = 0; k < N; k++) G[(size_t)k * M + m] = xz[k];
        }
        for (int k = 0; k < N; k++)
          for (int i = 0; i < M; i++) {
            double acc = 0.;
            for (int m = 0; m < M; m++) acc += Q[i * M + m] * G[(size_t)k * M + m];
            F[(size_t)k * M + i] = sq[i] * acc;
          }
      }
      if (Jp == 1) {
        double sum = 0.;
        for (long q = 0; q < (long)M * N; q++) sum += F[q];
        double dpm = sum / (double)((long)M * N);
        for (long q = 0; q < (long)M * N; q++) F[q] = F[q] - dpm;
      }
    }
    free(bml); free(G); free(fz); free(xz); free(bz);
  }
  /* DP = 0, DUMMY/L, backward FFT, ghost copies (direct.f:1035-1106) */
  memset(dp, 0, sizeof(double) * (size_t)s->ncell);
#pragma omp parallel
  {
    double *line = (double *)malloc(sizeof(double) * L);
#pragma omp for schedule(static)
    for (int k = 0; k < N; k++)
      for (int i = 0; i < M; i++) {
        for (int j = 0; j < L; j++) line[j] = spec[(size_t)j * M * N + (size_t)k * M + i] / (double)L;
        eo_rfftb(L, line);
        for (int j = 0; j < L; j++) A(dp, i + 2, j + 2, k + 2) = line[j];
      }
    free(line);
  }
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++) { A(dp, 1, j, k) = A(dp, 2, j, k); A(dp, NX, j, k) = A(dp, NX - 1, j, k); }
  for (int k = 1; k <= NZ; k++)
    for (int i = 1; i <= NX; i++) { A(dp, i, 1, k) = A(dp, i, NY - 1, k); A(dp, i, NY, k) = A(dp, i, 2, k); }
  free(spec); free(am); free(bm); free(cm); free(an); free(bn); free(cn);
  free(Q); free(lam); free(sq);
  return rc;
}

/* The operator DIRECT inverts, applied to the interior of x (ghosts ignored:
 * Neumann in x and z, periodic in y). */
void eo_apply_laplacian(eo_state *s, const double *x, double *out) {
  const eo_grid *g = s->g;
  int M = NX - 2, L = NY - 2, N = NZ - 2;
  double *am = (double *)malloc(sizeof(double) * M), *bm = (double *)malloc(sizeof(double) * M);
  double *cm = (double *)malloc(sizeof(double) * M), *an = (double *)malloc(sizeof(double) * N);
  double *bn = (double *)malloc(sizeof(double) * N), *cn = (double *)malloc(sizeof(double) * N);
  direct_coeffs(g, am, bm, cm, an, bn, cn);
  double r = 1. / g->delysq;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < N; k++)
    for (int j = 0; j < L; j++)
      for (int i = 0; i < M; i++) {
        int I = i + 2, J = j + 2, K = k + 2;
        int jm = (j == 0) ? L + 1 : J - 1, jp = (j == L - 1) ? 2 : J + 1;
        double c = A(x, I, J, K);
        double v = bm[i] * c + bn[k] * c;
        if (i > 0) v += am[i] * A(x, I - 1, J, K);
        if (i < M - 1) v += cm[i] * A(x, I + 1, J, K);
        if (k > 0) v += an[k] * A(x, I, J, K - 1);
        if (k < N - 1) v += cn[k] * A(x, I, J, K + 1);
        v += r * (A(x, I, jm, K) - 2. * c + A(x, I, jp, K));
        A(out, I, J, K) = v;
      }
  free(am); free(bm); free(cm); free(an); free(bn); free(cn);
}
