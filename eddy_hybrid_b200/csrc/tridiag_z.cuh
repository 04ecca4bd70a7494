// tridiag_z.cuh -- per-wavenumber line solves along the stretched z axis of
// the Poisson solve (the z direction of src/direct.f's block-tridiagonal
// systems after the x eigen-transform): for every (m, J) line
//   an(k) x(k-1) + (bn(k) + lambda_m - AK(J)) x(k) + cn(k) x(k+1) = g(k).
// Thomas elimination in FP64 arithmetic; the right-hand side and solution are
// stored as G (double for the plain form, float for the mixed form's
// correction solves); the eliminated coefficients c' and right-hand side dd
// as C (FP64 in the plain form; FP32 in the mixed form, whose solves feed an
// FP64-residual refinement and need only FP32 accuracy).  The mixed form
// reads c' from a table computed once per plan (k_tridiag_cprime) instead of
// writing it in every solve.
// The singular line (J = 0, m = m0, the constant x mode) is made compatible by
// removing its z-volume-weighted mean (computed by k_line_mean) and pinned by
// dropping its first equation; its first entry is set to zero.
// dd may alias g (plain form: in place).  Loads are issued in chunks of ZC
// planes ahead of the recurrence so each thread keeps several memory
// requests in flight.
#pragma once

// weighted mean of the singular line: out = sum_k g(m0,0,k) wz(k) / sum_k wz(k)
template <class G>
__global__ void k_line_mean(int M, int L, int N, int m0, const double *__restrict__ wz, const G *__restrict__ g,
                            double *out) {
  __shared__ double s1[256], s2[256];
  double a = 0., b = 0.;
  long long ML = (long long)M * L;
  for (int k = threadIdx.x; k < N; k += blockDim.x) {
    a += (double)g[m0 + ML * k] * wz[k];
    b += wz[k];
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s1[threadIdx.x] += s1[threadIdx.x + w];
      s2[threadIdx.x] += s2[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = s1[0] / s2[0];
}

// c'(k) of every line alone: the eliminated upper diagonal depends only on
// the line's shift and the z coefficients, not on the right-hand side, so a
// solve that reads it from here (PC below) does not store it.  Same
// arithmetic as the elimination in k_tridiag_lines.
template <class C>
__global__ void __launch_bounds__(128)
    k_tridiag_cprime(int M, int L, int N, int m0, const double *__restrict__ lam, const double *__restrict__ ak,
                     const double *__restrict__ an, const double *__restrict__ bn, const double *__restrict__ cn,
                     C *__restrict__ cpr) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)M * L) return;
  const int mi = (int)(t % M), J = (int)(t / M);
  const long long ML = (long long)M * L;
  const int s0 = (J == 0 && mi == m0) ? 1 : 0;
  const double shift = lam[mi] - ak[J];
  double pc = 0.;
  for (int k = s0; k < N; k++) {
    const double a = (k == s0) ? 0. : an[k];
    const double rden = 1.0 / ((bn[k] + shift) - a * pc);
    const double c = cn[k] * rden;
    cpr[t + ML * k] = (C)c;
    pc = c;
  }
}

// DB: issue the next chunk's loads before the current chunk's recurrence (two
// register buffers; pays off with FP32 storage, the FP64 form keeps one).
// PC: c' comes precomputed (k_tridiag_cprime) in cpr, which the elimination
// then only reads; otherwise the elimination writes it there.
// ZF: chunk of the forward sweep (one load per plane there against two in the
// back substitution, so a longer chunk keeps as many bytes in flight).
template <class G, class C = double, int ZC = 8, bool DB = true, bool PC = false, int ZF = ZC>
__global__ void __launch_bounds__(128)
    k_tridiag_lines(int M, int L, int N, int m0, const double *__restrict__ lam, const double *__restrict__ ak,
                    const double *__restrict__ an, const double *__restrict__ bn, const double *__restrict__ cn,
                    const double *__restrict__ cmean, G *g, C *cpr, C *dd) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)M * L) return;
  const int mi = (int)(t % M), J = (int)(t / M);
  const long long ML = (long long)M * L;
  const bool pin = (J == 0 && mi == m0);
  const int s0 = pin ? 1 : 0;
  const double shift = lam[mi] - ak[J];
  const double cm = pin ? cmean[0] : 0.;
  double pc = 0., pd = 0.;
  // forward elimination; the loads of the next chunk are issued before the
  // recurrence over the current one (two register buffers)
  G fa[ZF], fb[ZF];
  auto load_f = [&](G (&f)[ZF], int k0) {
#pragma unroll
    for (int q = 0; q < ZF; q++) f[q] = (k0 + q < N) ? g[t + ML * (k0 + q)] : G(0);
  };
  auto elim = [&](const G (&f)[ZF], int k0) {
#pragma unroll
    for (int q = 0; q < ZF; q++) {
      const int k = k0 + q;
      if (k < N) {
        const double a = (k == s0) ? 0. : an[k];
        const double rden = 1.0 / ((bn[k] + shift) - a * pc);
        const double c = cn[k] * rden;
        const double e = (((double)f[q] - cm) - a * pd) * rden;
        if (!PC) cpr[t + ML * k] = (C)c;
        dd[t + ML * k] = (C)e;
        pc = c;
        pd = e;
      }
    }
  };
  if (DB) {
    load_f(fa, s0);
    for (int k0 = s0; k0 < N; k0 += 2 * ZF) {
      if (k0 + ZF < N) load_f(fb, k0 + ZF);
      elim(fa, k0);
      if (k0 + ZF < N) {
        if (k0 + 2 * ZF < N) load_f(fa, k0 + 2 * ZF);
        elim(fb, k0 + ZF);
      }
    }
  } else {
    for (int k0 = s0; k0 < N; k0 += ZF) {
      load_f(fa, k0);
      elim(fa, k0);
    }
  }
  // back substitution, same double buffering (chunk k1, k1-1, ..., k1-ZC+1)
  double x = pd;
  g[t + ML * (N - 1)] = (G)x;
  C ca[ZC], ea[ZC], cb[ZC], eb[ZC];
  auto load_b = [&](C (&cv)[ZC], C (&ev)[ZC], int k1) {
#pragma unroll
    for (int q = 0; q < ZC; q++) {
      const int k = k1 - q;
      cv[q] = k >= s0 ? cpr[t + ML * k] : C(0);
      ev[q] = k >= s0 ? dd[t + ML * k] : C(0);
    }
  };
  auto subst = [&](const C (&cv)[ZC], const C (&ev)[ZC], int k1) {
#pragma unroll
    for (int q = 0; q < ZC; q++) {
      const int k = k1 - q;
      if (k >= s0) {
        x = (double)ev[q] - (double)cv[q] * x;
        g[t + ML * k] = (G)x;
      }
    }
  };
  if (DB) {
    if (N - 2 >= s0) load_b(ca, ea, N - 2);
    for (int k1 = N - 2; k1 >= s0; k1 -= 2 * ZC) {
      if (k1 - ZC >= s0) load_b(cb, eb, k1 - ZC);
      subst(ca, ea, k1);
      if (k1 - ZC >= s0) {
        if (k1 - 2 * ZC >= s0) load_b(ca, ea, k1 - 2 * ZC);
        subst(cb, eb, k1 - ZC);
      }
    }
  } else {
    for (int k1 = N - 2; k1 >= s0; k1 -= ZC) {
      load_b(ca, ea, k1);
      subst(ca, ea, k1);
    }
  }
  if (pin) g[t] = (G)0.;
}
