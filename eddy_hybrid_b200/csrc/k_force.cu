// k_force.cu -- the force on the immersed body by the control-volume approach
// of calcfrc (src/calcforce.f:3-779, Cartesian branch) on the device fields
// UO, VO, WO, P and the body's taguo flags: the momentum inside the control
// volume (its change over dt is the unsteady term) and the momentum and
// stress fluxes through its six faces.  Reductions: every block accumulates
// its grid-stride share of up to 14 terms per thread, reduces them in shared
// memory and writes its partials; one warp per group then sums the partials
// in block order (deterministic; against the reference's sequential sums the
// results differ by the reduction order only).  The host assembles the
// reference's output array from the 35 sums.
#include <cmath>

#include "eddy_internal.h"

namespace {

constexpr int CVB = 148;  // blocks per group (one per SM)
constexpr int CVT = 256;  // threads per block
constexpr int CVN = 14;   // terms per group at most

struct CvArgs {
  Dims d;
  DevMetrics m;
  const double *u, *v, *w, *p;
  const signed char *fu, *fv, *fw;  // the body's taguo flags; nullptr: all fluid
  int icb, ice, kcb, kce, kbflag, keflag;
  double ru1;
};

__device__ __forceinline__ int fl(const signed char *f, const Dims &d, int i, int j, int k) {
  return f ? (int)f[fidx(d, i, j, k)] : 0;
}

// the j = 1 branch's DWDY2 at (k, i), when that branch runs there
__device__ __forceinline__ bool left_dwdy2(const CvArgs &a, int k, int i, double &dwdy2) {
  const Dims &d = a.d;
  if (fl(a.fv, d, i, 1, k) <= 0 || fl(a.fw, d, i, 1, k) <= 0) {
    dwdy2 = (a.w[fidx(d, i, 2, k - 1)] - a.w[fidx(d, i, 1, k - 1)]) * a.m.bw[1];
    return true;
  }
  return false;
}

// the terms of index t of group g (0 volume, 1 inlet/outlet, 2 top/bottom,
// 3 the j = 1 and j = JY2 planes), in the reference's arithmetic
__device__ void cv_terms(const CvArgs &a, int g, long long t, double (&r)[CVN]) {
  const Dims &d = a.d;
  const DevMetrics &m = a.m;
  const int ni = a.ice - a.icb, nj = d.jy2 - d.jy1 + 1;
  auto U = [&](int i, int j, int k) { return a.u[fidx(d, i, j, k)]; };
  auto V = [&](int i, int j, int k) { return a.v[fidx(d, i, j, k)]; };
  auto W = [&](int i, int j, int k) { return a.w[fidx(d, i, j, k)]; };
  auto P = [&](int i, int j, int k) { return a.p[fidx(d, i, j, k)]; };
  const double ru1 = a.ru1;
  if (g == 0) {
    // momentum in the volume (:96-112)
    const int j = d.jy1 + (int)(t % nj), i = a.icb + 1 + (int)((t / nj) % ni);
    const int k = a.kcb + 1 + (int)(t / ((long long)nj * ni));
    const double dv = 1.0 / (m.bp[j] * m.ap[i] * m.cp[k]);
    if (fl(a.fu, d, i, j, k) <= 0 || fl(a.fu, d, i - 1, j, k) <= 0) r[0] += 0.5 * (U(i, j, k) + U(i - 1, j, k)) * dv;
    if (fl(a.fv, d, i, j, k) <= 0 || fl(a.fv, d, i, j - 1, k) <= 0) r[1] += 0.5 * (V(i, j, k) + V(i, j - 1, k)) * dv;
    if (fl(a.fw, d, i, j, k) <= 0 || fl(a.fw, d, i, j, k - 1) <= 0) r[2] += 0.5 * (W(i, j, k) + W(i, j, k - 1)) * dv;
  } else if (g == 1) {
    // x-y planes: inlet k = KCB, outlet k = KCE (:362-426)
    const int j = d.jy1 + (int)(t % nj), i = a.icb + 1 + (int)(t / nj);
    const double da = 1.0 / m.bp[j] / m.ap[i];
    for (int side = 0; side < 2; side++) {
      if (side == 0 ? !a.kbflag : !a.keflag) continue;
      const int k = side == 0 ? a.kcb : a.kce;
      const double sa = side == 0 ? -da : da;
      const double dwdx = (W(i + 1, j, k) - W(i - 1, j, k)) * m.aw[i] / 2.;
      const double dudz1 = (U(i, j, k + 1) - U(i, j, k)) * m.cw[k];
      const double dudz2 = (U(i - 1, j, k + 1) - U(i - 1, j, k)) * m.cw[k];
      const double dudz = 0.5 * (dudz1 + dudz2);
      const double sxz = dudz + dwdx;
      const double txz = ru1 * sxz;
      const double u1 = 0.25 * (U(i, j, k) + U(i, j, k + 1) + U(i - 1, j, k) + U(i - 1, j, k + 1));
      const double uw = u1 * W(i, j, k);
      const double dwdz = (W(i, j, k + 1) - W(i, j, k - 1)) * m.cw[k] / 2.;
      const double szz = 2. * ru1 * dwdz;
      const double pres = 0.5 * (P(i, j, k + 1) + P(i, j, k));
      const double tzz = pres - szz;
      const double wsq = W(i, j, k) * W(i, j, k);
      double *o = r + 7 * side;  // FX, F(1), F(2), FZ, F(3), F(4), F(5)
      o[0] += (uw - txz) * sa;
      o[1] += uw * sa;
      o[2] += -(txz * sa);
      o[3] += (wsq + tzz) * sa;
      o[4] += pres * sa;
      o[5] += -(szz * sa);
      o[6] += wsq * sa;
    }
  } else if (g == 2) {
    // y-z planes: top i = ICE, bottom i = ICB (:428-496)
    const int j = d.jy1 + (int)(t % nj), k = a.kcb + 1 + (int)(t / nj);
    const double da = 1.0 / m.bp[j] / m.cp[k];
    for (int side = 0; side < 2; side++) {
      const int i = side == 0 ? a.ice : a.icb;
      const double sa = side == 0 ? da : -da;
      const double dudx = (U(i + 1, j, k) - U(i - 1, j, k)) * m.au[i] / 2;
      const double sxx = 2. * ru1 * dudx;
      const double pres = 0.5 * (P(i + 1, j, k) + P(i, j, k));
      const double txx = pres - sxx;
      const double usq = U(i, j, k) * U(i, j, k);
      const double dudz = (U(i, j, k + 1) - U(i, j, k - 1)) * m.cu[k] / 2.;
      const double dwdx1 = (W(i + 1, j, k) - W(i, j, k)) * m.au[i];
      const double dwdx2 = (W(i + 1, j, k - 1) - W(i, j, k - 1)) * m.au[i];
      const double dwdx = 0.5 * (dwdx1 + dwdx2);
      const double w1 = 0.25 * (W(i, j, k) + W(i, j, k - 1) + W(i + 1, j, k) + W(i + 1, j, k - 1));
      const double uw = U(i, j, k) * w1;
      const double sxz = ru1 * (dudz + dwdx);
      double *o = r + 7 * side;  // FX, F(1), F(2), F(3), FZ, F(4), F(5)
      o[0] += (usq + txx) * sa;
      o[1] += usq * sa;
      o[2] += pres * sa;
      o[3] += -(sxx * sa);
      o[4] += (uw - sxz) * sa;
      o[5] += uw * sa;
      o[6] += -(sxz * sa);
    }
  } else {
    // x-z planes j = 1 and j = JY2 (:498-558), positions in the reference's
    // loop order (k outer, i inner)
    const int i = a.icb + 1 + (int)(t % ni), k = a.kcb + 1 + (int)(t / ni);
    const double da = 1. / m.cp[k] / m.ap[i];
    for (int side = 0; side < 2; side++) {
      const int j = side == 0 ? 1 : d.jy2;
      const double sa = side == 0 ? -da : da;
      if (fl(a.fu, d, i, j, k) <= 0 || fl(a.fv, d, i, j, k) <= 0) {
        const double dudy1 = (U(i, j + 1, k) - U(i, j, k)) * m.bu[j];
        const double dudy2 = (U(i - 1, j + 1, k) - U(i - 1, j, k)) * m.bu[j];
        const double dudy = 0.5 * (dudy1 + dudy2);
        const double dvdx = (V(i + 1, j, k) - V(i - 1, j, k)) * m.av[i] / 2.;
        const double sxy = ru1 * (dudy + dvdx);
        const double u1 = 0.25 * (U(i, j, k) + U(i - 1, j, k) + U(i, j + 1, k) + U(i - 1, j + 1, k));
        const double uv = V(i, j, k) * u1;
        r[2 * side] += (uv - sxy) * sa;
      }
      if (fl(a.fv, d, i, j, k) <= 0 || fl(a.fw, d, i, j, k) <= 0) {
        double dwdy1, dwdy2 = 0.;
        if (side == 0) {
          dwdy1 = (W(i, j + 1, k) - W(i, j, k)) * m.bw[j];
          left_dwdy2(a, k, i, dwdy2);
        } else {
          // as written the j = JY2 branch assigns DWDY1 twice and reads DWDY2
          // as the last j = 1 branch before it left it (this position's, else
          // the nearest earlier one in loop order; zero before any)
          dwdy1 = (W(i, j + 1, k - 1) - W(i, j, k - 1)) * m.bw[j];
          for (long long s = t; s >= 0; s--) {
            const int is = a.icb + 1 + (int)(s % ni), ks = a.kcb + 1 + (int)(s / ni);
            if (left_dwdy2(a, ks, is, dwdy2)) break;
          }
        }
        const double dwdy = 0.5 * (dwdy1 + dwdy2);
        const double dvdz = (V(i, j, k + 1) - V(i, j, k - 1)) * m.cu[k] / 2.;
        const double syz = ru1 * (dvdz + dwdy);
        const double w1 = 0.25 * (W(i, j, k) + W(i, j, k - 1) + W(i, j + 1, k) + W(i, j + 1, k - 1));
        const double vw = V(i, j, k) * w1;
        r[2 * side + 1] += (vw - syz) * sa;
      }
    }
  }
}

__global__ void __launch_bounds__(CVT) k_cv_sums(CvArgs a, long long n0, long long n1, long long n2, long long n3,
                                                double *part) {
  __shared__ double sh[CVN][CVT];
  const int g = blockIdx.y;
  const long long n = g == 0 ? n0 : g == 1 ? n1 : g == 2 ? n2 : n3;
  double r[CVN];
#pragma unroll
  for (int e = 0; e < CVN; e++) r[e] = 0.;
  for (long long t = (long long)blockIdx.x * CVT + threadIdx.x; t < n; t += (long long)CVB * CVT) cv_terms(a, g, t, r);
#pragma unroll
  for (int e = 0; e < CVN; e++) sh[e][threadIdx.x] = r[e];
  __syncthreads();
  for (int s = CVT / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
#pragma unroll
      for (int e = 0; e < CVN; e++) sh[e][threadIdx.x] += sh[e][threadIdx.x + s];
    __syncthreads();
  }
  if ((int)threadIdx.x < CVN) part[((long long)g * CVB + blockIdx.x) * CVN + threadIdx.x] = sh[threadIdx.x][0];
}

// term e of group g: the blocks' partials in block order
__global__ void k_cv_final(const double *part, double *res) {
  const int g = blockIdx.x, e = threadIdx.x;
  if (e >= CVN) return;
  double s = 0.;
  for (int b = 0; b < CVB; b++) s += part[((long long)g * CVB + b) * CVN + e];
  res[g * CVN + e] = s;
}

// closest (src/numrec.f:433-475) on xx(1..n)
int closest(const double *xx, int n, double x) {
  int jl = 0, ju = n + 1;
  if (x == xx[1]) {
    jl = 1;
  } else {
    while (ju - jl > 1) {
      const int jm = (ju + jl) / 2;
      if ((xx[n] > xx[1]) == (x > xx[jm])) jl = jm;
      else ju = jm;
    }
  }
  int j = jl;
  if (j > 0 && j < n) {
    if (std::fabs(x - xx[j]) > std::fabs(x - xx[j + 1])) j = jl + 1;
  } else if (j < 1) {
    j = 1;
  } else if (j > n) {
    j = n;
  }
  return j;
}

// locate (src/numrec.f:390-422) on xx(1..n)
int locate(const double *xx, int n, double x) {
  int jl = 0, ju = n + 1;
  if (xx[1] == x) return 1;
  while (ju - jl > 1) {
    const int jm = (ju + jl) / 2;
    if ((xx[n] > xx[1]) == (x > xx[jm])) jl = jm;
    else ju = jm;
  }
  return jl;
}

}  // namespace

extern "C" int eddy_body_force_cv(eddy_ctx *ctx, const double *cvlim, double dt, int icycle, double *out) {
  if (!ctx || !cvlim || !out || !(dt > 0.)) return EDDY_EINVAL;
  if (int rc = ib_join(ctx)) return rc;
  const Dims &d = ctx->d;
  const int NZ = d.nz;
  // the control volume (src/calcforce.f:44-94)
  const int icb = closest(ctx->h[0].data(), d.nx, cvlim[0]), ice = closest(ctx->h[0].data(), d.nx, cvlim[1]);
  int kcb = locate(ctx->h[12].data(), NZ - 1, cvlim[2]), kce = locate(ctx->h[12].data(), NZ - 1, cvlim[3]);
  int kbflag = 0, keflag = 0;
  if (kcb == 0 && kce == 0) {
    kcb = NZ;
    kce = 0;
  } else if (kcb == 0 && (kce > 0 && kce < NZ - 1)) {
    keflag = 1;
    kcb = 1;
    if (kce == 1) kce = 2;
  } else if ((kcb > 0 && kcb < NZ - 1) && (kce > 0 && kce < NZ - 1)) {
    kbflag = 1;
    keflag = 1;
    kcb = kcb + 1;
  } else if (kcb == 0 && kce == NZ - 1) {
    kcb = 1;
  } else if ((kcb > 0 && kcb < NZ - 1) && kce == NZ - 1) {
    kbflag = 1;
    kcb = kcb + 1;
  } else if (kcb == NZ - 1 && kce == NZ - 1) {
    kcb = NZ;
    kce = 0;
  }
  // every stencil reads one plane beyond its index: the faces must lie
  // inside the arrays
  if (icb < 2 || ice > d.nx - 1 || (kbflag && (kcb < 2 || kcb > NZ - 1)) || (keflag && (kce < 2 || kce > NZ - 1))) {
    ctx->err = "eddy_body_force_cv: the control volume reaches the domain's outer planes";
    return EDDY_EINVAL;
  }
  if (!ctx->cv_buf) EDDY_CUDA(cudaMalloc(&ctx->cv_buf, sizeof(double) * (4 * CVB * CVN + 4 * CVN)));
  CvArgs a{d, ctx->m, ctx->f[EDDY_UO], ctx->f[EDDY_VO], ctx->f[EDDY_WO], ctx->f[EDDY_P],
           ib_flag_dev(ctx, 0), ib_flag_dev(ctx, 1), ib_flag_dev(ctx, 2),
           icb, ice, kcb, kce, kbflag, keflag, ctx->sc.ru1};
  const long long ni = ice > icb ? ice - icb : 0, nj = d.jy2 - d.jy1 + 1, nk = kce > kcb ? kce - kcb : 0;
  double *part = ctx->cv_buf, *res = ctx->cv_buf + 4 * CVB * CVN;
  k_cv_sums<<<dim3(CVB, 4), CVT, 0, ctx->stream>>>(a, ni * nj * nk, ni * nj, nk * nj, nk * ni, part);
  EDDY_LAUNCHED(ctx);
  k_cv_final<<<4, 32, 0, ctx->stream>>>(part, res);
  EDDY_LAUNCHED(ctx);
  double h[4 * CVN];
  EDDY_CUDA(cudaMemcpyAsync(h, res, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  // the unsteady term (:113-124)
  double fbv[3] = {h[0], h[1], h[2]}, fbt[3];
  for (int c = 0; c < 3; c++) {
    fbt[c] = icycle == 0 ? 0. : (fbv[c] - ctx->cv_fb[c]) / dt;
    ctx->cv_fb[c] = fbv[c];
  }
  double fx[6] = {h[CVN + 0], h[CVN + 7], h[2 * CVN + 0], h[2 * CVN + 7], h[3 * CVN + 0], h[3 * CVN + 2]};
  double fz[6] = {h[CVN + 3], h[CVN + 10], h[2 * CVN + 4], h[2 * CVN + 11], h[3 * CVN + 1], h[3 * CVN + 3]};
  for (int e = 0; e < 56; e++) out[e] = 0.;
  for (int e = 0; e < 6; e++) {
    out[e] = fx[e];
    out[12 + e] = fz[e];
  }
  for (int c = 0; c < 3; c++) out[18 + c] = fbt[c];
  double sx = 0., sy = 0., sz = 0.;
  for (int e = 0; e < 6; e++) {
    sx = sx + fx[e];
    sz = sz + fz[e];
  }
  out[21] = -(sx + fbt[0]);
  out[22] = -(sy + fbt[1]);
  out[23] = -(sz + fbt[2]);
  // Finlet / Foutlet (1..5: UW, TXZ, PRES, SZZ, WSQ) and Ftop / Fbot (1..5:
  // USQ, PRES, SXX, UW, SXZ); (6), (7) the x and z subtotals (:562-569)
  const double *src[4] = {h + CVN, h + CVN + 7, h + 2 * CVN, h + 2 * CVN + 7};
  const int map[2][5] = {{1, 2, 4, 5, 6}, {1, 2, 3, 5, 6}};
  for (int q = 0; q < 4; q++) {
    double *ff = out + 24 + 8 * q;
    for (int e = 0; e < 5; e++) ff[e] = src[q][map[q / 2][e]];
    const int n1 = q < 2 ? 2 : 3;
    double x = 0., z = 0.;
    for (int e = 0; e < n1; e++) x = x + ff[e];
    for (int e = n1; e < 5; e++) z = z + ff[e];
    ff[5] = x;
    ff[6] = z;
  }
  return EDDY_OK;
}

extern "C" int eddy_body_force_cv_reset(eddy_ctx *ctx) {
  if (!ctx) return EDDY_EINVAL;
  for (int c = 0; c < 3; c++) ctx->cv_fb[c] = 0.;
  return EDDY_OK;
}
