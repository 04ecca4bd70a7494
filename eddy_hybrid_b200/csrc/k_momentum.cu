// k_momentum.cu -- momentum right-hand side fused with the RK predictor,
// boundary-condition plane fills, BOUNDINOUT, CORRECT and the pressure update.
//
// Plain FP64 form: compiled with -fmad=false so every expression rounds in the
// reference's operation order (src/rhs.f, src/timeindeg.f); the explicit
// (non Crank-Nicolson) branch of the Cartesian equations.
#include "eddy_internal.h"

#define A(a, i, j, k) (a)[fidx(d, (i), (j), (k))]

namespace {

constexpr int BX = 32, BY = 4, BZ = 2;

// ---------------------------------------------------------------------------
// u-momentum explicit RHS at a u point (src/rhs.f:77-172)
__device__ __forceinline__ double rhs_u(const Dims &d, const DevMetrics &m, double ru1,
                                        const double *__restrict__ uo, const double *__restrict__ vo,
                                        const double *__restrict__ wo, const double *__restrict__ tv,
                                        int i, int j, int k, long long q, int sy, long long sz) {
  const double *qr = uo;
  double qxp = (qr[q+1] + qr[q]) * 0.5;
  double qxm = (qr[q] + qr[q-1]) * 0.5;
  double uxp = (uo[q+1] + uo[q]) * 0.5;
  double uxm = (uo[q] + uo[q-1]) * 0.5;
  double uyp = (uo[q+sy] + uo[q]) * 0.5;
  double uym = (uo[q] + uo[q-sy]) * 0.5;
  double uzp = (uo[q+sz] + uo[q]) * 0.5;
  double uzm = (uo[q] + uo[q-sz]) * 0.5;
  double vxp = (vo[q+1] + vo[q]) * 0.5;
  double vxm = (vo[q+1-sy] + vo[q-sy]) * 0.5;
  double wxp = (wo[q+1] + wo[q]) * 0.5;
  double wxm = (wo[q+1-sz] + wo[q-sz]) * 0.5;
  double dqdxp = m.ap[i + 1] * (qr[q+1] - qr[q]);
  double dqdxm = m.ap[i] * (qr[q] - qr[q-1]);
  double dudyp = m.bv[j] * (uo[q+sy] - uo[q]);
  double dudym = m.bv[j - 1] * (uo[q] - uo[q-sy]);
  double dudzp = m.cw[k] * (uo[q+sz] - uo[q]);
  double dudzm = m.cw[k - 1] * (uo[q] - uo[q-sz]);
  double dvdxp = m.au[i] * (vo[q+1] - vo[q]);
  double dvdxm = m.au[i] * (vo[q+1-sy] - vo[q-sy]);
  double dwdxp = m.au[i] * (wo[q+1] - wo[q]);
  double dwdxm = m.au[i] * (wo[q+1-sz] - wo[q-sz]);
  double tvjp = 0.25 * (tv[q+1] + tv[q] + tv[q+1+sy] + tv[q+sy]);
  double tvjm = 0.25 * (tv[q+1] + tv[q] + tv[q+1-sy] + tv[q-sy]);
  double tvkp = 0.25 * (tv[q+1] + tv[q] + tv[q+1+sz] + tv[q+sz]);
  double tvkm = 0.25 * (tv[q+1] + tv[q] + tv[q+1-sz] + tv[q-sz]);
  double txxp = (ru1 + 2. * tv[q+1]) * dqdxp;
  double txxm = (ru1 + 2. * tv[q]) * dqdxm;
  double tyyp = (ru1 + tvjp) * dudyp;
  double tyym = (ru1 + tvjm) * dudym;
  double tzzp = (ru1 + tvkp) * dudzp;
  double tzzm = (ru1 + tvkm) * dudzm;
  double txyp = tvjp * dvdxp;
  double txym = tvjm * dvdxm;
  double txzp = tvkp * dwdxp;
  double txzm = tvkm * dwdxm;
  double h11 = -m.au[i] * (qxp * uxp - qxm * uxm);
  double h22 = -m.bu[j] * (vxp * uyp - vxm * uym);
  double h33 = -m.cu[k] * (wxp * uzp - wxm * uzm);
  double t11 = m.au[i] * (txxp - txxm);
  double t22 = m.bu[j] * (tyyp - tyym);
  double t33 = m.cu[k] * (tzzp - tzzm);
  double s22 = m.bu[j] * (txyp - txym);
  double s33 = m.cu[k] * (txzp - txzm);
  return h11 + h22 + h33 + t11 + t22 + t33 + s22 + s33;
}

// v-momentum (src/rhs.f:219-321)
__device__ __forceinline__ double rhs_v(const Dims &d, const DevMetrics &m, double ru1,
                                        const double *__restrict__ uo, const double *__restrict__ vo,
                                        const double *__restrict__ wo, const double *__restrict__ tv,
                                        int i, int j, int k, long long q, int sy, long long sz) {
  const double *qr = uo;
  double vxp = (vo[q+1] + vo[q]) * 0.5;
  double vxm = (vo[q] + vo[q-1]) * 0.5;
  double vyp = (vo[q+sy] + vo[q]) * 0.5;
  double vym = (vo[q] + vo[q-sy]) * 0.5;
  double vzp = (vo[q+sz] + vo[q]) * 0.5;
  double vzm = (vo[q] + vo[q-sz]) * 0.5;
  double qyp = (qr[q+sy] + qr[q]) * 0.5;
  double qym = (qr[q-1+sy] + qr[q-1]) * 0.5;
  double wyp = (wo[q+sy] + wo[q]) * 0.5;
  double wym = (wo[q+sy-sz] + wo[q-sz]) * 0.5;
  double dvdxp = m.au[i] * (vo[q+1] - vo[q]);
  double dvdxm = m.au[i - 1] * (vo[q] - vo[q-1]);
  double dvdyp = m.bp[j + 1] * (vo[q+sy] - vo[q]);
  double dvdym = m.bp[j] * (vo[q] - vo[q-sy]);
  double dvdzp = m.cw[k] * (vo[q+sz] - vo[q]);
  double dvdzm = m.cw[k - 1] * (vo[q] - vo[q-sz]);
  double dudyp = m.bv[j] * (uo[q+sy] - uo[q]);
  double dudym = m.bv[j] * (uo[q-1+sy] - uo[q-1]);
  double dwdyp = m.bv[j] * (wo[q+sy] - wo[q]);
  double dwdym = m.bv[j] * (wo[q+sy-sz] - wo[q-sz]);
  double tvip = 0.25 * (tv[q+sy] + tv[q] + tv[q+1+sy] + tv[q+1]);
  double tvim = 0.25 * (tv[q+sy] + tv[q] + tv[q-1+sy] + tv[q-1]);
  double tvkp = 0.25 * (tv[q+sy] + tv[q] + tv[q+sy+sz] + tv[q+sz]);
  double tvkm = 0.25 * (tv[q+sy] + tv[q] + tv[q+sy-sz] + tv[q-sz]);
  double txxp = (ru1 + tvip) * dvdxp;
  double txxm = (ru1 + tvim) * dvdxm;
  double tyyp = (ru1 + 2. * tv[q+sy]) * dvdyp;
  double tyym = (ru1 + 2. * tv[q]) * dvdym;
  double tzzp = (ru1 + tvkp) * dvdzp;
  double tzzm = (ru1 + tvkm) * dvdzm;
  double txyp = tvip * dudyp;
  double txym = tvim * dudym;
  double tyzp = tvkp * dwdyp;
  double tyzm = tvkm * dwdym;
  double h11 = -m.av[i] * (qyp * vxp - qym * vxm);
  double h22 = -m.bv[j] * (vyp * vyp - vym * vym);
  double h33 = -m.cv[k] * (wyp * vzp - wym * vzm);
  double t11 = m.av[i] * (txxp - txxm);
  double t22 = m.bv[j] * (tyyp - tyym);
  double t33 = m.cv[k] * (tzzp - tzzm);
  double s11 = m.av[i] * (txyp - txym);
  double s33 = m.cv[k] * (tyzp - tyzm);
  return h11 + h22 + h33 + t11 + t22 + t33 + s11 + s33;
}

// w-momentum (src/rhs.f:347-422)
__device__ __forceinline__ double rhs_w(const Dims &d, const DevMetrics &m, double ru1,
                                        const double *__restrict__ uo, const double *__restrict__ vo,
                                        const double *__restrict__ wo, const double *__restrict__ tv,
                                        int i, int j, int k, long long q, int sy, long long sz) {
  const double *qr = uo;
  double wxp = (wo[q+1] + wo[q]) * 0.5;
  double wxm = (wo[q] + wo[q-1]) * 0.5;
  double wyp = (wo[q+sy] + wo[q]) * 0.5;
  double wym = (wo[q] + wo[q-sy]) * 0.5;
  double wzp = (wo[q+sz] + wo[q]) * 0.5;
  double wzm = (wo[q] + wo[q-sz]) * 0.5;
  double qzp = (qr[q+sz] + qr[q]) * 0.5;
  double qzm = (qr[q-1+sz] + qr[q-1]) * 0.5;
  double vzp = (vo[q+sz] + vo[q]) * 0.5;
  double vzm = (vo[q-sy+sz] + vo[q-sy]) * 0.5;
  double dwdxp = m.au[i] * (wo[q+1] - wo[q]);
  double dwdxm = m.au[i - 1] * (wo[q] - wo[q-1]);
  double dwdyp = m.bv[j] * (wo[q+sy] - wo[q]);
  double dwdym = m.bv[j - 1] * (wo[q] - wo[q-sy]);
  double dwdzp = m.cp[k + 1] * (wo[q+sz] - wo[q]);
  double dwdzm = m.cp[k] * (wo[q] - wo[q-sz]);
  double dudzp = m.cw[k] * (uo[q+sz] - uo[q]);
  double dudzm = m.cw[k] * (uo[q-1+sz] - uo[q-1]);
  double dvdzp = m.cw[k] * (vo[q+sz] - vo[q]);
  double dvdzm = m.cw[k] * (vo[q-sy+sz] - vo[q-sy]);
  double tvip = 0.25 * (tv[q+sz] + tv[q] + tv[q+1+sz] + tv[q+1]);
  double tvim = 0.25 * (tv[q+sz] + tv[q] + tv[q-1+sz] + tv[q-1]);
  double tvjp = 0.25 * (tv[q+sz] + tv[q] + tv[q+sy+sz] + tv[q+sy]);
  double tvjm = 0.25 * (tv[q+sz] + tv[q] + tv[q-sy+sz] + tv[q-sy]);
  double txxp = (ru1 + tvip) * dwdxp;
  double txxm = (ru1 + tvim) * dwdxm;
  double tyyp = (ru1 + tvjp) * dwdyp;
  double tyym = (ru1 + tvjm) * dwdym;
  double tzzp = (ru1 + 2. * tv[q+sz]) * dwdzp;
  double tzzm = (ru1 + 2. * tv[q]) * dwdzm;
  double txzp = tvip * dudzp;
  double txzm = tvim * dudzm;
  double tyzp = tvjp * dvdzp;
  double tyzm = tvjm * dvdzm;
  double h11 = -m.aw[i] * (qzp * wxp - qzm * wxm);
  double h22 = -m.bw[j] * (vzp * wyp - vzm * wym);
  double h33 = -m.cw[k] * (wzp * wzp - wzm * wzm);
  double t11 = m.aw[i] * (txxp - txxm);
  double t22 = m.bw[j] * (tyyp - tyym);
  double t33 = m.cw[k] * (tzzp - tzzm);
  double s11 = m.aw[i] * (txzp - txzm);
  double s22 = m.bw[j] * (tyzp - tyzm);
  return h11 + h22 + h33 + t11 + t22 + t33 + s11 + s22;
}

// RHS + PREDICTORD + sponges over the whole array (ghost cells of u*,v*,w*
// are zero, as RHS leaves them, src/rhs.f:65-70).
__global__ void __launch_bounds__(BX *BY *BZ)
    k_rhs_predictord(Dims d, DevMetrics m, Scalars s, const double *__restrict__ uo,
                     const double *__restrict__ vo, const double *__restrict__ wo,
                     const double *__restrict__ tv, const double *__restrict__ p,
                     const double *__restrict__ dens, double *__restrict__ us, double *__restrict__ vs,
                     double *__restrict__ ws, double *__restrict__ ua, double *__restrict__ va,
                     double *__restrict__ wa, double alfxdt, double gamxdt, double rhoxdt) {
  int i = 1 + threadIdx.x + blockIdx.x * BX;
  int j = 1 + threadIdx.y + blockIdx.y * BY;
  int k = 1 + threadIdx.z + blockIdx.z * BZ;
  if (i > d.nx || j > d.ny || k > d.nz) return;
  long long q = fidx(d, i, j, k);
  const int sy = d.nx;
  const long long sz = (long long)d.nx * d.ny;
  const double coef = 0.5 * alfxdt, coefd = alfxdt;
  const bool kin = (k >= d.kz1 && k <= d.kz2), jin = (j >= d.jy1 && j <= d.jy2);
  // ---- u ----
  double uval = 0.0;
  if (kin && jin && i >= d.ibu && i <= d.ieu) {
    double ur = rhs_u(d, m, s.ru1, uo, vo, wo, tv, i, j, k, q, sy, sz);
    double ustar = uo[q] + gamxdt * ur + rhoxdt * ua[q] - alfxdt * m.au[i] * (p[q + 1] - p[q]) +
                   coef * 0.0 - alfxdt * s.dpdx;
    if (s.idens == 1)
      ustar = ustar - coefd * 0.50 * s.grav *
                          ((dens[q + 1] - m.dens_bg[i + d.nx * (j - 1)]) +
                           (dens[q] - m.dens_bg[(i - 1) + d.nx * (j - 1)]));
    ua[q] = ur;
    if (i >= d.ieu - s.vspngx1) ustar = ustar + m.dfxu[i] * (0. - ustar) * alfxdt * 1.0;
    if (s.ivspngl == 1) ustar = ustar + m.dfxul[k] * (0. - ustar) * alfxdt * 1.0;
    uval = ustar;
  }
  us[q] = uval;
  // ---- v ----
  double vval = 0.0;
  if (kin && j >= d.jbv && j <= d.jev && i >= d.ix1 && i <= d.ix2) {
    double vr = rhs_v(d, m, s.ru1, uo, vo, wo, tv, i, j, k, q, sy, sz);
    double vstar = vo[q] + gamxdt * vr + rhoxdt * va[q] - alfxdt * m.bv[j] * (p[q + sy] - p[q]) +
                   coef * 0.0 - alfxdt * s.dpdy;
    va[q] = vr;
    if (i >= d.ix2 - s.vspngx1) vstar = vstar + m.dfxw[i] * (0. - vstar) * alfxdt * 1.0;
    if (s.ivspngl == 1 && i >= d.ibu && i <= d.ieu && jin) vstar = vstar + m.dfxwl[k] * (0. - vstar) * alfxdt * 1.0;
    vval = vstar;
  }
  vs[q] = vval;
  // ---- w ----
  double wval = 0.0;
  if (k >= d.kbw && k <= d.kew && jin && i >= d.ix1 && i <= d.ix2) {
    double wr = rhs_w(d, m, s.ru1, uo, vo, wo, tv, i, j, k, q, sy, sz);
    double wstar = wo[q] + gamxdt * wr + rhoxdt * wa[q] - alfxdt * m.cw[k] * (p[q + sz] - p[q]) +
                   coef * 0.0 - alfxdt * s.dpdz;
    wa[q] = wr;
    if (i >= d.ix2 - s.vspngx1) wstar = wstar + m.dfxw[i] * (1. - wstar) * alfxdt * 1.0;
    if (s.ivspngl == 1) wstar = wstar + m.dfxwl[k] * (1. - wstar) * alfxdt * 1.0;
    wval = wstar;
  }
  ws[q] = wval;
}

// ---------------------------------------------------------------------------
// plane fill a(dst) = sgn*a(src) (or 0) over a whole plane of one axis.
__global__ void k_fill_plane(Dims d, double *a, int axis, int dst, int src, double sgn, int zero) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int n1 = axis == 0 ? d.ny : d.nx;
  int n2 = axis == 2 ? d.ny : d.nz;
  if (t >= n1 * n2) return;
  int a1 = 1 + t % n1, a2 = 1 + t / n1;
  long long qd, qs;
  if (axis == 0) { qd = fidx(d, dst, a1, a2); qs = fidx(d, src, a1, a2); }
  else if (axis == 1) { qd = fidx(d, a1, dst, a2); qs = fidx(d, a1, src, a2); }
  else { qd = fidx(d, a1, a2, dst); qs = fidx(d, a1, a2, src); }
  a[qd] = zero ? 0. : sgn * a[qs];
}

// deterministic single-block sum over the interior (i,j) of plane k of
// a(i,j,k)/(ap(i)bp(j)) (flux through a z plane, src/boundary.f:787-795)
__global__ void k_plane_flux(Dims d, DevMetrics m, const double *a, int k, double *out) {
  __shared__ double sf[1024], sa[1024];
  int mi = d.ix2 - d.ix1 + 1, mj = d.jy2 - d.jy1 + 1;
  double f = 0., ar = 0.;
  for (int t = threadIdx.x; t < mi * mj; t += blockDim.x) {
    int i = d.ix1 + t % mi, j = d.jy1 + t / mi;
    double areaij = 1.0 / (m.ap[i] * m.bp[j]);
    f = f + a[fidx(d, i, j, k)] * areaij;
    ar = ar + areaij;
  }
  sf[threadIdx.x] = f;
  sa[threadIdx.x] = ar;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      sf[threadIdx.x] += sf[threadIdx.x + w];
      sa[threadIdx.x] += sa[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sf[0];
    out[1] = sa[0];
  }
}

__global__ void k_inlet_plane(Dims d, double *ubc, double *vbc, double *wbc, const double *pu,
                              const double *pv, const double *pw) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.nx * d.ny) return;
  long long q = (long long)t;  // k = 1 plane
  ubc[q] = pu[t];
  vbc[q] = pv[t];
  wbc[q] = pw[t];
}

// 730 convective outflow, predictor (src/boundary.f:853-870); flux[0..1] inlet
__global__ void k_outlet_convective(Dims d, DevMetrics m, double *ubc, double *vbc, double *wbc,
                                    const double *uof, const double *vof, const double *wof,
                                    const double *flux_in, double alfxdt) {
  int mi = d.ix2 - d.ix1 + 1, mj = d.jy2 - d.jy1 + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= mi * mj) return;
  int i = d.ix1 + t % mi, j = d.jy1 + t / mi;
  double qin2 = flux_in[0] / flux_in[1];
  double coef = qin2 * alfxdt * m.cp[d.kz2];
  int NZ = d.nz, kz2 = d.kz2;
  long long qn = fidx(d, i, j, NZ), qk = fidx(d, i, j, kz2), qkm = fidx(d, i, j, kz2 - 1);
  ubc[qn] = uof[qn] - coef * (uof[qn] - uof[qk]);
  vbc[qn] = vof[qn] - coef * (vof[qn] - vof[qk]);
  wbc[qk] = wof[qk] - coef * (wof[qk] - wof[qkm]);
}

// y periodic ghost rows of three arrays over all i,k (src/boundary.f:862-867)
__global__ void k_yper3(Dims d, double *a, double *b, double *c) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.nx * d.nz) return;
  int i = 1 + t % d.nx, k = 1 + t / d.nx;
  double *arr[3] = {a, b, c};
  for (int s = 0; s < 3; s++) {
    double *x = arr[s];
    x[fidx(d, i, 1, k)] = x[fidx(d, i, d.ny - 1, k)];
    x[fidx(d, i, d.ny, k)] = x[fidx(d, i, 2, k)];
  }
}

// outflow mass balance (src/boundary.f:920-944)
__global__ void k_outlet_rescale(Dims d, double *wbc, const double *flux_in, const double *flux_out) {
  int mi = d.ix2 - d.ix1 + 1, mj = d.jy2 - d.jy1 + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= mi * mj) return;
  int i = d.ix1 + t % mi, j = d.jy1 + t / mi;
  long long q = fidx(d, i, j, d.kz2);
  double qin1 = flux_in[0], qout = flux_out[0];
  if (qout != 0.) {
    double c = qin1 / qout;
    wbc[q] = wbc[q] * c;
  } else {
    wbc[q] = qin1 / flux_out[1];
  }
}

// corrector 730/731 and 710 copies (src/boundary.f:947-980)
__global__ void k_outlet_corrector(Dims d, double *ubc, double *vbc, double *wbc, const double *uof,
                                   const double *vof, const double *wof, int t6) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.nx * d.ny) return;
  int i = 1 + t % d.nx, j = 1 + t / d.nx;
  long long qn = fidx(d, i, j, d.nz), qk = fidx(d, i, j, d.kz2);
  if (t6 == 730 || t6 == 731) {
    ubc[qn] = uof[qn];
    vbc[qn] = vof[qn];
    wbc[qk] = wof[qk];
  } else if (t6 == 710) {
    ubc[qn] = uof[qk];
    vbc[qn] = vof[qk];
    wbc[qk] = wof[qk];
  }
}

// CORRECT (src/timeindeg.f:981-1028)
__global__ void __launch_bounds__(BX *BY *BZ)
    k_correct(Dims d, DevMetrics m, const double *__restrict__ us, const double *__restrict__ vs,
              const double *__restrict__ ws, const double *__restrict__ dp, double *__restrict__ uo,
              double *__restrict__ vo, double *__restrict__ wo, double alfxdt) {
  int i = 1 + threadIdx.x + blockIdx.x * BX;
  int j = 1 + threadIdx.y + blockIdx.y * BY;
  int k = 1 + threadIdx.z + blockIdx.z * BZ;
  if (i > d.nx || j > d.ny || k > d.nz) return;
  long long q = fidx(d, i, j, k);
  const int sy = d.nx;
  const long long sz = (long long)d.nx * d.ny;
  bool kin = k >= d.kz1 && k <= d.kz2, jin = j >= d.jy1 && j <= d.jy2;
  if (kin && jin && i >= d.ibu && i <= d.ieu)
    uo[q] = us[q] - m.au[i] * (dp[q + 1] - dp[q]) * alfxdt;
  if (kin && j >= d.jbv && j <= d.jev && i >= d.ix1 && i <= d.ix2)
    vo[q] = vs[q] - m.bv[j] * (dp[q + sy] - dp[q]) * alfxdt;
  if (k >= d.kbw && k <= d.kew && jin && i >= d.ix1 && i <= d.ix2)
    wo[q] = ws[q] - m.cw[k] * (dp[q + sz] - dp[q]) * alfxdt;
}

// pref = sum_j (p+dp)(ix1,j,2) / (NY-2), summed in order (src/Eddy6.f:2802)
__global__ void k_pref(Dims d, const double *p, const double *dp, double *out) {
  double s = 0.;
  for (int j = d.jy1; j <= d.jy2; j++) {
    long long q = fidx(d, d.ix1, j, 2);
    s += p[q] + dp[q];
  }
  out[0] = s / (double)(d.ny - 2);
}

__global__ void __launch_bounds__(256) k_pupdate(Dims d, double *p, const double *dp, const double *pref) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= d.ncell) return;
  p[q] = (p[q] + dp[q]) - pref[0];
}

// final pressure ghosts: value of the mapped interior cell (the composition
// of the z, x, y fills of src/Eddy6.f:2911-2953)
__device__ __forceinline__ int map_axis(int a, int n, int lo, int hi, int periodic, int active) {
  if (!active) return a;
  if (a == 1) return periodic ? hi : lo;
  if (a == n) return periodic ? lo : hi;
  return a;
}

__global__ void k_pghost(Dims d, double *p) {
  // threads over all ghost cells of the 6 faces (grid-stride over the volume
  // surface via three plane sets)
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long sxy = (long long)d.nx * d.ny, sxz = (long long)d.nx * d.nz, syz = (long long)d.ny * d.nz;
  int i, j, k;
  if (t < 2 * sxy) {
    int f = (int)(t / sxy);
    long long r = t % sxy;
    i = 1 + (int)(r % d.nx); j = 1 + (int)(r / d.nx); k = f ? d.nz : 1;
  } else if (t < 2 * sxy + 2 * sxz) {
    long long u = t - 2 * sxy;
    int f = (int)(u / sxz);
    long long r = u % sxz;
    i = 1 + (int)(r % d.nx); k = 1 + (int)(r / d.nx); j = f ? d.ny : 1;
  } else if (t < 2 * sxy + 2 * sxz + 2 * syz) {
    long long u = t - 2 * sxy - 2 * sxz;
    int f = (int)(u / syz);
    long long r = u % syz;
    j = 1 + (int)(r % d.ny); k = 1 + (int)(r / d.ny); i = f ? d.nx : 1;
  } else {
    return;
  }
  int zact = d.itype[5] != 0 || d.itype[6] != 0;
  int zper = d.itype[5] == 500;
  int si = map_axis(i, d.nx, d.ix1, d.ix2, d.mp == 0, 1);
  int sj = map_axis(j, d.ny, d.jy1, d.jy2, d.lp == 0, 1);
  int sk = map_axis(k, d.nz, d.kz1, d.kz2, zper, zact);
  if (si == i && sj == j && sk == k) return;
  p[fidx(d, i, j, k)] = p[fidx(d, si, sj, sk)];
}

inline dim3 grid3(const Dims &d) {
  return dim3((d.nx + BX - 1) / BX, (d.ny + BY - 1) / BY, (d.nz + BZ - 1) / BZ);
}

int fill(eddy_ctx *ctx, double *a, int axis, int dst, int src, double sgn, int zero) {
  const Dims &d = ctx->d;
  int n = axis == 0 ? d.ny * d.nz : (axis == 1 ? d.nx * d.nz : d.nx * d.ny);
  k_fill_plane<<<(n + 255) / 256, 256, 0, ctx->stream>>>(d, a, axis, dst, src, sgn, zero);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

}  // namespace

int launch_fill_plane(eddy_ctx *ctx, double *a, int axis, int dst, int src, double sgn, int zero) {
  return fill(ctx, a, axis, dst, src, sgn, zero);
}

int launch_rhs_predictord(eddy_ctx *ctx, double alfxdt, double gamxdt, double rhoxdt) {
  const Dims &d = ctx->d;
  double **f = ctx->f;
  k_rhs_predictord<<<grid3(d), dim3(BX, BY, BZ), 0, ctx->stream>>>(
      d, ctx->m, ctx->sc, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], f[EDDY_TV], f[EDDY_P], f[EDDY_DENS],
      f[EDDY_US], f[EDDY_VS], f[EDDY_WS], f[EDDY_UA], f[EDDY_VA], f[EDDY_WA], alfxdt, gamxdt, rhoxdt);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

// BOUNDARY (src/boundary.f:7-66): wall types first, then periodic x/y.
int launch_boundary(eddy_ctx *ctx, double *u, double *v, double *w) {
  const Dims &d = ctx->d;
  int rc;
#define F(...) \
  if ((rc = fill(ctx, __VA_ARGS__)) != EDDY_OK) return rc
  for (int ib = 1; ib <= 6; ib++) {
    int t = d.itype[ib];
    if (t == 50 || t == 60) {
      double sg = (t == 50) ? -1. : 1.;
      switch (ib) {
        case 1: F(u, 0, 1, 0, 0., 1); F(v, 0, 1, d.ix1, sg, 0); F(w, 0, 1, d.ix1, sg, 0); break;
        case 2: F(u, 0, d.ix2, 0, 0., 1); F(v, 0, d.nx, d.ix2, sg, 0); F(w, 0, d.nx, d.ix2, sg, 0); break;
        case 3: F(u, 1, 1, d.jy1, sg, 0); F(v, 1, 1, 0, 0., 1); F(w, 1, 1, d.jy1, sg, 0); break;
        case 4: F(u, 1, d.ny, d.jy2, sg, 0); F(v, 1, d.jy2, 0, 0., 1); F(w, 1, d.ny, d.jy2, sg, 0); break;
        case 5: F(u, 2, 1, d.kz1, sg, 0); F(v, 2, 1, d.kz1, sg, 0); F(w, 2, 1, 0, 0., 1); break;
        case 6: F(u, 2, d.nz, d.kz2, sg, 0); F(v, 2, d.nz, d.kz2, sg, 0); F(w, 2, d.kz2, 0, 0., 1); break;
      }
    } else if (t == 82) {
      if (ib == 1) { F(u, 0, 1, d.ix1, 1., 0); F(v, 0, 1, d.ix1, -1., 0); F(w, 0, 1, d.ix1, -1., 0); }
      if (ib == 2) { F(u, 0, d.nx, d.ix2, 1., 0); F(v, 0, d.nx, d.ix2, 1., 0); F(w, 0, d.nx, d.ix2, 1., 0); }
    }
  }
  if (d.itype[1] == 500) {
    F(u, 0, 1, d.ix2, 1., 0); F(v, 0, 1, d.ix2, 1., 0); F(w, 0, 1, d.ix2, 1., 0);
    F(u, 0, d.nx, d.ix1, 1., 0); F(v, 0, d.nx, d.ix1, 1., 0); F(w, 0, d.nx, d.ix1, 1., 0);
  }
  if (d.itype[3] == 500) {
    F(u, 1, 1, d.jy2, 1., 0); F(v, 1, 1, d.jy2, 1., 0); F(w, 1, 1, d.jy2, 1., 0);
    F(u, 1, d.ny, d.jy1, 1., 0); F(v, 1, d.ny, d.jy1, 1., 0); F(w, 1, d.ny, d.jy1, 1., 0);
  }
#undef F
  return EDDY_OK;
}

// BOUNDINOUT (src/boundary.f:505-994) for inlet 305 and outlets 710/720/730.
int launch_boundinout(eddy_ctx *ctx, double *ubc, double *vbc, double *wbc, const double *uof,
                      const double *vof, const double *wof, double alfxdt, int idiv) {
  const Dims &d = ctx->d;
  cudaStream_t st = ctx->stream;
  double *fin = ctx->scal + 8, *fout = ctx->scal + 10;
  int n2 = d.nx * d.ny, nin = (d.ix2 - d.ix1 + 1) * (d.jy2 - d.jy1 + 1);
  int iinq = idiv;
  if (d.itype[5] == 305) {
    k_inlet_plane<<<(n2 + 255) / 256, 256, 0, st>>>(d, ubc, vbc, wbc, ctx->f[EDDY_PLANEU],
                                                    ctx->f[EDDY_PLANEV], ctx->f[EDDY_PLANEW]);
    EDDY_LAUNCHED(ctx);
  } else {
    iinq = 0;
  }
  int t6 = d.itype[6];
  if (idiv == 1) {
    if (t6 == 710 || t6 == 720) {
      ctx->err = "outlet types 710/720 are not on the restated hot path";
      return EDDY_EINVAL;
    }
    if (t6 != 730) return EDDY_OK;
    if (iinq != 1) {
      ctx->err = "convective outlet needs the 305 inlet flux";
      return EDDY_EINVAL;
    }
    k_plane_flux<<<1, 1024, 0, st>>>(d, ctx->m, wbc, 1, fin);
    EDDY_LAUNCHED(ctx);
    k_outlet_convective<<<(nin + 255) / 256, 256, 0, st>>>(d, ctx->m, ubc, vbc, wbc, uof, vof, wof, fin,
                                                           alfxdt);
    EDDY_LAUNCHED(ctx);
    k_yper3<<<(d.nx * d.nz + 255) / 256, 256, 0, st>>>(d, ubc, vbc, wbc);
    EDDY_LAUNCHED(ctx);
    k_plane_flux<<<1, 1024, 0, st>>>(d, ctx->m, wbc, d.kz2, fout);
    EDDY_LAUNCHED(ctx);
    k_outlet_rescale<<<(nin + 255) / 256, 256, 0, st>>>(d, wbc, fin, fout);
    EDDY_LAUNCHED(ctx);
  } else {
    if (t6 == 720) {
      ctx->err = "outlet type 720 is not on the restated hot path";
      return EDDY_EINVAL;
    }
    k_outlet_corrector<<<(n2 + 255) / 256, 256, 0, st>>>(d, ubc, vbc, wbc, uof, vof, wof, t6);
    EDDY_LAUNCHED(ctx);
  }
  return EDDY_OK;
}

int launch_correct(eddy_ctx *ctx, double alfxdt) {
  const Dims &d = ctx->d;
  double **f = ctx->f;
  k_correct<<<grid3(d), dim3(BX, BY, BZ), 0, ctx->stream>>>(d, ctx->m, f[EDDY_US], f[EDDY_VS], f[EDDY_WS],
                                                            f[EDDY_DP], f[EDDY_UO], f[EDDY_VO], f[EDDY_WO],
                                                            alfxdt);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

int launch_pressure_update(eddy_ctx *ctx) {
  const Dims &d = ctx->d;
  double *p = ctx->f[EDDY_P], *dp = ctx->f[EDDY_DP];
  k_pref<<<1, 1, 0, ctx->stream>>>(d, p, dp, ctx->scal);
  EDDY_LAUNCHED(ctx);
  k_pupdate<<<(unsigned)((d.ncell + 255) / 256), 256, 0, ctx->stream>>>(d, p, dp, ctx->scal);
  EDDY_LAUNCHED(ctx);
  long long nghost = 2LL * d.nx * d.ny + 2LL * d.nx * d.nz + 2LL * d.ny * d.nz;
  k_pghost<<<(unsigned)((nghost + 255) / 256), 256, 0, ctx->stream>>>(d, p);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}
