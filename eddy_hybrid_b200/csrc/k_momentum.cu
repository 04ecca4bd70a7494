// k_momentum.cu -- momentum right-hand side fused with the RK predictor,
// boundary-condition plane fills, BOUNDINOUT, CORRECT and the pressure update.
//
// Plain FP64 form: compiled with -fmad=false so every expression rounds in the
// reference's operation order (src/rhs.f, src/timeindeg.f); the explicit
// (non Crank-Nicolson) branch of the Cartesian equations.
#include "eddy_internal.h"
#include "tma_ring.cuh"

#define A(a, i, j, k) (a)[fidx(d, (i), (j), (k))]

namespace {

constexpr int BX = 32, BY = 4, BZ = 2;

// ---------------------------------------------------------------------------
// u-momentum explicit RHS at a u point (src/rhs.f:77-172)
template <class Acc>
__device__ __forceinline__ double rhs_u(const Acc &S, const DevMetrics &m, double ru1, int i, int j, int k) {
  double qxp = (S.u(1, 0, 0) + S.u(0, 0, 0)) * 0.5;
  double qxm = (S.u(0, 0, 0) + S.u(-1, 0, 0)) * 0.5;
  double uxp = (S.u(1, 0, 0) + S.u(0, 0, 0)) * 0.5;
  double uxm = (S.u(0, 0, 0) + S.u(-1, 0, 0)) * 0.5;
  double uyp = (S.u(0, 1, 0) + S.u(0, 0, 0)) * 0.5;
  double uym = (S.u(0, 0, 0) + S.u(0, -1, 0)) * 0.5;
  double uzp = (S.u(0, 0, 1) + S.u(0, 0, 0)) * 0.5;
  double uzm = (S.u(0, 0, 0) + S.u(0, 0, -1)) * 0.5;
  double vxp = (S.v(1, 0, 0) + S.v(0, 0, 0)) * 0.5;
  double vxm = (S.v(1, -1, 0) + S.v(0, -1, 0)) * 0.5;
  double wxp = (S.w(1, 0, 0) + S.w(0, 0, 0)) * 0.5;
  double wxm = (S.w(1, 0, -1) + S.w(0, 0, -1)) * 0.5;
  double dqdxp = m.ap[i + 1] * (S.u(1, 0, 0) - S.u(0, 0, 0));
  double dqdxm = m.ap[i] * (S.u(0, 0, 0) - S.u(-1, 0, 0));
  double dudyp = m.bv[j] * (S.u(0, 1, 0) - S.u(0, 0, 0));
  double dudym = m.bv[j - 1] * (S.u(0, 0, 0) - S.u(0, -1, 0));
  double dudzp = m.cw[k] * (S.u(0, 0, 1) - S.u(0, 0, 0));
  double dudzm = m.cw[k - 1] * (S.u(0, 0, 0) - S.u(0, 0, -1));
  double dvdxp = m.au[i] * (S.v(1, 0, 0) - S.v(0, 0, 0));
  double dvdxm = m.au[i] * (S.v(1, -1, 0) - S.v(0, -1, 0));
  double dwdxp = m.au[i] * (S.w(1, 0, 0) - S.w(0, 0, 0));
  double dwdxm = m.au[i] * (S.w(1, 0, -1) - S.w(0, 0, -1));
  double tvjp = 0.25 * (S.t(1, 0, 0) + S.t(0, 0, 0) + S.t(1, 1, 0) + S.t(0, 1, 0));
  double tvjm = 0.25 * (S.t(1, 0, 0) + S.t(0, 0, 0) + S.t(1, -1, 0) + S.t(0, -1, 0));
  double tvkp = 0.25 * (S.t(1, 0, 0) + S.t(0, 0, 0) + S.t(1, 0, 1) + S.t(0, 0, 1));
  double tvkm = 0.25 * (S.t(1, 0, 0) + S.t(0, 0, 0) + S.t(1, 0, -1) + S.t(0, 0, -1));
  double txxp = (ru1 + 2. * S.t(1, 0, 0)) * dqdxp;
  double txxm = (ru1 + 2. * S.t(0, 0, 0)) * dqdxm;
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
template <class Acc>
__device__ __forceinline__ double rhs_v(const Acc &S, const DevMetrics &m, double ru1, int i, int j, int k) {
  double vxp = (S.v(1, 0, 0) + S.v(0, 0, 0)) * 0.5;
  double vxm = (S.v(0, 0, 0) + S.v(-1, 0, 0)) * 0.5;
  double vyp = (S.v(0, 1, 0) + S.v(0, 0, 0)) * 0.5;
  double vym = (S.v(0, 0, 0) + S.v(0, -1, 0)) * 0.5;
  double vzp = (S.v(0, 0, 1) + S.v(0, 0, 0)) * 0.5;
  double vzm = (S.v(0, 0, 0) + S.v(0, 0, -1)) * 0.5;
  double qyp = (S.u(0, 1, 0) + S.u(0, 0, 0)) * 0.5;
  double qym = (S.u(-1, 1, 0) + S.u(-1, 0, 0)) * 0.5;
  double wyp = (S.w(0, 1, 0) + S.w(0, 0, 0)) * 0.5;
  double wym = (S.w(0, 1, -1) + S.w(0, 0, -1)) * 0.5;
  double dvdxp = m.au[i] * (S.v(1, 0, 0) - S.v(0, 0, 0));
  double dvdxm = m.au[i - 1] * (S.v(0, 0, 0) - S.v(-1, 0, 0));
  double dvdyp = m.bp[j + 1] * (S.v(0, 1, 0) - S.v(0, 0, 0));
  double dvdym = m.bp[j] * (S.v(0, 0, 0) - S.v(0, -1, 0));
  double dvdzp = m.cw[k] * (S.v(0, 0, 1) - S.v(0, 0, 0));
  double dvdzm = m.cw[k - 1] * (S.v(0, 0, 0) - S.v(0, 0, -1));
  double dudyp = m.bv[j] * (S.u(0, 1, 0) - S.u(0, 0, 0));
  double dudym = m.bv[j] * (S.u(-1, 1, 0) - S.u(-1, 0, 0));
  double dwdyp = m.bv[j] * (S.w(0, 1, 0) - S.w(0, 0, 0));
  double dwdym = m.bv[j] * (S.w(0, 1, -1) - S.w(0, 0, -1));
  double tvip = 0.25 * (S.t(0, 1, 0) + S.t(0, 0, 0) + S.t(1, 1, 0) + S.t(1, 0, 0));
  double tvim = 0.25 * (S.t(0, 1, 0) + S.t(0, 0, 0) + S.t(-1, 1, 0) + S.t(-1, 0, 0));
  double tvkp = 0.25 * (S.t(0, 1, 0) + S.t(0, 0, 0) + S.t(0, 1, 1) + S.t(0, 0, 1));
  double tvkm = 0.25 * (S.t(0, 1, 0) + S.t(0, 0, 0) + S.t(0, 1, -1) + S.t(0, 0, -1));
  double txxp = (ru1 + tvip) * dvdxp;
  double txxm = (ru1 + tvim) * dvdxm;
  double tyyp = (ru1 + 2. * S.t(0, 1, 0)) * dvdyp;
  double tyym = (ru1 + 2. * S.t(0, 0, 0)) * dvdym;
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
template <class Acc>
__device__ __forceinline__ double rhs_w(const Acc &S, const DevMetrics &m, double ru1, int i, int j, int k) {
  double wxp = (S.w(1, 0, 0) + S.w(0, 0, 0)) * 0.5;
  double wxm = (S.w(0, 0, 0) + S.w(-1, 0, 0)) * 0.5;
  double wyp = (S.w(0, 1, 0) + S.w(0, 0, 0)) * 0.5;
  double wym = (S.w(0, 0, 0) + S.w(0, -1, 0)) * 0.5;
  double wzp = (S.w(0, 0, 1) + S.w(0, 0, 0)) * 0.5;
  double wzm = (S.w(0, 0, 0) + S.w(0, 0, -1)) * 0.5;
  double qzp = (S.u(0, 0, 1) + S.u(0, 0, 0)) * 0.5;
  double qzm = (S.u(-1, 0, 1) + S.u(-1, 0, 0)) * 0.5;
  double vzp = (S.v(0, 0, 1) + S.v(0, 0, 0)) * 0.5;
  double vzm = (S.v(0, -1, 1) + S.v(0, -1, 0)) * 0.5;
  double dwdxp = m.au[i] * (S.w(1, 0, 0) - S.w(0, 0, 0));
  double dwdxm = m.au[i - 1] * (S.w(0, 0, 0) - S.w(-1, 0, 0));
  double dwdyp = m.bv[j] * (S.w(0, 1, 0) - S.w(0, 0, 0));
  double dwdym = m.bv[j - 1] * (S.w(0, 0, 0) - S.w(0, -1, 0));
  double dwdzp = m.cp[k + 1] * (S.w(0, 0, 1) - S.w(0, 0, 0));
  double dwdzm = m.cp[k] * (S.w(0, 0, 0) - S.w(0, 0, -1));
  double dudzp = m.cw[k] * (S.u(0, 0, 1) - S.u(0, 0, 0));
  double dudzm = m.cw[k] * (S.u(-1, 0, 1) - S.u(-1, 0, 0));
  double dvdzp = m.cw[k] * (S.v(0, 0, 1) - S.v(0, 0, 0));
  double dvdzm = m.cw[k] * (S.v(0, -1, 1) - S.v(0, -1, 0));
  double tvip = 0.25 * (S.t(0, 0, 1) + S.t(0, 0, 0) + S.t(1, 0, 1) + S.t(1, 0, 0));
  double tvim = 0.25 * (S.t(0, 0, 1) + S.t(0, 0, 0) + S.t(-1, 0, 1) + S.t(-1, 0, 0));
  double tvjp = 0.25 * (S.t(0, 0, 1) + S.t(0, 0, 0) + S.t(0, 1, 1) + S.t(0, 1, 0));
  double tvjm = 0.25 * (S.t(0, 0, 1) + S.t(0, 0, 0) + S.t(0, -1, 1) + S.t(0, -1, 0));
  double txxp = (ru1 + tvip) * dwdxp;
  double txxm = (ru1 + tvim) * dwdxm;
  double tyyp = (ru1 + tvjp) * dwdyp;
  double tyym = (ru1 + tvjm) * dwdym;
  double tzzp = (ru1 + 2. * S.t(0, 0, 1)) * dwdzp;
  double tzzm = (ru1 + 2. * S.t(0, 0, 0)) * dwdzm;
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

// RHS + PREDICTORD + sponges (src/rhs.f:4-438, src/timeindeg.f:1041-1265).
// A block owns a 32x8 tile of (i,j) columns and marches along k over a chunk
// of planes; planes of uo,vo,wo,tv,p,dens,ua,va,wa (one-cell halo in i and j)
// stream into the shared-memory ring of tma_ring.cuh.
constexpr int TX = 32, TY = 8, NFLD = 9, KCHUNK = 32;  // uo vo wo tv p dens ua va wa
using Acc9 = RingAcc<TX, TY, NFLD>;

struct MomAcc {
  const Acc9 &r;
  __device__ __forceinline__ double u(int di, int dj, int dk) const { return r.at(0, di, dj, dk); }
  __device__ __forceinline__ double v(int di, int dj, int dk) const { return r.at(1, di, dj, dk); }
  __device__ __forceinline__ double w(int di, int dj, int dk) const { return r.at(2, di, dj, dk); }
  __device__ __forceinline__ double t(int di, int dj, int dk) const { return r.at(3, di, dj, dk); }
};

__global__ void __launch_bounds__(TX *TY)
    k_rhs_predictord(Dims d, DevMetrics m, Scalars s, const __grid_constant__ TmaMaps<NFLD> maps,
                     double *__restrict__ us, double *__restrict__ vs, double *__restrict__ ws,
                     double *__restrict__ ua, double *__restrict__ va, double *__restrict__ wa, double alfxdt,
                     double gamxdt, double rhoxdt, int *err) {
  const double coef = 0.5 * alfxdt, coefd = alfxdt;
  tma_march<NFLD, TX, TY, KCHUNK>(
      d.ix1, d.ix2, d.jy1, d.jy2, d.kz1, d.kz2, maps, err, [&](int i, int j, int k, bool active, const Acc9 &R) {
        if (!active) return;
        MomAcc S{R};
        long long q = fidx(d, i, j, k);
        const bool jin = j >= d.jy1 && j <= d.jy2;
        const bool kin = (k >= d.kz1 && k <= d.kz2);
        // ---- u ----
        double uval = 0.0;
        if (kin && jin && i >= d.ibu && i <= d.ieu) {
          double ur = rhs_u(S, m, s.ru1, i, j, k);
          double ustar = R.at(0, 0, 0, 0) + gamxdt * ur + rhoxdt * R.at(6, 0, 0, 0) -
                         alfxdt * m.au[i] * (R.at(4, 1, 0, 0) - R.at(4, 0, 0, 0)) + coef * 0.0 - alfxdt * s.dpdx;
          if (s.idens == 1)
            ustar = ustar - coefd * 0.50 * s.grav *
                                ((R.at(5, 1, 0, 0) - m.dens_bg[i + d.nx * (j - 1)]) +
                                 (R.at(5, 0, 0, 0) - m.dens_bg[(i - 1) + d.nx * (j - 1)]));
          ua[q] = ur;
          if (i >= d.ieu - s.vspngx1) ustar = ustar + m.dfxu[i] * (0. - ustar) * alfxdt * 1.0;
          if (s.ivspngl == 1) ustar = ustar + m.dfxul[k] * (0. - ustar) * alfxdt * 1.0;
          uval = ustar;
        }
        us[q] = uval;
        // ---- v ----
        double vval = 0.0;
        if (kin && j >= d.jbv && j <= d.jev && i >= d.ix1 && i <= d.ix2) {
          double vr = rhs_v(S, m, s.ru1, i, j, k);
          double vstar = R.at(1, 0, 0, 0) + gamxdt * vr + rhoxdt * R.at(7, 0, 0, 0) -
                         alfxdt * m.bv[j] * (R.at(4, 0, 1, 0) - R.at(4, 0, 0, 0)) + coef * 0.0 - alfxdt * s.dpdy;
          va[q] = vr;
          if (i >= d.ix2 - s.vspngx1) vstar = vstar + m.dfxw[i] * (0. - vstar) * alfxdt * 1.0;
          if (s.ivspngl == 1 && i >= d.ibu && i <= d.ieu && jin)
            vstar = vstar + m.dfxwl[k] * (0. - vstar) * alfxdt * 1.0;
          vval = vstar;
        }
        vs[q] = vval;
        // ---- w ----
        double wval = 0.0;
        if (k >= d.kbw && k <= d.kew && jin && i >= d.ix1 && i <= d.ix2) {
          double wr = rhs_w(S, m, s.ru1, i, j, k);
          double wstar = R.at(2, 0, 0, 0) + gamxdt * wr + rhoxdt * R.at(8, 0, 0, 0) -
                         alfxdt * m.cw[k] * (R.at(4, 0, 0, 1) - R.at(4, 0, 0, 0)) + coef * 0.0 - alfxdt * s.dpdz;
          wa[q] = wr;
          if (i >= d.ix2 - s.vspngx1) wstar = wstar + m.dfxw[i] * (1. - wstar) * alfxdt * 1.0;
          if (s.ivspngl == 1) wstar = wstar + m.dfxwl[k] * (1. - wstar) * alfxdt * 1.0;
          wval = wstar;
        }
        ws[q] = wval;
      });
}

// ghost faces of u*,v*,w* are zero (RHS zeroes the whole arrays, src/rhs.f:65-70)
__global__ void k_zero_faces3(Dims d, double *a, double *b, double *c3) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long sxy = (long long)d.nx * d.ny, sxz = (long long)d.nx * d.nz, syz = (long long)d.ny * d.nz;
  int i, j, k;
  if (t < 2 * sxy) {
    long long r = t % sxy;
    i = 1 + (int)(r % d.nx); j = 1 + (int)(r / d.nx); k = (t / sxy) ? d.nz : 1;
  } else if (t < 2 * sxy + 2 * sxz) {
    long long u = t - 2 * sxy, r = u % sxz;
    i = 1 + (int)(r % d.nx); k = 1 + (int)(r / d.nx); j = (u / sxz) ? d.ny : 1;
  } else if (t < 2 * sxy + 2 * sxz + 2 * syz) {
    long long u = t - 2 * sxy - 2 * sxz, r = u % syz;
    j = 1 + (int)(r % d.ny); k = 1 + (int)(r / d.ny); i = (u / syz) ? d.nx : 1;
  } else {
    return;
  }
  long long q = fidx(d, i, j, k);
  a[q] = 0.;
  b[q] = 0.;
  c3[q] = 0.;
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
  TmaMaps<NFLD> maps;
  const double *src[NFLD] = {f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], f[EDDY_TV], f[EDDY_P], f[EDDY_DENS],
                             f[EDDY_UA], f[EDDY_VA], f[EDDY_WA]};
  for (int q = 0; q < NFLD; q++) {
    const CUtensorMap *mp = ctx_tensor_map(ctx, src[q], TX + 2, TY + 2);
    if (!mp) return EDDY_ECUDA;
    maps.m[q] = *mp;
  }
  size_t smem = ring_smem_bytes<NFLD, TX, TY>();
  EDDY_CUDA(cudaFuncSetAttribute(k_rhs_predictord, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 g((d.ix2 - d.ix1 + TX) / TX, (d.jy2 - d.jy1 + TY) / TY, (d.kz2 - d.kz1 + KCHUNK) / KCHUNK);
  k_rhs_predictord<<<g, dim3(TX, TY), smem, ctx->stream>>>(d, ctx->m, ctx->sc, maps, f[EDDY_US], f[EDDY_VS],
                                                          f[EDDY_WS], f[EDDY_UA], f[EDDY_VA], f[EDDY_WA], alfxdt,
                                                          gamxdt, rhoxdt, ctx->err_flag);
  EDDY_LAUNCHED(ctx);
  long long nghost = 2LL * d.nx * d.ny + 2LL * d.nx * d.nz + 2LL * d.ny * d.nz;
  k_zero_faces3<<<(unsigned)((nghost + 255) / 256), 256, 0, ctx->stream>>>(d, f[EDDY_US], f[EDDY_VS],
                                                                            f[EDDY_WS]);
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
