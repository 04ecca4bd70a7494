// k_implicit.cu -- Crank-Nicolson viscous (IMPLY) and convective (IMPLCY)
// terms along the periodic y axis (IMPLYDCMP = 0): INVERSEY
// (src/timeindeg.f:120-340) on the predicted velocities US, VS, WS and
// INVERSEYD / INVERSEYD_NEW (src/density.f:290-460) on the predicted density
// RS; and along x (IMPLX, IMPLCX; IMPLXDCMP = 0): INVERSEX
// (src/timeindeg.f:344-690) and INVERSEXD (src/density.f:129-290).
//
// Every (i,k) line of a component is one periodic tridiagonal system over the
// jy1..jy2 cells, (1 + D) x = r with D the C.N. half of the y diffusion.  One
// thread solves one line (threads along i: every row access is coalesced):
// the corner entries by Sherman-Morrison on top of a Thomas elimination, the
// published method of the reference's solver (src/numrec.f:754-800), in its
// operation order, so that with -fmad=false the result is the reference
// restatement's bit for bit.  The forward sweep writes the eliminated
// solution in place, the multipliers and the Sherman-Morrison vector to two
// scratch fields; two more sweeps finish the back substitution and the
// correction.  The flags scale their coefficients at run time: a flag of 0
// multiplies its terms by an exact zero, as the reference's rflag factors do.
// Cartesian: rp = ru = 1.
#include "eddy_internal.h"

namespace {

// row j of line (i,k): sub-, main and super-diagonal and an addend of the
// right-hand side.  fy = rflagy (IMPLY) scales the viscous coefficients, fc =
// rflagcy (IMPLCY) the convective ones (timeindeg.f:150-312)
struct RowV {  // v: viscosity 2 tv(j) and 2 tv(j+1) on the faces; convection about VO
  const double *__restrict__ tv, *__restrict__ bv, *__restrict__ bp, *__restrict__ vo;
  double coef, ru1, fy, fc;
  __device__ void operator()(const Dims &d, int i, int j, int k, double &a, double &b, double &c, double &r) const {
    const double tvjp = 2. * tv[fidx(d, i, j + 1, k)] + ru1, tvjm = 2. * tv[fidx(d, i, j, k)] + ru1;
    const double coefy = fy * coef * bv[j] / (1.0 * 1.0);
    const double ayv = -coefy * bp[j] * tvjm, cyv = -coefy * bp[j + 1] * tvjp, byv = -ayv - cyv;
    if (fc == 0.) {  // the convective terms are signed zeros: the same sums without their loads
      a = ayv;
      c = cyv;
      b = 1.0 + byv;
      r = 0.;
      return;
    }
    const double vm = vo[fidx(d, i, j - 1, k)], v0 = vo[fidx(d, i, j, k)], vp = vo[fidx(d, i, j + 1, k)];
    const double coefc = fc * coef * bv[j] / 1.0;
    const double ayc = -0.25 * coefc * (vm + v0) * 2.0, cyc = 0.25 * coefc * (vp + v0) * 2.0, byc = ayc + cyc;
    a = ayv + ayc;
    c = cyv + cyc;
    b = 1.0 + byv + byc;
    const double vyp = (vp + v0) * 0.5, vym = (v0 + vm) * 0.5;
    r = coefc * (vyp * vyp - vym * vym);
  }
};
struct RowW {  // w: edge viscosity averaged over four cells; convection about the provisional VS
  const double *__restrict__ tv, *__restrict__ bw, *__restrict__ bv, *__restrict__ vs;
  double coef, ru1, fy, fc;
  __device__ void operator()(const Dims &d, int i, int j, int k, double &a, double &b, double &c, double &r) const {
    const double tvjp = 0.25 * (tv[fidx(d, i, j, k + 1)] + tv[fidx(d, i, j, k)] + tv[fidx(d, i, j + 1, k + 1)] +
                                tv[fidx(d, i, j + 1, k)]) + ru1;
    const double tvjm = 0.25 * (tv[fidx(d, i, j, k + 1)] + tv[fidx(d, i, j, k)] + tv[fidx(d, i, j - 1, k + 1)] +
                                tv[fidx(d, i, j - 1, k)]) + ru1;
    const double coefy = fy * coef * bw[j] / (1.0 * 1.0);
    const double ayv = -coefy * bv[j - 1] * tvjm, cyv = -coefy * bv[j] * tvjp, byv = -ayv - cyv;
    if (fc == 0.) {
      a = ayv;
      c = cyv;
      b = 1.0 + byv;
      r = 0.;
      return;
    }
    const double vzp = (vs[fidx(d, i, j, k + 1)] + vs[fidx(d, i, j, k)]) * 0.5;
    const double vzm = (vs[fidx(d, i, j - 1, k + 1)] + vs[fidx(d, i, j - 1, k)]) * 0.5;
    const double coefc = fc * 0.5 * coef * bw[j] / 1.0;
    const double ayc = -coefc * vzm, cyc = coefc * vzp, byc = ayc + cyc;
    a = ayv + ayc;
    c = cyv + cyc;
    b = 1.0 + byv + byc;
    r = 0.;
  }
};
struct RowU {  // u (timeindeg.f:290-312); convection about the provisional VS
  const double *__restrict__ tv, *__restrict__ bu, *__restrict__ bv, *__restrict__ vs;
  double coef, ru1, fy, fc;
  __device__ void operator()(const Dims &d, int i, int j, int k, double &a, double &b, double &c, double &r) const {
    const double tvjp = 0.25 * (tv[fidx(d, i + 1, j, k)] + tv[fidx(d, i, j, k)] + tv[fidx(d, i + 1, j + 1, k)] +
                                tv[fidx(d, i, j + 1, k)]) + ru1;
    const double tvjm = 0.25 * (tv[fidx(d, i + 1, j, k)] + tv[fidx(d, i, j, k)] + tv[fidx(d, i + 1, j - 1, k)] +
                                tv[fidx(d, i, j - 1, k)]) + ru1;
    const double coefy = fy * coef * bu[j] / (1.0 * 1.0);
    const double ayv = -coefy * bv[j - 1] * tvjm, cyv = -coefy * bv[j] * tvjp, byv = -ayv - cyv;
    if (fc == 0.) {
      a = ayv;
      c = cyv;
      b = 1.0 + byv;
      r = 0.;
      return;
    }
    const double vxp = (vs[fidx(d, i + 1, j, k)] + vs[fidx(d, i, j, k)]) * 0.5;
    const double vxm = (vs[fidx(d, i + 1, j - 1, k)] + vs[fidx(d, i, j - 1, k)]) * 0.5;
    const double coefc = fc * 0.5 * coef * bu[j] / 1.0;
    const double ayc = -coefc * vxm, cyc = coefc * vxp, byc = ayc + cyc;
    a = ayv + ayc;
    c = cyv + cyc;
    b = 1.0 + byv + byc;
    r = 0.;
  }
};
struct RowD {  // density (density.f:425-440): both faces take 0.5 (tv(j) + tv(j+1)) + ru1/prn
  const double *__restrict__ tv, *__restrict__ bp;
  double coef, kmol;
  __device__ void operator()(const Dims &d, int i, int j, int k, double &a, double &b, double &c, double &r) const {
    const double tvjp = 0.5 * (tv[fidx(d, i, j, k)] + tv[fidx(d, i, j + 1, k)]) + kmol;
    const double tvjm = 0.5 * (tv[fidx(d, i, j, k)] + tv[fidx(d, i, j + 1, k)]) + kmol;
    const double coefy = 1.0 * coef * bp[j] / (1.0 * 1.0);
    a = -coefy * bp[j - 1] * tvjm;
    c = -coefy * bp[j] * tvjp;
    b = 1.0 + (-a - c);
    r = 0.;
  }
};
struct RowDN {  // density, INVERSEYD_NEW (density.f:322-352): faces 0.5 (tv(j) + tv(j+/-1)) + ru1/prn, convection by VO
  const double *__restrict__ tv, *__restrict__ bp, *__restrict__ bv, *__restrict__ vo;
  double coef, kmol, fy, fc;
  __device__ void operator()(const Dims &d, int i, int j, int k, double &a, double &b, double &c, double &r) const {
    const double tvjp = 0.5 * (tv[fidx(d, i, j, k)] + tv[fidx(d, i, j + 1, k)]) + kmol;
    const double tvjm = 0.5 * (tv[fidx(d, i, j, k)] + tv[fidx(d, i, j - 1, k)]) + kmol;
    const double coefy = fy * coef * bp[j] / (1.0 * 1.0);
    const double ayv = -coefy * bv[j - 1] * tvjm, cyv = -coefy * bv[j] * tvjp, byv = -ayv - cyv;
    const double vzp = vo[fidx(d, i, j, k)], vzm = vo[fidx(d, i, j - 1, k)];
    const double coefc = fc * 0.5 * coef * bp[j] / 1.0;
    const double ayc = -coefc * vzm, cyc = coefc * vzp, byc = ayc + cyc;
    a = ayv + ayc;
    c = cyv + cyc;
    b = 1.0 + byv + byc;
    r = 0.;
  }
};

// lines i in [i0, i0+ni), k in [k0, k0+nk); rows jy1..jy2 (n = jy2 - 1 >= 3);
// x: right-hand side in, solution out (in place); gam, z: scratch fields.
// Each sweep loads the next row's operands before the current row's
// dependent arithmetic (the loads do not depend on the recurrence), so every
// thread keeps two rows of loads in flight.
template <class Row>
__global__ void __launch_bounds__(128) k_cyclic_lines(Dims d, Row row, int i0, int ni, int k0, int nk,
                                                      double *__restrict__ x, double *__restrict__ gam,
                                                      double *__restrict__ z) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)ni * nk) return;
  const int i = i0 + (int)(t % ni), k = k0 + (int)(t / ni);
  const int n = d.jy2 - 1;
  const long long q0 = fidx(d, i, d.jy1, k), sj = d.nx;
  // forward elimination of A' x = r and A' z = (gamma, 0, .., 0, alpha), A'
  // the matrix with b1' = b1 - gamma, bn' = bn - alpha beta / gamma
  double beta = 0., gamma = 1., bet = 1., cprev = 0., xp = 0., zp = 0.;
  double a, b, c, dr;
  row(d, i, d.jy1, k, a, b, c, dr);
  double xr = x[q0];
  for (int r = 0; r < n; r++) {
    const long long q = q0 + sj * r;
    double an = 0., bn = 1., cn = 0., drn = 0., xrn = 0.;
    if (r + 1 < n) {
      row(d, i, d.jy1 + r + 1, k, an, bn, cn, drn);
      xrn = x[q + sj];
    }
    const double rr = xr + dr;
    if (r == 0) {
      beta = a;
      gamma = -b;
      bet = b - gamma;
      xp = rr / bet;
      zp = gamma / bet;
    } else {
      const double bb = r == n - 1 ? b - c * beta / gamma : b;
      const double g = cprev / bet;
      bet = bb - a * g;
      const double u = r == n - 1 ? c : 0.;
      xp = (rr - a * xp) / bet;
      zp = (u - a * zp) / bet;
      gam[q] = g;
    }
    x[q] = xp;
    z[q] = zp;
    cprev = c;
    a = an; b = bn; c = cn; dr = drn; xr = xrn;
  }
  // back substitution (the last row stands)
  const double xn = xp, zn = zp;
  if (n >= 2) {
    long long q = q0 + sj * (n - 2);
    double g = gam[q + sj], xq = x[q], zq = z[q];
    for (int r = n - 2; r >= 0; r--, q -= sj) {
      double gnx = 0., xnx = 0., znx = 0.;
      if (r > 0) {
        gnx = gam[q];
        xnx = x[q - sj];
        znx = z[q - sj];
      }
      xp = xq - g * xp;
      zp = zq - g * zp;
      x[q] = xp;
      z[q] = zp;
      g = gnx; xq = xnx; zq = znx;
    }
  }
  // Sherman-Morrison correction for the two corner entries
  const double fact = (xp + beta * xn / gamma) / (1. + zp + beta * zn / gamma);
  for (int r = 0; r < n; r++) {
    const long long q = q0 + sj * r;
    x[q] = x[q] - fact * z[q];
  }
}

template <class Row>
int lines(eddy_ctx *ctx, const Row &row, int i0, int i1, int k0, int k1, double *x) {
  const int ni = i1 - i0 + 1, nk = k1 - k0 + 1;
  if (ni <= 0 || nk <= 0) return EDDY_OK;
  const long long nl = (long long)ni * nk;
  k_cyclic_lines<Row><<<(unsigned)((nl + 127) / 128), 128, 0, ctx->stream>>>(ctx->d, row, i0, ni, k0, nk, x,
                                                                              ctx->f[EDDY_UB], ctx->f[EDDY_VB]);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

// ---- x lines (IMPLX or IMPLCX = 1) ----
// Every (j,k) line is one tridiagonal system over i1..i2 solved by tridag
// (src/numrec.f:783-802) in its operation order, one thread per line (the
// threads walk their lines in step; consecutive i of a line share a sector,
// so the strided rows stay cached).  The boundary tables of
// src/timeindeg.f:370-434 for one implicit region over the whole x range and
// slip walls (type 60) on both x boundaries: rdir = 0; u takes its wall
// value UB = 0 (BOUND060 zeroes the wall-normal velocity, rperb = 1); v, w
// and the density are Neumann (IBC = -1, src/setup.f:21-40: bdirb = 1,
// rdirb = 0, rperb = 0), so the first and last rows take b + a and b + c and
// every right-hand-side correction is a times an exact zero.
struct RowXU {  // u (timeindeg.f:441-486): viscosity 2 tv(i) and 2 tv(i+1); convection about UO
  const double *tv, *au, *ap, *uo;
  double coef, ru1, fx, fc;
  __device__ void operator()(const Dims &d, int i, int j, int k, double &a, double &b, double &c, double &r) const {
    const double tvip = 2. * tv[fidx(d, i + 1, j, k)] + ru1, tvim = 2. * tv[fidx(d, i, j, k)] + ru1;
    const double coefx = fx * coef * au[i];
    const double axv = -coefx * ap[i] * tvim, cxv = -coefx * ap[i + 1] * tvip, bxv = -axv - cxv;
    if (fc == 0.) {  // the convective terms are signed zeros: the same sums without their loads
      a = axv;
      c = cxv;
      b = 1.0 + bxv;
      r = 0.;
      return;
    }
    const double um = uo[fidx(d, i - 1, j, k)], u0 = uo[fidx(d, i, j, k)], up = uo[fidx(d, i + 1, j, k)];
    const double coefc = fc * coef * au[i] / 1.0;
    const double qxm = (u0 + um) * 0.5, qxp = (u0 + up) * 0.5;
    const double axc = -coefc * qxm, cxc = coefc * qxp, bxc = axc + cxc;
    a = axv + axc;
    c = cxv + cxc;
    b = 1.0 + bxv + bxc;
    const double uxp = (up + u0) * 0.5, uxm = (um + u0) * 0.5;
    r = coefc * (qxp * uxp - qxm * uxm);
  }
};
struct RowXV {  // v (timeindeg.f:528-560); convection about the provisional US
  const double *tv, *av, *au, *us;
  double coef, ru1, fx, fc;
  __device__ void operator()(const Dims &d, int i, int j, int k, double &a, double &b, double &c, double &r) const {
    const double tvip = 0.25 * (tv[fidx(d, i, j + 1, k)] + tv[fidx(d, i, j, k)] + tv[fidx(d, i + 1, j + 1, k)] +
                                tv[fidx(d, i + 1, j, k)]) + ru1;
    const double tvim = 0.25 * (tv[fidx(d, i, j + 1, k)] + tv[fidx(d, i, j, k)] + tv[fidx(d, i - 1, j + 1, k)] +
                                tv[fidx(d, i - 1, j, k)]) + ru1;
    const double coefx = fx * coef * av[i] / 1.0;
    const double axv = -coefx * au[i - 1] * tvim, cxv = -coefx * au[i] * tvip, bxv = -axv - cxv;
    if (fc == 0.) {  // the convective terms are signed zeros: the same sums without their loads
      a = axv;
      c = cxv;
      b = 1.0 + bxv;
      r = 0.;
      return;
    }
    const double coefc = fc * 0.5 * coef * av[i] / 1.0;
    const double qyp = 1.0 * (us[fidx(d, i, j + 1, k)] + us[fidx(d, i, j, k)]) * 0.5;
    const double qym = 1.0 * (us[fidx(d, i - 1, j + 1, k)] + us[fidx(d, i - 1, j, k)]) * 0.5;
    const double axc = -coefc * qym, cxc = coefc * qyp, bxc = axc + cxc;
    a = axv + axc;
    c = cxv + cxc;
    b = 1.0 + bxv + bxc;
    r = 0.;
  }
};
struct RowXW {  // w (timeindeg.f:594-626); convection about the provisional US
  const double *tv, *aw, *au, *us;
  double coef, ru1, fx, fc;
  __device__ void operator()(const Dims &d, int i, int j, int k, double &a, double &b, double &c, double &r) const {
    const double tvip = 0.25 * (tv[fidx(d, i, j, k + 1)] + tv[fidx(d, i, j, k)] + tv[fidx(d, i + 1, j, k + 1)] +
                                tv[fidx(d, i + 1, j, k)]) + ru1;
    const double tvim = 0.25 * (tv[fidx(d, i, j, k + 1)] + tv[fidx(d, i, j, k)] + tv[fidx(d, i - 1, j, k + 1)] +
                                tv[fidx(d, i - 1, j, k)]) + ru1;
    const double coefx = fx * coef * aw[i] / 1.0;
    const double axv = -coefx * au[i - 1] * tvim, cxv = -coefx * au[i] * tvip, bxv = -axv - cxv;
    if (fc == 0.) {  // the convective terms are signed zeros: the same sums without their loads
      a = axv;
      c = cxv;
      b = 1.0 + bxv;
      r = 0.;
      return;
    }
    const double coefc = fc * 0.5 * coef * aw[i] / 1.0;
    const double qzp = 1.0 * (us[fidx(d, i, j, k + 1)] + us[fidx(d, i, j, k)]) * 0.5;
    const double qzm = 1.0 * (us[fidx(d, i - 1, j, k + 1)] + us[fidx(d, i - 1, j, k)]) * 0.5;
    const double axc = -coefc * qzm, cxc = coefc * qzp, bxc = axc + cxc;
    a = axv + axc;
    c = cxv + cxc;
    b = 1.0 + bxv + bxc;
    r = 0.;
  }
};
struct RowXD {  // density (density.f:212-240): the molecular diffusivity ru1/prn on both faces
  const double *aw, *au;
  double coef, kmol, fx;
  __device__ void operator()(const Dims &d, int i, int j, int k, double &a, double &b, double &c, double &r) const {
    const double coefx = fx * coef * aw[i] / 1.0;
    a = -coefx * au[i - 1] * kmol;
    c = -coefx * au[i] * kmol;
    b = 1.0 + (-a - c);
    r = 0.;
  }
};

// lines j in [j0, j0+nj), k in [k0, k0+nk); rows i1..i2; NEU: Neumann walls
// (b + a on the first row, b + c on the last); x: right-hand side in,
// solution out (in place); gam: scratch field for the multipliers
template <class Row, bool NEU>
__global__ void __launch_bounds__(64) k_x_lines(Dims d, Row row, int i1, int i2, int j0, int nj, int k0, int nk,
                                                double *x, double *gam) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nj * nk) return;
  const int j = j0 + (int)(t % nj), k = k0 + (int)(t / nj);
  const long long q1 = fidx(d, i1, j, k);
  double bet = 1., up = 0., cprev = 0.;
  for (int i = i1; i <= i2; i++) {
    const long long q = q1 + (i - i1);
    double a, b, c, dr;
    row(d, i, j, k, a, b, c, dr);
    double r = x[q] + dr;
    if (i == i1) {
      if (NEU) b = b + 1.0 * a;
      r = r - a * 0.0;
    }
    if (i == i2) {
      if (NEU) b = b + 1.0 * c;
      r = r - c * 0.0;
    }
    if (i == i1) {
      bet = b;
      up = r / bet;
    } else {
      const double g = cprev / bet;
      gam[q] = g;
      bet = b - a * g;
      up = (r - a * up) / bet;
    }
    x[q] = up;
    cprev = c;
  }
  for (int i = i2 - 1; i >= i1; i--) {
    const long long q = q1 + (i - i1);
    up = x[q] - gam[q + 1] * up;
    x[q] = up;
  }
}

template <class Row, bool NEU>
int xlines(eddy_ctx *ctx, const Row &row, int i1, int i2, int j0, int j1, int k0, int k1, double *x, double *gam) {
  const int nj = j1 - j0 + 1, nk = k1 - k0 + 1;
  if (nj <= 0 || nk <= 0 || i2 < i1) return EDDY_OK;
  const long long nl = (long long)nj * nk;
  k_x_lines<Row, NEU><<<(unsigned)((nl + 63) / 64), 64, 0, ctx->stream>>>(ctx->d, row, i1, i2, j0, nj, k0, nk, x,
                                                                          gam);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

}  // namespace

// INVERSEX: u lines (i in [2, NX-2], j in [jy1, jy2], k in [kz1, kz2]), then v
// (i in [2, NX-1], j in [jbv, jev]) and w (i in [2, NX-1], k in [kbw, kew]);
// rflagx = IMPLX and rflagcx = IMPLCX: the u systems linearise the convection
// about UO, the v and w systems about the u lines' result in US (the launches
// run in that order on one stream); REFRESHBC is a no-op on one rank
int launch_inversex(eddy_ctx *ctx, double alfxdt) {
  const Dims &d = ctx->d;
  const DevMetrics &m = ctx->m;
  double **f = ctx->f;
  const double coef = 0.5 * alfxdt, ru1 = ctx->sc.ru1;
  int rc;
  const double fx = (double)ctx->sc.implx, fc = (double)ctx->sc.implcx;
  if ((rc = xlines<RowXU, false>(ctx, RowXU{f[EDDY_TV], m.au, m.ap, f[EDDY_UO], coef, ru1, fx, fc}, 2, d.nx - 2,
                                 d.jy1, d.jy2, d.kz1, d.kz2, f[EDDY_US], f[EDDY_UB])))
    return rc;
  if ((rc = xlines<RowXV, true>(ctx, RowXV{f[EDDY_TV], m.av, m.au, f[EDDY_US], coef, ru1, fx, fc}, 2, d.nx - 1,
                                d.jbv, d.jev, d.kz1, d.kz2, f[EDDY_VS], f[EDDY_VB])))
    return rc;
  return xlines<RowXW, true>(ctx, RowXW{f[EDDY_TV], m.aw, m.au, f[EDDY_US], coef, ru1, fx, fc}, 2, d.nx - 1, d.jy1,
                             d.jy2, d.kbw, d.kew, f[EDDY_WS], f[EDDY_WB]);
}

// INVERSEXD on RS: i in [2, NX-1], j in [jy1, jy2], k in [kbw, kew]
int launch_inversexd(eddy_ctx *ctx, double alfxdt) {
  const Dims &d = ctx->d;
  return xlines<RowXD, true>(ctx, RowXD{ctx->m.aw, ctx->m.au, 0.5 * alfxdt, ctx->sc.ru1 / ctx->sc.prn,
                                        (double)ctx->sc.implx},
                             2, d.nx - 1, d.jy1, d.jy2, d.kbw, d.kew, ctx->f[EDDY_RS], ctx->f[EDDY_UB]);
}

// INVERSEY: v lines (i in [2, NX-1], k in [kz1, kz2]), then w (i in [2, NX-1],
// k in [kbw, kew]), then u (i in [2, NX-2], k in [kz1, kz2]); REFRESHBC is a
// no-op on one rank with non-periodic z
int launch_inversey(eddy_ctx *ctx, double alfxdt) {
  const Dims &d = ctx->d;
  const DevMetrics &m = ctx->m;
  double **f = ctx->f;
  const double coef = 0.5 * alfxdt, ru1 = ctx->sc.ru1;
  int rc;
  const double fy = (double)ctx->sc.imply, fc = (double)ctx->sc.implcy;
  if ((rc = lines(ctx, RowV{f[EDDY_TV], m.bv, m.bp, f[EDDY_VO], coef, ru1, fy, fc}, 2, d.nx - 1, d.kz1, d.kz2,
                  f[EDDY_VS])))
    return rc;
  if ((rc = lines(ctx, RowW{f[EDDY_TV], m.bw, m.bv, f[EDDY_VS], coef, ru1, fy, fc}, 2, d.nx - 1, d.kbw, d.kew,
                  f[EDDY_WS])))
    return rc;
  return lines(ctx, RowU{f[EDDY_TV], m.bu, m.bv, f[EDDY_VS], coef, ru1, fy, fc}, 2, d.nx - 2, d.kz1, d.kz2,
               f[EDDY_US]);
}

// INVERSEYD_NEW on RS (IMPLY = IMPLCY = 1): i in [2, NX-1], k in [kbw, kew]
int launch_inverseyd_new(eddy_ctx *ctx, double alfxdt) {
  const Dims &d = ctx->d;
  const DevMetrics &m = ctx->m;
  return lines(ctx, RowDN{ctx->f[EDDY_TV], m.bp, m.bv, ctx->f[EDDY_VO], 0.5 * alfxdt, ctx->sc.ru1 / ctx->sc.prn,
                          (double)ctx->sc.imply, (double)ctx->sc.implcy},
               2, d.nx - 1, d.kbw, d.kew, ctx->f[EDDY_RS]);
}

// INVERSEYD on RS: i in [2, NX-1], k in [kbw, kew] (the reference's w range)
int launch_inverseyd(eddy_ctx *ctx, double alfxdt) {
  const Dims &d = ctx->d;
  return lines(ctx, RowD{ctx->f[EDDY_TV], ctx->m.bp, 0.5 * alfxdt, ctx->sc.ru1 / ctx->sc.prn}, 2, d.nx - 1, d.kbw, d.kew,
               ctx->f[EDDY_RS]);
}
