/*
 * eo_force.c -- oracle restatement of calcfrc (src/calcforce.f:3-779), the
 * force on the immersed body by the control-volume approach, Cartesian
 * branch (icyl = 0), one rank.  TEST INFRASTRUCTURE ONLY.
 *
 * The control volume is [xu(ICB), xu(ICE)] x y x [zw(KCB), zw(KCE)] with
 * ICB, ICE the faces closest to CVLIM(1:2) (closest, src/numrec.f:433) and
 * KCB, KCE located by bisection (locate, src/numrec.f:390; eo_locate of
 * eo_ib.c) and adjusted as the reference does when the volume reaches past
 * the domain.  Sums in the reference's loop order.
 */
#include <math.h>
#include <string.h>
#include "eddy_oracle.h"

#define NX (g->nx)
#define NY (g->ny)
#define NZ (g->nz)
#define IX(i, j, k) ((size_t)((i) - 1) + (size_t)NX * ((size_t)((j) - 1) + (size_t)NY * (size_t)((k) - 1)))
#define A(a, i, j, k) (a)[IX(i, j, k)]
#define FL(f, i, j, k) ((f) ? (int)(f)[IX(i, j, k)] : 0)

/* closest (src/numrec.f:433-475) on xx(1..n) */
int eo_closest(const double *xx, int n, double x) {
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
    if (fabs(x - xx[j]) > fabs(x - xx[j + 1])) j = jl + 1;
  } else if (j < 1) {
    j = 1;
  } else if (j > n) {
    j = n;
  }
  return j;
}

/* the control volume's index range and face flags (src/calcforce.f:44-94):
 * cv[0..5] = ICB, ICE, KCB, KCE, KBFLAG, KEFLAG */
void eo_cv_range(const eo_grid *g, const double cvlim[4], int cv[6]) {
  const int icb = eo_closest(g->xu, NX, cvlim[0]), ice = eo_closest(g->xu, NX, cvlim[1]);
  int kcb = eo_locate(g->zw, NZ - 1, cvlim[2]), kce = eo_locate(g->zw, NZ - 1, cvlim[3]);
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
  cv[0] = icb; cv[1] = ice; cv[2] = kcb; cv[3] = kce; cv[4] = kbflag; cv[5] = keflag;
}

/* calcfrc on UO, VO, WO, P with the body's taguo flags (none: all fluid).
 * fb: the control volume's momentum of the previous call, updated.
 * out[56]: FX(1..6), FY(1..6), FZ(1..6), the unsteady terms FBX, FBY, FBZ,
 * the totals -(SUM(F) + FB) per component, Finlet(1..8), Foutlet(1..8),
 * Ftop(1..8), Fbot(1..8) (src/calcforce.f:600-771). */
void eo_calcfrc(eo_state *s, const double cvlim[4], double dt, int icycle, double fb[3], double out[56]) {
  const eo_grid *g = s->g;
  const double *u = s->uo, *v = s->vo, *w = s->wo, *p = s->p;
  const double ru1 = s->prm.ru1;
  const double *ap = g->ap, *au = g->au, *av = g->av, *aw = g->aw;
  const double *bp = g->bp, *bu = g->bu, *bw = g->bw, *cp = g->cp, *cu = g->cu, *cw = g->cw;
  const signed char *fu = s->ib ? eo_ib_flags(s->ib, 0) : NULL;
  const signed char *fv = s->ib ? eo_ib_flags(s->ib, 1) : NULL;
  const signed char *fw = s->ib ? eo_ib_flags(s->ib, 2) : NULL;
  int cv[6];
  eo_cv_range(g, cvlim, cv);
  const int icb = cv[0], ice = cv[1], kcb = cv[2], kce = cv[3], kbflag = cv[4], keflag = cv[5];
  const int jy1 = g->jy1, jy2 = g->jy2;

  /* momentum in the control volume (:96-125) */
  double fbxc = 0., fbyc = 0., fbzc = 0.;
  for (int k = kcb + 1; k <= kce; k++)
    for (int i = icb + 1; i <= ice; i++)
      for (int j = jy1; j <= jy2; j++) {
        const double dv = 1.0 / (bp[j] * ap[i] * cp[k]);
        if (FL(fu, i, j, k) <= 0 || FL(fu, i - 1, j, k) <= 0) fbxc = fbxc + 0.5 * (A(u, i, j, k) + A(u, i - 1, j, k)) * dv;
        if (FL(fv, i, j, k) <= 0 || FL(fv, i, j - 1, k) <= 0) fbyc = fbyc + 0.5 * (A(v, i, j, k) + A(v, i, j - 1, k)) * dv;
        if (FL(fw, i, j, k) <= 0 || FL(fw, i, j, k - 1) <= 0) fbzc = fbzc + 0.5 * (A(w, i, j, k) + A(w, i, j, k - 1)) * dv;
      }
  double fbx, fby, fbz;
  if (icycle == 0) {
    fbx = 0.; fby = 0.; fbz = 0.;
  } else {
    fbx = (fbxc - fb[0]) / dt;
    fby = (fbyc - fb[1]) / dt;
    fbz = (fbzc - fb[2]) / dt;
  }
  fb[0] = fbxc; fb[1] = fbyc; fb[2] = fbzc;

  double fx[6] = {0}, fy[6] = {0}, fz[6] = {0}, fin[8] = {0}, fout[8] = {0}, ftop[8] = {0}, fbot[8] = {0};
  /* x-y planes: inlet (k = KCB) and outlet (k = KCE), :362-426 */
  for (int i = icb + 1; i <= ice; i++)
    for (int j = jy1; j <= jy2; j++) {
      const double da = 1.0 / bp[j] / ap[i];
      for (int side = 0; side < 2; side++) {
        if (side == 0 ? !kbflag : !keflag) continue;
        const int k = side == 0 ? kcb : kce;
        const double sa = side == 0 ? -da : da;
        const double dwdx = (A(w, i + 1, j, k) - A(w, i - 1, j, k)) * aw[i] / 2.;
        const double dudz1 = (A(u, i, j, k + 1) - A(u, i, j, k)) * cw[k];
        const double dudz2 = (A(u, i - 1, j, k + 1) - A(u, i - 1, j, k)) * cw[k];
        const double dudz = 0.5 * (dudz1 + dudz2);
        const double sxz = dudz + dwdx;
        const double txz = ru1 * sxz;
        const double u1 = 0.25 * (A(u, i, j, k) + A(u, i, j, k + 1) + A(u, i - 1, j, k) + A(u, i - 1, j, k + 1));
        const double uw = u1 * A(w, i, j, k);
        double *ff = side == 0 ? fin : fout;
        fx[side] = fx[side] + (uw - txz) * sa;
        ff[0] = ff[0] + uw * sa;
        ff[1] = ff[1] - txz * sa;
        const double dwdz = (A(w, i, j, k + 1) - A(w, i, j, k - 1)) * cw[k] / 2.;
        const double szz = 2. * ru1 * dwdz;
        const double pres = 0.5 * (A(p, i, j, k + 1) + A(p, i, j, k));
        const double tzz = pres - szz;
        const double wsq = A(w, i, j, k) * A(w, i, j, k);
        fz[side] = fz[side] + (wsq + tzz) * sa;
        ff[2] = ff[2] + pres * sa;
        ff[3] = ff[3] - szz * sa;
        ff[4] = ff[4] + wsq * sa;
      }
    }
  /* y-z planes: top (i = ICE, :428-461) and bottom (i = ICB, :463-496) */
  for (int side = 0; side < 2; side++) {
    const int i = side == 0 ? ice : icb;
    double *ff = side == 0 ? ftop : fbot;
    for (int k = kcb + 1; k <= kce; k++)
      for (int j = jy1; j <= jy2; j++) {
        const double da = 1.0 / bp[j] / cp[k];
        const double sa = side == 0 ? da : -da;
        const double dudx = (A(u, i + 1, j, k) - A(u, i - 1, j, k)) * au[i] / 2;
        const double sxx = 2. * ru1 * dudx;
        const double pres = 0.5 * (A(p, i + 1, j, k) + A(p, i, j, k));
        const double txx = pres - sxx;
        const double usq = A(u, i, j, k) * A(u, i, j, k);
        fx[2 + side] = fx[2 + side] + (usq + txx) * sa;
        ff[0] = ff[0] + usq * sa;
        ff[1] = ff[1] + pres * sa;
        ff[2] = ff[2] - sxx * sa;
        const double dudz = (A(u, i, j, k + 1) - A(u, i, j, k - 1)) * cu[k] / 2.;
        const double dwdx1 = (A(w, i + 1, j, k) - A(w, i, j, k)) * au[i];
        const double dwdx2 = (A(w, i + 1, j, k - 1) - A(w, i, j, k - 1)) * au[i];
        const double dwdx = 0.5 * (dwdx1 + dwdx2);
        const double w1 = 0.25 * (A(w, i, j, k) + A(w, i, j, k - 1) + A(w, i + 1, j, k) + A(w, i + 1, j, k - 1));
        const double uw = A(u, i, j, k) * w1;
        const double sxz = ru1 * (dudz + dwdx);
        fz[2 + side] = fz[2 + side] + (uw - sxz) * sa;
        ff[3] = ff[3] + uw * sa;
        ff[4] = ff[4] - sxz * sa;
      }
  }
  /* x-z planes j = 1 and j = JY2 (:498-558).  As written, the j = JY2 branch
   * assigns DWDY1 twice and reads DWDY2 as the j = 1 branch (or an earlier
   * iteration) left it; it starts at zero here (undefined in the reference) */
  double dwdy2 = 0.;
  for (int k = kcb + 1; k <= kce; k++)
    for (int i = icb + 1; i <= ice; i++) {
      const double da = 1. / cp[k] / ap[i];
      int j = 1;
      if (FL(fu, i, j, k) <= 0 || FL(fv, i, j, k) <= 0) {
        const double dudy1 = (A(u, i, j + 1, k) - A(u, i, j, k)) * bu[j];
        const double dudy2 = (A(u, i - 1, j + 1, k) - A(u, i - 1, j, k)) * bu[j];
        const double dudy = 0.5 * (dudy1 + dudy2);
        const double dvdx = (A(v, i + 1, j, k) - A(v, i - 1, j, k)) * av[i] / 2.;
        const double sxy = ru1 * (dudy + dvdx);
        const double u1 = 0.25 * (A(u, i, j, k) + A(u, i - 1, j, k) + A(u, i, j + 1, k) + A(u, i - 1, j + 1, k));
        const double uv = A(v, i, j, k) * u1;
        fx[4] = fx[4] + (uv - sxy) * (-da);
      }
      if (FL(fv, i, j, k) <= 0 || FL(fw, i, j, k) <= 0) {
        const double dvdz = (A(v, i, j, k + 1) - A(v, i, j, k - 1)) * cu[k] / 2.;
        const double dwdy1 = (A(w, i, j + 1, k) - A(w, i, j, k)) * bw[j];
        dwdy2 = (A(w, i, j + 1, k - 1) - A(w, i, j, k - 1)) * bw[j];
        const double dwdy = 0.5 * (dwdy1 + dwdy2);
        const double syz = ru1 * (dvdz + dwdy);
        const double w1 = 0.25 * (A(w, i, j, k) + A(w, i, j, k - 1) + A(w, i, j + 1, k) + A(w, i, j + 1, k - 1));
        const double vw = A(v, i, j, k) * w1;
        fz[4] = fz[4] + (vw - syz) * (-da);
      }
      j = jy2;
      if (FL(fu, i, j, k) <= 0 || FL(fv, i, j, k) <= 0) {
        const double dudy1 = (A(u, i, j + 1, k) - A(u, i, j, k)) * bu[j];
        const double dudy2 = (A(u, i - 1, j + 1, k) - A(u, i - 1, j, k)) * bu[j];
        const double dudy = 0.5 * (dudy1 + dudy2);
        const double dvdx = (A(v, i + 1, j, k) - A(v, i - 1, j, k)) * av[i] / 2.;
        const double sxy = ru1 * (dudy + dvdx);
        const double u1 = 0.25 * (A(u, i, j, k) + A(u, i - 1, j, k) + A(u, i, j + 1, k) + A(u, i - 1, j + 1, k));
        const double uv = A(v, i, j, k) * u1;
        fx[5] = fx[5] + (uv - sxy) * da;
      }
      if (FL(fv, i, j, k) <= 0 || FL(fw, i, j, k) <= 0) {
        const double dwdy1 = (A(w, i, j + 1, k - 1) - A(w, i, j, k - 1)) * bw[j];
        const double dwdy = 0.5 * (dwdy1 + dwdy2);
        const double dvdz = (A(v, i, j, k + 1) - A(v, i, j, k - 1)) * cu[k] / 2.;
        const double syz = ru1 * (dvdz + dwdy);
        const double w1 = 0.25 * (A(w, i, j, k) + A(w, i, j, k - 1) + A(w, i, j + 1, k) + A(w, i, j + 1, k - 1));
        const double vw = A(v, i, j, k) * w1;
        fz[5] = fz[5] + (vw - syz) * da;
      }
    }
  /* :562-569 */
  double *ffs[4] = {fin, fout, ftop, fbot};
  for (int q = 0; q < 4; q++) {
    double *ff = ffs[q];
    const int n1 = q < 2 ? 2 : 3;  /* inlet/outlet: x terms 1..2, z terms 3..5; top/bottom: 1..3, 4..5 */
    double a = 0., b = 0.;
    for (int e = 0; e < n1; e++) a = a + ff[e];
    for (int e = n1; e < 5; e++) b = b + ff[e];
    ff[5] = a;
    ff[6] = b;
  }
  memcpy(out, fx, sizeof fx);
  memcpy(out + 6, fy, sizeof fy);
  memcpy(out + 12, fz, sizeof fz);
  out[18] = fbx; out[19] = fby; out[20] = fbz;
  double sx = 0., sy = 0., sz = 0.;
  for (int e = 0; e < 6; e++) { sx = sx + fx[e]; sy = sy + fy[e]; sz = sz + fz[e]; }
  out[21] = -(sx + fbx); out[22] = -(sy + fby); out[23] = -(sz + fbz);
  memcpy(out + 24, fin, sizeof fin);
  memcpy(out + 32, fout, sizeof fout);
  memcpy(out + 40, ftop, sizeof ftop);
  memcpy(out + 48, fbot, sizeof fbot);
}
