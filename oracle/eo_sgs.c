/*
 * eo_sgs.c -- oracle restatement of the dynamic eddy-viscosity procedure
 * TURVIS (src/vt.f:16-442) with STRAIN (:955-1018), FILTERSIZE (:1096-1127),
 * filter3d (:1132-1268) and BOUNDTURB (:700-950).  TEST INFRASTRUCTURE ONLY.
 *
 * Whole-array Fortran statements are restated over the whole array, so the
 * ghost layers hold exactly what the reference leaves there.  Scratch roles
 * follow the driver's call (src/Eddy6.f:3017): MXX..MXZ = US,VS,WS,UB,VB,WB,
 * GB = DP, LM/TV double as filter work arrays.  Cartesian (icyl=0), y periodic
 * (LP=0), z not periodic (NP=1): the y-average branch (:296-318).
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
#define WH(a, i, d) a[(i)*3 + (d) + 1]

void eo_filtersize(eo_state *s) {
  const eo_grid *g = s->g;
  const double ppp = 2. / 3.;
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= NX; i++)
        A(s->dxdydz, i, j, k) = pow(fabs(1.0) / (g->ap[i] * g->bp[j] * g->cp[k]), ppp);
  if (g->lp == 0)
    for (int k = 1; k <= NZ; k++)
      for (int i = 1; i <= NX; i++) {
        A(s->dxdydz, i, 1, k) = A(s->dxdydz, i, NY - 1, k);
        A(s->dxdydz, i, NY, k) = A(s->dxdydz, i, 2, k);
      }
}

void eo_strain(eo_state *s, const double *uc, const double *vc, const double *wc) {
  const eo_grid *g = s->g;
  const double *au = g->au, *bv = g->bv, *cw = g->cw;
#pragma omp parallel for schedule(static)
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ix1; i <= g->ix2; i++) {
        double dudxp = au[i] * (A(uc, i + 1, j, k) - A(uc, i, j, k));
        double dudxm = au[i - 1] * (A(uc, i, j, k) - A(uc, i - 1, j, k));
        double dudyp = bv[j] * (A(uc, i, j + 1, k) - A(uc, i, j, k));
        double dudym = bv[j - 1] * (A(uc, i, j, k) - A(uc, i, j - 1, k));
        double dudzp = cw[k] * (A(uc, i, j, k + 1) - A(uc, i, j, k));
        double dudzm = cw[k - 1] * (A(uc, i, j, k) - A(uc, i, j, k - 1));
        double dvdxp = au[i] * (A(vc, i + 1, j, k) - A(vc, i, j, k));
        double dvdxm = au[i - 1] * (A(vc, i, j, k) - A(vc, i - 1, j, k));
        double dvdyp = bv[j] * (A(vc, i, j + 1, k) - A(vc, i, j, k));
        double dvdym = bv[j - 1] * (A(vc, i, j, k) - A(vc, i, j - 1, k));
        double dvdzp = cw[k] * (A(vc, i, j, k + 1) - A(vc, i, j, k));
        double dvdzm = cw[k - 1] * (A(vc, i, j, k) - A(vc, i, j, k - 1));
        double dwdxp = au[i] * (A(wc, i + 1, j, k) - A(wc, i, j, k));
        double dwdxm = au[i - 1] * (A(wc, i, j, k) - A(wc, i - 1, j, k));
        double dwdyp = bv[j] * (A(wc, i, j + 1, k) - A(wc, i, j, k));
        double dwdym = bv[j - 1] * (A(wc, i, j, k) - A(wc, i, j - 1, k));
        double dwdzp = cw[k] * (A(wc, i, j, k + 1) - A(wc, i, j, k));
        double dwdzm = cw[k - 1] * (A(wc, i, j, k) - A(wc, i, j, k - 1));
        double sxx = 0.5 * (dudxp + dudxm);
        double syy = 0.5 * (dvdyp + dvdym);
        double szz = 0.5 * (dwdzp + dwdzm);
        double sxy = 0.25 * (dudyp + dudym + dvdxp + dvdxm);
        double sxz = 0.25 * (dudzp + dudzm + dwdxp + dwdxm);
        double syz = 0.25 * (dwdyp + dwdym + dvdzp + dvdzm);
        A(s->sxx, i, j, k) = sxx; A(s->syy, i, j, k) = syy; A(s->szz, i, j, k) = szz;
        A(s->sxy, i, j, k) = sxy; A(s->sxz, i, j, k) = sxz; A(s->syz, i, j, k) = syz;
        A(s->g_s, i, j, k) = sqrt(2. * (sxx * sxx + syy * syy + szz * szz) +
                                  4. * (sxy * sxy + syz * syz + sxz * sxz));
      }
}

/* filter3d (vt.f:1132-1268), LP = 0, NP = 1 branch; f may alias fb. */
void eo_filter3d(eo_state *s, const double *f, double *fb, double *wk1, double *wk2) {
  const eo_grid *g = s->g;
  const double *whx = g->whx, *whz = g->whz;
  int ix1 = g->ix1, ix2 = g->ix2, kz1 = g->kz1, kz2 = g->kz2;
  size_t n = (size_t)s->ncell;
  memset(wk1, 0, n * sizeof(double));
  memset(wk2, 0, n * sizeof(double));
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++) {
      for (int i = ix1 + 1; i <= ix2 - 1; i++)
        A(wk1, i, j, k) = WH(whx, i, -1) * A(f, i - 1, j, k) + WH(whx, i, 0) * A(f, i, j, k) +
                          WH(whx, i, 1) * A(f, i + 1, j, k);
      A(wk1, ix1, j, k) = WH(whx, ix1, -1) * A(f, ix1, j, k) + WH(whx, ix1, 0) * A(f, ix1 + 1, j, k) +
                          WH(whx, ix1, 1) * A(f, ix1 + 2, j, k);
      A(wk1, ix2, j, k) = WH(whx, ix2, -1) * A(f, ix2, j, k) + WH(whx, ix2, 0) * A(f, ix2 - 1, j, k) +
                          WH(whx, ix2, 1) * A(f, ix2 - 2, j, k);
    }
  /* y: LP = 0 */
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= NZ; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = 1; i <= NX; i++)
        A(wk2, i, j, k) = 0.25 * A(wk1, i, j - 1, k) + 0.50 * A(wk1, i, j, k) + 0.25 * A(wk1, i, j + 1, k);
  /* z: NP = 1 */
#pragma omp parallel for schedule(static)
  for (int k = kz1 + 1; k <= kz2 - 1; k++)
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= NX; i++)
        A(fb, i, j, k) = WH(whz, k, -1) * A(wk2, i, j, k - 1) + WH(whz, k, 0) * A(wk2, i, j, k) +
                         WH(whz, k, 1) * A(wk2, i, j, k + 1);
  for (int j = 1; j <= NY; j++)
    for (int i = 1; i <= NX; i++) {
      if (s->prm.itype[5] > 0)
        A(fb, i, j, kz1) = WH(whz, kz1, -1) * A(wk2, i, j, kz1) + WH(whz, kz1, 0) * A(wk2, i, j, kz1 + 1) +
                           WH(whz, kz1, 1) * A(wk2, i, j, kz1 + 2);
      else
        A(fb, i, j, kz1) = WH(whz, kz1, -1) * A(wk2, i, j, kz1 - 1) + WH(whz, kz1, 0) * A(wk2, i, j, kz1) +
                           WH(whz, kz1, 1) * A(wk2, i, j, kz1 + 1);
      if (s->prm.itype[6] > 0)
        A(fb, i, j, kz2) = WH(whz, kz2, -1) * A(wk2, i, j, kz2) + WH(whz, kz2, 0) * A(wk2, i, j, kz2 - 1) +
                           WH(whz, kz2, 1) * A(wk2, i, j, kz2 - 2);
      else
        A(fb, i, j, kz2) = WH(whz, kz2, -1) * A(wk2, i, j, kz2 - 1) + WH(whz, kz2, 0) * A(wk2, i, j, kz2) +
                           WH(whz, kz2, 1) * A(wk2, i, j, kz2 + 1);
    }
}

/* BOUNDTURB (vt.f:700-757): iflg 0 for ILM/TV, 1 for IMM */
static void boundturb(eo_state *s, double *vt, int iflg) {
  const eo_grid *g = s->g;
  const int *it = s->prm.itype;
  int IM = NX, JM = NY, KM = NZ;
  for (int ib = 1; ib <= 6; ib++) {
    int t = it[ib];
    int mode = 0; /* 1 wall (negate), 2 grad (copy) */
    if (iflg == 0) {
      if (t > 700) mode = 2;
      else if (t != 0 && t != 500 && t != 300) mode = 1;
    } else {
      if (t != 0 && t != 500 && t != 300) mode = 2;
    }
    if (!mode) continue;
    double sg = (mode == 1) ? -1. : 1.;
    switch (ib) {
      case 1: for (int k = 1; k <= KM; k++) for (int j = 1; j <= JM; j++) A(vt, 1, j, k) = sg * A(vt, 2, j, k); break;
      case 2: for (int k = 1; k <= KM; k++) for (int j = 1; j <= JM; j++) A(vt, IM, j, k) = sg * A(vt, g->ix2, j, k); break;
      case 3: for (int k = 1; k <= KM; k++) for (int i = 1; i <= IM; i++) A(vt, i, 1, k) = sg * A(vt, i, 2, k); break;
      case 4: for (int k = 1; k <= KM; k++) for (int i = 1; i <= IM; i++) A(vt, i, JM, k) = sg * A(vt, i, g->jy2, k); break;
      case 5: for (int j = 1; j <= JM; j++) for (int i = 1; i <= IM; i++) A(vt, i, j, 1) = sg * A(vt, i, j, 2); break;
      case 6: for (int j = 1; j <= JM; j++) for (int i = 1; i <= IM; i++) A(vt, i, j, KM) = sg * A(vt, i, j, g->kz2); break;
    }
  }
  for (int ib = 1; ib <= 4; ib++) {
    if (it[ib] != 500) continue;
    switch (ib) {
      case 1: for (int k = 1; k <= KM; k++) for (int j = 1; j <= JM; j++) A(vt, 1, j, k) = A(vt, g->ix2, j, k); break;
      case 2: for (int k = 1; k <= KM; k++) for (int j = 1; j <= JM; j++) A(vt, IM, j, k) = A(vt, 2, j, k); break;
      case 3: for (int k = 1; k <= KM; k++) for (int i = 1; i <= IM; i++) A(vt, i, 1, k) = A(vt, i, g->jy2, k); break;
      case 4: for (int k = 1; k <= KM; k++) for (int i = 1; i <= IM; i++) A(vt, i, JM, k) = A(vt, i, 2, k); break;
    }
  }
}

static void per_y(const eo_grid *g, double *a) {
  for (int k = 1; k <= NZ; k++)
    for (int i = 1; i <= NX; i++) {
      A(a, i, 1, k) = A(a, i, g->jy2, k);
      A(a, i, NY, k) = A(a, i, 2, k);
    }
}

void eo_turvis(eo_state *s) {
  const eo_grid *g = s->g;
  size_t n = (size_t)s->ncell;
  int IM = NX, JM = NY, KM = NZ, ix1 = g->ix1, ix2 = g->ix2, jy1 = g->jy1, jy2 = g->jy2, kz1 = g->kz1, kz2 = g->kz2;
  double *uo = s->uo, *vo = s->vo, *wo = s->wo, *uc = s->uc, *vc = s->vc, *wc = s->wc;
  /* centred velocities (vt.f:64-74) */
  for (int k = 1; k <= KM; k++)
    for (int j = 1; j <= JM; j++) {
      for (int i = ix1; i <= ix2; i++) A(uc, i, j, k) = 0.5 * (A(uo, i - 1, j, k) + A(uo, i, j, k));
      A(uc, 1, j, k) = 2. * A(uo, 1, j, k) - A(uc, ix1, j, k);
      A(uc, IM, j, k) = 2. * A(uo, ix2, j, k) - A(uc, ix2, j, k);
    }
  for (int k = 1; k <= KM; k++)
    for (int i = 1; i <= IM; i++) {
      for (int j = jy1; j <= jy2; j++) A(vc, i, j, k) = 0.5 * (A(vo, i, j - 1, k) + A(vo, i, j, k));
      A(vc, i, 1, k) = 2. * A(vo, i, 1, k) - A(vc, i, jy1, k);
      A(vc, i, JM, k) = 2. * A(vo, i, jy2, k) - A(vc, i, jy2, k);
    }
  for (int j = 1; j <= JM; j++)
    for (int i = 1; i <= IM; i++) {
      for (int k = kz1; k <= kz2; k++) A(wc, i, j, k) = 0.5 * (A(wo, i, j, k - 1) + A(wo, i, j, k));
      A(wc, i, j, 1) = 2. * A(wo, i, j, 1) - A(wc, i, j, kz1);
      A(wc, i, j, KM) = 2. * A(wo, i, j, kz2) - A(wc, i, j, kz2);
    }
  eo_strain(s, uc, vc, wc);
  double *G = s->g_s, *dx = s->dxdydz;
  if (s->prm.isgs == 1) {
    double css = s->prm.css;
    for (size_t q = 0; q < n; q++) s->tv[q] = css * css * 1.0 * dx[q] * G[q];
  } else {
    double *sxx = s->sxx, *syy = s->syy, *szz = s->szz, *sxy = s->sxy, *syz = s->syz, *sxz = s->sxz;
    double *mxx = s->us, *myy = s->vs, *mzz = s->ws, *mxy = s->ub, *myz = s->vb, *mxz = s->wb;
    double *gb = s->dp, *lm = s->lm, *mm = s->mm, *tv = s->tv;
    if (g->lp == 0) {
      per_y(g, sxx); per_y(g, syy); per_y(g, szz); per_y(g, sxy); per_y(g, sxz); per_y(g, syz); per_y(g, G);
    }
    for (size_t q = 0; q < n; q++) {
      mxx[q] = G[q] * sxx[q]; myy[q] = G[q] * syy[q]; mzz[q] = G[q] * szz[q];
      mxy[q] = G[q] * sxy[q]; myz[q] = G[q] * syz[q]; mxz[q] = G[q] * sxz[q];
    }
    eo_filter3d(s, mxx, mxx, lm, tv); eo_filter3d(s, myy, myy, lm, tv); eo_filter3d(s, mzz, mzz, lm, tv);
    eo_filter3d(s, mxy, mxy, lm, tv); eo_filter3d(s, myz, myz, lm, tv); eo_filter3d(s, mxz, mxz, lm, tv);
    eo_filter3d(s, sxx, sxx, lm, tv); eo_filter3d(s, syy, syy, lm, tv); eo_filter3d(s, szz, szz, lm, tv);
    eo_filter3d(s, sxy, sxy, lm, tv); eo_filter3d(s, syz, syz, lm, tv); eo_filter3d(s, sxz, sxz, lm, tv);
    eo_filter3d(s, G, gb, lm, tv);
    const double C = 1.0, R = 6.;
    for (size_t q = 0; q < n; q++) {
      mxx[q] = C * dx[q] * (R * gb[q] * sxx[q] - mxx[q]);
      myy[q] = C * dx[q] * (R * gb[q] * syy[q] - myy[q]);
      mzz[q] = C * dx[q] * (R * gb[q] * szz[q] - mzz[q]);
      mxy[q] = C * dx[q] * (R * gb[q] * sxy[q] - mxy[q]);
      myz[q] = C * dx[q] * (R * gb[q] * syz[q] - myz[q]);
      mxz[q] = C * dx[q] * (R * gb[q] * sxz[q] - mxz[q]);
    }
    for (size_t q = 0; q < n; q++)
      mm[q] = mxx[q] * mxx[q] + myy[q] * myy[q] + mzz[q] * mzz[q] +
              2. * (mxy[q] * mxy[q] + myz[q] * myz[q] + mxz[q] * mxz[q]);
    eo_filter3d(s, uc, sxx, lm, tv); eo_filter3d(s, vc, syy, lm, tv); eo_filter3d(s, wc, szz, lm, tv);
    for (size_t q = 0; q < n; q++) gb[q] = uc[q] * uc[q];
    eo_filter3d(s, gb, gb, lm, tv);
    for (size_t q = 0; q < n; q++) mxx[q] = (gb[q] - sxx[q] * sxx[q]) * mxx[q];
    for (size_t q = 0; q < n; q++) gb[q] = vc[q] * vc[q];
    eo_filter3d(s, gb, gb, lm, tv);
    for (size_t q = 0; q < n; q++) myy[q] = (gb[q] - syy[q] * syy[q]) * myy[q];
    for (size_t q = 0; q < n; q++) gb[q] = wc[q] * wc[q];
    eo_filter3d(s, gb, gb, lm, tv);
    for (size_t q = 0; q < n; q++) mzz[q] = (gb[q] - szz[q] * szz[q]) * mzz[q];
    for (size_t q = 0; q < n; q++) gb[q] = uc[q] * vc[q];
    eo_filter3d(s, gb, gb, lm, tv);
    for (size_t q = 0; q < n; q++) mxy[q] = (gb[q] - sxx[q] * syy[q]) * mxy[q];
    for (size_t q = 0; q < n; q++) gb[q] = vc[q] * wc[q];
    eo_filter3d(s, gb, gb, lm, tv);
    for (size_t q = 0; q < n; q++) myz[q] = (gb[q] - syy[q] * szz[q]) * myz[q];
    for (size_t q = 0; q < n; q++) gb[q] = uc[q] * wc[q];
    eo_filter3d(s, gb, gb, lm, tv);
    for (size_t q = 0; q < n; q++) mxz[q] = (gb[q] - sxx[q] * szz[q]) * mxz[q];
    for (size_t q = 0; q < n; q++) lm[q] = mxx[q] + myy[q] + mzz[q] + 2. * (mxy[q] + myz[q] + mxz[q]);
    /* homogeneous (y) average, LP = 0, NP != 0 (vt.f:296-318) */
    double *ilm = s->ilm, *imm = s->imm;
    for (size_t q = 0; q < n; q++) if (lm[q] < 0.) lm[q] = 0.;
    for (int k = kz1; k <= kz2; k++)
      for (int i = ix1; i <= ix2; i++) {
        double sm = 0., sl = 0.;
        for (int j = jy1; j <= jy2; j++) { sm += A(mm, i, j, k); sl += A(lm, i, j, k); }
        double am = sm / (double)(JM - 2), al = sl / (double)(JM - 2);
        for (int j = 1; j <= JM; j++) { A(imm, i, j, k) = am; A(ilm, i, j, k) = al; }
      }
    boundturb(s, ilm, 0);
    boundturb(s, imm, 1);
    for (size_t q = 0; q < n; q++) if (ilm[q] < 0) ilm[q] = 0.;
    double se = sqrt(s->prm.eps);
    for (size_t q = 0; q < n; q++) {
      tv[q] = 0.;
      if (imm[q] > se) tv[q] = (ilm[q] / imm[q]) * dx[q] * G[q];
      if (tv[q] < 0.0) tv[q] = 0.0;
    }
  }
  boundturb(s, s->tv, 0);
}
