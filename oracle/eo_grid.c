/*
 * eo_grid.c -- oracle restatement of the reference grid/metric builder and of
 * the set-up routines that feed the hot path.  TEST INFRASTRUCTURE ONLY.
 *
 *   eo_grid_create  : src/grid.f:8-483 (igrid=1 x from file, uniform y,
 *                     kgrid=1 z from file), src/setup.f:2-75 (index bounds),
 *                     src/inpall.f:166-172 (MP/LP/NP),
 *                     src/vt.f:1374-1434 (filter weights),
 *                     src/Initialize.f:129-271 (sponge profiles),
 *                     src/hybrid.f:143 (background density; Cartesian form).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "eddy_oracle.h"

static double *alloc1(int n) { return (double *)calloc((size_t)n + 2, sizeof(double)); }

eo_grid *eo_grid_create(const eo_params *p, const double *xu_faces, double ymin,
                        double ymax, const double *zw_faces) {
  eo_grid *g = (eo_grid *)calloc(1, sizeof(eo_grid));
  int nx = p->nx, ny = p->ny, nz = p->nz;
  g->nx = nx; g->ny = ny; g->nz = nz;
  g->xu = alloc1(nx); g->xc = alloc1(nx); g->ap = alloc1(nx); g->au = alloc1(nx);
  g->av = alloc1(nx); g->aw = alloc1(nx);
  g->yv = alloc1(ny); g->yc = alloc1(ny); g->bp = alloc1(ny); g->bu = alloc1(ny);
  g->bv = alloc1(ny); g->bw = alloc1(ny);
  g->zw = alloc1(nz); g->zc = alloc1(nz); g->cp = alloc1(nz); g->cu = alloc1(nz);
  g->cv = alloc1(nz); g->cw = alloc1(nz);
  g->whx = (double *)calloc((size_t)3 * (nx + 2), sizeof(double));
  g->why = (double *)calloc((size_t)3 * (ny + 2), sizeof(double));
  g->whz = (double *)calloc((size_t)3 * (nz + 2), sizeof(double));
  g->dfxu = alloc1(nx); g->dfxw = alloc1(nx); g->dfxd = alloc1(nx);
  g->dfxul = alloc1(nz); g->dfxwl = alloc1(nz); g->dfxdl = alloc1(nz);
  g->dens_bg = (double *)calloc((size_t)nx * ny, sizeof(double));

  double *xu = g->xu, *xc = g->xc, *ap = g->ap, *au = g->au, *av = g->av, *aw = g->aw;
  /* ---- x: non-uniform grid read from file (grid.f:21-46) ---- */
  int ix1 = 2, ix2 = nx - 1;
  for (int i = 1; i <= ix2; i++) xu[i] = xu_faces[i - 1];
  xu[nx] = 2. * xu[ix2] - xu[ix2 - 1];
  for (int i = ix1; i <= ix2; i++) xc[i] = .5 * (xu[i - 1] + xu[i]);
  xc[1] = 2. * xu[1] - xc[2];
  xc[nx] = 2. * xu[ix2] - xc[ix2];
  for (int i = ix1; i <= ix2; i++) au[i] = 2. / (xu[i + 1] - xu[i - 1]);
  au[1] = 2. / (-3. * xu[1] + 4. * xu[2] - xu[3]);
  au[ix2] = 2. / (3. * xu[ix2] - 4. * xu[ix2 - 1] + xu[ix2 - 2]);
  au[nx] = au[ix2];
  for (int i = ix1; i <= ix2; i++) ap[i] = 1. / (xu[i] - xu[i - 1]);
  ap[1] = ap[ix1];
  ap[nx] = ap[ix2];
  for (int i = ix1; i <= ix2; i++) av[i] = 2. / (xc[i + 1] - xc[i - 1]);
  av[1] = 2. / (-3. * xc[1] + 4. * xc[2] - xc[3]);
  av[nx] = 2. / (3. * xc[nx] - 4. * xc[nx - 1] + xc[nx - 2]);
  for (int i = 1; i <= nx; i++) aw[i] = av[i];

  /* ---- y: uniform grid (grid.f:64-83) ---- */
  int jy1 = 2, jy2 = ny - 1;
  double ylen = ymax - ymin;
  double dely = ylen / (double)(ny - 2);
  double rdely = 1. / dely;
  for (int j = 1; j <= ny; j++) {
    g->yv[j] = (double)(j - 1) * dely + ymin;
    g->bp[j] = rdely; g->bu[j] = rdely; g->bv[j] = rdely; g->bw[j] = rdely;
  }
  g->dely = dely;
  g->delysq = dely * dely;

  /* ---- z: non-uniform grid read from file (grid.f:87-112) ---- */
  int kz1 = 2, kz2 = nz - 1;
  double *zw = g->zw, *zc = g->zc;
  for (int k = 1; k <= kz2; k++) zw[k] = zw_faces[k - 1];
  zw[nz] = 2. * zw[kz2] - zw[kz2 - 1];
  for (int k = kz1; k <= kz2; k++) zc[k] = .5 * (zw[k - 1] + zw[k]);
  zc[1] = 2. * zw[1] - zc[2];
  zc[nz] = 2. * zw[kz2] - zc[kz2];
  for (int k = kz1; k <= kz2; k++) g->cw[k] = 2. / (zw[k + 1] - zw[k - 1]);
  g->cw[1] = 2. / (-3. * zw[1] + 4. * zw[2] - zw[3]);
  g->cw[kz2] = 2. / (3. * zw[kz2] - 4. * zw[kz2 - 1] + zw[kz2 - 2]);
  /* grid.f:112 assigns cwg(nzg) = cw(kz2) from the still-empty COMMON array */
  g->cw[nz] = 0.;
  for (int k = kz1; k <= kz2; k++) g->cp[k] = 1. / (zw[k] - zw[k - 1]);
  g->cp[1] = g->cp[kz1];
  g->cp[nz] = g->cp[kz2];
  for (int k = kz1; k <= kz2; k++) g->cv[k] = 2. / (zc[k + 1] - zc[k - 1]);
  g->cv[1] = 2. / (-3. * zc[1] + 4. * zc[2] - zc[3]);
  g->cv[nz] = 2. / (3. * zc[nz] - 4. * zc[nz - 1] + zc[nz - 2]);
  for (int k = 1; k <= nz; k++) g->cu[k] = g->cv[k];
  /* grid.f:162-173 recompute the centres (same values) */
  for (int j = jy1; j <= jy2; j++) g->yc[j] = 0.5 * (g->yv[j] + g->yv[j - 1]);
  g->yc[jy1 - 1] = 2. * g->yv[jy1 - 1] - g->yc[jy1];
  g->yc[jy2 + 1] = 2. * g->yv[jy2] - g->yc[jy2];

  /* ---- index bounds (setup.f, inpall.f:166-172) ---- */
  g->ix1 = ix1; g->ix2 = ix2; g->jy1 = jy1; g->jy2 = jy2; g->kz1 = kz1; g->kz2 = kz2;
  g->ib1 = ix1 - 1; g->ib2 = ix2 + 1; g->jb1 = jy1 - 1; g->jb2 = jy2 + 1;
  g->kb1 = kz1 - 1; g->kb2 = kz2 + 1;
  g->ibu = ix1;
  g->ieu = (p->itype[2] == 500) ? ix2 : ix2 - 1;
  g->jbv = jy1;
  g->jev = (p->itype[4] == 500) ? jy2 : jy2 - 1;
  g->kbw = kz1;
  g->kew = (p->itype[6] == 500 || p->itype[6] == 0) ? kz2 : kz2 - 1;
  g->mp = (p->itype[2] == 500) ? 0 : 1;
  g->lp = (p->itype[4] == 500) ? 0 : 1;
  g->np = (p->itype[6] == 500) ? 0 : 1;

  /* ---- filter weights (vt.f:1374-1434); index [i*3 + d+1] ---- */
  double *whx = g->whx, *why = g->why, *whz = g->whz;
#define WH(a, i, d) a[(i)*3 + (d) + 1]
  for (int i = ix1; i <= ix2; i++) WH(whx, i, 0) = 0.50;
  for (int i = ix1 + 1; i <= ix2 - 1; i++) {
    WH(whx, i, -1) = 0.25 * av[i] / au[i];
    WH(whx, i, 1) = 0.25 * av[i] / au[i - 1];
  }
  WH(whx, ix1, -1) = 0.50 * av[ix1 + 1] / au[ix1] + 0.25 * av[ix1 + 1] / au[ix1 + 1];
  WH(whx, ix1, 1) = -0.25 * av[ix1 + 1] / au[ix1];
  WH(whx, ix2, -1) = 0.50 * av[ix2 - 1] / au[ix2 - 1] + 0.25 * av[ix2 - 1] / au[ix2 - 2];
  WH(whx, ix2, 1) = -0.25 * av[ix2 - 1] / au[ix2 - 1];
  for (int j = jy1; j <= jy2; j++) WH(why, j, 0) = 0.50;
  for (int j = jy1 + 1; j <= jy2 - 1; j++) {
    WH(why, j, -1) = 0.25 * g->bw[j] / g->bv[j];
    WH(why, j, 1) = 0.25 * g->bw[j] / g->bv[j - 1];
  }
  WH(why, jy1, -1) = 0.50 * g->bw[jy1 + 1] / g->bv[jy1] + 0.25 * g->bw[jy1 + 1] / g->bv[jy1 + 1];
  WH(why, jy1, 1) = -0.25 * g->bw[jy1 + 1] / g->bv[jy1];
  WH(why, jy2, -1) = 0.50 * g->bw[jy2 - 1] / g->bv[jy2 - 1] + 0.25 * g->bw[jy2 - 1] / g->bv[jy2 - 2];
  WH(why, jy2, 1) = -0.25 * g->bw[jy2 - 1] / g->bv[jy2 - 1];
  for (int k = kz1; k <= kz2; k++) {
    WH(whz, k, 0) = 0.50;
    WH(whz, k, -1) = 0.25 * g->cu[k] / g->cw[k];
    WH(whz, k, 1) = 0.25 * g->cu[k] / g->cw[k - 1];
  }
  if (p->itype[5] != 0) {
    WH(whz, kz1, -1) = 0.50 * g->cu[kz1 + 1] / g->cw[kz1] + 0.25 * g->cu[kz1 + 1] / g->cw[kz1 + 1];
    WH(whz, kz1, 1) = -0.25 * g->cu[kz1 + 1] / g->cw[kz1];
  }
  if (p->itype[6] != 0) {
    WH(whz, kz2, -1) = 0.50 * g->cu[kz2 - 1] / g->cw[kz2 - 1] + 0.25 * g->cu[kz2 - 1] / g->cw[kz2 - 2];
    WH(whz, kz2, 1) = -0.25 * g->cu[kz2 - 1] / g->cw[kz2 - 1];
  }
#undef WH

  /* ---- sponge profiles (Initialize.f:129-271) ---- */
  int ibu = g->ibu, ieu = g->ieu, nzg = nz;
  int vx1 = p->vspngx1, vin = p->vspngx3in, vout = p->vspngx3out;
  int dx1 = p->dspngx1, din = p->dspngx3in, dout = p->dspngx3out;
  for (int i = ibu; i <= ieu; i++) {
    g->dfxu[i] = 0.0;
    if (i >= ieu - vx1 && vx1 > 0) {
      double r = (xu[i] - xu[ieu - vx1]) / (xu[ieu] - xu[ieu - vx1]);
      g->dfxu[i] = 5.0 * (r * r);
    }
  }
  for (int i = ix1; i <= ix2; i++) {
    g->dfxw[i] = 0.0;
    if (i >= ix2 - vx1 && vx1 > 0) {
      double r = (xc[i] - xc[ix2 - vx1]) / (xc[ix2] - xc[ix2 - vx1]);
      g->dfxw[i] = 5.0 * (r * r);
    }
  }
  double *dfxug = alloc1(nzg), *dfxwg = alloc1(nzg), *dfxdg = alloc1(nzg);
  for (int k = nzg; k >= 1; k--) {
    dfxug[k] = 0.0;
    if (k <= vin + 1 && vin > 0) {
      double r = (zc[k] - zc[vin + 1]) / (zc[2] - zc[vin + 1]);
      dfxug[k] = 20.0 * (r * r);
    }
  }
  for (int k = nzg; k >= 1; k--) {
    dfxwg[k] = 0.0;
    if (k <= vin + 1 && vin > 0) {
      double r = (zw[k] - zw[vin + 1]) / (zw[2] - zw[vin + 1]);
      dfxwg[k] = 20.0 * (r * r);
    }
  }
  for (int k = 1; k <= nzg; k++) {
    if (k >= nzg - vout && vout > 0) {
      double r = (zc[k - 2] - zc[nzg - vout]) / (zc[nzg - 2] - zc[nzg - dout]);
      dfxug[k] = 10.0 * (r * r);
    }
  }
  for (int k = 1; k <= nzg; k++) {
    if (k >= nzg - vout && vout > 0) {
      double r = (zw[k - 2] - zw[nzg - dout]) / (zw[nzg - 2] - zw[nzg - dout]);
      dfxwg[k] = 10.0 * (r * r);
    }
  }
  g->ivspngl = 0;
  for (int k = kz1; k <= kz2; k++) {
    g->dfxul[k] = dfxug[k];
    g->dfxwl[k] = dfxwg[k];
    if (g->dfxwl[k] > 0.0) g->ivspngl = 1;
  }
  for (int k = 1; k <= nzg; k++) dfxdg[k] = 0.0;
  for (int k = 1; k <= nzg; k++) {
    if (k >= nzg - dout && dout > 0) {
      double r = (zc[k - 2] - zc[nzg - dout]) / (zc[nzg - 2] - zc[nzg - dout]);
      dfxdg[k] = 100.0 * (r * r);
    }
  }
  for (int k = nzg; k >= 1; k--) {
    if (k <= din + 1 && din > 0) {
      double r = (zc[k] - zc[din + 1]) / (zc[2] - zc[din + 1]);
      dfxdg[k] = 100.0 * (r * r);
    }
  }
  g->idspngl = 0;
  for (int k = kz1; k <= kz2; k++) {
    g->dfxdl[k] = dfxdg[k];
    if (g->dfxdl[k] > 0.0) g->idspngl = 1;
  }
  for (int i = ibu; i <= ieu; i++) {
    if (i >= ieu - dx1 && dx1 > 0) {
      double r = (xc[i] - xc[ieu - dx1]) / (xc[ieu] - xc[ieu - dx1]);
      g->dfxd[i] = 5.0 * (r * r);
    }
  }
  free(dfxug); free(dfxwg); free(dfxdg);

  /* ---- background density: hybrid.f:143 denP1*rp(i)*sin(yc(j)) is the
   * vertical coordinate of the cylindrical cross-section; the Cartesian
   * restatement takes x as the vertical, so dens_bg = denP1*xc(i). ---- */
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++)
      g->dens_bg[(i - 1) + (size_t)nx * (j - 1)] = p->denP1 * xc[i];
  return g;
}

void eo_grid_free(eo_grid *g) {
  if (!g) return;
  double *arrs[] = {g->xu, g->xc, g->ap, g->au, g->av, g->aw, g->yv, g->yc,
                    g->bp, g->bu, g->bv, g->bw, g->zw, g->zc, g->cp, g->cu,
                    g->cv, g->cw, g->whx, g->why, g->whz, g->dfxu, g->dfxw,
                    g->dfxul, g->dfxwl, g->dfxd, g->dfxdl, g->dens_bg};
  for (size_t i = 0; i < sizeof(arrs) / sizeof(arrs[0]); i++) free(arrs[i]);
  free(g);
}

int eo_grid_get(const eo_grid *g, int which, double *out, int n) {
  const double *src = NULL;
  int len = 0, off = 1;
  switch (which) {
    case 0: src = g->xu; len = g->nx; break;
    case 1: src = g->xc; len = g->nx; break;
    case 2: src = g->ap; len = g->nx; break;
    case 3: src = g->au; len = g->nx; break;
    case 4: src = g->av; len = g->nx; break;
    case 5: src = g->aw; len = g->nx; break;
    case 6: src = g->yv; len = g->ny; break;
    case 7: src = g->yc; len = g->ny; break;
    case 8: src = g->bp; len = g->ny; break;
    case 9: src = g->bu; len = g->ny; break;
    case 10: src = g->bv; len = g->ny; break;
    case 11: src = g->bw; len = g->ny; break;
    case 12: src = g->zw; len = g->nz; break;
    case 13: src = g->zc; len = g->nz; break;
    case 14: src = g->cp; len = g->nz; break;
    case 15: src = g->cu; len = g->nz; break;
    case 16: src = g->cv; len = g->nz; break;
    case 17: src = g->cw; len = g->nz; break;
    case 18: src = g->whx; len = 3 * (g->nx + 1); off = 0; break;
    case 19: src = g->why; len = 3 * (g->ny + 1); off = 0; break;
    case 20: src = g->whz; len = 3 * (g->nz + 1); off = 0; break;
    case 21: src = g->dfxu; len = g->nx; break;
    case 22: src = g->dfxw; len = g->nx; break;
    case 23: src = g->dfxul; len = g->nz; break;
    case 24: src = g->dfxwl; len = g->nz; break;
    case 25: src = g->dfxd; len = g->nx; break;
    case 26: src = g->dfxdl; len = g->nz; break;
    case 27: src = g->dens_bg; len = g->nx * g->ny; off = 0; break;
    default: return -1;
  }
  if (n < len) return -2;
  memcpy(out, src + off, sizeof(double) * (size_t)len);
  return len;
}
