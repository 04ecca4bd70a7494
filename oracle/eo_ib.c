/*
 * eo_ib.c -- immersed-boundary restatement (TEST INFRASTRUCTURE ONLY: the
 * checker for the CUDA immersed-boundary kernels).
 *
 * Follows, for one body in a Cartesian domain on a single rank:
 *   LIMIMB            src/object.f:713-800   body index limits from centroids
 *   TAG3D_MOD         src/rt.f:2704-3020     ray casting along z, IMBDCMP=0
 *   segtriint         src/rt.f:1179-1226     segment/triangle
 *   intersect_triangle src/rt.f:1263-1330    Moller-Trumbore, det eps 1e-18,
 *                                            u+v-1 > 1e-7 edge tolerance
 *   LOCATE            src/numrec.f:390-422   bisection (restated)
 *   taguo             src/devel.f:8-110      interior / forcing / fluid flags
 *   flagp             src/matint.f:135-260   pressure flags
 *   forcpts           src/matint.f:3388-3430 forcing-point list (k, j, i order)
 *   norm_intr         src/matint.f:1404-1690 normal-direction stencil
 *   grid_intr         src/matint.f:800-1160  grid-line stencil (26 directions)
 *   closest_intr      src/matint.f:1693-1985 closest-point stencil
 *   tri_closest_pt    src/rt.f:2525-2700     (published region method)
 *   ray_face_int,     src/rt.f:1395-1845, 2054-2155 ray / cell-face tests
 *   ray_poly_int, ray_xzface_int, point_poly_clasf, ray_seg_int, plane_tri
 *   vec_ijkext_gridpoint src/devel.f:5296-5410
 *   fluidface, closest src/matint.f:4124-4170, src/numrec.f:425-474
 *   recheckface       src/devel.f:8107-8175
 *   geom_mod          src/devel.f:9265-9800  dependency loops
 *   interp_cellface   src/interp.f:3-82      face interpolation (forcing)
 *   mtrx              src/devel.f:1159-1290  2x2 systems
 *   ludcmp / lubksb   src/numrec.f:22-118    LU with implicit partial pivoting
 *                                            (the published Crout algorithm,
 *                                            restated for n = 2)
 *   momforc_mod2      src/momforc.f:1248-1485 explicit forcing
 *   velinterior       src/momforc.f:186-300
 *   correctpres_mod2  src/momforc.f:1617-1760, correctdens_mod2 :1762
 *   presinterior      src/devel.f:1525, densinterior src/momforc.f:574
 *   RBM, ubd/vbd/wbd  src/rbm.f:2-40,168-309 (translation at a constant velocity)
 *
 * Restatement choices (the same in the CUDA path):
 *  * TAG3D's 2-D kd-tree (ANN committee4) only prunes the triangles tested
 *    against a column; here every triangle whose xy bounding box contains the
 *    column is tested, which is the set the reference's bounding-box test
 *    accepts when the search radius covers the triangle.
 *  * geom_mod (ivelrcn = 0) is restated with its three stencils and their
 *    order: the normal direction (mrk 1), the grid line (mrk 2), the closest
 *    point (mrk 3), each over the 3-D nearest-centroid candidate lists of
 *    sizes 3, 5, nntr3d (ANN committee3), computed exactly here (ties by
 *    triangle index; ANN's tie order is not specified).  Points whose
 *    stencil touches a forcing point wait for a later dependency loop under
 *    the reference's mimdif / ndif rules; points left without a stencil are
 *    dropped (the velocity flag becomes fluid, the pressure flag interior).
 *  * Faces and cells that would reach past the arrays count as missed (the
 *    reference bounds-checks i and j only; no case here reaches them).
 *  * The body translates at a constant velocity: ubd/vbd/wbd are constants.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "eddy_oracle.h"
#ifdef _OPENMP
#include <omp.h>
#endif

#define NCR 16
#define NNTR3D 25
#define NFLU 30

static long IDX(const eo_grid *g, int i, int j, int k) {
  return (long)(i - 1) + (long)g->nx * ((long)(j - 1) + (long)g->ny * (long)(k - 1));
}

/* ---- table search with the contract of LOCATE (src/numrec.f:390-422) ----
 * Position of x in the monotone table xx[1..n] (1-based): for an ascending
 * table the number of entries below x, i.e. j with xx[j] < x <= xx[j+1]
 * (0 below the table, n above it); for a descending one the number of
 * entries >= x; x equal to the first entry gives 1.  A partition-point
 * binary search over the predicate "entry m lies before x". */
int eo_locate(const double *xx, int n, double x) {
  if (xx[1] == x) return 1;
  const int asc = xx[n] > xx[1];
  int first = 1, count = n;
  while (count > 0) {
    const int step = count / 2, m = first + step;
    if ((x > xx[m]) == asc) {
      first = m + 1;
      count -= step + 1;
    } else {
      count = step;
    }
  }
  return first - 1;
}

/* ---- intersect_triangle (src/rt.f:1263-1330) ---- */
static void sub3(double *r, const double *a, const double *b) {
  r[0] = a[0] - b[0];
  r[1] = a[1] - b[1];
  r[2] = a[2] - b[2];
}
static void cross3(double *r, const double *x, const double *y) {
  r[0] = x[1] * y[2] - y[1] * x[2];
  r[1] = x[2] * y[0] - y[2] * x[0];
  r[2] = x[0] * y[1] - y[0] * x[1];
}
static double dot3(const double *x, const double *y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; }

static int intersect_triangle(const double *orig, const double *dir, const double *v0, const double *v1,
                              const double *v2, double *t, double *u, double *v) {
  double e1[3], e2[3], pv[3], tv[3], qv[3];
  *t = 0.;
  *u = 0.;
  *v = 0.;
  sub3(e1, v1, v0);
  sub3(e2, v2, v0);
  cross3(pv, dir, e2);
  double det = dot3(e1, pv);
  if (det > -1.0e-18 && det < 1.0e-18) return 2;
  double inv = 1.0 / det;
  sub3(tv, orig, v0);
  *u = dot3(tv, pv) * inv;
  if (*u < 0.0 || *u > 1.0) return 3;
  cross3(qv, tv, e1);
  *v = dot3(dir, qv) * inv;
  if (*v < 0.0 || (*u + *v - 1.) > 1.e-07) return 3;
  *t = dot3(e2, qv) * inv;
  return 1;
}

/* segtriint (src/rt.f:1179-1226): 1 and the point when segment p1->p2 meets
 * triangle (a,b,c) */
int eo_segtriint(const double *p1, const double *p2, const double *a, const double *b, const double *c,
                 double *xm) {
  double q[3] = {p1[0], p1[1], p1[2]}, r[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
  double t, u, v;
  int code = intersect_triangle(q, r, a, b, c, &t, &u, &v);
  if (code == 1 && (t > 1.0 || t < 0.0)) return 0;
  if (code == 2) code = intersect_triangle(q, r, a, c, b, &t, &u, &v);
  xm[0] = q[0] + t * r[0];
  xm[1] = q[1] + t * r[1];
  xm[2] = q[2] + t * r[2];
  return code == 1;
}

/* ---- state ---- */
struct eo_ib {
  const eo_grid *g;
  int nb;
  double *v, *c, *n;  /* vertices [nb][3][3], centroids [nb][3], normals [nb][3] */
  double vel[3];
  int lim[6];         /* imin imax jmin jmax kmin kmax */
  signed char *tag[4];  /* TAG3D IBS per variable u, v, w, p */
  signed char *flag[5]; /* taguo flags u, v, w, tv; flagp p */
  eo_ib_set set[4];     /* stencils u, v, w, p */
  int nntr3d, nflu, itagy;
  int every; /* 1: move + regenerate every substep, 0: once per step */
  int brute; /* 1: exhaustive searches (cross-check of the binned ones) */
  /* xy bins of the triangles' bounding boxes (TAG3D candidates) and 3-D bins
   * of the centroids (nearest-centroid lists); rebuilt at every regeneration */
  double bx0, by0, bx1, by1, bhx, bhy;
  int bnx, bny, *bstart, *blist;
  double c0[3], ch[3];
  int cn[3], *cstart, *clist;
};

eo_ib *eo_ib_create(const eo_grid *g, int nb, const double *vert, const double *normals, const double *vel) {
  eo_ib *ib = (eo_ib *)calloc(1, sizeof(eo_ib));
  ib->g = g;
  ib->nb = nb;
  ib->v = (double *)malloc(sizeof(double) * 9 * nb);
  ib->c = (double *)malloc(sizeof(double) * 3 * nb);
  ib->n = (double *)malloc(sizeof(double) * 3 * nb);
  memcpy(ib->v, vert, sizeof(double) * 9 * nb);
  memcpy(ib->n, normals, sizeof(double) * 3 * nb);
  for (int t = 0; t < nb; t++)
    for (int d = 0; d < 3; d++) {
      const double *tv = ib->v + 9 * t;
      ib->c[3 * t + d] = ((tv[d] + tv[3 + d]) + tv[6 + d]) / 3.0;
    }
  for (int d = 0; d < 3; d++) ib->vel[d] = vel[d];
  long nc = (long)g->nx * g->ny * g->nz;
  for (int q = 0; q < 4; q++) ib->tag[q] = (signed char *)calloc(nc, 1);
  for (int q = 0; q < 5; q++) ib->flag[q] = (signed char *)calloc(nc, 1);
  ib->nntr3d = NNTR3D;
  ib->nflu = NFLU;
  ib->itagy = 0;
  return ib;
}

static void set_free(eo_ib_set *s) {
  free(s->i); free(s->j); free(s->k); free(s->di); free(s->dj); free(s->dk);
  free(s->lev); free(s->indx); free(s->xn); free(s->yn); free(s->zn); free(s->lu); free(s->lev_start);
  free(s->mrk); free(s->dir); free(s->xe); free(s->ye); free(s->ze);
  memset(s, 0, sizeof(*s));
}

void eo_ib_free(eo_ib *ib) {
  if (!ib) return;
  free(ib->v); free(ib->c); free(ib->n);
  free(ib->bstart); free(ib->blist); free(ib->cstart); free(ib->clist);
  for (int q = 0; q < 4; q++) { free(ib->tag[q]); set_free(&ib->set[q]); }
  for (int q = 0; q < 5; q++) free(ib->flag[q]);
  free(ib);
}

/* coordinates of variable q: 0 u (xu, yc, zc), 1 v (xc, yv, zc), 2 w (xc, yc, zw), 3 p (xc, yc, zc) */
static void var_axes(const eo_grid *g, int q, const double **x, const double **y, const double **z) {
  *x = (q == 0) ? g->xu : g->xc;
  *y = (q == 1) ? g->yv : g->yc;
  *z = (q == 2) ? g->zw : g->zc;
}

/* ---- LIMIMB (src/object.f:713-800), Cartesian, single rank ---- */
void eo_ib_limimb(eo_ib *ib) {
  const eo_grid *g = ib->g;
  double mnx = 1e300, mxx = -1e300, mnz = 1e300, mxz = -1e300;
  for (int t = 0; t < ib->nb; t++) {
    mnx = fmin(mnx, ib->c[3 * t]);
    mxx = fmax(mxx, ib->c[3 * t]);
    mnz = fmin(mnz, ib->c[3 * t + 2]);
    mxz = fmax(mxz, ib->c[3 * t + 2]);
  }
  int imin = eo_locate(g->xu, g->nx, mnx), imax = eo_locate(g->xu, g->nx, mxx);
  int kmin = g->nz, kmax = 1;
  if (mnz < g->zw[g->nz] && mxz >= g->zc[1]) {
    kmin = eo_locate(g->zw, g->nz, mnz);
    kmax = eo_locate(g->zw, g->nz, mxz);
  }
  imin -= 3;
  imax += 3;
  if (imin < 1) imin = 1;
  if (imax > g->nx - 1) imax = g->nx - 1;
  if (kmax >= kmin) {
    kmin -= 3;
    kmax += 3;
  }
  if (kmin < 1) kmin = 1; /* ITYPE(5) /= 500 */
  if (kmax > g->nz) kmax = g->nz;
  ib->lim[0] = imin; ib->lim[1] = imax;
  ib->lim[2] = 2; ib->lim[3] = g->ny - 1;
  ib->lim[4] = kmin; ib->lim[5] = kmax;
}

/* ---- exact spatial bins (the reference prunes with ANN kd-trees; the
 * candidate sets here are supersets filtered by the same exact tests, visited
 * in ascending triangle order, so results equal the exhaustive search) ---- */
static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static void build_bins(eo_ib *ib) {
  const int nb = ib->nb;
  free(ib->bstart); free(ib->blist); free(ib->cstart); free(ib->clist);
  ib->bstart = ib->blist = ib->cstart = ib->clist = NULL;
  if (nb == 0) return;
  /* xy bins over the union of the triangles' xy boxes */
  double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
  for (int t = 0; t < nb; t++)
    for (int a = 0; a < 3; a++) {
      const double *p = ib->v + 9 * t + 3 * a;
      x0 = fmin(x0, p[0]); x1 = fmax(x1, p[0]); y0 = fmin(y0, p[1]); y1 = fmax(y1, p[1]);
    }
  int m = (int)ceil(sqrt((double)nb));
  m = clampi(m, 1, 2048);
  ib->bx0 = x0; ib->by0 = y0; ib->bx1 = x1; ib->by1 = y1;
  ib->bhx = (x1 - x0) / m; ib->bhy = (y1 - y0) / m;
  if (!(ib->bhx > 0)) ib->bhx = 1.0;
  if (!(ib->bhy > 0)) ib->bhy = 1.0;
  ib->bnx = m; ib->bny = m;
  ib->bstart = (int *)calloc((size_t)m * m + 1, sizeof(int));
  for (int pass = 0; pass < 2; pass++) {
    int *fill = pass ? (int *)calloc((size_t)m * m, sizeof(int)) : NULL;
    for (int t = 0; t < nb; t++) {
      const double *a = ib->v + 9 * t, *b = a + 3, *c = a + 6;
      double tx0 = fmin(fmin(a[0], b[0]), c[0]), tx1 = fmax(fmax(a[0], b[0]), c[0]);
      double ty0 = fmin(fmin(a[1], b[1]), c[1]), ty1 = fmax(fmax(a[1], b[1]), c[1]);
      int i0 = clampi((int)floor((tx0 - x0) / ib->bhx), 0, m - 1), i1 = clampi((int)floor((tx1 - x0) / ib->bhx), 0, m - 1);
      int j0 = clampi((int)floor((ty0 - y0) / ib->bhy), 0, m - 1), j1 = clampi((int)floor((ty1 - y0) / ib->bhy), 0, m - 1);
      for (int jb = j0; jb <= j1; jb++)
        for (int ibn = i0; ibn <= i1; ibn++) {
          int cell = jb * m + ibn;
          if (pass == 0) ib->bstart[cell + 1]++;
          else ib->blist[ib->bstart[cell] + fill[cell]++] = t;
        }
    }
    if (pass == 0) {
      for (int cidx = 0; cidx < m * m; cidx++) ib->bstart[cidx + 1] += ib->bstart[cidx];
      ib->blist = (int *)malloc(sizeof(int) * (size_t)(ib->bstart[m * m] > 0 ? ib->bstart[m * m] : 1));
    } else {
      free(fill);
    }
  }
  /* 3-D centroid bins, about four centroids per occupied cell of a shell */
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int t = 0; t < nb; t++)
    for (int d = 0; d < 3; d++) { lo[d] = fmin(lo[d], ib->c[3 * t + d]); hi[d] = fmax(hi[d], ib->c[3 * t + d]); }
  int n1 = clampi((int)ceil(sqrt((double)nb / 4.0)), 1, 512);
  int ntot = 1;
  for (int d = 0; d < 3; d++) {
    ib->c0[d] = lo[d];
    ib->cn[d] = n1;
    ib->ch[d] = (hi[d] - lo[d]) / n1;
    if (!(ib->ch[d] > 0)) ib->ch[d] = 1.0;
    ntot *= n1;
  }
  ib->cstart = (int *)calloc((size_t)ntot + 1, sizeof(int));
  ib->clist = (int *)malloc(sizeof(int) * (size_t)nb);
  int *cell = (int *)malloc(sizeof(int) * (size_t)nb);
  for (int t = 0; t < nb; t++) {
    int ci[3];
    for (int d = 0; d < 3; d++) ci[d] = clampi((int)floor((ib->c[3 * t + d] - ib->c0[d]) / ib->ch[d]), 0, n1 - 1);
    cell[t] = (ci[2] * n1 + ci[1]) * n1 + ci[0];
    ib->cstart[cell[t] + 1]++;
  }
  for (int cidx = 0; cidx < ntot; cidx++) ib->cstart[cidx + 1] += ib->cstart[cidx];
  int *fill = (int *)calloc((size_t)ntot, sizeof(int));
  for (int t = 0; t < nb; t++) ib->clist[ib->cstart[cell[t]] + fill[cell[t]]++] = t;
  free(fill);
  free(cell);
}

/* ---- TAG3D_MOD (src/rt.f:2704-3020) for variable q ---- */
void eo_ib_tag(eo_ib *ib, int q) {
  const eo_grid *g = ib->g;
  const double *X, *Y, *Z;
  var_axes(g, q, &X, &Y, &Z);
  signed char *ibs = ib->tag[q];
  long nc = (long)g->nx * g->ny * g->nz;
  for (long t = 0; t < nc; t++) ibs[t] = 1;
  const double zmin = g->zw[1], zmax = g->zw[g->nz - 1], zlen = zmax - zmin;
  const double rzmin = fmin(zmin - zlen, -1.0e8), rzmax = fmax(zmax + zlen, 1.0e8);
  const int ni = ib->lim[1] - ib->lim[0] + 1, nj = g->ny - 2;
#pragma omp parallel for schedule(dynamic, 16)
  for (int col = 0; col < ni * nj; col++) {
      const int i = ib->lim[0] + col / nj, j = 2 + col % nj;
      const double xcc = X[i], ycc = Y[j];
      double zc_[NCR], zo[NCR];
      int nc_ = 0;
      /* candidate triangles: all of them, or the xy bin of the column */
      int cb = 0, ce = ib->nb;
      const int *cl = NULL;
      if (!ib->brute) {
        cb = ce = 0;
        /* a triangle whose xy box holds the column was binned over a range
         * of bins that contains the column's (floor is monotone) */
        if (ib->nb > 0 && xcc >= ib->bx0 && xcc <= ib->bx1 && ycc >= ib->by0 && ycc <= ib->by1) {
          int bi = clampi((int)floor((xcc - ib->bx0) / ib->bhx), 0, ib->bnx - 1);
          int bj = clampi((int)floor((ycc - ib->by0) / ib->bhy), 0, ib->bny - 1);
          cb = ib->bstart[bj * ib->bnx + bi];
          ce = ib->bstart[bj * ib->bnx + bi + 1];
          cl = ib->blist;
        }
      }
      for (int ct = cb; ct < ce; ct++) {
        const int t = cl ? cl[ct] : ct;
        const double *a = ib->v + 9 * t, *b = a + 3, *c = a + 6;
        if (ycc >= fmin(fmin(a[1], b[1]), c[1]) && ycc <= fmax(fmax(a[1], b[1]), c[1]) &&
            xcc >= fmin(fmin(a[0], b[0]), c[0]) && xcc <= fmax(fmax(a[0], b[0]), c[0])) {
          double p1[3] = {xcc, ycc, rzmin}, p2[3] = {xcc, ycc, rzmax}, xm[3];
          if (eo_segtriint(p1, p2, a, b, c, xm)) {
            if (nc_ < NCR) zc_[nc_] = xm[2];
            nc_++;
          }
        }
      }
      if (nc_ > NCR) nc_ = NCR;
      /* selection sort ascending; ties take the last minimum (.le.) */
      for (int i1 = 0; i1 < nc_; i1++) {
        double ztmin = 1.0e10;
        int isave = 0;
        for (int i2 = 0; i2 < nc_; i2++)
          if (zc_[i2] <= ztmin) {
            ztmin = zc_[i2];
            isave = i2;
          }
        zo[i1] = ztmin;
        zc_[isave] = 2.0e10;
      }
      /* drop crossings within 1e-6 of an earlier one */
      double zz[NCR];
      for (int i1 = 0; i1 < nc_; i1++) zz[i1] = zo[i1];
      int ncl = 0;
      for (int i1 = 0; i1 < nc_; i1++) {
        int ndp = 0;
        for (int i2 = 0; i2 < nc_; i2++)
          if (fabs(zz[i2] - zz[i1]) < 1.e-06 && i1 > i2) ndp++;
        if (ndp == 0) zo[ncl++] = zz[i1];
      }
      if (ncl == 1) ncl = 0;
      for (int ic = 0; ic + 1 < ncl; ic += 2) {
        int k1 = eo_locate(Z, g->nz, zo[ic]);
        int k2 = eo_locate(Z, g->nz, zo[ic + 1]);
        if (k2 > k1)
          for (int k = k1 + 1; k <= k2; k++) ibs[IDX(g, i, j, k)] = -1;
      }
    }
  /* y periodic ghosts over the body's k range */
  for (int k = ib->lim[4]; k <= ib->lim[5]; k++)
    for (int i = ib->lim[0]; i <= ib->lim[1]; i++) {
      ibs[IDX(g, i, 1, k)] = ibs[IDX(g, i, g->ny - 1, k)];
      ibs[IDX(g, i, g->ny, k)] = ibs[IDX(g, i, 2, k)];
    }
}

/* ---- taguo (src/devel.f:8-110): flago 1 interior, -1 forcing, 0 fluid ---- */
void eo_ib_taguo(eo_ib *ib, int q, int fq) {
  const eo_grid *g = ib->g;
  const signed char *f = ib->tag[q];
  signed char *fo = ib->flag[fq];
  long nc = (long)g->nx * g->ny * g->nz;
  memset(fo, 0, nc);
  const int *L = ib->lim;
  for (int k = L[4]; k <= L[5]; k++)
    for (int j = L[2]; j <= L[3]; j++)
      for (int i = L[0]; i <= L[1]; i++)
        if (f[IDX(g, i, j, k)] == -1) fo[IDX(g, i, j, k)] = 1;
  for (int k = 1; k <= g->nz; k++)
    for (int i = 1; i <= g->nx; i++) {
      fo[IDX(g, i, 1, k)] = fo[IDX(g, i, g->ny - 1, k)];
      fo[IDX(g, i, g->ny, k)] = fo[IDX(g, i, 2, k)];
    }
  const int nn = ib->itagy == 0 ? 2 : 0;
  const int k1 = L[4] > 2 ? L[4] : 2, k2 = L[5] < g->nz - 1 ? L[5] : g->nz - 1;
  for (int k = k1; k <= k2; k++)
    for (int j = L[2]; j <= L[3]; j++)
      for (int i = (L[0] > 2 ? L[0] : 2); i <= L[1]; i++) {
        int c = f[IDX(g, i, j, k)];
        int nb[6] = {c + f[IDX(g, i + 1, j, k)], c + f[IDX(g, i - 1, j, k)], c + f[IDX(g, i, j, k + 1)],
                     c + f[IDX(g, i, j, k - 1)], c + f[IDX(g, i, j - 1, k)], c + f[IDX(g, i, j + 1, k)]};
        long prod = 1;
        for (int m = 0; m < 6 - nn; m++) prod *= nb[m];
        if (prod == 0 && c == 1) fo[IDX(g, i, j, k)] = -1;
      }
  for (int k = 1; k <= g->nz; k++)
    for (int i = 1; i <= g->nx; i++) {
      fo[IDX(g, i, 1, k)] = fo[IDX(g, i, g->ny - 1, k)];
      fo[IDX(g, i, g->ny, k)] = fo[IDX(g, i, 2, k)];
    }
}

/* ---- flagp (src/matint.f:135-260) ---- */
void eo_ib_flagp(eo_ib *ib) {
  const eo_grid *g = ib->g;
  const signed char *fu = ib->flag[0], *fv = ib->flag[1], *fw = ib->flag[2];
  signed char *fp = ib->flag[4];
  long nc = (long)g->nx * g->ny * g->nz;
  memset(fp, 0, nc);
  const int *L = ib->lim;
  for (int pass = 0; pass < 2; pass++) {
    int ka = pass == 0 ? L[4] : (L[4] > 2 ? L[4] : 2);
    int kb = pass == 0 ? 1 : L[5];
    for (int k = ka; k <= kb; k++)
      for (int j = L[2]; j <= L[3]; j++)
        for (int i = (L[0] > 2 ? L[0] : 2); i <= L[1]; i++) {
          int it[6], n;
          if (pass == 0) {
            it[0] = fu[IDX(g, i, j, k)]; it[1] = fu[IDX(g, i - 1, j, k)]; it[2] = fw[IDX(g, i, j, k)];
            it[3] = fv[IDX(g, i, j, k)]; it[4] = fv[IDX(g, i, j - 1, k)];
            n = 5;
          } else {
            it[0] = fu[IDX(g, i, j, k)]; it[1] = fu[IDX(g, i - 1, j, k)]; it[2] = fw[IDX(g, i, j, k)];
            it[3] = fw[IDX(g, i, j, k - 1)]; it[4] = fv[IDX(g, i, j, k)]; it[5] = fv[IDX(g, i, j - 1, k)];
            n = 6;
          }
          int ifld = 0, ibdy = 0, ibnd = 0;
          for (int m = 0; m < n; m++) {
            ifld += it[m] == 0;
            ibdy += it[m] > 0;
            ibnd += it[m] < 0;
          }
          signed char *o = &fp[IDX(g, i, j, k)];
          if ((ibdy + ibnd) != 0 && ifld != 0) *o = -1;
          if (ifld == 0 && ibnd != 0) *o = -1;
          if (ifld == 0 && ibnd == 0 && ibdy != 0) *o = 1;
        }
  }
}

/* ---- exact k nearest centroids (ties by triangle index): the first k of
 * all centroids ordered by (squared distance, index) ---- */
static void topk_insert(double *best, int *bi, int *m, int k, double d2, int t) {
  if (*m == k && (d2 > best[k - 1] || (d2 == best[k - 1] && t > bi[k - 1]))) return;
  int p = *m < k ? *m : k - 1;
  while (p > 0 && (best[p - 1] > d2 || (best[p - 1] == d2 && bi[p - 1] > t))) {
    best[p] = best[p - 1];
    bi[p] = bi[p - 1];
    p--;
  }
  best[p] = d2;
  bi[p] = t;
  if (*m < k) (*m)++;
}

static void knn(const eo_ib *ib, const double *q, int k, int *out) {
  double best[NNTR3D];
  int bi[NNTR3D];
  int m = 0;
  if (ib->brute || !ib->cstart) {
    for (int t = 0; t < ib->nb; t++) {
      const double *c = ib->c + 3 * t;
      double dx = c[0] - q[0], dy = c[1] - q[1], dz = c[2] - q[2];
      topk_insert(best, bi, &m, k, dx * dx + dy * dy + dz * dz, t);
    }
  } else {
    /* rings of cells around the query's cell until no unvisited centroid can
     * come closer than the k-th found (strictly, with a rounding margin) */
    const int *n = ib->cn;
    int ci[3];
    for (int d = 0; d < 3; d++) ci[d] = clampi((int)floor((q[d] - ib->c0[d]) / ib->ch[d]), 0, n[d] - 1);
    for (int r = 0;; r++) {
      int lo[3], hi[3], full = 1;
      for (int d = 0; d < 3; d++) {
        lo[d] = ci[d] - r; hi[d] = ci[d] + r;
        if (lo[d] > 0 || hi[d] < n[d] - 1) full = 0;
      }
      for (int z = lo[2] < 0 ? 0 : lo[2]; z <= (hi[2] > n[2] - 1 ? n[2] - 1 : hi[2]); z++)
        for (int y = lo[1] < 0 ? 0 : lo[1]; y <= (hi[1] > n[1] - 1 ? n[1] - 1 : hi[1]); y++)
          for (int x = lo[0] < 0 ? 0 : lo[0]; x <= (hi[0] > n[0] - 1 ? n[0] - 1 : hi[0]); x++) {
            if (x != lo[0] && x != hi[0] && y != lo[1] && y != hi[1] && z != lo[2] && z != hi[2]) continue;
            int cell = (z * n[1] + y) * n[0] + x;
            for (int e = ib->cstart[cell]; e < ib->cstart[cell + 1]; e++) {
              const int t = ib->clist[e];
              const double *c = ib->c + 3 * t;
              double dx = c[0] - q[0], dy = c[1] - q[1], dz = c[2] - q[2];
              topk_insert(best, bi, &m, k, dx * dx + dy * dy + dz * dz, t);
            }
          }
      if (full) break;
      /* distance from q to the nearest face of the visited box that has
       * cells beyond it */
      double dmin = 1e300;
      for (int d = 0; d < 3; d++) {
        if (lo[d] > 0) dmin = fmin(dmin, q[d] - (ib->c0[d] + lo[d] * ib->ch[d]));
        if (hi[d] < n[d] - 1) dmin = fmin(dmin, (ib->c0[d] + (hi[d] + 1) * ib->ch[d]) - q[d]);
      }
      if (m == k && dmin > 0 && best[k - 1] * (1.0 + 1e-9) < dmin * dmin) break;
    }
  }
  for (int a = 0; a < m; a++) out[a] = bi[a];
  for (int a = m; a < k; a++) out[a] = -1;
}

static const int GIND[26][3] = {
    {1, 0, 0},  {-1, 0, 0}, {0, 0, 1},   {0, 0, -1},  {1, 0, 1},   {1, 0, -1},  {-1, 0, 1},
    {-1, 0, -1}, {0, 1, 0},  {0, -1, 0},  {1, 1, 0},   {-1, 1, 0},  {0, 1, 1},   {0, 1, -1},
    {1, 1, 1},  {1, 1, -1}, {-1, 1, 1},  {-1, 1, -1}, {1, -1, 0},  {-1, -1, 0}, {0, -1, 1},
    {0, -1, -1}, {1, -1, 1}, {1, -1, -1}, {-1, -1, 1}, {-1, -1, -1}};

static double unitdot(const double *x, const double *xn, const double *nrm) {
  double a[3] = {x[0] - xn[0], x[1] - xn[1], x[2] - xn[2]};
  double ma = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  a[0] = a[0] / ma; a[1] = a[1] / ma; a[2] = a[2] / ma;
  double b[3] = {nrm[0], nrm[1], nrm[2]};
  double mb = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
  b[0] = b[0] / mb; b[1] = b[1] / mb; b[2] = b[2] / mb;
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* ---- face and ray primitives of the stencil searches (Cartesian) ----
 * Sums start from zero as the reference's DOTPROD / DOTPRODUCT / vecmag do
 * (src/triinter.f:119, src/rt.f:2101,2164). */
static double dotz3(const double *a, const double *b) {
  double s = 0.;
  s = s + a[0] * b[0];
  s = s + a[1] * b[1];
  s = s + a[2] * b[2];
  return s;
}

static double magz3(const double *a) {
  double s = 0.;
  s = s + a[0] * a[0];
  s = s + a[1] * a[1];
  s = s + a[2] * a[2];
  return sqrt(s);
}

/* ray_seg_int (src/rt.f:2054-2096): ray p + a q (a >= 0) against the segment
 * r + b s (0 <= b <= 1) */
static int ray_seg(const double *p, const double *q, const double *r, const double *s) {
  double f[2] = {s[1], -s[0]};
  const double d0 = (0. + f[0] * q[0]) + f[1] * q[1];
  if (d0 == 0.) return 0;
  const double g[2] = {r[0] - p[0], r[1] - p[1]};
  const double a = ((0. + f[0] * g[0]) + f[1] * g[1]) / d0;
  if (!(a >= 0.)) return 0;
  f[0] = q[1];
  f[1] = -q[0];
  const double b = ((0. + f[0] * g[0]) + f[1] * g[1]) / d0;
  return b >= 0.0 && b <= 1.0;
}

/* point_poly_clasf (src/rt.f:1590-1625): crossings of the ray towards
 * (1000, 0) with the edges v1-v2, v2-v3, v3-v4 of the 4-vertex polygon (the
 * closing edge v4-v1 is not tested, as in the reference); odd is inside */
static int point_in_face(double x, double y, const double V[4][3], int u, int v) {
  const double p[2] = {x, y}, q[2] = {1000., 0.};
  int cross = 0;
  for (int e = 0; e < 3; e++) {
    const double r[2] = {V[e][u], V[e][v]};
    const double s[2] = {V[e + 1][u] - V[e][u], V[e + 1][v] - V[e][v]};
    cross += ray_seg(p, q, r, s);
  }
  return cross % 2;
}

/* plane_tri + cross (src/rt.f:2130-2155, 1250-1259): A x + B y + C z + D = 0
 * through the first three vertices */
static void face_plane(const double V[4][3], double *pn, double *dd) {
  double s1[3], s2[3];
  for (int a = 0; a < 3; a++) {
    s1[a] = V[1][a] - V[0][a];
    s2[a] = V[2][a] - V[0][a];
  }
  pn[0] = s1[1] * s2[2] - s2[1] * s1[2];
  pn[1] = s1[2] * s2[0] - s2[2] * s1[0];
  pn[2] = s1[0] * s2[1] - s2[0] * s1[1];
  *dd = -((pn[0] * V[0][0] + pn[1] * V[0][1]) + pn[2] * V[0][2]);
}

/* ray_poly_int (src/rt.f:1507-1580): plane hit at t >= 0, then the polygon
 * test in the coordinate plane picked by the largest (signed) normal entry */
static int ray_poly(const double *q, const double *r, const double V[4][3], double *xi) {
  double pn[3], dd;
  face_plane(V, pn, &dd);
  const double vd = dotz3(pn, r);
  if (vd == 0.) return 0;
  const double v1 = -(dotz3(pn, q) + dd);
  const double t = v1 / vd;
  if (!(t >= 0.)) return 0;
  xi[0] = q[0] + t * r[0];
  xi[1] = q[1] + t * r[1];
  xi[2] = q[2] + t * r[2];
  int dir = 0;
  if (pn[1] > pn[dir]) dir = 1;
  if (pn[2] > pn[dir]) dir = 2;
  if (dir == 0) return point_in_face(xi[1], xi[2], V, 1, 2);
  if (dir == 1) return point_in_face(xi[0], xi[2], V, 0, 2);
  return point_in_face(xi[0], xi[1], V, 0, 1);
}

/* ray_xzface_int (src/rt.f:1740-1845), Cartesian: plane hit at t >= 0 inside
 * the x and z ranges of the face */
static int ray_xzface(const double *q, const double *r, const double V[4][3], double *xi) {
  double pn[3], dd;
  face_plane(V, pn, &dd);
  const double vd = dotz3(pn, r);
  if (vd == 0.) return 0;
  const double v1 = -(dotz3(pn, q) + dd);
  const double t = v1 / vd;
  if (t < 0.) return 0;
  xi[0] = q[0] + t * r[0];
  xi[1] = q[1] + t * r[1];
  xi[2] = q[2] + t * r[2];
  double rmin = V[0][0], rmax = V[1][0], zmin = V[0][2], zmax = V[3][2];
  if (rmin > rmax) { const double a = rmin; rmin = rmax; rmax = a; }
  if (zmin > zmax) { const double a = zmin; zmin = zmax; zmax = a; }
  if (xi[0] < rmin || xi[0] > rmax) return 0;
  if (xi[2] < zmin || xi[2] > zmax) return 0;
  return 1;
}

/* ray_face_int (src/rt.f:1395-1500), Cartesian: the ray q + t r against the
 * face of cell (i, j, k) normal to axis dir (1..3).  Faces that would reach
 * past the arrays count as missed (the reference checks i and j only). */
static int ray_face(const eo_grid *g, const double *X, const double *Y, const double *Z, const double *q,
                    const double *r, int i, int j, int k, int dir, double *xi) {
  if (i < 1 || i > g->nx || j < 1 || j > g->ny) return 0;
  if (k < 1 || k > g->nz) return 0;
  const int i1 = dir == 1 ? i : i + 1, j1 = dir == 2 ? j : j + 1, k1 = dir == 3 ? k : k + 1;
  if (i1 > g->nx || j1 > g->ny || k1 > g->nz) return 0;
  double V[4][3];
  if (dir == 1) {
    const double v[4][3] = {{X[i], Y[j], Z[k]}, {X[i], Y[j1], Z[k]}, {X[i], Y[j1], Z[k1]}, {X[i], Y[j], Z[k1]}};
    memcpy(V, v, sizeof(V));
    return ray_poly(q, r, V, xi);
  }
  if (dir == 2) {
    const double v[4][3] = {{X[i], Y[j], Z[k]}, {X[i1], Y[j], Z[k]}, {X[i1], Y[j], Z[k1]}, {X[i], Y[j], Z[k1]}};
    memcpy(V, v, sizeof(V));
    return ray_xzface(q, r, V, xi);
  }
  const double v[4][3] = {{X[i], Y[j], Z[k]}, {X[i1], Y[j], Z[k]}, {X[i1], Y[j1], Z[k]}, {X[i], Y[j1], Z[k]}};
  memcpy(V, v, sizeof(V));
  return ray_poly(q, r, V, xi);
}

/* vec_ijkext_gridpoint (src/devel.f:5296-5410), Cartesian: the cell whose
 * face normal to axis dir the ray from a grid point along r crosses first */
static void ray_cell(const double *r, int dir, int *e) {
  const int pi = !(r[0] < 0), pj = !(r[1] < 0), pk = !(r[2] < 0);
  if (dir == 1) {
    e[0] = pi ? 1 : -1; e[1] = pj ? 0 : -1; e[2] = pk ? 0 : -1;
  } else if (dir == 2) {
    e[0] = pi ? 0 : -1; e[1] = pj ? 1 : -1; e[2] = pk ? 0 : -1;
  } else {
    e[0] = pi ? 0 : -1; e[1] = pj ? 0 : -1; e[2] = pk ? 1 : -1;
  }
}

/* fluidface (src/matint.f:4124-4170): 1 all four nodes fluid, 0 a forcing
 * node, -1 a body node; faces reaching past the arrays give 0 */
static int fluid_face(const eo_grid *g, const signed char *flag, int i, int j, int k, int dir) {
  if (i < 1 || i > g->nx || j < 1 || j > g->ny) return 0;
  const int i1 = dir == 1 ? i : i + 1, j1 = dir == 2 ? j : j + 1, k1 = dir == 3 ? k : k + 1;
  if (k < 1 || i1 > g->nx || j1 > g->ny || k1 > g->nz) return 0;
  int t[4];
  if (dir == 1) {
    t[0] = flag[IDX(g, i, j, k)]; t[1] = flag[IDX(g, i, j1, k)];
    t[2] = flag[IDX(g, i, j, k1)]; t[3] = flag[IDX(g, i, j1, k1)];
  } else if (dir == 2) {
    t[0] = flag[IDX(g, i, j, k)]; t[1] = flag[IDX(g, i1, j, k)];
    t[2] = flag[IDX(g, i, j, k1)]; t[3] = flag[IDX(g, i1, j, k1)];
  } else {
    t[0] = flag[IDX(g, i, j, k)]; t[1] = flag[IDX(g, i1, j, k)];
    t[2] = flag[IDX(g, i, j1, k)]; t[3] = flag[IDX(g, i1, j1, k)];
  }
  int any = 0, pos = 0;
  for (int a = 0; a < 4; a++) {
    any |= t[a] != 0;
    pos |= t[a] > 0;
  }
  return pos ? -1 : (any ? 0 : 1);
}

/* closest (src/numrec.f:425-474): the entry of the monotone table nearest
 * to x, from the LOCATE position and its upper neighbour */
static int closest_entry(const double *xx, int n, double x) {
  int j = eo_locate(xx, n, x);
  if (j > 0 && j < n) {
    if (fabs(x - xx[j]) > fabs(x - xx[j + 1])) j = j + 1;
  } else if (j < 1) {
    j = 1;
  } else if (j > n) {
    j = n;
  }
  return j;
}

/* the cell face normal to axis dir holding point xp: the nearest node along
 * dir, the LOCATE cells along the other two (recheckface / interp_cellface) */
static void face_of_point(const eo_grid *g, const double *X, const double *Y, const double *Z, const double *xp,
                          int dir, int *i, int *j, int *k) {
  *i = dir == 1 ? closest_entry(X, g->nx, xp[0]) : eo_locate(X, g->nx, xp[0]);
  *j = dir == 2 ? closest_entry(Y, g->ny, xp[1]) : eo_locate(Y, g->ny, xp[1]);
  *k = dir == 3 ? closest_entry(Z, g->nz, xp[2]) : eo_locate(Z, g->nz, xp[2]);
}

/* recheckface (src/devel.f:8107-8175), Cartesian: 1 fluid face, -1 a forcing
 * node, -2 a body node */
static int recheck_face(const eo_grid *g, const double *X, const double *Y, const double *Z, const signed char *flag,
                        const double *xp, int dir) {
  int i, j, k;
  face_of_point(g, X, Y, Z, xp, dir, &i, &j, &k);
  const int f = fluid_face(g, flag, i, j, k, dir);
  return f == 0 ? -1 : (f == -1 ? -2 : f);
}

/* tri_closest_pt (src/rt.f:2525-2700): the point of triangle (v0, v1, v2)
 * nearest to p, by the published region decomposition of the (s, t)
 * parameter plane (D. Eberly, "Distance Between Point and Triangle in 3D",
 * Geometric Tools); only s and t are needed, not the distance */
static void tri_nearest(const double *tv, const double *p, double *out) {
  double e0[3], e1[3], df[3];
  for (int a = 0; a < 3; a++) {
    e0[a] = tv[3 + a] - tv[a];
    e1[a] = tv[6 + a] - tv[a];
    df[a] = tv[a] - p[a];
  }
  const double a00 = dotz3(e0, e0), a01 = dotz3(e0, e1), a11 = dotz3(e1, e1);
  const double b0 = dotz3(e0, df), b1 = dotz3(e1, df);
  const double det = fabs(a00 * a11 - a01 * a01);
  double s = a01 * b1 - a11 * b0, t = a01 * b0 - a00 * b1;
  if (s + t <= det) {
    if (s < 0) {
      if (t < 0) { /* region 4 */
        if (b0 < 0.0) {
          t = 0.0;
          s = (-b0 >= a00) ? 1.0 : -b0 / a00;
        } else {
          s = 0.0;
          if (b1 > 0.0)
            t = 0.0;
          else if (-b1 >= a11)
            t = 1.0;
          else
            t = -b1 / a11;
        }
      } else { /* region 3 */
        s = 0.0;
        if (b1 >= 0.0)
          t = 0.0;
        else if (-b1 > a11)
          t = 1.0;
        else
          t = -b1 / a11;
      }
    } else if (t < 0.0) { /* region 5 */
      t = 0.0;
      if (b0 >= 0.0)
        s = 0.0;
      else if (-b0 >= a00)
        s = 1.0;
      else
        s = -b0 / a00;
    } else { /* region 0 */
      const double inv = 1.0 / det;
      s = s * inv;
      t = t * inv;
    }
  } else {
    if (s < 0.0) { /* region 2 */
      const double tmp0 = a01 + b0, tmp1 = a11 + b1;
      if (tmp1 > tmp0) {
        const double numer = tmp1 - tmp0, denom = a00 - 2.0 * a01 + a11;
        if (numer >= denom) {
          s = 1.0; t = 0.0;
        } else {
          s = numer / denom; t = 1.0 - s;
        }
      } else {
        s = 0.0;
        if (tmp1 <= 0.0)
          t = 1.0;
        else if (b1 >= 0.0)
          t = 0.0;
        else
          t = -b1 / a11;
      }
    } else if (t < 0.0) { /* region 6 */
      const double tmp0 = a01 + b1, tmp1 = a00 + b0;
      if (tmp1 > tmp0) {
        const double numer = tmp1 - tmp0, denom = a00 - 2.0 * a01 + a11;
        if (numer >= denom) {
          t = 1.0; s = 0.0;
        } else {
          t = numer / denom; s = 1.0 - t;
        }
      } else {
        t = 0.0;
        if (tmp1 < 0.0)
          s = 1.0;
        else if (b0 >= 0.0)
          s = 0.0;
        else
          s = -b0 / a00;
      }
    } else { /* region 1 */
      const double numer = a11 + b1 - a01 - b0;
      if (numer <= 0.0) {
        s = 0.0; t = 1.0;
      } else {
        const double denom = a00 - 2.0 * a01 + a11;
        if (numer >= denom) {
          s = 1.0; t = 0.0;
        } else {
          s = numer / denom; t = 1.0 - s;
        }
      }
    }
  }
  for (int a = 0; a < 3; a++) out[a] = (tv[a] + s * e0[a]) + t * e1[a];
}

/* one stencil search's result: body point xn, extension point xe on a fluid
 * face normal to axis dir, triangle fp (0-based, -1 none) */
typedef struct {
  double xn[3], xe[3];
  int dir, fp;
} eo_hit;

/* the first fluid face the ray q + t r crosses: tried along x, then y, then
 * z (the z cell side from the sign of sz), as norm_intr and closest_intr do.
 * Returns the fluidface code of the face found (1, 0, -1), or 2 when the ray
 * meets none of the three; xe and dir of the face found. */
static int ray_first_face(const eo_grid *g, const double *X, const double *Y, const double *Z,
                          const signed char *flag, const double *q, const double *r, int im, int jm, int km,
                          double *xe, int *dir) {
  int e[3];
  for (int d = 1; d <= 3; d++) {
    ray_cell(r, d, e);
    if (ray_face(g, X, Y, Z, q, r, im + e[0], jm + e[1], km + e[2], d, xe)) {
      *dir = d;
      return fluid_face(g, flag, im + e[0], jm + e[1], km + e[2], d);
    }
  }
  return 2;
}

/* norm_intr (src/matint.f:1404-1690): the normal of each candidate triangle
 * through the point (segment of 10 normals each way); the first triangle the
 * segment crosses whose normal ray from the point meets a face that is fluid
 * (1) or holds a forcing node (-1) decides.  Returns 1, -1, -2 (only faces
 * with body nodes), 0 (no triangle crossed, or no face met). */
static int norm_intr(const eo_ib *ib, int q, const signed char *flag, int im, int jm, int km, const int *inn, int nn,
                     eo_hit *h) {
  const eo_grid *g = ib->g;
  const double *X, *Y, *Z;
  var_axes(g, q, &X, &Y, &Z);
  const double p0[3] = {X[im], Y[jm], Z[km]};
  int res = 0;
  for (int in = 0; in < nn; in++) {
    const int n = inn[in];
    if (n < 0) continue;
    const double *un = ib->n + 3 * n;
    const double s1[3] = {p0[0] - 10.0 * -un[0], p0[1] - 10.0 * -un[1], p0[2] - 10.0 * -un[2]};
    const double s2[3] = {p0[0] + 10.0 * -un[0], p0[1] + 10.0 * -un[1], p0[2] + 10.0 * -un[2]};
    double xm[3];
    if (!eo_segtriint(s1, s2, ib->v + 9 * n, ib->v + 9 * n + 3, ib->v + 9 * n + 6, xm)) continue;
    const double r[3] = {fabs(10.0) * un[0], fabs(10.0) * un[1], fabs(10.0) * un[2]};
    h->fp = n;
    double xe[3];
    int dir = 0;
    const int f = ray_first_face(g, X, Y, Z, flag, p0, r, im, jm, km, xe, &dir);
    if (f == 1 || f == 0) {
      memcpy(h->xn, xm, sizeof(xm));
      memcpy(h->xe, xe, sizeof(xe));
      h->dir = dir;
      return f == 1 ? 1 : -1;
    }
    if (f == -1) res = -2;
  }
  return res;
}

/* closest_intr (src/matint.f:1693-1985): for every candidate triangle its
 * nearest point to the point, and the ray from that point through the
 * forcing point (turned to the triangle's outward side) to the first face it
 * meets; the first fluid face among the candidates decides, else the first
 * face holding a forcing node.  fp ends as the last candidate, as in the
 * reference.  Returns 1, -1, -2 (faces with body nodes only, or none met), 0
 * (no candidate). */
static int closest_intr(const eo_ib *ib, int q, const signed char *flag, int im, int jm, int km, const int *inn,
                        int nn, eo_hit *h) {
  const eo_grid *g = ib->g;
  const double *X, *Y, *Z;
  var_axes(g, q, &X, &Y, &Z);
  const double p0[3] = {X[im], Y[jm], Z[km]};
  int ibint = 0, nrec = 0, sel = -1, first = -1;
  for (int in = 0; in < nn; in++) {
    const int n = inn[in];
    if (n < 0) continue;
    const double *un = ib->n + 3 * n;
    double pn[3];
    tri_nearest(ib->v + 9 * n, p0, pn);
    ibint++;
    const double d[3] = {p0[0] - pn[0], p0[1] - pn[1], p0[2] - pn[2]};
    const double mag = magz3(d);
    double r[3] = {fabs(100.0) * d[0] / mag, fabs(100.0) * d[1] / mag, fabs(100.0) * d[2] / mag};
    if (dotz3(d, un) < 0) {
      r[0] = -r[0]; r[1] = -r[1]; r[2] = -r[2];
    }
    h->fp = n;
    double xe[3];
    int dir = 0;
    const int f = ray_first_face(g, X, Y, Z, flag, p0, r, im, jm, km, xe, &dir);
    if (f == 1 || f == 0) {
      nrec++;
      if (first < 0) {
        first = 0;
        memcpy(h->xn, pn, sizeof(pn));
        memcpy(h->xe, xe, sizeof(xe));
        h->dir = dir;
        sel = f == 1;
      }
      if (f == 1 && sel == 0) {
        /* the first fluid face wins over an earlier forcing-node face */
        memcpy(h->xn, pn, sizeof(pn));
        memcpy(h->xe, xe, sizeof(xe));
        h->dir = dir;
        sel = 1;
      }
    }
  }
  if (nrec == 0) return ibint == 0 ? 0 : -2;
  return sel ? 1 : -1;
}

/* interp_cellface (src/interp.f:3-82), Cartesian: bilinear interpolation of
 * a on the cell face normal to axis dir through xp; y indices periodic
 * (index_bnd, src/matint.f:4377-4405) */
static double interp_face(const eo_grid *g, const double *X, const double *Y, const double *Z, const double *a,
                          const double *xp, int dir) {
  int i, j, k;
  face_of_point(g, X, Y, Z, xp, dir, &i, &j, &k);
  /* cells inside the tables (a face point always lies inside them) */
  i = clampi(i, 1, dir == 1 ? g->nx : g->nx - 1);
  j = clampi(j, 1, dir == 2 ? g->ny : g->ny - 1);
  k = clampi(k, 1, dir == 3 ? g->nz : g->nz - 1);
  int jj[2] = {j, j + 1};
  for (int b = 0; b < 2; b++) {
    if (jj[b] <= 1)
      jj[b] = g->ny - 2 + jj[b];
    else if (jj[b] >= g->ny)
      jj[b] = jj[b] - g->ny + 2;
  }
  if (dir == 1) {
    const double b1 = (xp[1] - Y[j]) / (Y[j + 1] - Y[j]), c1 = (xp[2] - Z[k]) / (Z[k + 1] - Z[k]);
    return (((1 - b1) * (1 - c1) * a[IDX(g, i, jj[0], k)] + b1 * (1 - c1) * a[IDX(g, i, jj[1], k)]) +
            (1 - b1) * c1 * a[IDX(g, i, jj[0], k + 1)]) +
           b1 * c1 * a[IDX(g, i, jj[1], k + 1)];
  }
  if (dir == 2) {
    const double a1 = (xp[0] - X[i]) / (X[i + 1] - X[i]), c1 = (xp[2] - Z[k]) / (Z[k + 1] - Z[k]);
    return (((1 - a1) * (1 - c1) * a[IDX(g, i, jj[0], k)] + a1 * (1 - c1) * a[IDX(g, i + 1, jj[0], k)]) +
            (1 - a1) * c1 * a[IDX(g, i, jj[0], k + 1)]) +
           a1 * c1 * a[IDX(g, i + 1, jj[0], k + 1)];
  }
  const double a1 = (xp[0] - X[i]) / (X[i + 1] - X[i]), b1 = (xp[1] - Y[j]) / (Y[j + 1] - Y[j]);
  return (((1 - a1) * (1 - b1) * a[IDX(g, i, jj[0], k)] + a1 * (1 - b1) * a[IDX(g, i + 1, jj[0], k)]) +
          (1 - a1) * b1 * a[IDX(g, i, jj[1], k)]) +
         a1 * b1 * a[IDX(g, i + 1, jj[1], k)];
}

/* grid_intr (src/matint.f:800-1160), igrdint = 1: the 26 grid directions in
 * the order of the criterion isrt (0: fluid, then forcing neighbours; 1: the
 * fluid neighbours by the cosine of the direction with the normal of
 * triangle fp; 2: the same for fluid and forcing neighbours), the first
 * candidate triangle the 10x extended grid segment crosses with the
 * extension point on its outward side.  Returns 1 (fluid extension point),
 * -1 (a forcing point), 0 (no crossing), -2 (inward crossings only); on 1
 * and -1 the body point xn, the offsets dd (as reals in ext) and the
 * triangle fp. */
int eo_ib_grid_intr(const eo_ib *ib, int q, const signed char *flag, int im, int jm, int km, const int *inn,
                    int nn, int isrt, double *xn, double *ext, int *fp) {
  const eo_grid *g = ib->g;
  const double *X, *Y, *Z;
  var_axes(g, q, &X, &Y, &Z);
  const double p0[3] = {X[im], Y[jm], Z[km]};
  double crit[26];
  int ord[26];
  for (int i = 0; i < 26; i++) {
    const int f = flag[IDX(g, im + GIND[i][0], jm + GIND[i][1], km + GIND[i][2])];
    crit[i] = -2.0;
    if (isrt == 0) {
      if (f == 0)
        crit[i] = 1.0;
      else if (f < 0)
        crit[i] = 0.5;
    } else if ((isrt == 1 && f == 0) || (isrt == 2 && f <= 0)) {
      double r[3] = {X[im + GIND[i][0]] - p0[0], Y[jm + GIND[i][1]] - p0[1], Z[km + GIND[i][2]] - p0[2]};
      const double m = magz3(r);
      r[0] = r[0] / m; r[1] = r[1] / m; r[2] = r[2] / m;
      crit[i] = dotz3(r, ib->n + 3 * *fp);
    }
  }
  int nphy = 0;
  for (int i = 0; i < 26; i++) {
    int b = 0;
    for (int m = 1; m < 26; m++)
      if (crit[m] > crit[b]) b = m;
    ord[i] = b;
    crit[b] = -10.0;
    if (flag[IDX(g, im + GIND[i][0], jm + GIND[i][1], km + GIND[i][2])] <= 0) nphy++;
  }
  int intrs = 0, ibint = 0;
  double xint[26][3];
  int tri[26], dir[26], icand[26];
  for (int i = 0; i < nphy; i++) {
    const int ii = ord[i];
    const int id = GIND[ii][0], jd = GIND[ii][1], kd = GIND[ii][2];
    const int fext = flag[IDX(g, im + id, jm + jd, km + kd)];
    if (fext > 0) continue;
    const double pe[3] = {X[im + id], Y[jm + jd], Z[km + kd]};
    double r[3] = {pe[0] - p0[0], pe[1] - p0[1], pe[2] - p0[2]};
    r[0] = r[0] * 10.0; r[1] = r[1] * 10.0; r[2] = r[2] * 10.0;
    const double s1[3] = {p0[0] - r[0], p0[1] - r[1], p0[2] - r[2]};
    const double s2[3] = {p0[0] + r[0], p0[1] + r[1], p0[2] + r[2]};
    for (int in = 0; in < nn; in++) {
      const int n = inn[in];
      if (n < 0) continue;
      const double *a = ib->v + 9 * n;
      double xm[3];
      if (eo_segtriint(s1, s2, a, a + 3, a + 6, xm)) {
        ibint++;
        if (unitdot(pe, p0, ib->n + 3 * n) > 0.0) {
          xint[intrs][0] = xm[0]; xint[intrs][1] = xm[1]; xint[intrs][2] = xm[2];
          tri[intrs] = n;
          dir[intrs] = ii;
          icand[intrs] = fext < 0;
          intrs++;
          break;
        }
      }
    }
  }
  if (intrs == 0) return ibint == 0 ? 0 : -2;
  double best = 0.;
  int bsel = -1;
  for (int m = 0; m < intrs; m++) {
    const int ii = dir[m];
    const double pe[3] = {X[im + GIND[ii][0]], Y[jm + GIND[ii][1]], Z[km + GIND[ii][2]]};
    double ds = unitdot(pe, p0, ib->n + 3 * tri[m]);
    ds = ds + (double)flag[IDX(g, im + GIND[ii][0], jm + GIND[ii][1], km + GIND[ii][2])] * (double)(m + 1);
    if (bsel < 0 || ds > best) {
      best = ds;
      bsel = m;
    }
  }
  xn[0] = xint[bsel][0]; xn[1] = xint[bsel][1]; xn[2] = xint[bsel][2];
  ext[0] = GIND[dir[bsel]][0]; ext[1] = GIND[dir[bsel]][1]; ext[2] = GIND[dir[bsel]][2];
  *fp = tri[bsel];
  return icand[bsel] ? -1 : 1;
}

/* one forcing point's search state across the dependency loops (geom_mod):
 * mrk (0 new; 1, 2, 3 valid; -1, -2, -3 waiting on the normal, grid-line or
 * closest-point stencil), the triangle fp, the face axis dir, the candidate
 * list stage icm (lists of 3, 5, nntr3d nearest centroids), the body point
 * and the extension (face coordinates for mrk 1, 3; grid offsets for 2) */
typedef struct {
  int mrk, fp, dir, icm;
  double xn[3], ext[3];
} eo_pt;

/* geom_mod's treatment of one point in loop ilp (src/devel.f:9470-9755):
 * the normal-direction stencil for a new point, else the grid-line stencil,
 * else the closest-point stencil; waiting points are rechecked against the
 * working flags.  Returns the new mrk (0: not valid, the point is dropped). */
static int geom_point(const eo_ib *ib, int q, const signed char *fw, int im, int jm, int km, const int *inn,
                      int ilp, int mimdif, int ndif, eo_pt *st) {
  const eo_grid *g = ib->g;
  const double *X, *Y, *Z;
  var_axes(g, q, &X, &Y, &Z);
  const int nfu = ib->nflu;
  const int sizes[3] = {3, 5, ib->nntr3d};
  int intrs = 0;
  if (st->mrk == -1) {
    intrs = recheck_face(g, X, Y, Z, fw, st->ext, st->dir);
  } else if (st->mrk == 0) {
    for (int icm = 0; icm < 3; icm++) {
      st->icm = icm;
      eo_hit h;
      h.fp = st->fp;
      intrs = norm_intr(ib, q, fw, im, jm, km, inn, sizes[icm], &h);
      st->fp = h.fp;
      if (intrs == 1 || intrs == -1) {
        memcpy(st->xn, h.xn, sizeof(h.xn));
        memcpy(st->ext, h.xe, sizeof(h.xe));
        st->dir = h.dir;
      }
      if (intrs != 0) break;
    }
    if (intrs == 0) st->fp = -1;
  }
  if (im <= 2) intrs = 0;
  if (intrs == 1) return 1;
  if (intrs == -1 && ilp < nfu && mimdif != 0) return -1;
  int gintrs = 0;
  if (st->mrk == -2 && ndif < 3) {
    gintrs = fw[IDX(g, im + (int)st->ext[0], jm + (int)st->ext[1], km + (int)st->ext[2])] == 0 ? 1 : -1;
  } else {
    int srt = 0;
    if (st->fp >= 0) srt = ndif < 2 ? 1 : 2;
    int icm = st->icm;
    while (icm < 3) {
      gintrs = eo_ib_grid_intr(ib, q, fw, im, jm, km, inn, sizes[icm], srt, st->xn, st->ext, &st->fp);
      if (gintrs != 0 && gintrs != -2) break;
      icm++;
      if (icm < 3) st->icm = icm;
    }
  }
  if (gintrs == 1) return 2;
  if (gintrs == -1 && ilp < nfu) return -2;
  int cintrs;
  if (st->mrk == -3) {
    cintrs = recheck_face(g, X, Y, Z, fw, st->ext, st->dir);
  } else {
    eo_hit h;
    h.fp = st->fp;
    cintrs = closest_intr(ib, q, fw, im, jm, km, inn, sizes[st->icm], &h);
    st->fp = h.fp;
    if (cintrs == 1 || cintrs == -1) {
      memcpy(st->xn, h.xn, sizeof(h.xn));
      memcpy(st->ext, h.xe, sizeof(h.xe));
      st->dir = h.dir;
    }
  }
  if (cintrs == 1) return 3;
  if (cintrs == -1 && ilp < nfu && ndif < 2) return -3;
  return 0;
}

/* ---- ludcmp/lubksb for n = 2 (implicit partial pivoting, Crout) ---- */
void eo_lu2(double *a /* column-major a11 a21 a12 a22 */, int *indx) {
  double A[2][2] = {{a[0], a[2]}, {a[1], a[3]}};
  double vv[2];
  for (int i = 0; i < 2; i++) {
    double aamax = 0.;
    for (int j = 0; j < 2; j++)
      if (fabs(A[i][j]) > aamax) aamax = fabs(A[i][j]);
    vv[i] = 1. / aamax;
  }
  /* column 1 */
  double aamax = 0.;
  int imax = 0;
  for (int i = 0; i < 2; i++) {
    double sum = A[i][0];
    double dum = vv[i] * fabs(sum);
    if (dum >= aamax) {
      imax = i;
      aamax = dum;
    }
  }
  if (imax != 0) {
    for (int k = 0; k < 2; k++) {
      double dum = A[imax][k];
      A[imax][k] = A[0][k];
      A[0][k] = dum;
    }
    vv[imax] = vv[0];
  }
  indx[0] = imax;
  if (A[0][0] == 0.) A[0][0] = 1.0e-20;
  {
    double dum = 1. / A[0][0];
    A[1][0] = A[1][0] * dum;
  }
  /* column 2 */
  {
    double sum = A[1][1];
    sum = sum - A[1][0] * A[0][1];
    A[1][1] = sum;
  }
  indx[1] = 1;
  if (A[1][1] == 0.) A[1][1] = 1.0e-20;
  a[0] = A[0][0]; a[1] = A[1][0]; a[2] = A[0][1]; a[3] = A[1][1];
}

void eo_lusolve2(const double *a, const int *indx, double *b) {
  double A[2][2] = {{a[0], a[2]}, {a[1], a[3]}};
  int ii = -1;
  for (int i = 0; i < 2; i++) {
    int ll = indx[i];
    double sum = b[ll];
    b[ll] = b[i];
    if (ii >= 0) {
      for (int j = ii; j <= i - 1; j++) sum = sum - A[i][j] * b[j];
    } else if (sum != 0.) {
      ii = i;
    }
    b[i] = sum;
  }
  for (int i = 1; i >= 0; i--) {
    double sum = b[i];
    for (int j = i + 1; j < 2; j++) sum = sum - A[i][j] * b[j];
    b[i] = sum / A[i][i];
  }
}

/* ---- forcpts + geom_mod + mtrx, variable q (flag fq) ----
 * The dependency loops of geom_mod (src/devel.f:9420-9770) on one rank:
 * mimdif is the change in the number of points treated from one loop to the
 * next and ndif counts the loops without change; a loop treats its points
 * against the working flags of the previous loops, then the points it made
 * valid become fluid in those flags (physical_mrk2flag1_mod) and the y ghost
 * planes are refreshed.  Points are treated in forcpts order; the output is
 * ordered by the loop that made a point valid, then forcpts order
 * (rord_forcpts1). */
void eo_ib_geom(eo_ib *ib, int q, int fq, int imn) {
  const eo_grid *g = ib->g;
  const double *X, *Y, *Z;
  var_axes(g, q, &X, &Y, &Z);
  eo_ib_set *S = &ib->set[q];
  set_free(S);
  signed char *flagu = ib->flag[fq];
  const int *L = ib->lim;
  const int k1 = L[4] > 2 ? L[4] : 2, k2 = L[5] < g->nz - 1 ? L[5] : g->nz - 1;
  /* forcpts: (k, j, i) order */
  int cap = 1024, n = 0;
  int *pi = (int *)malloc(sizeof(int) * cap), *pj = (int *)malloc(sizeof(int) * cap),
      *pk = (int *)malloc(sizeof(int) * cap);
  for (int k = k1; k <= k2; k++)
    for (int j = L[2]; j <= L[3]; j++)
      for (int i = (L[0] > 2 ? L[0] : 2); i <= L[1]; i++)
        if (flagu[IDX(g, i, j, k)] == -1) {
          if (n == cap) {
            cap *= 2;
            pi = (int *)realloc(pi, sizeof(int) * cap);
            pj = (int *)realloc(pj, sizeof(int) * cap);
            pk = (int *)realloc(pk, sizeof(int) * cap);
          }
          pi[n] = i; pj[n] = j; pk[n] = k;
          n++;
        }
  const long nc = (long)g->nx * g->ny * g->nz;
  const int n1 = n > 0 ? n : 1;
  signed char *fw = (signed char *)malloc(nc);
  memcpy(fw, flagu, nc);
  eo_pt *st = (eo_pt *)calloc(n1, sizeof(eo_pt));
  int *lev = (int *)calloc(n1, sizeof(int)), *inn = (int *)malloc(sizeof(int) * NNTR3D * n1);
  int *pend = (int *)malloc(sizeof(int) * n1), *nxt = (int *)malloc(sizeof(int) * n1);
  int *res = (int *)malloc(sizeof(int) * n1), *out = (int *)malloc(sizeof(int) * n1);
  /* the nearest-centroid lists: sorted by (distance, index), so the lists
   * of 3 and 5 are prefixes of the nntr3d list */
#pragma omp parallel for schedule(dynamic, 8)
  for (int p = 0; p < n; p++) {
    const double qv[3] = {X[pi[p]], Y[pj[p]], Z[pk[p]]};
    knn(ib, qv, ib->nntr3d, inn + NNTR3D * p);
    st[p].fp = -1;
  }
  const signed char inonvld = (signed char)(imn == 0 ? 1 : 0);
  int np = n, prev = 0, ndif = 0, nlev = 0;
  for (int a = 0; a < n; a++) pend[a] = a;
  for (int ilp = 1; ilp <= ib->nflu; ilp++) {
    const int mimdif = np - prev;
    prev = np;
    if (mimdif == 0) ndif++;
    if (np == 0) break;
    /* the points of one loop are independent: the working flags change
     * only between loops */
#pragma omp parallel for schedule(dynamic, 4)
    for (int a = 0; a < np; a++) {
      const int p = pend[a];
      out[a] = geom_point(ib, q, fw, pi[p], pj[p], pk[p], inn + NNTR3D * p, ilp, mimdif, ndif, st + p);
    }
    int nres = 0, nn2 = 0;
    for (int a = 0; a < np; a++) {
      const int p = pend[a];
      st[p].mrk = out[a];
      if (out[a] > 0) {
        lev[p] = ilp;
        res[nres++] = p;
      } else if (out[a] < 0) {
        nxt[nn2++] = p;
      } else {
        flagu[IDX(g, pi[p], pj[p], pk[p])] = inonvld;
      }
    }
    if (nres > 0) nlev = ilp;
    for (int a = 0; a < nres; a++) fw[IDX(g, pi[res[a]], pj[res[a]], pk[res[a]])] = 0;
    for (int k = 1; k <= g->nz; k++)
      for (int i = 1; i <= g->nx; i++) {
        fw[IDX(g, i, 1, k)] = fw[IDX(g, i, g->ny - 1, k)];
        fw[IDX(g, i, g->ny, k)] = fw[IDX(g, i, 2, k)];
      }
    int *t = pend; pend = nxt; nxt = t;
    np = nn2;
  }
  /* outputs ordered by level, then forcpts order */
  int nv = 0;
  for (int a = 0; a < n; a++) nv += st[a].mrk > 0;
  S->n = nv;
  S->nlev = nlev;
  const int m1 = nv > 0 ? nv : 1;
  S->i = (int *)malloc(sizeof(int) * m1); S->j = (int *)malloc(sizeof(int) * m1); S->k = (int *)malloc(sizeof(int) * m1);
  S->di = (int *)malloc(sizeof(int) * m1); S->dj = (int *)malloc(sizeof(int) * m1); S->dk = (int *)malloc(sizeof(int) * m1);
  S->lev = (int *)malloc(sizeof(int) * m1); S->indx = (int *)malloc(sizeof(int) * 2 * m1);
  S->xn = (double *)malloc(sizeof(double) * m1); S->yn = (double *)malloc(sizeof(double) * m1);
  S->zn = (double *)malloc(sizeof(double) * m1); S->lu = (double *)malloc(sizeof(double) * 4 * m1);
  S->mrk = (int *)malloc(sizeof(int) * m1); S->dir = (int *)malloc(sizeof(int) * m1);
  S->xe = (double *)malloc(sizeof(double) * m1); S->ye = (double *)malloc(sizeof(double) * m1);
  S->ze = (double *)malloc(sizeof(double) * m1);
  S->lev_start = (int *)malloc(sizeof(int) * (nlev + 2));
  int o = 0;
  for (int l = 1; l <= nlev; l++) {
    S->lev_start[l - 1] = o;
    for (int a = 0; a < n; a++) {
      if (st[a].mrk <= 0 || lev[a] != l) continue;
      const eo_pt *s = st + a;
      const int grid = s->mrk == 2;
      S->i[o] = pi[a]; S->j[o] = pj[a]; S->k[o] = pk[a];
      S->di[o] = grid ? (int)s->ext[0] : 0; S->dj[o] = grid ? (int)s->ext[1] : 0; S->dk[o] = grid ? (int)s->ext[2] : 0;
      S->xe[o] = grid ? 0. : s->ext[0]; S->ye[o] = grid ? 0. : s->ext[1]; S->ze[o] = grid ? 0. : s->ext[2];
      S->mrk[o] = s->mrk;
      S->dir[o] = grid ? 0 : s->dir;
      S->lev[o] = l;
      S->xn[o] = s->xn[0]; S->yn[o] = s->xn[1]; S->zn[o] = s->xn[2];
      /* mtrx (src/devel.f:1159-1290), Cartesian: the extension point is the
       * grid point for mrk = 2, the face point otherwise */
      const double xu = X[pi[a]], yu = Y[pj[a]], zu = Z[pk[a]];
      double x1, y1, z1;
      if (grid) {
        x1 = X[pi[a] + S->di[o]]; y1 = Y[pj[a] + S->dj[o]]; z1 = Z[pk[a] + S->dk[o]];
      } else {
        x1 = s->ext[0]; y1 = s->ext[1]; z1 = s->ext[2];
      }
      const double is1 = imn == 1 ? -1. : 1.;
      double so = sqrt(((xu - S->xn[o]) * (xu - S->xn[o]) + (yu - S->yn[o]) * (yu - S->yn[o])) +
                       (zu - S->zn[o]) * (zu - S->zn[o])) * is1;
      double s1 = sqrt(((xu - x1) * (xu - x1) + (yu - y1) * (yu - y1)) + (zu - z1) * (zu - z1)) * 1.0;
      double *A = S->lu + 4 * o;
      if (imn != 0) {
        A[0] = 1.; A[2] = so;
      } else {
        A[0] = 0.; A[2] = 1.0;
      }
      A[1] = 1.; A[3] = s1;
      eo_lu2(A, S->indx + 2 * o);
      o++;
    }
  }
  S->lev_start[nlev] = o;
  free(pi); free(pj); free(pk); free(fw); free(st); free(lev); free(inn); free(pend); free(nxt); free(res); free(out);
}

/* the whole regeneration for the current body position (src/Eddy6.f:2163-2380) */
void eo_ib_regen(eo_ib *ib) {
  eo_ib_limimb(ib);
  build_bins(ib);
  for (int q = 0; q < 4; q++) {
    eo_ib_tag(ib, q);
    eo_ib_taguo(ib, q, q);
  }
  for (int q = 0; q < 3; q++) eo_ib_geom(ib, q, q, 1);
  eo_ib_flagp(ib);
  eo_ib_geom(ib, 3, 4, 0);
}

/* RBM: translation over tmove (src/rbm.f:2-40 with a constant velocity) */
void eo_ib_move(eo_ib *ib, double tmove) {
  for (int t = 0; t < ib->nb; t++) {
    double *tv = ib->v + 9 * t;
    for (int a = 0; a < 3; a++)
      for (int d = 0; d < 3; d++) tv[3 * a + d] = tv[3 * a + d] + ib->vel[d] * tmove;
    for (int d = 0; d < 3; d++) ib->c[3 * t + d] = ((tv[d] + tv[3 + d]) + tv[6 + d]) / 3.0;
  }
}

static void yper(const eo_grid *g, double *a) {
  for (int k = 1; k <= g->nz; k++)
    for (int i = 1; i <= g->nx; i++) {
      a[IDX(g, i, 1, k)] = a[IDX(g, i, g->ny - 1, k)];
      a[IDX(g, i, g->ny, k)] = a[IDX(g, i, 2, k)];
    }
}

/* momforc_mod2 explicit (src/momforc.f:1400-1470) / correctpres_mod2 with a
 * zero normal gradient (src/momforc.f:1690-1705): the extension value is the
 * grid point's (mrk 2) or interpolated on the fluid face (mrk 1, 3); levels
 * in order, y periodic planes after each */
void eo_ib_force(eo_ib *ib, int q, double *a, double b0) {
  const eo_grid *g = ib->g;
  const double *X, *Y, *Z;
  var_axes(g, q, &X, &Y, &Z);
  eo_ib_set *S = &ib->set[q];
  for (int l = 0; l < S->nlev; l++) {
    for (int o = S->lev_start[l]; o < S->lev_start[l + 1]; o++) {
      double ae;
      if (S->mrk[o] == 2) {
        int i1 = S->i[o] + S->di[o], j1 = S->j[o] + S->dj[o], k1 = S->k[o] + S->dk[o];
        if (j1 <= 1)
          j1 = g->ny - 2 + j1;
        else if (j1 >= g->ny)
          j1 = j1 - g->ny + 2;
        ae = a[IDX(g, i1, j1, k1)];
      } else {
        /* normal-direction and closest-point stencils: the value on the
         * fluid face (interp_cellface) */
        const double xe[3] = {S->xe[o], S->ye[o], S->ze[o]};
        ae = interp_face(g, X, Y, Z, a, xe, S->dir[o]);
      }
      double b[2] = {b0, ae};
      eo_lusolve2(S->lu + 4 * o, S->indx + 2 * o, b);
      a[IDX(g, S->i[o], S->j[o], S->k[o])] = b[0];
    }
    yper(g, a);
  }
}

/* momforc_mod2 with impl = 1 (src/momforc.f:1280-1372): the stencil values
 * come from UB (the explicit estimate us + alfxdt/2 C.N. part); each forcing
 * point takes us + b(1) - ub, which ub then takes too (later levels read it);
 * the y ghost planes of us are refreshed after every level */
void eo_ib_force_impl(eo_ib *ib, int q, double *us, double *ub, double b0) {
  const eo_grid *g = ib->g;
  const double *X, *Y, *Z;
  var_axes(g, q, &X, &Y, &Z);
  eo_ib_set *S = &ib->set[q];
  for (int l = 0; l < S->nlev; l++) {
    for (int o = S->lev_start[l]; o < S->lev_start[l + 1]; o++) {
      double ae;
      if (S->mrk[o] == 2) {
        int i1 = S->i[o] + S->di[o], j1 = S->j[o] + S->dj[o], k1 = S->k[o] + S->dk[o];
        if (j1 <= 1)
          j1 = g->ny - 2 + j1;
        else if (j1 >= g->ny)
          j1 = j1 - g->ny + 2;
        ae = ub[IDX(g, i1, j1, k1)];
      } else {
        const double xe[3] = {S->xe[o], S->ye[o], S->ze[o]};
        ae = interp_face(g, X, Y, Z, ub, xe, S->dir[o]);
      }
      double b[2] = {b0, ae};
      eo_lusolve2(S->lu + 4 * o, S->indx + 2 * o, b);
      const size_t c = IDX(g, S->i[o], S->j[o], S->k[o]);
      us[c] = us[c] + b[0] - ub[c];
      ub[c] = us[c];
    }
    yper(g, us);
  }
}

/* velinterior with impl = 1 (src/momforc.f:235-248): us - ub + the body
 * velocity at flag == 1 */
void eo_ib_interior_impl(eo_ib *ib, int fq, double *us, const double *ub, double value) {
  const eo_grid *g = ib->g;
  const int *L = ib->lim;
  const signed char *f = ib->flag[fq];
  for (int k = L[4]; k <= L[5]; k++)
    for (int j = L[2]; j <= L[3]; j++)
      for (int i = L[0]; i <= L[1]; i++)
        if (f[IDX(g, i, j, k)] == 1) us[IDX(g, i, j, k)] = us[IDX(g, i, j, k)] - ub[IDX(g, i, j, k)] + value;
  yper(g, us);
}

/* velinterior / presinterior / densinterior / tvinterior: value at flag == 1 */
void eo_ib_interior(eo_ib *ib, int fq, double *a, double value) {
  const eo_grid *g = ib->g;
  const int *L = ib->lim;
  const signed char *f = ib->flag[fq];
  for (int k = L[4]; k <= L[5]; k++)
    for (int j = L[2]; j <= L[3]; j++)
      for (int i = L[0]; i <= L[1]; i++)
        if (f[IDX(g, i, j, k)] == 1) a[IDX(g, i, j, k)] = value;
  yper(g, a);
}

/* ---- accessors ---- */
const int *eo_ib_limits(const eo_ib *ib) { return ib->lim; }
const double *eo_ib_velocity(const eo_ib *ib) { return ib->vel; }
void eo_ib_set_cadence(eo_ib *ib, int every) { ib->every = every ? 1 : 0; }
void eo_ib_set_brute(eo_ib *ib, int brute) { ib->brute = brute ? 1 : 0; }
int eo_ib_every(const eo_ib *ib) { return ib->every; }
const signed char *eo_ib_tags(const eo_ib *ib, int q) { return ib->tag[q]; }
const signed char *eo_ib_flags(const eo_ib *ib, int fq) { return ib->flag[fq]; }
const eo_ib_set *eo_ib_stencils(const eo_ib *ib, int q) { return &ib->set[q]; }
void eo_ib_body(const eo_ib *ib, double *v, double *c) {
  if (v) memcpy(v, ib->v, sizeof(double) * 9 * ib->nb);
  if (c) memcpy(c, ib->c, sizeof(double) * 3 * ib->nb);
}
