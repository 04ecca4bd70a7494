/*
 * eo_core.c -- oracle restatement of the pointwise/stencil parts of the
 * fractional step.  TEST INFRASTRUCTURE ONLY.  Compiled with
 * -ffp-contract=off so every expression keeps the reference's operation order.
 *
 * Cartesian branch only (icyl=0, ru=rp=1).  The viscous terms along y may be
 * Crank-Nicolson implicit (IMPLY = 1, over the whole x range): RHS then keeps
 * them out of the explicit part and returns them as the C.N. parts ut,vt,wt
 * (src/rhs.f:175-191), INVERSEY/INVERSEYD solve the periodic y lines; the
 * other implicit options (implx, implcx, implcy) are 0.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "eddy_oracle.h"

#ifdef _OPENMP
#include <omp.h>
#endif

#define NX (g->nx)
#define NY (g->ny)
#define NZ (g->nz)
#define IX(i, j, k) ((size_t)((i) - 1) + (size_t)NX * ((size_t)((j) - 1) + (size_t)NY * (size_t)((k) - 1)))
#define A(a, i, j, k) (a)[IX(i, j, k)]
#define DBG(i, j) g->dens_bg[(size_t)((i) - 1) + (size_t)NX * (size_t)((j) - 1)]

void eo_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

uint64_t eo_splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

double eo_uniform(uint64_t seed, uint64_t counter) {
  uint64_t h = eo_splitmix64(eo_splitmix64(seed) ^ counter);
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

static double *zalloc(long n) { return (double *)calloc((size_t)n, sizeof(double)); }

eo_state *eo_state_create(const eo_params *p, const eo_grid *g) {
  eo_state *s = (eo_state *)calloc(1, sizeof(eo_state));
  s->prm = *p;
  s->g = (eo_grid *)g;
  long n = (long)p->nx * p->ny * p->nz;
  s->ncell = n;
  double **f3[] = {&s->uo, &s->vo, &s->wo, &s->p, &s->dp, &s->dens, &s->tv,
                   &s->us, &s->vs, &s->ws, &s->ua, &s->va, &s->wa, &s->ub,
                   &s->vb, &s->wb, &s->rha, &s->rhb, &s->rs, &s->g_s, &s->sxx,
                   &s->syy, &s->szz, &s->sxy, &s->syz, &s->sxz, &s->ilm,
                   &s->imm, &s->lm, &s->mm, &s->uc, &s->vc, &s->wc, &s->dxdydz,
                   &s->cles};
  for (size_t i = 0; i < sizeof(f3) / sizeof(f3[0]); i++) *f3[i] = zalloc(n);
  long n2 = (long)p->nx * p->ny;
  s->planeU = zalloc(n2); s->planeV = zalloc(n2); s->planeW = zalloc(n2);
  s->planeD = zalloc(n2);
  return s;
}

void eo_state_free(eo_state *s) {
  if (!s) return;
  double *f3[] = {s->uo, s->vo, s->wo, s->p, s->dp, s->dens, s->tv, s->us,
                  s->vs, s->ws, s->ua, s->va, s->wa, s->ub, s->vb, s->wb,
                  s->rha, s->rhb, s->rs, s->g_s, s->sxx, s->syy, s->szz,
                  s->sxy, s->syz, s->sxz, s->ilm, s->imm, s->lm, s->mm, s->uc,
                  s->vc, s->wc, s->dxdydz, s->cles, s->planeU, s->planeV,
                  s->planeW, s->planeD};
  for (size_t i = 0; i < sizeof(f3) / sizeof(f3[0]); i++) free(f3[i]);
  free(s->feed);
  free(s);
}

double *eo_field(eo_state *s, int id) {
  switch (id) {
    case EO_UO: return s->uo; case EO_VO: return s->vo; case EO_WO: return s->wo;
    case EO_P: return s->p; case EO_DP: return s->dp; case EO_DENS: return s->dens;
    case EO_TV: return s->tv; case EO_US: return s->us; case EO_VS: return s->vs;
    case EO_WS: return s->ws; case EO_UA: return s->ua; case EO_VA: return s->va;
    case EO_WA: return s->wa; case EO_UB: return s->ub; case EO_VB: return s->vb;
    case EO_WB: return s->wb; case EO_RHA: return s->rha; case EO_RHB: return s->rhb;
    case EO_RS: return s->rs; case EO_PLANEU: return s->planeU;
    case EO_PLANEV: return s->planeV; case EO_PLANEW: return s->planeW;
    case EO_PLANED: return s->planeD;
    default: return NULL;
  }
}

static long field_len(eo_state *s, int id) {
  if (id >= EO_PLANEU && id <= EO_PLANED) return (long)s->prm.nx * s->prm.ny;
  return s->ncell;
}
int eo_set(eo_state *s, int id, const double *src) {
  double *d = eo_field(s, id);
  if (!d) return -1;
  memcpy(d, src, sizeof(double) * (size_t)field_len(s, id));
  return 0;
}
int eo_get(eo_state *s, int id, double *dst) {
  double *d = eo_field(s, id);
  if (!d) return -1;
  memcpy(dst, d, sizeof(double) * (size_t)field_len(s, id));
  return 0;
}

/* ------------------------------------------------------------------------
 * RHS: src/rhs.f:4-438 (icyl=0; rflagx = IMPLX, rflagy = IMPLY, rflagcx =
 * IMPLCX, rflagcy = IMPLCY: ut,vt,wt take the C.N. parts).
 * ut,vt,wt and ur,vr,wr are zeroed over the whole array first (rhs.f:65-70);
 * qr = uo (rhs.f:58).
 * ---------------------------------------------------------------------- */
void eo_rhs(eo_state *s, const double *uo, const double *vo, const double *wo,
            const double *tv, double *ut, double *vt, double *wt, double *ur,
            double *vr, double *wr, double *qr) {
  const eo_grid *g = s->g;
  const double ru1 = s->prm.ru1;
  const double *ap = g->ap, *au = g->au, *av = g->av, *aw = g->aw;
  const double *bp = g->bp, *bu = g->bu, *bv = g->bv, *bw = g->bw;
  const double *cp = g->cp, *cu = g->cu, *cv = g->cv, *cw = g->cw;
  long n = s->ncell;
  /* rflag* of src/rhs.f:49-52 with ruimplx = rvimplx = ruimply = rvimply = 1
   * (IMPLXDCMP = IMPLYDCMP = 0) */
  const double rflagx = (double)s->prm.implx, rflagcx = (double)s->prm.implcx, rflagy = (double)s->prm.imply,
               rflagcy = (double)s->prm.implcy;
  memcpy(qr, uo, sizeof(double) * (size_t)n);
  memset(ut, 0, sizeof(double) * (size_t)n); memset(ur, 0, sizeof(double) * (size_t)n);
  memset(vt, 0, sizeof(double) * (size_t)n); memset(vr, 0, sizeof(double) * (size_t)n);
  memset(wt, 0, sizeof(double) * (size_t)n); memset(wr, 0, sizeof(double) * (size_t)n);
  /* u component (rhs.f:77-205) */
#pragma omp parallel for schedule(static)
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ibu; i <= g->ieu; i++) {
        double qxp = (A(qr, i + 1, j, k) + A(qr, i, j, k)) * 0.5;
        double qxm = (A(qr, i, j, k) + A(qr, i - 1, j, k)) * 0.5;
        double uxp = (A(uo, i + 1, j, k) + A(uo, i, j, k)) * 0.5;
        double uxm = (A(uo, i, j, k) + A(uo, i - 1, j, k)) * 0.5;
        double uyp = (A(uo, i, j + 1, k) + A(uo, i, j, k)) * 0.5;
        double uym = (A(uo, i, j, k) + A(uo, i, j - 1, k)) * 0.5;
        double uzp = (A(uo, i, j, k + 1) + A(uo, i, j, k)) * 0.5;
        double uzm = (A(uo, i, j, k) + A(uo, i, j, k - 1)) * 0.5;
        double vxp = (A(vo, i + 1, j, k) + A(vo, i, j, k)) * 0.5;
        double vxm = (A(vo, i + 1, j - 1, k) + A(vo, i, j - 1, k)) * 0.5;
        double wxp = (A(wo, i + 1, j, k) + A(wo, i, j, k)) * 0.5;
        double wxm = (A(wo, i + 1, j, k - 1) + A(wo, i, j, k - 1)) * 0.5;
        double dqdxp = ap[i + 1] * (A(qr, i + 1, j, k) - A(qr, i, j, k));
        double dqdxm = ap[i] * (A(qr, i, j, k) - A(qr, i - 1, j, k));
        double dudyp = bv[j] * (A(uo, i, j + 1, k) - A(uo, i, j, k));
        double dudym = bv[j - 1] * (A(uo, i, j, k) - A(uo, i, j - 1, k));
        double dudzp = cw[k] * (A(uo, i, j, k + 1) - A(uo, i, j, k));
        double dudzm = cw[k - 1] * (A(uo, i, j, k) - A(uo, i, j, k - 1));
        double dvdxp = au[i] * (A(vo, i + 1, j, k) - A(vo, i, j, k));
        double dvdxm = au[i] * (A(vo, i + 1, j - 1, k) - A(vo, i, j - 1, k));
        double dwdxp = au[i] * (A(wo, i + 1, j, k) - A(wo, i, j, k));
        double dwdxm = au[i] * (A(wo, i + 1, j, k - 1) - A(wo, i, j, k - 1));
        double tvjp = 0.25 * (A(tv, i + 1, j, k) + A(tv, i, j, k) + A(tv, i + 1, j + 1, k) + A(tv, i, j + 1, k));
        double tvjm = 0.25 * (A(tv, i + 1, j, k) + A(tv, i, j, k) + A(tv, i + 1, j - 1, k) + A(tv, i, j - 1, k));
        double tvkp = 0.25 * (A(tv, i + 1, j, k) + A(tv, i, j, k) + A(tv, i + 1, j, k + 1) + A(tv, i, j, k + 1));
        double tvkm = 0.25 * (A(tv, i + 1, j, k) + A(tv, i, j, k) + A(tv, i + 1, j, k - 1) + A(tv, i, j, k - 1));
        double txxp = (ru1 + 2. * A(tv, i + 1, j, k)) * dqdxp;
        double txxm = (ru1 + 2. * A(tv, i, j, k)) * dqdxm;
        double tyyp = (ru1 + tvjp) * dudyp;
        double tyym = (ru1 + tvjm) * dudym;
        double tzzp = (ru1 + tvkp) * dudzp;
        double tzzm = (ru1 + tvkm) * dudzm;
        double txyp = tvjp * dvdxp;
        double txym = tvjm * dvdxm;
        double txzp = tvkp * dwdxp;
        double txzm = tvkm * dwdxm;
        double h11 = -au[i] * (qxp * uxp - qxm * uxm);
        double h22 = -bu[j] * (vxp * uyp - vxm * uym);
        double h33 = -cu[k] * (wxp * uzp - wxm * uzm);
        double t11 = au[i] * (txxp - txxm);
        double t22 = bu[j] * (tyyp - tyym);
        double t33 = cu[k] * (tzzp - tzzm);
        double s22 = bu[j] * (txyp - txym);
        double s33 = cu[k] * (txzp - txzm);
        A(ur, i, j, k) = (1. - rflagcx * 1.) * h11 + (1. - rflagcy * 1.) * h22 + h33 + (1. - rflagx * 1.) * t11 +
                         (1. - rflagy * 1.) * t22 + t33 + s22 + s33;
        A(ut, i, j, k) = rflagx * 1. * t11 + rflagy * 1. * t22 + rflagcx * 1. * h11 + rflagcy * 1. * h22;
      }
  /* v component (rhs.f:219-335) */
#pragma omp parallel for schedule(static)
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jbv; j <= g->jev; j++)
      for (int i = g->ix1; i <= g->ix2; i++) {
        double vxp = (A(vo, i + 1, j, k) + A(vo, i, j, k)) * 0.5;
        double vxm = (A(vo, i, j, k) + A(vo, i - 1, j, k)) * 0.5;
        double vyp = (A(vo, i, j + 1, k) + A(vo, i, j, k)) * 0.5;
        double vym = (A(vo, i, j, k) + A(vo, i, j - 1, k)) * 0.5;
        double vzp = (A(vo, i, j, k + 1) + A(vo, i, j, k)) * 0.5;
        double vzm = (A(vo, i, j, k) + A(vo, i, j, k - 1)) * 0.5;
        double qyp = (A(qr, i, j + 1, k) + A(qr, i, j, k)) * 0.5;
        double qym = (A(qr, i - 1, j + 1, k) + A(qr, i - 1, j, k)) * 0.5;
        double wyp = (A(wo, i, j + 1, k) + A(wo, i, j, k)) * 0.5;
        double wym = (A(wo, i, j + 1, k - 1) + A(wo, i, j, k - 1)) * 0.5;
        double dvdxp = au[i] * (A(vo, i + 1, j, k) - A(vo, i, j, k));
        double dvdxm = au[i - 1] * (A(vo, i, j, k) - A(vo, i - 1, j, k));
        double dvdyp = bp[j + 1] * (A(vo, i, j + 1, k) - A(vo, i, j, k));
        double dvdym = bp[j] * (A(vo, i, j, k) - A(vo, i, j - 1, k));
        double dvdzp = cw[k] * (A(vo, i, j, k + 1) - A(vo, i, j, k));
        double dvdzm = cw[k - 1] * (A(vo, i, j, k) - A(vo, i, j, k - 1));
        double dudyp = bv[j] * (A(uo, i, j + 1, k) - A(uo, i, j, k));
        double dudym = bv[j] * (A(uo, i - 1, j + 1, k) - A(uo, i - 1, j, k));
        double dwdyp = bv[j] * (A(wo, i, j + 1, k) - A(wo, i, j, k));
        double dwdym = bv[j] * (A(wo, i, j + 1, k - 1) - A(wo, i, j, k - 1));
        double tvip = 0.25 * (A(tv, i, j + 1, k) + A(tv, i, j, k) + A(tv, i + 1, j + 1, k) + A(tv, i + 1, j, k));
        double tvim = 0.25 * (A(tv, i, j + 1, k) + A(tv, i, j, k) + A(tv, i - 1, j + 1, k) + A(tv, i - 1, j, k));
        double tvkp = 0.25 * (A(tv, i, j + 1, k) + A(tv, i, j, k) + A(tv, i, j + 1, k + 1) + A(tv, i, j, k + 1));
        double tvkm = 0.25 * (A(tv, i, j + 1, k) + A(tv, i, j, k) + A(tv, i, j + 1, k - 1) + A(tv, i, j, k - 1));
        double txxp = (ru1 + tvip) * dvdxp;
        double txxm = (ru1 + tvim) * dvdxm;
        double tyyp = (ru1 + 2. * A(tv, i, j + 1, k)) * dvdyp;
        double tyym = (ru1 + 2. * A(tv, i, j, k)) * dvdym;
        double tzzp = (ru1 + tvkp) * dvdzp;
        double tzzm = (ru1 + tvkm) * dvdzm;
        double txyp = tvip * dudyp;
        double txym = tvim * dudym;
        double tyzp = tvkp * dwdyp;
        double tyzm = tvkm * dwdym;
        double h11 = -av[i] * (qyp * vxp - qym * vxm);
        double h22 = -bv[j] * (vyp * vyp - vym * vym);
        double h33 = -cv[k] * (wyp * vzp - wym * vzm);
        double t11 = av[i] * (txxp - txxm);
        double t22 = bv[j] * (tyyp - tyym);
        double t33 = cv[k] * (tzzp - tzzm);
        double s11 = av[i] * (txyp - txym);
        double s33 = cv[k] * (tyzp - tyzm);
        A(vr, i, j, k) = (1. - rflagcx * 1.) * h11 + (1. - rflagcy * 1.) * h22 + h33 + (1. - rflagx * 1.) * t11 +
                         (1. - rflagy * 1.) * t22 + t33 + s11 + s33;
        A(vt, i, j, k) = rflagx * 1. * t11 + rflagy * 1. * t22 + rflagcx * 1. * h11 + rflagcy * 1. * h22;
      }
  /* w component (rhs.f:347-428) */
#pragma omp parallel for schedule(static)
  for (int k = g->kbw; k <= g->kew; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ix1; i <= g->ix2; i++) {
        double wxp = (A(wo, i + 1, j, k) + A(wo, i, j, k)) * 0.5;
        double wxm = (A(wo, i, j, k) + A(wo, i - 1, j, k)) * 0.5;
        double wyp = (A(wo, i, j + 1, k) + A(wo, i, j, k)) * 0.5;
        double wym = (A(wo, i, j, k) + A(wo, i, j - 1, k)) * 0.5;
        double wzp = (A(wo, i, j, k + 1) + A(wo, i, j, k)) * 0.5;
        double wzm = (A(wo, i, j, k) + A(wo, i, j, k - 1)) * 0.5;
        double qzp = (A(qr, i, j, k + 1) + A(qr, i, j, k)) * 0.5;
        double qzm = (A(qr, i - 1, j, k + 1) + A(qr, i - 1, j, k)) * 0.5;
        double vzp = (A(vo, i, j, k + 1) + A(vo, i, j, k)) * 0.5;
        double vzm = (A(vo, i, j - 1, k + 1) + A(vo, i, j - 1, k)) * 0.5;
        double dwdxp = au[i] * (A(wo, i + 1, j, k) - A(wo, i, j, k));
        double dwdxm = au[i - 1] * (A(wo, i, j, k) - A(wo, i - 1, j, k));
        double dwdyp = bv[j] * (A(wo, i, j + 1, k) - A(wo, i, j, k));
        double dwdym = bv[j - 1] * (A(wo, i, j, k) - A(wo, i, j - 1, k));
        double dwdzp = cp[k + 1] * (A(wo, i, j, k + 1) - A(wo, i, j, k));
        double dwdzm = cp[k] * (A(wo, i, j, k) - A(wo, i, j, k - 1));
        double dudzp = cw[k] * (A(uo, i, j, k + 1) - A(uo, i, j, k));
        double dudzm = cw[k] * (A(uo, i - 1, j, k + 1) - A(uo, i - 1, j, k));
        double dvdzp = cw[k] * (A(vo, i, j, k + 1) - A(vo, i, j, k));
        double dvdzm = cw[k] * (A(vo, i, j - 1, k + 1) - A(vo, i, j - 1, k));
        double tvip = 0.25 * (A(tv, i, j, k + 1) + A(tv, i, j, k) + A(tv, i + 1, j, k + 1) + A(tv, i + 1, j, k));
        double tvim = 0.25 * (A(tv, i, j, k + 1) + A(tv, i, j, k) + A(tv, i - 1, j, k + 1) + A(tv, i - 1, j, k));
        double tvjp = 0.25 * (A(tv, i, j, k + 1) + A(tv, i, j, k) + A(tv, i, j + 1, k + 1) + A(tv, i, j + 1, k));
        double tvjm = 0.25 * (A(tv, i, j, k + 1) + A(tv, i, j, k) + A(tv, i, j - 1, k + 1) + A(tv, i, j - 1, k));
        double txxp = (ru1 + tvip) * dwdxp;
        double txxm = (ru1 + tvim) * dwdxm;
        double tyyp = (ru1 + tvjp) * dwdyp;
        double tyym = (ru1 + tvjm) * dwdym;
        double tzzp = (ru1 + 2. * A(tv, i, j, k + 1)) * dwdzp;
        double tzzm = (ru1 + 2. * A(tv, i, j, k)) * dwdzm;
        double txzp = tvip * dudzp;
        double txzm = tvim * dudzm;
        double tyzp = tvjp * dvdzp;
        double tyzm = tvjm * dvdzm;
        double h11 = -aw[i] * (qzp * wxp - qzm * wxm);
        double h22 = -bw[j] * (vzp * wyp - vzm * wym);
        double h33 = -cw[k] * (wzp * wzp - wzm * wzm);
        double t11 = aw[i] * (txxp - txxm);
        double t22 = bw[j] * (tyyp - tyym);
        double t33 = cw[k] * (tzzp - tzzm);
        double s11 = aw[i] * (txzp - txzm);
        double s22 = bw[j] * (tyzp - tyzm);
        A(wr, i, j, k) = (1. - rflagcx * 1.) * h11 + (1. - rflagcy * 1.) * h22 + h33 + (1. - rflagx * 1.) * t11 +
                         (1. - rflagy * 1.) * t22 + t33 + s11 + s22;
        A(wt, i, j, k) = rflagx * 1. * t11 + rflagy * 1. * t22 + rflagcx * 1. * h11 + rflagcy * 1. * h22;
      }
}

/* ------------------------------------------------------------------------
 * PREDICTORD: src/timeindeg.f:1041-1265.  Cartesian buoyancy: gravity acts
 * along x (the sin(yc) factor of the cylindrical form is 1, the cos(yv) factor
 * on v is 0).  Sponges: timeindeg.f:1117-1143,1185-1211,1245-1263.
 * ---------------------------------------------------------------------- */
void eo_predictord(eo_state *s, double alfxdt, double gamxdt, double rhoxdt) {
  const eo_grid *g = s->g;
  const eo_params *pr = &s->prm;
  double coef = 0.5 * alfxdt, coefd = alfxdt;
  double *uo = s->uo, *vo = s->vo, *wo = s->wo, *p = s->p, *dens = s->dens;
  double *ua = s->ua, *va = s->va, *wa = s->wa, *ub = s->ub, *vb = s->vb,
         *wb = s->wb, *us = s->us, *vs = s->vs, *ws = s->ws;
  const double *au = g->au, *bv = g->bv, *cw = g->cw;
  int vx1 = pr->vspngx1;
#pragma omp parallel for schedule(static)
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ibu; i <= g->ieu; i++) {
        double ustar = A(uo, i, j, k) + gamxdt * A(ub, i, j, k) + rhoxdt * A(ua, i, j, k) -
                       alfxdt * au[i] * (A(p, i + 1, j, k) - A(p, i, j, k)) + coef * A(us, i, j, k) -
                       alfxdt * pr->dpdx;
        if (pr->idens == 1)
          ustar = ustar - coefd * 0.50 * pr->grav *
                              ((A(dens, i + 1, j, k) - DBG(i + 1, j)) + (A(dens, i, j, k) - DBG(i, j)));
        A(ua, i, j, k) = A(ub, i, j, k);
        A(ub, i, j, k) = A(us, i, j, k);
        A(us, i, j, k) = ustar;
      }
#pragma omp parallel for schedule(static)
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ieu - vx1; i <= g->ieu; i++)
        A(us, i, j, k) = A(us, i, j, k) + g->dfxu[i] * (0. - A(us, i, j, k)) * alfxdt * 1.0;
  if (g->ivspngl == 1) {
#pragma omp parallel for schedule(static)
    for (int k = g->kz1; k <= g->kz2; k++)
      for (int j = g->jy1; j <= g->jy2; j++)
        for (int i = g->ibu; i <= g->ieu; i++)
          A(us, i, j, k) = A(us, i, j, k) + g->dfxul[k] * (0. - A(us, i, j, k)) * alfxdt * 1.0;
  }
#pragma omp parallel for schedule(static)
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jbv; j <= g->jev; j++)
      for (int i = g->ix1; i <= g->ix2; i++) {
        double vstar = A(vo, i, j, k) + gamxdt * A(vb, i, j, k) + rhoxdt * A(va, i, j, k) -
                       alfxdt * bv[j] * (A(p, i, j + 1, k) - A(p, i, j, k)) + coef * A(vs, i, j, k) -
                       alfxdt * pr->dpdy;
        A(va, i, j, k) = A(vb, i, j, k);
        A(vb, i, j, k) = A(vs, i, j, k);
        A(vs, i, j, k) = vstar;
      }
#pragma omp parallel for schedule(static)
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jbv; j <= g->jev; j++)
      for (int i = g->ix2 - vx1; i <= g->ix2; i++)
        A(vs, i, j, k) = A(vs, i, j, k) + g->dfxw[i] * (0. - A(vs, i, j, k)) * alfxdt * 1.0;
  if (g->ivspngl == 1) {
#pragma omp parallel for schedule(static)
    for (int k = g->kz1; k <= g->kz2; k++)
      for (int j = g->jy1; j <= g->jy2; j++)
        for (int i = g->ibu; i <= g->ieu; i++)
          A(vs, i, j, k) = A(vs, i, j, k) + g->dfxwl[k] * (0. - A(vs, i, j, k)) * alfxdt * 1.0;
  }
#pragma omp parallel for schedule(static)
  for (int k = g->kbw; k <= g->kew; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ix1; i <= g->ix2; i++) {
        double wstar = A(wo, i, j, k) + gamxdt * A(wb, i, j, k) + rhoxdt * A(wa, i, j, k) -
                       alfxdt * cw[k] * (A(p, i, j, k + 1) - A(p, i, j, k)) + coef * A(ws, i, j, k) -
                       alfxdt * pr->dpdz;
        A(wa, i, j, k) = A(wb, i, j, k);
        A(wb, i, j, k) = A(ws, i, j, k);
        A(ws, i, j, k) = wstar;
      }
#pragma omp parallel for schedule(static)
  for (int k = g->kbw; k <= g->kew; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ix2 - vx1; i <= g->ix2; i++)
        A(ws, i, j, k) = A(ws, i, j, k) + g->dfxw[i] * (1. - A(ws, i, j, k)) * alfxdt * 1.0;
  if (g->ivspngl == 1) {
#pragma omp parallel for schedule(static)
    for (int k = g->kbw; k <= g->kew; k++)
      for (int j = g->jy1; j <= g->jy2; j++)
        for (int i = g->ix1; i <= g->ix2; i++)
          A(ws, i, j, k) = A(ws, i, j, k) + g->dfxwl[k] * (1. - A(ws, i, j, k)) * alfxdt * 1.0;
  }
}

/* ------------------------------------------------------------------------
 * BOUNDARY: src/boundary.f:7-66 with BOUND050 (:69), BOUND060 (:125),
 * BOUND082 (:372), BOUND500 (:409).  Whole-plane assignments as written.
 * ---------------------------------------------------------------------- */
static void fill_x_plane(const eo_grid *g, double *a, int idst, int isrc, double sgn, int zero) {
  for (int k = 1; k <= NZ; k++)
    for (int j = 1; j <= NY; j++) A(a, idst, j, k) = zero ? 0. : sgn * A(a, isrc, j, k);
}
static void fill_y_plane(const eo_grid *g, double *a, int jdst, int jsrc, double sgn, int zero) {
  for (int k = 1; k <= NZ; k++)
    for (int i = 1; i <= NX; i++) A(a, i, jdst, k) = zero ? 0. : sgn * A(a, i, jsrc, k);
}
static void fill_z_plane(const eo_grid *g, double *a, int kdst, int ksrc, double sgn, int zero) {
  for (int j = 1; j <= NY; j++)
    for (int i = 1; i <= NX; i++) A(a, i, j, kdst) = zero ? 0. : sgn * A(a, i, j, ksrc);
}

void eo_boundary(eo_state *s, double *u, double *v, double *w) {
  const eo_grid *g = s->g;
  const int *it = s->prm.itype;
  for (int ib = 1; ib <= 6; ib++) {
    int t = it[ib];
    if (t == 50 || t == 60) {
      double sg = (t == 50) ? -1. : 1.;
      switch (ib) {
        case 1: fill_x_plane(g, u, g->ib1, 0, 0, 1); fill_x_plane(g, v, g->ib1, g->ix1, sg, 0);
                fill_x_plane(g, w, g->ib1, g->ix1, sg, 0); break;
        case 2: fill_x_plane(g, u, g->ix2, 0, 0, 1); fill_x_plane(g, v, g->ib2, g->ix2, sg, 0);
                fill_x_plane(g, w, g->ib2, g->ix2, sg, 0); break;
        case 3: fill_y_plane(g, u, g->jb1, g->jy1, sg, 0); fill_y_plane(g, v, g->jb1, 0, 0, 1);
                fill_y_plane(g, w, g->jb1, g->jy1, sg, 0); break;
        case 4: fill_y_plane(g, u, g->jb2, g->jy2, sg, 0); fill_y_plane(g, v, g->jy2, 0, 0, 1);
                fill_y_plane(g, w, g->jb2, g->jy2, sg, 0); break;
        case 5: fill_z_plane(g, u, g->kb1, g->kz1, sg, 0); fill_z_plane(g, v, g->kb1, g->kz1, sg, 0);
                fill_z_plane(g, w, g->kb1, 0, 0, 1); break;
        case 6: fill_z_plane(g, u, g->kb2, g->kz2, sg, 0); fill_z_plane(g, v, g->kb2, g->kz2, sg, 0);
                fill_z_plane(g, w, g->kz2, 0, 0, 1); break;
      }
    } else if (t == 82) {
      if (ib == 1) {
        fill_x_plane(g, u, g->ib1, g->ix1, 1., 0); fill_x_plane(g, v, g->ib1, g->ix1, -1., 0);
        fill_x_plane(g, w, g->ib1, g->ix1, -1., 0);
      } else if (ib == 2) {
        fill_x_plane(g, u, g->ib2, g->ix2, 1., 0); fill_x_plane(g, v, g->ib2, g->ix2, 1., 0);
        fill_x_plane(g, w, g->ib2, g->ix2, 1., 0);
      }
    }
  }
  for (int ib = 1; ib <= 3; ib += 2) {
    if (it[ib] != 500) continue;
    if (ib == 1) {
      fill_x_plane(g, u, g->ib1, g->ix2, 1., 0); fill_x_plane(g, v, g->ib1, g->ix2, 1., 0);
      fill_x_plane(g, w, g->ib1, g->ix2, 1., 0);
      fill_x_plane(g, u, g->ib2, g->ix1, 1., 0); fill_x_plane(g, v, g->ib2, g->ix1, 1., 0);
      fill_x_plane(g, w, g->ib2, g->ix1, 1., 0);
    } else {
      fill_y_plane(g, u, g->jb1, g->jy2, 1., 0); fill_y_plane(g, v, g->jb1, g->jy2, 1., 0);
      fill_y_plane(g, w, g->jb1, g->jy2, 1., 0);
      fill_y_plane(g, u, g->jb2, g->jy1, 1., 0); fill_y_plane(g, v, g->jb2, g->jy1, 1., 0);
      fill_y_plane(g, w, g->jb2, g->jy1, 1., 0);
    }
  }
}

/* ------------------------------------------------------------------------
 * BOUNDINOUT: src/boundary.f:505-994, inlet 305 (hybrid plane, :694) and
 * outlets 710/720/730 (:806-958).  x-boundary mass correction (types 80-82)
 * is not part of the restated configurations.
 * ---------------------------------------------------------------------- */
void eo_boundinout(eo_state *s, double *ubc, double *vbc, double *wbc,
                   const double *uof, const double *vof, const double *wof,
                   double alfxdt, int idiv) {
  const eo_grid *g = s->g;
  const int *it = s->prm.itype;
  int iinq = idiv, iouq = idiv;
  double qin1 = 0., qin2 = 0., area = 0., qinxg = 0.;
  if (it[5] == 305) {
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= NX; i++) {
        size_t q = (size_t)(i - 1) + (size_t)NX * (j - 1);
        A(ubc, i, j, g->kb1) = s->planeU[q];
        A(vbc, i, j, g->kb1) = s->planeV[q];
        A(wbc, i, j, g->kb1) = s->planeW[q];
      }
  } else {
    iinq = 0;
  }
  if (iinq == 1) {
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ix1; i <= g->ix2; i++) {
        double areaij = 1.0 / (g->ap[i] * g->bp[j]);
        qin1 = qin1 + A(wbc, i, j, g->kb1) * areaij;
        area = area + areaij;
      }
    qin2 = qin1 / area;
  }
  if (idiv == 1) {
    int t6 = it[6];
    if (t6 == 710) {
      for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++) A(wbc, i, j, g->kz2) = A(wbc, i, j, g->kz2 - 1);
    } else if (t6 == 720) {
      double c = g->cp[g->kz2 - 1] / g->cp[g->kz2];
      for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++)
          A(wbc, i, j, g->kz2) = (1 + c) * A(wbc, i, j, g->kz2 - 1) - c * A(wbc, i, j, g->kz2 - 2);
    } else if (t6 == 730) {
    } else {
      iouq = 0;
    }
    if (iouq == 1) {
      qin1 = qin1 + qinxg;
      if (t6 == 730) {
        double coef = qin2 * alfxdt * g->cp[g->kz2];
        int kz2 = g->kz2;
        for (int j = g->jy1; j <= g->jy2; j++)
          for (int i = g->ix1; i <= g->ix2; i++) {
            A(ubc, i, j, NZ) = A(uof, i, j, NZ) - coef * (A(uof, i, j, NZ) - A(uof, i, j, kz2));
            A(vbc, i, j, NZ) = A(vof, i, j, NZ) - coef * (A(vof, i, j, NZ) - A(vof, i, j, kz2));
            A(wbc, i, j, kz2) = A(wof, i, j, kz2) - coef * (A(wof, i, j, kz2) - A(wof, i, j, kz2 - 1));
          }
        fill_y_plane(g, ubc, 1, NY - 1, 1., 0); fill_y_plane(g, ubc, NY, 2, 1., 0);
        fill_y_plane(g, vbc, 1, NY - 1, 1., 0); fill_y_plane(g, vbc, NY, 2, 1., 0);
        fill_y_plane(g, wbc, 1, NY - 1, 1., 0); fill_y_plane(g, wbc, NY, 2, 1., 0);
      }
      double a2 = 0., qout = 0.;
      for (int j = g->jy1; j <= g->jy2; j++)
        for (int i = g->ix1; i <= g->ix2; i++) {
          double areaij = 1.0 / (g->ap[i] * g->bp[j]);
          qout = qout + A(wbc, i, j, g->kz2) * areaij;
          a2 = a2 + areaij;
        }
      s->qin_last = qin1;
      s->qout_last = qout;
      if (qout != 0.) {
        double c = qin1 / qout;
        for (int j = g->jy1; j <= g->jy2; j++)
          for (int i = g->ix1; i <= g->ix2; i++) A(wbc, i, j, g->kz2) = A(wbc, i, j, g->kz2) * c;
      } else {
        for (int j = g->jy1; j <= g->jy2; j++)
          for (int i = g->ix1; i <= g->ix2; i++) A(wbc, i, j, g->kz2) = qin1 / a2;
      }
    }
  } else {
    int t6 = it[6];
    if (t6 == 710) {
      for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++) {
          A(ubc, i, j, NZ) = A(uof, i, j, g->kz2);
          A(vbc, i, j, NZ) = A(vof, i, j, g->kz2);
          A(wbc, i, j, g->kz2) = A(wof, i, j, g->kz2);
        }
    } else if (t6 == 720) {
      double c = g->cw[g->kz2 - 1] / g->cw[g->kz2];
      for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++) {
          A(ubc, i, j, NZ) = (1 + c) * A(uof, i, j, g->kz2) - c * A(uof, i, j, g->kz2 - 1);
          A(vbc, i, j, NZ) = (1 + c) * A(vof, i, j, g->kz2) - c * A(vof, i, j, g->kz2 - 1);
          A(wbc, i, j, g->kz2) = A(wof, i, j, g->kz2);
        }
    } else if (t6 == 730 || t6 == 731) {
      for (int j = 1; j <= NY; j++)
        for (int i = 1; i <= NX; i++) {
          A(ubc, i, j, NZ) = A(uof, i, j, NZ);
          A(vbc, i, j, NZ) = A(vof, i, j, NZ);
          A(wbc, i, j, g->kz2) = A(wof, i, j, g->kz2);
        }
    }
  }
}

/* DIVERGENCE: src/timeindeg.f:908-977 (rp=ru=1) */
void eo_divergence(eo_state *s, const double *us, const double *vs, const double *ws, double *div) {
  const eo_grid *g = s->g;
#pragma omp parallel for schedule(static)
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ix1; i <= g->ix2; i++)
        A(div, i, j, k) = (g->ap[i] * (A(us, i, j, k) - A(us, i - 1, j, k)) +
                           g->bp[j] * (A(vs, i, j, k) - A(vs, i, j - 1, k)) +
                           g->cp[k] * (A(ws, i, j, k) - A(ws, i, j, k - 1)));
}

/* CORRECT: src/timeindeg.f:981-1028: (us,vs,ws,dp) -> (uo,vo,wo) */
void eo_correct(eo_state *s, double alfxdt) {
  s->alfxdt_last = alfxdt;
  const eo_grid *g = s->g;
  double *uo = s->uo, *vo = s->vo, *wo = s->wo, *us = s->us, *vs = s->vs, *ws = s->ws, *dp = s->dp;
#pragma omp parallel for schedule(static)
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ibu; i <= g->ieu; i++)
        A(uo, i, j, k) = A(us, i, j, k) - g->au[i] * (A(dp, i + 1, j, k) - A(dp, i, j, k)) * alfxdt;
#pragma omp parallel for schedule(static)
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jbv; j <= g->jev; j++)
      for (int i = g->ix1; i <= g->ix2; i++)
        A(vo, i, j, k) = A(vs, i, j, k) - g->bv[j] * (A(dp, i, j + 1, k) - A(dp, i, j, k)) * alfxdt;
#pragma omp parallel for schedule(static)
  for (int k = g->kbw; k <= g->kew; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ix1; i <= g->ix2; i++)
        A(wo, i, j, k) = A(ws, i, j, k) - g->cw[k] * (A(dp, i, j, k + 1) - A(dp, i, j, k)) * alfxdt;
}

/* Pressure update, reference value and ghost fills: src/Eddy6.f:2772-2853
 * followed by :2911-2953 (explicit scheme, ibm=0). */
void eo_pressure_update(eo_state *s) {
  const eo_grid *g = s->g;
  const int *it = s->prm.itype;
  double *p = s->p, *dp = s->dp;
  for (long q = 0; q < s->ncell; q++) p[q] = p[q] + dp[q];
  /* implicit y terms: the extra pressure correction (src/Eddy6.f:2775-2785;
   * rp = 1, RVIMPLY = 1); every right-hand value is the pre-update P */
  if (s->prm.imply == 1) {
    const double c = 0.5 * s->alfxdt_last * s->prm.ru1 / ((g->dely * 1.0) * (g->dely * 1.0));
#pragma omp parallel for schedule(static)
    for (int k = 2; k <= g->kz2; k++)
      for (int j = 2; j <= g->jy2; j++)
        for (int i = 2; i <= g->ix2; i++)
          A(p, i, j, k) = A(p, i, j, k) -
                          c * ((A(dp, i, j - 1, k) - 2. * A(dp, i, j, k)) + A(dp, i, j + 1, k)) * 1.0;
  }
  /* implicit x terms (src/Eddy6.f:2787-2795; rp = ru = 1, RVIMPLX = 1) */
  if (s->prm.implx == 1) {
    const double c = 0.5 * s->alfxdt_last * s->prm.ru1;
#pragma omp parallel for schedule(static)
    for (int k = 2; k <= g->kz2; k++)
      for (int j = 2; j <= g->jy2; j++)
        for (int i = 2; i <= g->ix2; i++)
          A(p, i, j, k) = A(p, i, j, k) - c * g->ap[i] / 1.0 *
                                              ((A(dp, i + 1, j, k) - A(dp, i, j, k)) * g->au[i] * 1.0 -
                                               (A(dp, i, j, k) - A(dp, i - 1, j, k)) * g->au[i - 1] * 1.0) *
                                              1.0;
  }
  double pref = 0.;
  for (int j = g->jy1; j <= g->jy2; j++) pref += A(p, g->ix1, j, 2);
  pref = pref / (double)(NY - 2);
  s->pref_last = pref;
  for (long q = 0; q < s->ncell; q++) p[q] = p[q] - pref;
  /* immersed body: pressure at the pressure forcing points and inside
   * (correctpres_mod2 + presinterior, :2881-2897; their effect on the ghost
   * planes is recomputed by the passes below) */
  if (s->ib) {
    eo_ib_force(s->ib, 3, p, 0.0);
    eo_ib_interior(s->ib, 4, p, 0.0);
  }
  /* first ghost pass (:2814-2853) */
  if (g->mp == 0) { fill_x_plane(g, p, 1, g->ix2, 1., 0); fill_x_plane(g, p, NX, g->ix1, 1., 0); }
  else { fill_x_plane(g, p, 1, g->ix1, -1., 0); fill_x_plane(g, p, NX, g->ix2, -1., 0); }
  if (g->lp == 0) { fill_y_plane(g, p, 1, g->jy2, 1., 0); fill_y_plane(g, p, NY, g->jy1, 1., 0); }
  else { fill_y_plane(g, p, 1, g->jy1, 1., 0); fill_y_plane(g, p, NY, g->jy2, 1., 0); }
  if (it[5] == 500) fill_z_plane(g, p, 1, g->kz2, 1., 0);
  if (it[6] == 500) fill_z_plane(g, p, NZ, g->kz1, 1., 0);
  if (it[5] != 0 && it[5] != 500) fill_z_plane(g, p, 1, g->kz1, 1., 0);
  if (it[6] != 0 && it[6] != 500) fill_z_plane(g, p, NZ, g->kz2, 1., 0);
  /* second ghost pass (:2911-2953) */
  if (it[5] != 0 && it[5] != 500) fill_z_plane(g, p, 1, g->kz1, 1., 0);
  if (it[6] != 0 && it[6] != 500) fill_z_plane(g, p, NZ, g->kz2, 1., 0);
  if (g->mp == 0) { fill_x_plane(g, p, 1, g->ix2, 1., 0); fill_x_plane(g, p, NX, g->ix1, 1., 0); }
  else { fill_x_plane(g, p, 1, g->ix1, 1., 0); fill_x_plane(g, p, NX, g->ix2, 1., 0); }
  if (g->lp == 0) { fill_y_plane(g, p, 1, g->jy2, 1., 0); fill_y_plane(g, p, NY, g->jy1, 1., 0); }
  else { fill_y_plane(g, p, 1, g->jy1, 1., 0); fill_y_plane(g, p, NY, g->jy2, 1., 0); }
}

/* RHS_DENSITY: src/rhs_density.f:4-175 (rr -> rhb, rt -> rs: the explicit
 * part and the C.N. part, the y diffusion when IMPLY = 1) */
void eo_rhs_density(eo_state *s) {
  const eo_grid *g = s->g;
  double *uo = s->uo, *vo = s->vo, *wo = s->wo, *dens = s->dens, *kv = s->tv;
  double *rr = s->rhb, *rt = s->rs;
  double repr1 = s->prm.ru1 / s->prm.prn;
  const double rflagx = (double)s->prm.implx, rflagcx = (double)s->prm.implcx, rflagy = (double)s->prm.imply,
               rflagcy = (double)s->prm.implcy;
  memset(rr, 0, sizeof(double) * (size_t)s->ncell);
#pragma omp parallel for schedule(static)
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ix1; i <= g->ix2; i++) {
        double qxp = A(uo, i, j, k), qxm = A(uo, i - 1, j, k);
        double rxp = (A(dens, i + 1, j, k) + A(dens, i, j, k)) * 0.5;
        double rxm = (A(dens, i, j, k) + A(dens, i - 1, j, k)) * 0.5;
        double vyp = A(vo, i, j, k), vym = A(vo, i, j - 1, k);
        double ryp = (A(dens, i, j + 1, k) + A(dens, i, j, k)) * 0.5;
        double rym = (A(dens, i, j, k) + A(dens, i, j - 1, k)) * 0.5;
        double wzp = A(wo, i, j, k), wzm = A(wo, i, j, k - 1);
        double rzp = (A(dens, i, j, k + 1) + A(dens, i, j, k)) * 0.5;
        double rzm = (A(dens, i, j, k) + A(dens, i, j, k - 1)) * 0.5;
        double drdxp = g->au[i] * (A(dens, i + 1, j, k) - A(dens, i, j, k));
        double drdxm = g->au[i - 1] * (A(dens, i, j, k) - A(dens, i - 1, j, k));
        double drdyp = g->bv[j] * (A(dens, i, j + 1, k) - A(dens, i, j, k));
        double drdym = g->bv[j - 1] * (A(dens, i, j, k) - A(dens, i, j - 1, k));
        double drdzp = g->cw[k] * (A(dens, i, j, k + 1) - A(dens, i, j, k));
        double drdzm = g->cw[k - 1] * (A(dens, i, j, k) - A(dens, i, j, k - 1));
        double kvip = 0.5 * (A(kv, i + 1, j, k) + A(kv, i, j, k));
        double kvim = 0.5 * (A(kv, i - 1, j, k) + A(kv, i, j, k));
        double kvjp = 0.5 * (A(kv, i, j + 1, k) + A(kv, i, j, k));
        double kvjm = 0.5 * (A(kv, i, j - 1, k) + A(kv, i, j, k));
        double kvkp = 0.5 * (A(kv, i, j, k + 1) + A(kv, i, j, k));
        double kvkm = 0.5 * (A(kv, i, j, k - 1) + A(kv, i, j, k));
        double txxp = (repr1 + kvip) * drdxp;
        double txxm = (repr1 + kvim) * drdxm;
        double tyyp = (repr1 + kvjp) * drdyp;
        double tyym = (repr1 + kvjm) * drdym;
        double tzzp = (repr1 + kvkp) * drdzp;
        double tzzm = (repr1 + kvkm) * drdzm;
        double h11 = -g->ap[i] * (rxp * qxp - rxm * qxm);
        double h22 = -g->bp[j] * (ryp * vyp - rym * vym);
        double h33 = -g->cp[k] * (rzp * wzp - rzm * wzm);
        double t11 = g->ap[i] * (txxp - txxm);
        double t22 = g->bp[j] * (tyyp - tyym);
        double t33 = g->cp[k] * (tzzp - tzzm);
        A(rr, i, j, k) = (1. - rflagcx * 1.) * h11 + (1. - rflagcy * 1.) * h22 + h33 + (1. - rflagx * 1.) * t11 +
                         (1. - rflagy * 1.) * t22 + t33;
        A(rt, i, j, k) = rflagx * 1. * t11 + rflagy * 1. * t22 + rflagcx * 1. * h11 + rflagcy * 1. * h22;
      }
}

/* BOUNDARY_DENS: src/boundary.f:2001-2197 (types 50, 82, 500) */
void eo_boundary_dens(eo_state *s, double *d) {
  const eo_grid *g = s->g;
  const int *it = s->prm.itype;
  for (int ib = 1; ib <= 6; ib++) {
    int t = it[ib];
    if (t == 50) {
      if (ib == 1) for (int k = 1; k <= NZ; k++) for (int j = 1; j <= NY; j++)
            A(d, g->ib1, j, k) = 2.0 * (0.5) - A(d, g->ib1 + 1, j, k);
      if (ib == 2) for (int k = 1; k <= NZ; k++) for (int j = 1; j <= NY; j++)
            A(d, g->ib2, j, k) = 2.0 * (-0.5) - A(d, g->ib2 - 1, j, k);
    } else if (t == 80 || t == 82) {
      if (ib == 1) fill_x_plane(g, d, g->ib1, g->ix1, 1., 0);
      if (ib == 2) {
        /* cylindrical background-gradient term vanishes for rp = 1 */
        fill_x_plane(g, d, g->ix2, g->ix2 - 1, 1., 0);
        fill_x_plane(g, d, g->ib2, g->ix2, 1., 0);
      }
    }
  }
  for (int ib = 1; ib <= 5; ib += 2) {
    if (it[ib] != 500) continue;
    if (ib == 1) { fill_x_plane(g, d, g->ib1, g->ix2, 1., 0); fill_x_plane(g, d, g->ib2, g->ix1, 1., 0); }
    if (ib == 3) { fill_y_plane(g, d, g->jb1, g->jy2, 1., 0); fill_y_plane(g, d, g->jb2, g->jy1, 1., 0); }
    if (ib == 5) { fill_z_plane(g, d, g->kb1, g->kz2, 1., 0); fill_z_plane(g, d, g->kb2, g->kz1, 1., 0); }
  }
}

/* BOUNDINOUTD: src/boundary.f:2241-2281 */
void eo_boundinoutd(eo_state *s, double *d) {
  const eo_grid *g = s->g;
  const int *it = s->prm.itype;
  if (it[5] == 305) {
    for (int j = 1; j <= NY; j++)
      for (int i = 1; i <= NX; i++) A(d, i, j, g->kb1) = s->planeD[(size_t)(i - 1) + (size_t)NX * (j - 1)];
    fill_z_plane(g, d, 2, 1, 1., 0);
  }
  if (it[6] == 730) {
    fill_z_plane(g, d, g->kz2, g->kz2 - 1, 1., 0);
    fill_z_plane(g, d, NZ, g->kz2, 1., 0);
  }
  if (it[6] == 710) fill_z_plane(g, d, g->kz2, g->kz2 - 1, 1., 0);
}

/* DENSITY: src/density.f:6-127 (INVERSEYD with IMPLY = 1, INVERSEXD with
 * IMPLX = 1) */
void eo_density(eo_state *s, double alfxdt, double gamxdt, double rhoxdt) {
  const eo_grid *g = s->g;
  double *dens = s->dens, *rha = s->rha, *rhb = s->rhb, *rs = s->rs;
  double coef = 0.5 * alfxdt;
#pragma omp parallel for schedule(static)
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ix1; i <= g->ix2; i++) {
        A(dens, i, j, k) = A(dens, i, j, k) + gamxdt * A(rhb, i, j, k) + rhoxdt * A(rha, i, j, k) +
                           coef * A(rs, i, j, k);
        A(rha, i, j, k) = A(rhb, i, j, k);
        A(rhb, i, j, k) = A(rs, i, j, k);
        A(rs, i, j, k) = A(dens, i, j, k);
      }
  for (long q = 0; q < s->ncell; q++) rhb[q] = rs[q] + 0.5 * alfxdt * rhb[q];
  eo_boundary_dens(s, rhb);
  /* implicit y diffusion, then the whole array is copied (density.f:96-100):
   * ghost cells take RS's, which nothing above writes but BOUNDARY_DENS */
  if (s->prm.imply == 1 && s->prm.implcy == 1) {
    eo_inverseyd_new(s, alfxdt);
    memcpy(dens, rs, sizeof(double) * (size_t)s->ncell);
  } else if (s->prm.imply == 1) {
    eo_inverseyd(s, alfxdt);
    memcpy(dens, rs, sizeof(double) * (size_t)s->ncell);
  }
  /* implicit x diffusion (density.f:101-104) */
  if (s->prm.implx == 1 || s->prm.implcx == 1) {
    eo_inversexd(s, alfxdt);
    memcpy(dens, rs, sizeof(double) * (size_t)s->ncell);
  }
  if (g->idspngl == 1) {
#pragma omp parallel for schedule(static)
    for (int k = g->kz1; k <= g->kz2; k++)
      for (int j = g->jy1; j <= g->jy2; j++)
        for (int i = g->ix1; i <= g->ix2; i++)
          A(dens, i, j, k) = A(dens, i, j, k) + g->dfxdl[k] * (DBG(i, j) - A(dens, i, j, k)) * alfxdt * 1.0;
  }
#pragma omp parallel for schedule(static)
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ix2 - s->prm.dspngx1; i <= g->ix2; i++)
        A(dens, i, j, k) = A(dens, i, j, k) + g->dfxd[i] * (DBG(i, j) - A(dens, i, j, k)) * alfxdt * 1.0;
}


/* ---- Crank-Nicolson y lines ----
 * cyclic: the Sherman-Morrison treatment of the two corner entries on top of
 * the Thomas elimination (the published method of src/numrec.f:754-800),
 * with its operation order: gamma = -b1, b1' = b1 - gamma,
 * bn' = bn - alpha*beta/gamma; solve A' x = r and A' z = (gamma,0..0,alpha);
 * x -= z (x1 + beta xn / gamma) / (1 + z1 + beta zn / gamma). */
static void thomas(const double *a, const double *b, const double *c, const double *r, double *u, int n,
                   double *gam) {
  double bet = b[0];
  u[0] = r[0] / bet;
  for (int j = 1; j < n; j++) {
    gam[j] = c[j - 1] / bet;
    bet = b[j] - a[j] * gam[j];
    u[j] = (r[j] - a[j] * u[j - 1]) / bet;
  }
  for (int j = n - 2; j >= 0; j--) u[j] = u[j] - gam[j + 1] * u[j + 1];
}

void eo_cyclic(const double *a, const double *b, const double *c, double alpha, double beta, const double *r,
               double *x, int n, double *work) {
  double *bb = work, *u = work + n, *z = work + 2 * n, *gam = work + 3 * n;
  const double gamma = -b[0];
  bb[0] = b[0] - gamma;
  bb[n - 1] = b[n - 1] - alpha * beta / gamma;
  for (int i = 1; i < n - 1; i++) bb[i] = b[i];
  thomas(a, bb, c, r, x, n, gam);
  u[0] = gamma;
  u[n - 1] = alpha;
  for (int i = 1; i < n - 1; i++) u[i] = 0.;
  thomas(a, bb, c, u, z, n, gam);
  const double fact = (x[0] + beta * x[n - 1] / gamma) / (1. + z[0] + beta * z[n - 1] / gamma);
  for (int i = 0; i < n; i++) x[i] = x[i] - fact * z[i];
}

/* INVERSEY (src/timeindeg.f:120-340), Cartesian (rp = ru = 1), IMPLYDCMP = 0:
 * v lines for i in [2, NX-1], w lines for i in [2, NX-1] and k in [kbw, kew],
 * u lines for i in [2, NX-2]; j periodic over [jy1, jy2].  rflagy = IMPLY
 * scales the viscous coefficients, rflagcy = IMPLCY the convective ones: the
 * v lines linearise about VO (and take the explicit half back on the right-
 * hand side), the w and u lines about the provisional VS the v lines just
 * produced.  REFRESHBC is a no-op on one rank with non-periodic z. */
void eo_inversey(eo_state *s, double alfxdt) {
  const eo_grid *g = s->g;
  const double coef = 0.5 * alfxdt, ru1 = s->prm.ru1;
  const double rflagy = (double)s->prm.imply, rflagcy = (double)s->prm.implcy;
  const int n = g->jy2 - 1;
  double *us = s->us, *vs = s->vs, *ws = s->ws;
  const double *tv = s->tv, *vo = s->vo;
  const double *bp = g->bp, *bu = g->bu, *bv = g->bv, *bw = g->bw;
#pragma omp parallel
  {
    double *ay = malloc(sizeof(double) * n), *by = malloc(sizeof(double) * n), *cy = malloc(sizeof(double) * n),
           *ry = malloc(sizeof(double) * n), *x = malloc(sizeof(double) * n), *wk = malloc(sizeof(double) * 4 * n);
    /* v */
#pragma omp for schedule(static) collapse(2)
    for (int k = g->kz1; k <= g->kz2; k++)
      for (int i = 2; i <= NX - 1; i++) {
        for (int j = g->jbv; j <= g->jev; j++) {
          const int jj = j - 2;
          const double tvjp = 2. * A(tv, i, j + 1, k) + ru1, tvjm = 2. * A(tv, i, j, k) + ru1;
          ry[jj] = A(vs, i, j, k);
          double coefy = rflagy * coef * bv[j] / (1.0 * 1.0);
          const double ayv = -coefy * bp[j] * tvjm, cyv = -coefy * bp[j + 1] * tvjp, byv = -ayv - cyv;
          coefy = rflagcy * coef * bv[j] / 1.0;
          const double ayc = -0.25 * coefy * (A(vo, i, j - 1, k) + A(vo, i, j, k)) * 2.0;
          const double cyc = 0.25 * coefy * (A(vo, i, j + 1, k) + A(vo, i, j, k)) * 2.0;
          const double byc = ayc + cyc;
          ay[jj] = ayv + ayc;
          cy[jj] = cyv + cyc;
          by[jj] = 1.0 + byv + byc;
          const double vyp = (A(vo, i, j + 1, k) + A(vo, i, j, k)) * 0.5;
          const double vym = (A(vo, i, j, k) + A(vo, i, j - 1, k)) * 0.5;
          ry[jj] = ry[jj] + coefy * (vyp * vyp - vym * vym);
        }
        eo_cyclic(ay, by, cy, cy[n - 1], ay[0], ry, x, n, wk);
        for (int j = g->jbv; j <= g->jev; j++) A(vs, i, j, k) = x[j - 2];
      }
    /* w */
#pragma omp for schedule(static) collapse(2)
    for (int k = g->kbw; k <= g->kew; k++)
      for (int i = 2; i <= NX - 1; i++) {
        for (int j = g->jy1; j <= g->jy2; j++) {
          const int jj = j - 2;
          const double tvjp =
              0.25 * (A(tv, i, j, k + 1) + A(tv, i, j, k) + A(tv, i, j + 1, k + 1) + A(tv, i, j + 1, k)) + ru1;
          const double tvjm =
              0.25 * (A(tv, i, j, k + 1) + A(tv, i, j, k) + A(tv, i, j - 1, k + 1) + A(tv, i, j - 1, k)) + ru1;
          ry[jj] = A(ws, i, j, k);
          double coefy = rflagy * coef * bw[j] / (1.0 * 1.0);
          const double ayv = -coefy * bv[j - 1] * tvjm, cyv = -coefy * bv[j] * tvjp, byv = -ayv - cyv;
          const double vzp = (A(vs, i, j, k + 1) + A(vs, i, j, k)) * 0.5;
          const double vzm = (A(vs, i, j - 1, k + 1) + A(vs, i, j - 1, k)) * 0.5;
          coefy = rflagcy * 0.5 * coef * bw[j] / 1.0;
          const double ayc = -coefy * vzm, cyc = coefy * vzp, byc = ayc + cyc;
          ay[jj] = ayv + ayc;
          cy[jj] = cyv + cyc;
          by[jj] = 1.0 + byv + byc;
        }
        eo_cyclic(ay, by, cy, cy[n - 1], ay[0], ry, x, n, wk);
        for (int j = g->jy1; j <= g->jy2; j++) A(ws, i, j, k) = x[j - 2];
      }
    /* u */
#pragma omp for schedule(static) collapse(2)
    for (int k = g->kz1; k <= g->kz2; k++)
      for (int i = 2; i <= NX - 2; i++) {
        for (int j = g->jy1; j <= g->jy2; j++) {
          const int jj = j - 2;
          const double tvjp =
              0.25 * (A(tv, i + 1, j, k) + A(tv, i, j, k) + A(tv, i + 1, j + 1, k) + A(tv, i, j + 1, k)) + ru1;
          const double tvjm =
              0.25 * (A(tv, i + 1, j, k) + A(tv, i, j, k) + A(tv, i + 1, j - 1, k) + A(tv, i, j - 1, k)) + ru1;
          ry[jj] = A(us, i, j, k);
          double coefy = rflagy * coef * bu[j] / (1.0 * 1.0);
          const double ayv = -coefy * bv[j - 1] * tvjm, cyv = -coefy * bv[j] * tvjp, byv = -ayv - cyv;
          const double vxp = (A(vs, i + 1, j, k) + A(vs, i, j, k)) * 0.5;
          const double vxm = (A(vs, i + 1, j - 1, k) + A(vs, i, j - 1, k)) * 0.5;
          coefy = rflagcy * 0.5 * coef * bu[j] / 1.0;
          const double ayc = -coefy * vxm, cyc = coefy * vxp, byc = ayc + cyc;
          ay[jj] = ayv + ayc;
          cy[jj] = cyv + cyc;
          by[jj] = 1.0 + byv + byc;
        }
        eo_cyclic(ay, by, cy, cy[n - 1], ay[0], ry, x, n, wk);
        for (int j = g->jy1; j <= g->jy2; j++) A(us, i, j, k) = x[j - 2];
      }
    free(ay); free(by); free(cy); free(ry); free(x); free(wk);
  }
}

/* INVERSEYD_NEW (src/density.f:290-380), IMPLY = IMPLCY = 1: the y diffusion
 * with the face diffusivities 0.5 (tv(j) + tv(j+/-1)) + ru1/prn and the
 * convection by VO, k in [kbw, kew], i in [2, NX-1] */
void eo_inverseyd_new(eo_state *s, double alfxdt) {
  const eo_grid *g = s->g;
  const double coef = 0.5 * alfxdt, kmol = s->prm.ru1 / s->prm.prn;
  const double rflagy = (double)s->prm.imply, rflagcy = (double)s->prm.implcy;
  const int n = g->jy2 - 1;
  double *rs = s->rs;
  const double *tv = s->tv, *vo = s->vo, *bp = g->bp, *bv = g->bv;
#pragma omp parallel
  {
    double *ay = malloc(sizeof(double) * n), *by = malloc(sizeof(double) * n), *cy = malloc(sizeof(double) * n),
           *ry = malloc(sizeof(double) * n), *x = malloc(sizeof(double) * n), *wk = malloc(sizeof(double) * 4 * n);
#pragma omp for schedule(static) collapse(2)
    for (int k = g->kbw; k <= g->kew; k++)
      for (int i = 2; i <= NX - 1; i++) {
        for (int j = g->jy1; j <= g->jy2; j++) {
          const int jj = j - 2;
          const double tvjp = 0.5 * (A(tv, i, j, k) + A(tv, i, j + 1, k)) + kmol;
          const double tvjm = 0.5 * (A(tv, i, j, k) + A(tv, i, j - 1, k)) + kmol;
          ry[jj] = A(rs, i, j, k);
          double coefy = rflagy * coef * bp[j] / (1.0 * 1.0);
          const double ayv = -coefy * bv[j - 1] * tvjm, cyv = -coefy * bv[j] * tvjp, byv = -ayv - cyv;
          const double vzp = A(vo, i, j, k), vzm = A(vo, i, j - 1, k);
          coefy = rflagcy * 0.5 * coef * bp[j] / 1.0;
          const double ayc = -coefy * vzm, cyc = coefy * vzp, byc = ayc + cyc;
          ay[jj] = ayv + ayc;
          cy[jj] = cyv + cyc;
          by[jj] = 1.0 + byv + byc;
        }
        eo_cyclic(ay, by, cy, cy[n - 1], ay[0], ry, x, n, wk);
        for (int j = g->jy1; j <= g->jy2; j++) A(rs, i, j, k) = x[j - 2];
      }
    free(ay); free(by); free(cy); free(ry); free(x); free(wk);
  }
}

/* INVERSEYD (src/density.f:383-460) on RS: k in [kbw, kew], i in [2, NX-1],
 * and, as there, the same face diffusivity 0.5(tv(j) + tv(j+1)) + ru1/prn on
 * both sides of a cell */
void eo_inverseyd(eo_state *s, double alfxdt) {
  const eo_grid *g = s->g;
  const double coef = 0.5 * alfxdt, rflagy = 1.0, kmol = s->prm.ru1 / s->prm.prn;
  const int n = g->jy2 - 1;
  double *rs = s->rs;
  const double *tv = s->tv, *bp = g->bp;
#pragma omp parallel
  {
    double *ay = malloc(sizeof(double) * n), *by = malloc(sizeof(double) * n), *cy = malloc(sizeof(double) * n),
           *ry = malloc(sizeof(double) * n), *x = malloc(sizeof(double) * n), *wk = malloc(sizeof(double) * 4 * n);
#pragma omp for schedule(static) collapse(2)
    for (int k = g->kbw; k <= g->kew; k++)
      for (int i = 2; i <= NX - 1; i++) {
        for (int j = g->jy1; j <= g->jy2; j++) {
          const int jj = j - 2;
          const double tvjp = 0.5 * (A(tv, i, j, k) + A(tv, i, j + 1, k)) + kmol;
          const double tvjm = 0.5 * (A(tv, i, j, k) + A(tv, i, j + 1, k)) + kmol;
          ry[jj] = A(rs, i, j, k);
          const double coefy = rflagy * coef * bp[j] / (1.0 * 1.0);
          const double ayv = -coefy * bp[j - 1] * tvjm, cyv = -coefy * bp[j] * tvjp, byv = -ayv - cyv;
          ay[jj] = ayv;
          cy[jj] = cyv;
          by[jj] = 1.0 + byv;
        }
        eo_cyclic(ay, by, cy, cy[n - 1], ay[0], ry, x, n, wk);
        for (int j = g->jy1; j <= g->jy2; j++) A(rs, i, j, k) = x[j - 2];
      }
    free(ay); free(by); free(cy); free(ry); free(x); free(wk);
  }
}

/* ---- Crank-Nicolson x lines ----
 * Boundary tables of INVERSEX / INVERSEXD (src/timeindeg.f:370-434,
 * src/density.f:150-204) for the one implicit region of IMPLXDCMP = 0
 * (i1 = 2 = IBU, i2 = NX-1 = IX2, src/inpall.f:703-709) and non-periodic x:
 * rdir = 0 on both sides; u takes its wall value from UB (rperb = 1); v and w
 * (and the density, on w's row) are Dirichlet (rdirb 2, bdirb -1) where
 * IBC = 1 and Neumann (rdirb 0, bdirb 1) otherwise, IBC as src/setup.f:18-49
 * sets it from ITYPE.  Index [q][side], q = 0 u, 1 v, 2 w. */
typedef struct {
  double rdir[3][2], rperb[3][2], rdirb[3][2], bdirb[3][2], bneub[3][2];
} xbc_tables;

static int ibc_of(int itype, int side, int q) {
  if (side == 0) {
    if (itype == 50 || itype == 300) return 1;
    if (itype == 60) return q == 0 ? 1 : -1;
    if (itype == 81) return q == 1 ? -1 : 1;
    return 1;
  }
  if (itype == 50) return 1;
  if (itype == 60 || itype == 80) return q == 0 ? 1 : -1;
  if (itype == 81) return q == 1 ? -1 : 1;
  return 1;
}

static void x_tables(const eo_state *s, xbc_tables *t) {
  for (int q = 0; q < 3; q++)
    for (int sd = 0; sd < 2; sd++) {
      t->rdir[q][sd] = 0.;
      t->rperb[q][sd] = q == 0 ? 1. : 0.;
      t->bneub[q][sd] = 0.;
      if (q == 0) {
        t->rdirb[q][sd] = 0.;
        t->bdirb[q][sd] = 0.;
      } else if (ibc_of(s->prm.itype[1 + sd], sd, q) == 1) {
        t->rdirb[q][sd] = 2.;
        t->bdirb[q][sd] = -1.;
      } else {
        t->rdirb[q][sd] = 0.;
        t->bdirb[q][sd] = 1.;
      }
    }
}

/* the boundary planes of UB, VB, WB before the x lines, IBM = 0
 * (src/Eddy6.f:2582-2591): UB(IX1) = US(IX1) + alfxdt/2 UB(IX1), the same at
 * IX2 and for v, w, then BOUNDARY twice; UB.. hold the C.N. parts of RHS */
void eo_inversex_walls(eo_state *s, double alfxdt) {
  const eo_grid *g = s->g;
  double *b[3] = {s->ub, s->vb, s->wb};
  const double *st[3] = {s->us, s->vs, s->ws};
  const int is[2] = {g->ix1, g->ix2};
  for (int q = 0; q < 3; q++)
    for (int e = 0; e < 2; e++)
      for (int k = 1; k <= NZ; k++)
        for (int j = 1; j <= NY; j++) A(b[q], is[e], j, k) = A(st[q], is[e], j, k) + 0.5 * alfxdt * A(b[q], is[e], j, k);
  eo_boundary(s, s->ub, s->vb, s->wb);
  eo_boundary(s, s->ub, s->vb, s->wb);
}

/* INVERSEX (src/timeindeg.f:344-690), Cartesian (rp = ru = 1), rflagx =
 * IMPLX and rflagcx = IMPLCX (the u lines linearised about UO, with the
 * explicit flux back on the right-hand side; the v and w lines about the
 * provisional US), IMPLXDCMP = 0: u lines for i in [2, NX-2], then
 * v lines (j in [jbv, jev]) and w lines (k in [kbw, kew]) for i in [2, NX-1];
 * tridag (src/numrec.f:783-802) on each.  REFRESHBC is a no-op on one rank
 * with non-periodic z. */
void eo_inversex(eo_state *s, double alfxdt) {
  const eo_grid *g = s->g;
  const double coef = 0.5 * alfxdt, ru1 = s->prm.ru1;
  const double rflagx = (double)s->prm.implx, rflagcx = (double)s->prm.implcx;
  double *us = s->us, *vs = s->vs, *ws = s->ws;
  const double *ub = s->ub, *vb = s->vb, *wb = s->wb, *tv = s->tv, *uo = s->uo;
  const double *ap = g->ap, *au = g->au, *av = g->av, *aw = g->aw;
  xbc_tables t;
  x_tables(s, &t);
  const int nmax = NX;
#pragma omp parallel
  {
    double *ax = malloc(sizeof(double) * nmax), *bx = malloc(sizeof(double) * nmax),
           *cx = malloc(sizeof(double) * nmax), *rx = malloc(sizeof(double) * nmax),
           *x = malloc(sizeof(double) * nmax), *gam = malloc(sizeof(double) * nmax);
    /* u */
#pragma omp for schedule(static) collapse(2)
    for (int k = g->kz1; k <= g->kz2; k++)
      for (int j = g->jy1; j <= g->jy2; j++) {
        const int i1 = 2, i2 = NX - 2, n = i2 - i1 + 1;
        for (int i = i1; i <= i2; i++) {
          const int ii = i - i1;
          const double tvip = 2. * A(tv, i + 1, j, k) + ru1, tvim = 2. * A(tv, i, j, k) + ru1;
          rx[ii] = A(us, i, j, k);
          double coefx = rflagx * coef * au[i];
          const double axv = -coefx * ap[i] * tvim, cxv = -coefx * ap[i + 1] * tvip, bxv = -axv - cxv;
          /* convective terms about UO (timeindeg.f:466-486) */
          coefx = rflagcx * coef * au[i] / 1.0;
          const double qxm = (A(uo, i, j, k) + A(uo, i - 1, j, k)) * 0.5;
          const double qxp = (A(uo, i, j, k) + A(uo, i + 1, j, k)) * 0.5;
          const double axc = -coefx * qxm, cxc = coefx * qxp, bxc = axc + cxc;
          ax[ii] = axv + axc;
          cx[ii] = cxv + cxc;
          bx[ii] = 1.0 + bxv + bxc;
          const double uxp = (A(uo, i + 1, j, k) + A(uo, i, j, k)) * 0.5;
          const double uxm = (A(uo, i - 1, j, k) + A(uo, i, j, k)) * 0.5;
          rx[ii] = rx[ii] + coefx * (qxp * uxp - qxm * uxm);
        }
        rx[0] = rx[0] - ax[0] * (A(us, i1 - 1, j, k) * t.rdir[0][0] + A(ub, i1 - 1, j, k) * t.rperb[0][0]);
        rx[n - 1] =
            rx[n - 1] - cx[n - 1] * (A(us, i2 + 1, j, k) * t.rdir[0][1] + A(ub, i2 + 1, j, k) * t.rperb[0][1]);
        thomas(ax, bx, cx, rx, x, n, gam);
        for (int i = i1; i <= i2; i++) A(us, i, j, k) = x[i - i1];
      }
    /* v */
#pragma omp for schedule(static) collapse(2)
    for (int k = g->kz1; k <= g->kz2; k++)
      for (int j = g->jbv; j <= g->jev; j++) {
        const int i1 = 2, i2 = NX - 1, n = i2 - i1 + 1;
        for (int i = i1; i <= i2; i++) {
          const int ii = i - i1;
          const double tvip =
              0.25 * (A(tv, i, j + 1, k) + A(tv, i, j, k) + A(tv, i + 1, j + 1, k) + A(tv, i + 1, j, k)) + ru1;
          const double tvim =
              0.25 * (A(tv, i, j + 1, k) + A(tv, i, j, k) + A(tv, i - 1, j + 1, k) + A(tv, i - 1, j, k)) + ru1;
          rx[ii] = A(vs, i, j, k);
          double coefx = rflagx * coef * av[i] / 1.0;
          const double axv = -coefx * au[i - 1] * tvim, cxv = -coefx * au[i] * tvip, bxv = -axv - cxv;
          /* convective terms about the provisional US (timeindeg.f:545-556) */
          coefx = rflagcx * 0.5 * coef * av[i] / 1.0;
          const double qyp = 1.0 * (A(us, i, j + 1, k) + A(us, i, j, k)) * 0.5;
          const double qym = 1.0 * (A(us, i - 1, j + 1, k) + A(us, i - 1, j, k)) * 0.5;
          const double axc = -coefx * qym, cxc = coefx * qyp, bxc = axc + cxc;
          ax[ii] = axv + axc;
          cx[ii] = cxv + cxc;
          bx[ii] = 1.0 + bxv + bxc;
        }
        bx[0] = bx[0] + (t.bdirb[1][0] + t.bneub[1][0]) * ax[0];
        bx[n - 1] = bx[n - 1] + (t.bdirb[1][1] + t.bneub[1][1]) * cx[n - 1];
        rx[0] = rx[0] - ax[0] * (A(vs, i1 - 1, j, k) * t.rdir[1][0] + A(vb, i1 - 1, j, k) * t.rperb[1][0] +
                                 0.5 * (A(vb, i1, j, k) + A(vb, i1 - 1, j, k)) * t.rdirb[1][0]);
        rx[n - 1] = rx[n - 1] - cx[n - 1] * (A(vs, i2 + 1, j, k) * t.rdir[1][1] + A(vb, i2 + 1, j, k) * t.rperb[1][1] +
                                             0.5 * (A(vb, i2, j, k) + A(vb, i2 + 1, j, k)) * t.rdirb[1][1]);
        thomas(ax, bx, cx, rx, x, n, gam);
        for (int i = i1; i <= i2; i++) A(vs, i, j, k) = x[i - i1];
      }
    /* w */
#pragma omp for schedule(static) collapse(2)
    for (int k = g->kbw; k <= g->kew; k++)
      for (int j = g->jy1; j <= g->jy2; j++) {
        const int i1 = 2, i2 = NX - 1, n = i2 - i1 + 1;
        for (int i = i1; i <= i2; i++) {
          const int ii = i - i1;
          const double tvip =
              0.25 * (A(tv, i, j, k + 1) + A(tv, i, j, k) + A(tv, i + 1, j, k + 1) + A(tv, i + 1, j, k)) + ru1;
          const double tvim =
              0.25 * (A(tv, i, j, k + 1) + A(tv, i, j, k) + A(tv, i - 1, j, k + 1) + A(tv, i - 1, j, k)) + ru1;
          rx[ii] = A(ws, i, j, k);
          double coefx = rflagx * coef * aw[i] / 1.0;
          const double axv = -coefx * au[i - 1] * tvim, cxv = -coefx * au[i] * tvip, bxv = -axv - cxv;
          /* convective terms about the provisional US (timeindeg.f:610-622) */
          coefx = rflagcx * 0.5 * coef * aw[i] / 1.0;
          const double qzp = 1.0 * (A(us, i, j, k + 1) + A(us, i, j, k)) * 0.5;
          const double qzm = 1.0 * (A(us, i - 1, j, k + 1) + A(us, i - 1, j, k)) * 0.5;
          const double axc = -coefx * qzm, cxc = coefx * qzp, bxc = axc + cxc;
          ax[ii] = axv + axc;
          cx[ii] = cxv + cxc;
          bx[ii] = 1.0 + bxv + bxc;
        }
        bx[0] = bx[0] + (t.bdirb[2][0] + t.bneub[2][0]) * ax[0];
        bx[n - 1] = bx[n - 1] + (t.bdirb[2][1] + t.bneub[2][1]) * cx[n - 1];
        rx[0] = rx[0] - ax[0] * (A(ws, i1 - 1, j, k) * t.rdir[2][0] + A(wb, i1 - 1, j, k) * t.rperb[2][0] +
                                 0.5 * (A(wb, i1, j, k) + A(wb, i1 - 1, j, k)) * t.rdirb[2][0]);
        rx[n - 1] = rx[n - 1] - cx[n - 1] * (A(ws, i2 + 1, j, k) * t.rdir[2][1] + A(wb, i2 + 1, j, k) * t.rperb[2][1] +
                                             0.5 * (A(wb, i2, j, k) + A(wb, i2 + 1, j, k)) * t.rdirb[2][1]);
        thomas(ax, bx, cx, rx, x, n, gam);
        for (int i = i1; i <= i2; i++) A(ws, i, j, k) = x[i - i1];
      }
    free(ax); free(bx); free(cx); free(rx); free(x); free(gam);
  }
}

/* INVERSEXD (src/density.f:129-290) on RS with RHB (the explicit predicted
 * density after BOUNDARY_DENS) for the wall values: k in [kbw, kew],
 * i in [2, NX-1], w's boundary row, and, as there, the molecular diffusivity
 * ru1/prn alone on both faces (the eddy diffusivity's x part, dropped from
 * the explicit right-hand side with IMPLX = 1, is not restored here) */
void eo_inversexd(eo_state *s, double alfxdt) {
  const eo_grid *g = s->g;
  const double coef = 0.5 * alfxdt, rflagx = (double)s->prm.implx, kmol = s->prm.ru1 / s->prm.prn;
  double *rs = s->rs;
  const double *rhb = s->rhb, *au = g->au, *aw = g->aw;
  xbc_tables t;
  x_tables(s, &t);
  const int nmax = NX;
#pragma omp parallel
  {
    double *ax = malloc(sizeof(double) * nmax), *bx = malloc(sizeof(double) * nmax),
           *cx = malloc(sizeof(double) * nmax), *rx = malloc(sizeof(double) * nmax),
           *x = malloc(sizeof(double) * nmax), *gam = malloc(sizeof(double) * nmax);
#pragma omp for schedule(static) collapse(2)
    for (int k = g->kbw; k <= g->kew; k++)
      for (int j = g->jy1; j <= g->jy2; j++) {
        const int i1 = 2, i2 = NX - 1, n = i2 - i1 + 1;
        for (int i = i1; i <= i2; i++) {
          const int ii = i - i1;
          const double tvip = kmol, tvim = kmol;
          rx[ii] = A(rs, i, j, k);
          const double coefx = rflagx * coef * aw[i] / 1.0;
          const double axv = -coefx * au[i - 1] * tvim, cxv = -coefx * au[i] * tvip, bxv = -axv - cxv;
          ax[ii] = axv;
          cx[ii] = cxv;
          bx[ii] = 1.0 + bxv;
        }
        bx[0] = bx[0] + (t.bdirb[2][0] + t.bneub[2][0]) * ax[0];
        bx[n - 1] = bx[n - 1] + (t.bdirb[2][1] + t.bneub[2][1]) * cx[n - 1];
        rx[0] = rx[0] - ax[0] * (A(rs, i1 - 1, j, k) * t.rdir[2][0] + A(rhb, i1 - 1, j, k) * t.rperb[2][0] +
                                 0.5 * (A(rhb, i1, j, k) + A(rhb, i1 - 1, j, k)) * t.rdirb[2][0]);
        rx[n - 1] = rx[n - 1] - cx[n - 1] * (A(rs, i2 + 1, j, k) * t.rdir[2][1] + A(rhb, i2 + 1, j, k) * t.rperb[2][1] +
                                             0.5 * (A(rhb, i2, j, k) + A(rhb, i2 + 1, j, k)) * t.rdirb[2][1]);
        thomas(ax, bx, cx, rx, x, n, gam);
        for (int i = i1; i <= i2; i++) A(rs, i, j, k) = x[i - i1];
      }
    free(ax); free(bx); free(cx); free(rx); free(x); free(gam);
  }
}
