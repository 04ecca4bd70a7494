/*
 * eo_step.c -- oracle restatement of the driver's time-advance sequence,
 * src/Eddy6.f:2095-3049 for ibm=0, explicit viscous terms, single rank.
 * TEST INFRASTRUCTURE ONLY.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "eddy_oracle.h"

/* RK3 / AB2 coefficients, src/inpall.f:218-235 */
static void scheme(int ischm, double gam[3], double rho[3], double alf[3]) {
  if (ischm == 1) {
    gam[0] = 1.5; gam[1] = 0.; gam[2] = 0.;
    rho[0] = -0.5; rho[1] = 0.; rho[2] = 0.;
  } else {
    gam[0] = 8. / 15.; gam[1] = 5. / 12.; gam[2] = 3. / 4.;
    rho[0] = 0.; rho[1] = -17. / 60.; rho[2] = -5. / 12.;
  }
  for (int q = 0; q < 3; q++) alf[q] = gam[q] + rho[q];
}

static int g_poisson_method = 0;

void eo_substep(eo_state *s, int is, double dtm1) {
  double gam[3], rho[3], alf[3];
  scheme(s->prm.ischm, gam, rho, alf);
  double alfxdt = alf[is] * dtm1, gamxdt = gam[is] * dtm1, rhoxdt = rho[is] * dtm1;
  /* moving body: RBM, then new stencils (:2163-2380); every substep over
   * alfxdt, or once per step (first substep) over the whole step */
  if (s->ib && (eo_ib_every(s->ib) || is == 0)) {
    eo_ib_move(s->ib, eo_ib_every(s->ib) ? alfxdt : dtm1);
    eo_ib_regen(s->ib);
  }
  /* Eddy6.f:2453 */
  eo_rhs(s, s->uo, s->vo, s->wo, s->tv, s->us, s->vs, s->ws, s->ub, s->vb, s->wb, s->dp);
  /* :2484 */
  eo_predictord(s, alfxdt, gamxdt, rhoxdt);
  const int implicit = s->prm.imply == 1 || s->prm.implx == 1;
  /* momentum forcing and body velocity inside (:2526-2575) */
  if (s->ib && implicit) {
    /* :2495-2520: UB = US + alfxdt/2 UB (UB holds the C.N. parts), its
     * boundary conditions, then the forcing of US from it (impl = 1) */
    for (long q = 0; q < s->ncell; q++) {
      s->ub[q] = s->us[q] + 0.5 * alfxdt * s->ub[q];
      s->vb[q] = s->vs[q] + 0.5 * alfxdt * s->vb[q];
      s->wb[q] = s->ws[q] + 0.5 * alfxdt * s->wb[q];
    }
    eo_boundary(s, s->ub, s->vb, s->wb);
    eo_boundinout(s, s->ub, s->vb, s->wb, s->uo, s->vo, s->wo, alfxdt, 1);
    eo_boundary(s, s->ub, s->vb, s->wb);
    const double *vel = eo_ib_velocity(s->ib);
    eo_ib_force_impl(s->ib, 0, s->us, s->ub, vel[0]);
    eo_ib_force_impl(s->ib, 1, s->vs, s->vb, vel[1]);
    eo_ib_force_impl(s->ib, 2, s->ws, s->wb, vel[2]);
    eo_ib_interior_impl(s->ib, 0, s->us, s->ub, vel[0]);
    eo_ib_interior_impl(s->ib, 1, s->vs, s->vb, vel[1]);
    eo_ib_interior_impl(s->ib, 2, s->ws, s->wb, vel[2]);
  } else if (s->ib) {
    const double *vel = eo_ib_velocity(s->ib);
    eo_ib_force(s->ib, 0, s->us, vel[0]);
    eo_ib_force(s->ib, 1, s->vs, vel[1]);
    eo_ib_force(s->ib, 2, s->ws, vel[2]);
    eo_ib_interior(s->ib, 0, s->us, vel[0]);
    eo_ib_interior(s->ib, 1, s->vs, vel[1]);
    eo_ib_interior(s->ib, 2, s->ws, vel[2]);
  }
  /* Crank-Nicolson y, then x lines (:2582-2607; the IBM = 0 planes of UB
   * only without a body) */
  const int cx = s->prm.implx == 1 || s->prm.implcx == 1, cy = s->prm.imply == 1 || s->prm.implcy == 1;
  if (cx && !s->ib) eo_inversex_walls(s, alfxdt);
  if (cy) eo_inversey(s, alfxdt);
  if (cx) eo_inversex(s, alfxdt);
  /* :2689-2704 */
  eo_boundary(s, s->us, s->vs, s->ws);
  eo_boundinout(s, s->us, s->vs, s->ws, s->uo, s->vo, s->wo, alfxdt, 1);
  eo_boundary(s, s->us, s->vs, s->ws);
  /* :2712-2715 */
  eo_divergence(s, s->us, s->vs, s->ws, s->dp);
  for (long q = 0; q < s->ncell; q++) s->dp[q] = s->dp[q] / alfxdt;
  /* :2722 */
  eo_direct(s, g_poisson_method);
  /* :2738-2761 */
  eo_correct(s, alfxdt);
  eo_boundary(s, s->uo, s->vo, s->wo);
  eo_boundinout(s, s->uo, s->vo, s->wo, s->us, s->vs, s->ws, alfxdt, 0);
  eo_boundary(s, s->uo, s->vo, s->wo);
  /* :2772-2853, :2911-2953 */
  eo_pressure_update(s);
  /* :2957-2969 */
  if (s->prm.idens == 1) {
    eo_boundinoutd(s, s->dens);
    eo_boundary_dens(s, s->dens);
    eo_rhs_density(s);
    eo_boundary_dens(s, s->rhb);
    eo_boundary_dens(s, s->rs);
    eo_density(s, alfxdt, gamxdt, rhoxdt);
    eo_boundinoutd(s, s->dens);
    eo_boundary_dens(s, s->dens);
    /* correctdens_mod2 + densinterior (:2972-2983) */
    if (s->ib) {
      eo_ib_force(s->ib, 3, s->dens, 0.0);
      eo_ib_interior(s->ib, 4, s->dens, 0.0);
    }
  }
}

void eo_state_set_ib(eo_state *s, eo_ib *ib) { s->ib = ib; }

/* sequence_hybrid (src/hybrid.f:224-232): icycle_feed = start + stride*c -
 * stride*floor(c/num)*num, i.e. position c - num*floor(c/num) of the feed */
int eo_feed_position(int c, int n) {
  const int nfc = (int)floor((double)c / (double)n);
  return c - nfc * n;
}

/* the plane of cycle c into planeU..planeD; i >= iref from the last plane
 * (src/hybrid.f:250-258) */
static void feed_load(eo_state *s, int c) {
  if (!s->feed || s->feed_n <= 0) return;
  const int nx = s->prm.nx, ny = s->prm.ny;
  const long n2 = (long)nx * ny;
  const double *src = s->feed + (long)eo_feed_position(c, s->feed_n) * 4 * n2;
  const double *ref = s->feed + (long)(s->feed_n - 1) * 4 * n2;
  double *dst[4] = {s->planeU, s->planeV, s->planeW, s->planeD};
  for (int f = 0; f < 4; f++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        const long q = (long)(i - 1) + (long)nx * (j - 1);
        dst[f][q] = i >= s->feed_iref ? ref[f * n2 + q] : src[f * n2 + q];
      }
}

void eo_feed_set(eo_state *s, int n, const double *planes, int iref, int nstep) {
  free(s->feed);
  s->feed = NULL;
  s->feed_n = 0;
  if (n <= 0) return;
  const long n2 = (long)s->prm.nx * s->prm.ny;
  s->feed = (double *)malloc(sizeof(double) * 4 * n2 * n);
  memcpy(s->feed, planes, sizeof(double) * 4 * n2 * n);
  s->feed_n = n;
  s->feed_iref = iref;
  s->icycle = nstep;
  feed_load(s, nstep - 1);
}

void eo_step(eo_state *s, double dtm1, int nsteps, int poisson_method) {
  double gam[3], rho[3], alf[3];
  scheme(s->prm.ischm, gam, rho, alf);
  g_poisson_method = poisson_method;
  int nsub = (s->prm.ischm == 1) ? 1 : 3;
  for (int n = 0; n < nsteps; n++) {
    double tlevel = s->time;
    s->icycle++; /* do icycle=1+nstep,... (:2095) */
    for (int is = 0; is < nsub; is++) {
      eo_substep(s, is, dtm1);
      feed_load(s, s->icycle); /* sequence_hybrid after each substep (:2985-2991) */
      double sa = 0.;
      for (int q = 0; q <= is; q++) sa += alf[q];
      tlevel = s->time + sa * dtm1;
    }
    s->time = tlevel;
    /* :3008-3019 */
    if (s->prm.isgs != 0) eo_turvis(s);
    /* tvinterior (:3040-3042) */
    if (s->ib && s->prm.isgs != 0) eo_ib_interior(s->ib, 3, s->tv, 0.0);
  }
}

/* Start-from-scratch initialisation after the fields are set (src/Eddy6.f
 * :582-617 ghost fills, :620 sponge set-up (in eo_grid_create), :752-756
 * inflow/outflow, :1718-1726 filter size and initial TURVIS). */
void eo_initialize(eo_state *s, double dtm1) {
  double gam[3], rho[3], alf[3];
  scheme(s->prm.ischm, gam, rho, alf);
  const eo_grid *g = s->g;
  eo_boundary(s, s->uo, s->vo, s->wo);
  eo_boundary_dens(s, s->dens);
  /* pressure ghosts (:585-617) */
  int nx = g->nx, ny = g->ny, nz = g->nz;
  double *p = s->p;
#define PA(i, j, k) p[(size_t)((i)-1) + (size_t)nx * ((size_t)((j)-1) + (size_t)ny * (size_t)((k)-1))]
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++) {
      if (g->mp == 0) { PA(1, j, k) = PA(g->ix2, j, k); PA(nx, j, k) = PA(g->ix1, j, k); }
      else { PA(1, j, k) = -PA(g->ix1, j, k); PA(nx, j, k) = -PA(g->ix2, j, k); }
    }
  for (int k = 1; k <= nz; k++)
    for (int i = 1; i <= nx; i++) {
      if (g->lp == 0) { PA(i, 1, k) = PA(i, g->jy2, k); PA(i, ny, k) = PA(i, g->jy1, k); }
      else { PA(i, 1, k) = PA(i, g->jy1, k); PA(i, ny, k) = PA(i, g->jy2, k); }
    }
  const int *it = s->prm.itype;
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++) {
      if (it[5] == 500) PA(i, j, 1) = PA(i, j, g->kz2);
      if (it[6] == 500) PA(i, j, nz) = PA(i, j, g->kz1);
      if (it[5] != 0 && it[5] != 500) PA(i, j, 1) = PA(i, j, g->kz1);
      if (it[6] != 0 && it[6] != 500) PA(i, j, nz) = PA(i, j, g->kz2);
    }
#undef PA
  double alfxdt = alf[0] * dtm1;
  eo_boundinout(s, s->uo, s->vo, s->wo, s->uo, s->vo, s->wo, alfxdt, 1);
  eo_boundary(s, s->uo, s->vo, s->wo);
  if (s->prm.idens == 1) eo_boundinoutd(s, s->dens);
  if (s->prm.isgs != 0) {
    eo_filtersize(s);
    eo_turvis(s);
  }
}

/* ---- one call per C-ABI entry point of the product, for kernel-level parity
 * tests (same sequences as include/eddy_b200.h documents) ---- */
void eo_call_rhs_predictord(eo_state *s, double alfxdt, double gamxdt, double rhoxdt) {
  eo_rhs(s, s->uo, s->vo, s->wo, s->tv, s->us, s->vs, s->ws, s->ub, s->vb, s->wb, s->dp);
  eo_predictord(s, alfxdt, gamxdt, rhoxdt);
}
void eo_call_boundary(eo_state *s, int set) {
  if (set == 0) eo_boundary(s, s->us, s->vs, s->ws);
  else eo_boundary(s, s->uo, s->vo, s->wo);
}
void eo_call_boundinout(eo_state *s, int idiv, double alfxdt) {
  if (idiv == 1) eo_boundinout(s, s->us, s->vs, s->ws, s->uo, s->vo, s->wo, alfxdt, 1);
  else eo_boundinout(s, s->uo, s->vo, s->wo, s->us, s->vs, s->ws, alfxdt, 0);
}
int eo_call_direct(eo_state *s, double alfxdt, int method) {
  eo_divergence(s, s->us, s->vs, s->ws, s->dp);
  for (long q = 0; q < s->ncell; q++) s->dp[q] = s->dp[q] / alfxdt;
  return eo_direct(s, method);
}
void eo_call_density(eo_state *s, double alfxdt, double gamxdt, double rhoxdt) {
  eo_boundinoutd(s, s->dens);
  eo_boundary_dens(s, s->dens);
  eo_rhs_density(s);
  eo_boundary_dens(s, s->rhb);
  eo_boundary_dens(s, s->rs);
  eo_density(s, alfxdt, gamxdt, rhoxdt);
  eo_boundinoutd(s, s->dens);
  eo_boundary_dens(s, s->dens);
}
double eo_max_divergence(eo_state *s) {
  const eo_grid *g = s->g;
  double mx = 0.;
  int nx = g->nx, ny = g->ny;
#define OA(a, i, j, k) (a)[(size_t)((i)-1) + (size_t)nx * ((size_t)((j)-1) + (size_t)ny * (size_t)((k)-1))]
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ix1; i <= g->ix2; i++) {
        double dv = (g->ap[i] * (OA(s->uo, i, j, k) - OA(s->uo, i - 1, j, k)) +
                     g->bp[j] * (OA(s->vo, i, j, k) - OA(s->vo, i, j - 1, k)) +
                     g->cp[k] * (OA(s->wo, i, j, k) - OA(s->wo, i, j, k - 1)));
        if (fabs(dv) > mx) mx = fabs(dv);
      }
#undef OA
  return mx;
}

/* CALCFL (src/timestep.f:2-78), Cartesian: CONST = 2, rp = 1, the implicit
 * flags RFLAGX = IMPLX, RFLAGY = IMPLY, RFLAGCX = IMPLCX, RFLAGCY = IMPLCY;
 * returns CFLM over the interior */
double eo_calcfl(eo_state *s) {
  const eo_grid *g = s->g;
  const double cst = 2., rflagx = (double)s->prm.implx, rflagcx = (double)s->prm.implcx,
               rflagcy = (double)s->prm.implcy, rflagy = (double)s->prm.imply;
  const int nx = g->nx, ny = g->ny;
  double cflm = 0.;
  for (int k = g->kz1; k <= g->kz2; k++)
    for (int j = g->jy1; j <= g->jy2; j++)
      for (int i = g->ix1; i <= g->ix2; i++) {
        const size_t q = (size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)ny * (size_t)(k - 1));
        const double cflx = (1. - rflagcx * 1.) * 0.5 * fabs(s->uo[q - 1] + s->uo[q]) * g->ap[i];
        const double cfly = (1. - rflagcy * 1.) * 0.5 * fabs(s->vo[q - nx] + s->vo[q]) * g->bp[j] / 1.0;
        const double cflz = 0.5 * fabs(s->wo[q - (size_t)nx * ny] + s->wo[q]) * g->cp[k];
        const double totvx = s->prm.ru1 + s->tv[q];
        const double cflvx = (1. - rflagx * 1.) * (g->ap[i] * g->ap[i]);
        const double by = g->bp[j] / 1.0;
        const double cflvy = (1. - rflagy * 1.) * (by * by);
        const double cflvz = g->cp[k] * g->cp[k];
        double c = fmax(fmax(fmax(cflx, cfly), fmax(cflz, cst * totvx * cflvx)),
                        fmax(cst * totvx * cflvy, cst * totvx * cflvz));
        cflm = fmax(cflm, c);
      }
  return cflm;
}
