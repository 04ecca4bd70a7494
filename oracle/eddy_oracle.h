/*
 * eddy_oracle.h -- CPU FP64 restatement of the eddy-hybrid fractional-step
 * time advance.  TEST INFRASTRUCTURE ONLY: this library is the checker that the
 * CUDA path is compared against.  Nothing in the product library links or calls
 * it; only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * it.
 *
 * Axes and layout follow the reference exactly (src/common.h, src/Eddy6.f:428):
 * arrays are Fortran column-major (NX,NY,NZ) with x fastest, 1-based indices,
 * one ghost layer each side.  x = x_ref (stretched, walls), y = y_ref (uniform,
 * periodic, the FFT axis), z = z_ref (stretched, streamwise inflow/outflow).
 *
 * Parity status: the reference is Fortran and cannot be compiled here (no
 * Fortran compiler; its default Poisson kernel BLKTRI exists only as a
 * prebuilt object that is off limits).  The FFT is pinned against
 * scipy.fftpack (which is FFTPACK, the library the reference ships in
 * src/fftpack.f); the Poisson solve is pinned by manufactured solutions and by
 * an independent block-tridiagonal elimination; the step is pinned by
 * invariants (divergence after projection, Taylor-Green decay).  Everything
 * else is parity-unpinned restatement of the cited Fortran lines.
 */
#ifndef EDDY_ORACLE_H
#define EDDY_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nx, ny, nz;          /* NX, NY, NZ incl. ghosts */
  int itype[7];            /* BC types, itype[1..6] as src/common.h ITYPE */
  int ischm;               /* 3 = low-storage RK3, 1 = AB2 (src/inpall.f:218) */
  int isgs;                /* 0 = none, 1 = Smagorinsky, 2 = dynamic (y average) */
  int idens;               /* 1 = Boussinesq density */
  double ru1;              /* 1/Re */
  double prn;              /* Prandtl */
  double denP1;            /* background density gradient */
  double grav;             /* gravity magnitude (after GRAVITY ramp) */
  double dpdx, dpdy, dpdz; /* imposed pressure gradients */
  double eps;              /* dynamic-model cutoff (IMM > sqrt(eps)) */
  double css;              /* Smagorinsky constant */
  int vspngx1, dspngx1, vspngx3in, vspngx3out, dspngx3in, dspngx3out;
  int imply;               /* 1: Crank-Nicolson viscous terms along y (INVERSEY/INVERSEYD) */
  int implx;               /* 1: Crank-Nicolson viscous terms along x (INVERSEX/INVERSEXD) */
  int implcx, implcy;      /* 1: Crank-Nicolson convective terms along x / y */
} eo_params;

/* 1-D metric arrays (src/common.h:51-54), 1-based: arrays have n+1 entries. */
typedef struct {
  int nx, ny, nz;
  int ix1, ix2, jy1, jy2, kz1, kz2;
  int ib1, ib2, jb1, jb2, kb1, kb2;
  int ibu, ieu, jbv, jev, kbw, kew;
  int mp, lp, np;
  double *xu, *xc, *ap, *au, *av, *aw;
  double *yv, *yc, *bp, *bu, *bv, *bw;
  double *zw, *zc, *cp, *cu, *cv, *cw;
  double *whx, *why, *whz;    /* filter weights (n+1)*3, index [i*3 + (d+1)] */
  double *dfxu, *dfxw, *dfxul, *dfxwl, *dfxd, *dfxdl; /* sponge profiles */
  int ivspngl, idspngl;
  double *dens_bg;            /* (NX,NY) background density */
  double dely, delysq;
} eo_grid;

/* Grid (src/grid.f:8-483) from face coordinates.  xu_faces has nx-1 entries
 * (the contents of a stretched-grid file: faces 1..ix2), zw_faces nz-1; y is
 * uniform on [ymin,ymax]. */
eo_grid *eo_grid_create(const eo_params *p, const double *xu_faces,
                        double ymin, double ymax, const double *zw_faces);
void eo_grid_free(eo_grid *g);
/* Copy 1-D arrays out (for checking the product's metric builder). which:
 * 0 xu 1 xc 2 ap 3 au 4 av 5 aw 6 yv 7 yc 8 bp 9 bu 10 bv 11 bw 12 zw 13 zc
 * 14 cp 15 cu 16 cv 17 cw 18 whx 19 why 20 whz 21 dfxu 22 dfxw 23 dfxul
 * 24 dfxwl 25 dfxd 26 dfxdl 27 dens_bg */
int eo_grid_get(const eo_grid *g, int which, double *out, int n);

/* Solver state: every 3-D field of the reference driver that the step
 * touches (src/Eddy6.f:428-454). */
typedef struct {
  eo_params prm;
  eo_grid *g;
  long ncell;
  double *uo, *vo, *wo, *p, *dp, *dens, *tv;
  double *us, *vs, *ws, *ua, *va, *wa, *ub, *vb, *wb;
  double *rha, *rhb, *rs;
  /* SGS scratch + persistent arrays (src/Eddy6.f:441-449) */
  double *g_s, *sxx, *syy, *szz, *sxy, *syz, *sxz, *ilm, *imm, *lm, *mm,
      *uc, *vc, *wc, *dxdydz, *cles;
  double *planeU, *planeV, *planeW, *planeD; /* (NX,NY) inflow planes */
  /* hybrid inflow sequence (src/hybrid.f:213-260): feed_n planes of u, v, w,
   * rho in feed order ([n][4][NX*NY]); x indices >= feed_iref take the last
   * plane (the reference plane); icycle is the driver's step counter */
  double *feed;
  int feed_n, feed_iref, icycle;
  double time;
  double alfxdt_last; /* alfxdt of the last CORRECT (the pressure update's implicit correction) */
  double pref_last;
  double qin_last, qout_last;
  struct eo_ib *ib;  /* immersed body (NULL: none) */
} eo_state;

eo_state *eo_state_create(const eo_params *p, const eo_grid *g);
void eo_state_free(eo_state *s);
/* field ids for get/set */
enum {
  EO_UO = 0, EO_VO, EO_WO, EO_P, EO_DP, EO_DENS, EO_TV, EO_US, EO_VS, EO_WS,
  EO_UA, EO_VA, EO_WA, EO_UB, EO_VB, EO_WB, EO_RHA, EO_RHB, EO_RS,
  EO_PLANEU, EO_PLANEV, EO_PLANEW, EO_PLANED, EO_NFIELDS
};
double *eo_field(eo_state *s, int id);
int eo_set(eo_state *s, int id, const double *src);
int eo_get(eo_state *s, int id, double *dst);

/* ---- individual subroutines (each mirrors one reference routine) ---- */
void eo_rhs(eo_state *s, const double *uo, const double *vo, const double *wo,
            const double *tv, double *ut, double *vt, double *wt, double *ur,
            double *vr, double *wr, double *qr);
void eo_predictord(eo_state *s, double alfxdt, double gamxdt, double rhoxdt);
void eo_boundary(eo_state *s, double *u, double *v, double *w);
void eo_boundinout(eo_state *s, double *ubc, double *vbc, double *wbc,
                   const double *uof, const double *vof, const double *wof,
                   double alfxdt, int idiv);
void eo_divergence(eo_state *s, const double *us, const double *vs,
                   const double *ws, double *div);
void eo_correct(eo_state *s, double alfxdt);
void eo_pressure_update(eo_state *s);
void eo_rhs_density(eo_state *s);
void eo_density(eo_state *s, double alfxdt, double gamxdt, double rhoxdt);
/* INVERSEY (src/timeindeg.f:120-340) on US,VS,WS and INVERSEYD
 * (src/density.f:383-460) on RS: the Crank-Nicolson y lines, IMPLY = 1 */
void eo_inversey(eo_state *s, double alfxdt);
/* CALCFL (src/timestep.f:2-78): CFLM over the interior */
double eo_calcfl(eo_state *s);
void eo_inverseyd(eo_state *s, double alfxdt);
void eo_inverseyd_new(eo_state *s, double alfxdt);
void eo_inversex_walls(eo_state *s, double alfxdt);
void eo_inversex(eo_state *s, double alfxdt);
void eo_inversexd(eo_state *s, double alfxdt);
/* calcfrc (src/calcforce.f:3-779), Cartesian, and its index helpers */
int eo_closest(const double *xx, int n, double x);
void eo_cv_range(const eo_grid *g, const double cvlim[4], int cv[6]);
void eo_calcfrc(eo_state *s, const double cvlim[4], double dt, int icycle, double fb[3], double out[56]);
/* periodic tridiagonal system (cyclic, src/numrec.f:754-779): n unknowns,
 * a sub-, b main, c super-diagonal, alpha = A(n,1), beta = A(1,n); work >= 4n */
void eo_cyclic(const double *a, const double *b, const double *c, double alpha, double beta, const double *r,
               double *x, int n, double *work);
void eo_boundary_dens(eo_state *s, double *d);
void eo_boundinoutd(eo_state *s, double *d);
void eo_turvis(eo_state *s);
void eo_filtersize(eo_state *s);
void eo_filter3d(eo_state *s, const double *f, double *fb, double *wk1,
                 double *wk2);
void eo_strain(eo_state *s, const double *uc, const double *vc,
               const double *wc);

/* ---- FFT in FFTPACK packed order (src/fftpack.f RFFTF/RFFTB) ---- */
void eo_rfftf(int n, double *r);   /* forward, unnormalised */
void eo_rfftb(int n, double *r);   /* backward, unnormalised */

/* ---- Poisson (src/direct.f:2-1118) ---- */
/* Solve in place on s->dp (input divergence/alfxdt in interior). method 0 =
 * per-wavenumber eigen-transform along x + tridiagonal along z, method 1 =
 * block-tridiagonal elimination (small sizes only, independent check). */
int eo_direct(eo_state *s, int method);
/* Apply the discrete operator the reference's DIRECT inverts (x: AP AU, y:
 * periodic uniform, z: CP CW, Neumann when mp/np=1) to x (interior), write
 * interior of out. */
void eo_apply_laplacian(eo_state *s, const double *x, double *out);

/* ---- one time step (src/Eddy6.f:2095-3049, ibm=0 path) ---- */
void eo_substep(eo_state *s, int is, double dtm1);
void eo_step(eo_state *s, double dtm1, int nsteps, int poisson_method);
void eo_set_threads(int n);
void eo_initialize(eo_state *s, double dtm1);
/* one call per product C-ABI entry point (kernel-level parity tests) */
void eo_call_rhs_predictord(eo_state *s, double alfxdt, double gamxdt, double rhoxdt);
void eo_call_boundary(eo_state *s, int set);
void eo_call_boundinout(eo_state *s, int idiv, double alfxdt);
int eo_call_direct(eo_state *s, double alfxdt, int method);
void eo_call_density(eo_state *s, double alfxdt, double gamxdt, double rhoxdt);
double eo_max_divergence(eo_state *s);

/* ---- immersed boundary (eo_ib.c; src/rt.f, devel.f, matint.f, momforc.f) ---- */
typedef struct eo_ib eo_ib;
/* stencils of one variable, ordered by dependency level */
typedef struct {
  int n, nlev;
  int *i, *j, *k;       /* forcing points (1-based) */
  int *di, *dj, *dk;    /* mrk 2: extension point offsets (grid-line stencil), else 0 */
  int *lev;             /* dependency loop (1-based) */
  int *indx;            /* [n][2] LU pivots (0-based rows) */
  double *xn, *yn, *zn; /* body intersection */
  double *lu;           /* [n][4] LU factors, column-major a11 a21 a12 a22 */
  int *lev_start;       /* [nlev+1] offsets of each level */
  int *mrk;             /* stencil kind: 1 normal direction, 2 grid line, 3 closest point */
  int *dir;             /* mrk 1, 3: axis (1..3) normal to the fluid face crossed */
  double *xe, *ye, *ze; /* mrk 1, 3: extension point on that face (interp_cellface) */
} eo_ib_set;
/* vert [nb][3][3] (x,y,z of vertices a,b,c), normals [nb][3], vel[3] */
eo_ib *eo_ib_create(const eo_grid *g, int nb, const double *vert, const double *normals, const double *vel);
void eo_ib_free(eo_ib *ib);
void eo_ib_limimb(eo_ib *ib);
void eo_ib_tag(eo_ib *ib, int q);
void eo_ib_taguo(eo_ib *ib, int q, int fq);
void eo_ib_flagp(eo_ib *ib);
void eo_ib_geom(eo_ib *ib, int q, int fq, int imn);
void eo_ib_regen(eo_ib *ib);
void eo_ib_move(eo_ib *ib, double tmove);
void eo_ib_force(eo_ib *ib, int q, double *a, double b0);
void eo_ib_interior(eo_ib *ib, int fq, double *a, double value);
void eo_ib_force_impl(eo_ib *ib, int q, double *us, double *ub, double b0);
void eo_ib_interior_impl(eo_ib *ib, int fq, double *us, const double *ub, double value);
const int *eo_ib_limits(const eo_ib *ib);
const signed char *eo_ib_tags(const eo_ib *ib, int q);
const signed char *eo_ib_flags(const eo_ib *ib, int fq);
const eo_ib_set *eo_ib_stencils(const eo_ib *ib, int q);
void eo_ib_body(const eo_ib *ib, double *v, double *c);
const double *eo_ib_velocity(const eo_ib *ib);
void eo_ib_set_cadence(eo_ib *ib, int every);
/* 1: exhaustive candidate and nearest-centroid searches instead of the
 * binned ones (same results; a cross-check) */
void eo_ib_set_brute(eo_ib *ib, int brute);
int eo_ib_every(const eo_ib *ib);
int eo_locate(const double *xx1, int n, double x);
int eo_segtriint(const double *p1, const double *p2, const double *a, const double *b, const double *c,
                 double *xm);
void eo_lu2(double *a, int *indx);
void eo_lusolve2(const double *a, const int *indx, double *b);
int eo_ib_grid_intr(const eo_ib *ib, int q, const signed char *flag, int im, int jm, int km, const int *inn,
                    int nn, int isrt, double *xn, double *ext, int *fp);
/* attach a body to the solver: the substep then moves it, regenerates the
 * stencils and applies the forcing (src/Eddy6.f:2163-2380, 2526-2575,
 * 2881-2897, 2972-2983) */
void eo_state_set_ib(eo_state *s, eo_ib *ib);
/* hybrid inflow sequence: n planes of (u, v, w, rho) in feed order, each
 * NX*NY (Fortran order), copied in; the cells i >= iref take the last plane
 * (sequence_hybrid, src/hybrid.f:250-258; the reference has iref = 116); the
 * step counter is set to nstep and the plane of cycle nstep - 1 loaded, as
 * the start-up call src/Eddy6.f:806-814 does.  eo_step then loads the plane
 * of the current cycle after every substep (src/Eddy6.f:2985-2991). */
void eo_feed_set(eo_state *s, int n, const double *planes, int iref, int nstep);
/* the sequence position of cycle c (sequence_hybrid's icycle_feed, as a
 * 0-based position in feed order) */
int eo_feed_position(int c, int n);

/* ---- deterministic noise: SplitMix64 counter generator ---- */
uint64_t eo_splitmix64(uint64_t x);
double eo_uniform(uint64_t seed, uint64_t counter);

#ifdef __cplusplus
}
#endif
#endif
