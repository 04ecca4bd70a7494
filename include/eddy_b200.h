/*
 * eddy_b200.h -- C ABI of the B200 (sm_100a) fractional-step time advance.
 *
 * Drop-in boundary for the reference's Fortran driver (src/Eddy6.f).  Every
 * entry point returns an int status (EDDY_OK = 0); none exits or traps.
 * Fields live on the GPU inside an opaque context; host arrays are touched
 * only by eddy_upload/eddy_download (Fortran column-major (NX,NY,NZ) FP64 with
 * ghost layers, exactly the driver's ALLOCATEd arrays, src/Eddy6.f:428-454).
 * All work is enqueued on the context's CUDA stream; eddy_sync and
 * eddy_download are the only calls that block.  A context is used by one host
 * thread at a time.
 *
 * Axes follow the reference: x = x_ref (stretched), y = y_ref (uniform,
 * periodic, FFT axis), z = z_ref (stretched).  Boundary types supported on
 * the hot path: 60 (slip wall) and 82 (the stratified-wave condition of
 * BOUND082) on x, 500 on y, 305 (hybrid inlet plane) and 730 (convective
 * outlet) on z.
 */
#ifndef EDDY_B200_H
#define EDDY_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum {
  EDDY_OK = 0,
  EDDY_EINVAL = 1,      /* bad argument / unsupported configuration */
  EDDY_ECUDA = 2,       /* CUDA error */
  EDDY_ENAN = 3,        /* non-finite value detected */
  EDDY_ESINGULAR = 4,   /* singular pivot in a line solve */
  EDDY_ENOCONV = 5,     /* refinement did not converge */
  EDDY_ETIMEOUT = 6,    /* a bounded device-side wait expired */
  EDDY_ENOMEM = 7
};

/* Precision forms. */
enum { EDDY_PLAIN_FP64 = 0, EDDY_MIXED = 1 };

/* Field ids for upload/download; numbering matches the reference names. */
enum {
  EDDY_UO = 0, EDDY_VO, EDDY_WO, EDDY_P, EDDY_DP, EDDY_DENS, EDDY_TV,
  EDDY_US, EDDY_VS, EDDY_WS, EDDY_UA, EDDY_VA, EDDY_WA, EDDY_UB, EDDY_VB,
  EDDY_WB, EDDY_RHA, EDDY_RHB, EDDY_RS,
  EDDY_PLANEU, EDDY_PLANEV, EDDY_PLANEW, EDDY_PLANED, /* (NX,NY) planes */
  EDDY_NFIELDS
};

/* Run parameters.  Names follow the reference's COMMON blocks
 * (src/common.h:77-112) and the sponge module (src/Initialize.f:139-153). */
typedef struct {
  int nx, ny, nz;            /* NX, NY, NZ including one ghost layer each side */
  int itype[7];              /* ITYPE(1..6) in itype[1..6]; itype[0] unused */
  int ischm;                 /* 3 = RK3, 1 = AB2 (src/inpall.f:218-235) */
  int isgs;                  /* 0 none, 1 Smagorinsky, 2 dynamic (y average) */
  int idens;                 /* 1 = Boussinesq density equation */
  double ru1, prn, denP1, grav, dpdx, dpdy, dpdz, eps, css;
  int vspngx1, dspngx1, vspngx3in, vspngx3out, dspngx3in, dspngx3out;
  int precision;             /* EDDY_PLAIN_FP64 or EDDY_MIXED */
  int refine_sweeps;         /* mixed form: FP64-residual refinement sweeps (1-3) */
  int closure;               /* 0 = dynamic TURVIS, 1 = learned MLP closure */
  int imply;                 /* IMPLY (src/inpall.f:42): 1 = the viscous terms along y
                                Crank-Nicolson implicit (INVERSEY src/timeindeg.f:120,
                                INVERSEYD src/density.f:383), over the whole x range
                                (IMPLYDCMP = 0); plain form.  With an immersed body
                                the velocity forcing runs before the line solves,
                                from the explicit estimate (src/Eddy6.f:2495-2575). */
  int implx;                 /* IMPLX: 1 = the viscous terms along x Crank-Nicolson
                                implicit (INVERSEX src/timeindeg.f:344, INVERSEXD
                                src/density.f:129) over the whole x range
                                (IMPLXDCMP = 0), with slip walls (type 60) on both
                                x boundaries; plain form. */
  int implcx, implcy;        /* IMPLCX, IMPLCY: 1 = the convective terms along x / y
                                Crank-Nicolson implicit inside the same line solves
                                (linearised about UO / VO and the provisional US /
                                VS as src/timeindeg.f:120-690 does; INVERSEYD_NEW,
                                src/density.f:290, for the density when IMPLY and
                                IMPLCY are both 1); plain form.  With a body and
                                neither IMPLX nor IMPLY the forcing runs before
                                the line solves, on US. */
} eddy_params;

typedef struct eddy_ctx eddy_ctx;

/* Create a context on CUDA device `device`.  Builds the metric arrays the way
 * src/grid.f:8-483 does from face coordinates (x: nx-1 faces, z: nz-1 faces,
 * the contents of the reference's grid files; y uniform on [ymin,ymax]),
 * the sponge profiles (src/Initialize.f:129-271) and the Poisson plan
 * (src/direct.f:121-585).  Replaces the driver's Grid/SETUP/SPONGE_SETUP
 * calls (src/Eddy6.f:463,531,620). */
int eddy_create(eddy_ctx **out, const eddy_params *prm, const double *xu_faces,
                double ymin, double ymax, const double *zw_faces, int device);
int eddy_destroy(eddy_ctx *ctx);

/* Copy a field between the host (Fortran-ordered FP64) and the device. */
int eddy_upload(eddy_ctx *ctx, int field, const double *host);
int eddy_download(eddy_ctx *ctx, int field, double *host);
/* Restart files in the layout of the reference's IOSCALAR (src/io.f:114-200,
 * serial case; written at src/Eddy6.f:3391-3408, read at :780-803):
 * Fortran unformatted sequential records with 4-byte length markers --
 * (NX, NY, NZ, 1) int32, one record of NX*NY float64 per z plane, nstep
 * int32, TIME float64, (DTM1, grav) float64.  Host-only functions on a
 * Fortran-ordered (NX,NY,NZ) array; reading refuses a file of another grid
 * or a truncated one with EDDY_EINVAL. */
int eddy_ioscalar_write(const char *path, int nx, int ny, int nz, const double *a, int nstep, double time,
                        double dtm1, double grav);
int eddy_ioscalar_read(const char *path, int nx, int ny, int nz, double *a, int *nstep, double *time,
                       double *dtm1, double *grav);
/* The same from and to a device field (one of the (NX,NY,NZ) fields; grav
 * written is the context's).  A restart is UO, VO, WO, P, TV and DENS
 * (the reference's set); stepping continues from them without
 * eddy_initialize.  Null out-pointers are skipped. */
int eddy_save_field(eddy_ctx *ctx, int field, const char *path, int nstep, double time, double dtm1);
int eddy_load_field(eddy_ctx *ctx, int field, const char *path, int *nstep, double *time, double *dtm1,
                    double *grav);
/* The hybrid inlet's inflow planes (src/hybrid.f:162-260).  A plane file in
 * the layout read_hybrid reads (Fortran unformatted records: icycle; TIME,
 * DTM1, grav, rho, Re, Pr; dir, -, index; zcg, zwg; NX, -, NY; xc, xu; yc,
 * yv; planeU, planeV, planeW, planeP, planeD), host-only; a file of another
 * grid or a truncated one is refused with EDDY_EINVAL; null outputs are
 * skipped. */
int eddy_read_hybrid_plane(const char *path, int nx, int ny, double *u, double *v, double *w, double *p, double *d,
                           int *icycle, double *time);
/* The sequence of n inflow planes, planes[n][4][NX*NY] (u, v, w, rho in feed
 * order, Fortran-ordered planes: the contents of the files start_feed,
 * start_feed + stride_feed, ..., end_feed), kept on the device.  Sets the
 * step counter to nstep and loads the plane of cycle nstep - 1, as the
 * start-up call src/Eddy6.f:806-814 does; every eddy_substep then loads the
 * plane of the current cycle (sequence_hybrid after each substep,
 * src/Eddy6.f:2985-2991: position c - n floor(c/n) of the feed), the cells
 * i >= iref from the last plane (the reference's steady far field; it has
 * iref = 116; NX + 1 turns that off).  eddy_step advances the
 * counter at the start of each step (src/Eddy6.f:2095); a driver stepping
 * with eddy_substep sets it with eddy_inflow_cycle before each step.  n = 0
 * removes the sequence (the inlet planes then stay as uploaded). */
int eddy_inflow_sequence(eddy_ctx *ctx, int n, const double *planes, int iref, int nstep);
int eddy_inflow_cycle(eddy_ctx *ctx, int icycle);
/* Read one of the 1-D metric arrays the context built (same numbering as the
 * oracle: 0 xu 1 xc 2 ap 3 au 4 av 5 aw 6 yv 7 yc 8 bp 9 bu 10 bv 11 bw
 * 12 zw 13 zc 14 cp 15 cu 16 cv 17 cw 18 whx 19 why 20 whz 21 dfxu 22 dfxw
 * 23 dfxul 24 dfxwl 25 dfxd 26 dfxdl 27 dens_bg); returns length or <0. */
int eddy_get_metric(eddy_ctx *ctx, int which, double *out, int n);
/* Host-only: the same metric arrays without a context or a GPU (the
 * reference's Grid subroutine, src/grid.f:8). */
int eddy_grid_metric(const eddy_params *prm, const double *xu_faces, double ymin, double ymax,
                     const double *zw_faces, int which, double *out, int n);

/* ---- one entry per reference subroutine on the hot path ---- */
/* RHS (src/rhs.f:4) fused with PREDICTORD (src/timeindeg.f:1041): uo,vo,wo,
 * tv,p,dens,ua.. -> us,vs,ws (u*), ua,va,wa (new explicit RHS). */
int eddy_rhs_predictord(eddy_ctx *ctx, double alfxdt, double gamxdt, double rhoxdt);
/* INVERSEY (src/timeindeg.f:120-340): the Crank-Nicolson y lines of US, VS,
 * WS after the predictor, the viscous (imply) and convective (implcy) parts;
 * one of the two must be on.  The density's INVERSEYD (src/density.f:383) or
 * INVERSEYD_NEW (src/density.f:290, imply and implcy) runs inside
 * eddy_density. */
int eddy_inversey(eddy_ctx *ctx, double alfxdt);
/* INVERSEX (src/timeindeg.f:344-690): the Crank-Nicolson x lines of US, then
 * VS and WS, the viscous (implx) and convective (implcx) parts; one of the two
 * must be on (after eddy_inversey when both axes are, as src/Eddy6.f:2597-2607
 * orders them).  INVERSEXD (src/density.f:129) runs inside eddy_density when
 * implx or implcx is 1. */
int eddy_inversex(eddy_ctx *ctx, double alfxdt);
/* BOUNDARY (src/boundary.f:7) on the provisional (set=0: US,VS,WS) or the
 * corrected (set=1: UO,VO,WO) velocity. */
int eddy_boundary(eddy_ctx *ctx, int set);
/* BOUNDINOUT (src/boundary.f:505); idiv=1 predictor on US.. (old UO..),
 * idiv=0 corrector on UO.. (from US..). */
int eddy_boundinout(eddy_ctx *ctx, int idiv, double alfxdt);
/* DIVERGENCE (src/timeindeg.f:908) / alfxdt then DIRECT (src/direct.f:2):
 * solves for DP on the device. */
int eddy_direct(eddy_ctx *ctx, double alfxdt);
/* CORRECT (src/timeindeg.f:981). */
int eddy_correct(eddy_ctx *ctx, double alfxdt);
/* P=P+DP, reference value, ghost fills (src/Eddy6.f:2772-2853,2911-2953). */
int eddy_pressure_update(eddy_ctx *ctx);
/* BOUNDINOUTD/BOUNDARY_DENS/RHS_DENSITY/DENSITY sequence (src/Eddy6.f
 * :2957-2969; src/rhs_density.f:4; src/density.f:6). */
int eddy_density(eddy_ctx *ctx, double alfxdt, double gamxdt, double rhoxdt);
/* TURVIS dynamic procedure (src/vt.f:16) incl. FILTERSIZE (src/vt.f:1096). */
int eddy_turvis(eddy_ctx *ctx);

/* ---- driver twin (src/Eddy6.f:2095-3049) ---- */
/* Start-from-scratch initialisation after uploading the initial fields
 * (src/Eddy6.f:582-765, 1718-1726). */
int eddy_initialize(eddy_ctx *ctx, double dt);
/* One RK substep is (0-based) of the step, time step dt. */
int eddy_substep(eddy_ctx *ctx, int is, double dt);
/* nsteps full steps (3 RK substeps + eddy viscosity update each). */
int eddy_step(eddy_ctx *ctx, double dt, int nsteps);

/* Standalone Poisson solve of the operator DIRECT inverts: rhs is an
 * (NX,NY,NZ) device or host array (interior used); the solution is written to
 * sol (same shape, DIRECT's ghost convention).  `on_device` selects pointer
 * space.  In the mixed form the solve is FP32 transforms wrapped in
 * refine_sweeps FP64-residual iterative-refinement sweeps. */
int eddy_poisson_solve(eddy_ctx *ctx, const double *rhs, double *sol, int on_device);

/* ---- immersed boundary (src/rt.f, src/devel.f, src/matint.f, src/momforc.f,
 * src/rbm.f) ---- */
/* Attach a triangulated body (replaces the STL read of src/object.f and the
 * motion law of src/rbm.f): nb triangles, vertices [nb][3][3] (x,y,z of the
 * three vertices), unit outward normals [nb][3], translation velocity [3].
 * nb = 0 detaches.  With a body attached, eddy_substep moves it, regenerates
 * tags and stencils and applies the forcing (the IBM > 1 path). */
int eddy_ib_set_body(eddy_ctx *ctx, int nb, const double *vertices, const double *normals,
                     const double *velocity);
/* Regeneration cadence: every_substep = 1 moves the body over alfxdt and
 * regenerates at every substep (the reference's IBM > 1 path,
 * src/Eddy6.f:2163); 0 (the default) moves it over the whole step and
 * regenerates once, at the first substep. */
int eddy_ib_set_cadence(eddy_ctx *ctx, int every_substep);
/* RBM (src/rbm.f:2): translate the body over tmove. */
int eddy_ib_move(eddy_ctx *ctx, double tmove);
/* LIMIMB, TAG3D_MOD, taguo, geom_mod + mtrx, flagp for the current body
 * position (src/Eddy6.f:2184-2380). */
int eddy_ib_regen(eddy_ctx *ctx);
/* momforc_mod2 on US, VS, WS then velinterior (src/Eddy6.f:2526-2575). */
int eddy_ib_momforc(eddy_ctx *ctx);
/* field EDDY_P: correctpres_mod2 + presinterior (src/Eddy6.f:2881-2897);
 * EDDY_DENS: correctdens_mod2 + densinterior (:2972-2983). */
int eddy_ib_correct(eddy_ctx *ctx, int field);
/* int8 (NX,NY,NZ): which 0..3 = TAG3D results on the u, v, w, p grids
 * (-1 inside, 1 outside); 4..7 = taguo flags u, v, w, tv and 8 = flagp
 * (1 interior, -1 forcing point, 0 fluid). */
int eddy_ib_flags(eddy_ctx *ctx, int which, signed char *out);
/* body index box (LIMIMB): imin imax jmin jmax kmin kmax */
int eddy_ib_limits(eddy_ctx *ctx, int *lim6);
/* Stencils of set q (0 u, 1 v, 2 w, 3 p), ordered by dependency loop: n, the
 * number of loops, forcing points ijk[3n] (1-based), extension offsets
 * dijk[3n] (grid-line stencils; 0 for the others), loop lev[n], body
 * intersection xn[3n], LU factors lu[4n] (column-major a11 a21 a12 a22) and
 * pivots indx[2n] (geom_mod + mtrx, src/devel.f:9265-9800, 1159-1290).  Null
 * arrays are skipped (call once with nulls for n). */
int eddy_ib_stencils(eddy_ctx *ctx, int q, int *n, int *nlev, int *ijk, int *dijk, int *lev, double *xn,
                     double *lu, int *indx);
/* The kind of each stencil of set q, in the order of eddy_ib_stencils:
 * mrk[n] (1 along the body normal, norm_intr src/matint.f:1404; 2 along a
 * grid line, grid_intr :800; 3 through the closest body point, closest_intr
 * :1693), and for kinds 1 and 3 the axis dir[n] (1..3) normal to the fluid
 * cell face the stencil's ray crosses and the crossing point xe[3n], where
 * the forcing interpolates (interp_cellface, src/interp.f:3); dir and xe
 * are 0 for kind 2.  Null arrays are skipped. */
int eddy_ib_stencil_kinds(eddy_ctx *ctx, int q, int *mrk, int *dir, double *xe);

/* Mixed form only (no counterpart in the reference): max |d - L phi| of the
 * last refined Poisson solve before each sweep s, out[s] for s < min(n, 4);
 * entries past refine_sweeps are 0.  EDDY_EINVAL in the plain form. */
int eddy_refine_residuals(eddy_ctx *ctx, double *out, int n);

/* Diagnostics: max |div u| of (UO,VO,WO) over the interior (src/info.f:32). */
int eddy_max_divergence(eddy_ctx *ctx, double *out);
/* CALCFL (src/timestep.f:2-78), Cartesian: the interior maximum of the
 * per-cell max of the convective constraints |u|/dx and the viscous ones
 * 2 (ru1 + tv)/dx^2 per axis (each dropped with its implicit flag); the
 * reference's constant-CFL run takes DTM1 = CFLC / CFLM (src/Eddy6.f:2118). */
int eddy_cfl(eddy_ctx *ctx, double *cflm);
/* SCRINFO's extrema (src/info.f:5-164): min and max of a field over the
 * interior. */
int eddy_field_extrema(eddy_ctx *ctx, int field, double *vmin, double *vmax);

/* Simulation time TIME: eddy_step advances it by dt per step (the RK3 and
 * AB2 coefficients sum to one); set it when starting from a restart. */
int eddy_set_time(eddy_ctx *ctx, double time);
int eddy_get_time(eddy_ctx *ctx, double *time);
/* Time probes on the device (rec_timeprobes_all, src/stats.f:132-185,
 * called every step at src/Eddy6.f:3640): n probe cells ijk[3n] (1-based,
 * the contents of probes.input, src/stats.f:48-66) and room for `capacity`
 * samples.  After every step of eddy_step the cell values of UO, VO, WO and
 * P at each probe are recorded with TIME, on the device; samples past the
 * capacity are dropped.  eddy_probes_read copies up to max_samples samples,
 * out[s][probe][5] = (time, u, v, w, p), consumes them, and returns in
 * *nsamples the number recorded before the read.  n = 0 removes the probes. */
int eddy_probes_set(eddy_ctx *ctx, int n, const int *ijk, int capacity);
int eddy_probes_read(eddy_ctx *ctx, double *out, int max_samples, int *nsamples);
/* One plane of a 3-D field, computed on the device and copied to out
 * (WRITE_PLANES / yface_velocity, src/Planes.f:1-543, without the file):
 * center 0 or 2 the cell values, 1 the average of u over (i-1, i) x (j,
 * j+1), 3 of w over (k-1, k) x (j, j+1) (both 0 outside i, k = 2..N-1 and j
 * = 1..NY-1), 4 the average over (j, j+1) (0 at j = NY); axis 1 the (j, k)
 * plane at i = index (out[NY*NZ]), 2 the (i, k) plane at j = index
 * (out[NX*NZ]), 3 the (i, j) plane at k = index (out[NX*NY]); Fortran order. */
int eddy_plane(eddy_ctx *ctx, int field, int center, int axis, int index, double *out);
/* calcfrc (src/calcforce.f:3-779, Cartesian branch): the force on the body
 * by the control-volume approach on UO, VO, WO, P and the body's flags (no
 * body: all fluid).  cvlim = CVLIM (x1, x2, z1, z2): the volume spans the x
 * faces closest to x1, x2 (closest, src/numrec.f:433) and the z faces that
 * locate (src/numrec.f:390) finds for z1, z2, adjusted as the reference does
 * where it reaches past the domain; faces on the outermost planes are refused
 * (EDDY_EINVAL).  The volume's momentum is kept in the context between calls:
 * the unsteady term is (now - previous) / dt, zero when icycle == 0 (FB of
 * the reference; eddy_body_force_cv_reset clears it).  out[56]: FX(1..6),
 * FY(1..6) (zero in Cartesian coordinates), FZ(1..6) (inlet, outlet, top,
 * bottom, j = 1, j = JY2 faces), the unsteady terms (3), the force on the
 * body -(SUM(F) + unsteady) per component (3), Finlet(1..8), Foutlet(1..8),
 * Ftop(1..8), Fbot(1..8) as the reference writes them to its force files. */
int eddy_body_force_cv(eddy_ctx *ctx, const double *cvlim, double dt, int icycle, double *out);
int eddy_body_force_cv_reset(eddy_ctx *ctx);

/* Kernel-category timing with CUDA events on the context stream (the
 * device-side counterpart of the reference's CLOCK array, src/info.f:350 and
 * src/Eddy6.f:2104-2990).  Categories: 0 RHS+predictor, 1 boundary fills,
 * 2 divergence+forward FFT, 3 forward transform, 4 z line solves,
 * 5 backward transform, 6 backward FFT, 7 CORRECT, 8 pressure update,
 * 9 density, 10 eddy viscosity, 11 refinement residual + forward FFT,
 * 12 FP64/FP32 copies (mixed form), 13 immersed-body regeneration, 14
 * immersed-body forcing, 15 Crank-Nicolson line solves of the velocities
 * (INVERSEY / INVERSEX; the density's run inside category 9).
 * eddy_profile_read synchronises, adds the window's elapsed times per
 * category to ms[16] / counts[16] (cumulative since the mask was set) and
 * starts a new window. */
int eddy_profile_enable(eddy_ctx *ctx, unsigned mask);
int eddy_profile_read(eddy_ctx *ctx, double *ms, long long *counts);

/* Largest grid (NX*NY*NZ, ghost layers included) eddy_max_divergence_noalloc
 * accepts: the size its fixed device scratch array was built for. */
#define EDDY_NOALLOC_MAX_CELLS (1 << 28)

/* No counterpart in the reference.  max |div u| over the interior, like
 * eddy_max_divergence, for callers that cannot call cudaMalloc (memory owned
 * by another allocator, code where allocation is not allowed, or no solver
 * context at all).  Allocates nothing: its scratch is a fixed 512 KiB
 * file-scope device array that every GPU loading this library holds until
 * the process exits.  u, v, w: device arrays (NX,NY,NZ), Fortran order;
 * ap, bp, cp: device copies of the 1-D metric arrays AP(1:NX), BP(1:NY),
 * CP(1:NZ); out: device pointer to one double that receives the result;
 * stream: cudaStream_t (NULL = default stream).  Asynchronous: read out after
 * synchronising the stream.  Returns EDDY_EINVAL when NX*NY*NZ exceeds
 * EDDY_NOALLOC_MAX_CELLS.  The first call in a CUDA context (per device,
 * the primary context in the runtime API) looks up the scratch array's
 * device address for that context, so make that first call before any
 * stream capture.  A launch error left pending on the calling thread by
 * earlier work is cleared on entry; EDDY_ECUDA reports this call's own
 * launches.  All calls share the one scratch array (each call writes
 * every slot it reads, so nothing needs clearing): calls that overlap on the
 * GPU race and must be ordered by the caller. */
int eddy_max_divergence_noalloc(int nx, int ny, int nz, const double *u, const double *v,
                                const double *w, const double *ap, const double *bp,
                                const double *cp, double *out, void *stream);

/* Diagnostic, no counterpart in the reference: one thread of a kernel waits
 * on a barrier that nothing ever completes, through the bounded wait that all
 * of this library's kernels use; *gave_up = 1 when the wait returned without
 * the barrier completing (it should: every wait gives up after 2 s of wall
 * time), *seconds = how long it waited.  Allocates 16 bytes of device memory
 * for the result; takes about 2 s. */
int eddy_selftest_wait_bound(int device, int *gave_up, double *seconds);

/* ---- learned closure (tensor-core MLP), no counterpart in the reference's
 * code: it stands in for the dynamic procedure of src/vt.f:172-431 ---- */
/* Self-test of the BF16 tensor-core GEMM used by the closure's training:
 * D[MxN] (+)= A[MxK] * B[NxK]^T, host arrays (bf16 bit patterns, f32 D). */
int eddy_umma_gemm_bf16(eddy_ctx *ctx, int M, int N, int K, const uint16_t *A, const uint16_t *B,
                        float *D, int acc);

/* Network parameters.  meta (50 floats): feature mean[12], 1/std[12], the
 * training envelope lo[12], hi[12] in normalised units, output scales s_nu,
 * s_kappa.  theta (10448 floats): W1[64][16] b1[64] W2[64][64] b2[64]
 * W3[64][64] b3[64] W4[16][64] b4[16] (inputs 12-15 and outputs 2-15 pad). */
int eddy_closure_set(eddy_ctx *ctx, const float *meta, const float *theta);
int eddy_closure_get(eddy_ctx *ctx, float *meta, float *theta);
/* Raw features (n x 12: 9 velocity gradients * Delta, |grad rho| * Delta,
 * N^2, wall distance) and targets nu_t/Delta (from the current TV) of the
 * given 0-based interior cell indices (i fastest). */
int eddy_closure_harvest(eddy_ctx *ctx, const long long *cells, int n, float *X, float *T);
/* Gradient of the batch loss (n multiple of 128) at the current parameters. */
int eddy_closure_grad(eddy_ctx *ctx, const float *X, const float *Y, int n, float *grad, double *loss);
/* Adam training on the GPU (own tensor-core forward/backward kernels). */
int eddy_closure_train(eddy_ctx *ctx, const float *X, const float *Y, long long n, int epochs, int batch,
                       float lr, unsigned long long seed, double *loss_hist);
/* nu_t -> TV and kappa_t over the field with the fused tensor-core MLP;
 * returns the number of cells outside the training envelope (they take the
 * last dynamic-model value). */
int eddy_closure_apply(eddy_ctx *ctx, long long *out_of_envelope);
/* Recompute the dynamic model (TURVIS) and keep it as the fallback. */
int eddy_closure_refresh_fallback(eddy_ctx *ctx);
int eddy_download_kappa(eddy_ctx *ctx, double *host);

int eddy_sync(eddy_ctx *ctx);
/* Copy the last error message (NUL-terminated, truncated to len). */
int eddy_last_error(eddy_ctx *ctx, char *buf, int len);
/* Number of kernels this context has launched since creation. */
int64_t eddy_launch_count(eddy_ctx *ctx);
/* The context's CUDA stream (cudaStream_t) for callers that synchronise. */
void *eddy_stream(eddy_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
