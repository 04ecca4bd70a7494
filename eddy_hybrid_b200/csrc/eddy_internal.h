// eddy_internal.h -- context layout and kernel launch declarations shared by
// the CUDA translation units of libeddy_b200.so.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <thread>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/eddy_b200.h"

// 1-D metric arrays on the device, indexed 1-based like the Fortran
// (entry 0 unused), sizes nx+2 / ny+2 / nz+2.
struct DevMetrics {
  double *ap, *au, *av, *aw;
  double *bp, *bu, *bv, *bw;
  double *cp, *cu, *cv, *cw;
  double *whx, *why, *whz;  // [i*3 + d+1]
  double *dfxu, *dfxw, *dfxul, *dfxwl, *dfxd, *dfxdl;
  double *dens_bg;  // (NX,NY)
};

// Integer bounds (src/setup.f, src/inpall.f:166-172) and scalars the kernels
// read; passed by value.
struct Dims {
  int nx, ny, nz;
  int ix1, ix2, jy1, jy2, kz1, kz2;
  int ibu, ieu, jbv, jev, kbw, kew;
  int mp, lp, np;
  int itype[7];
  long long ncell;  // nx*ny*nz
};

struct Scalars {
  double ru1, prn, grav, dpdx, dpdy, dpdz, eps, css;
  int vspngx1, dspngx1, ivspngl, idspngl, idens, isgs;
  int imply;  // IMPLY: Crank-Nicolson viscous terms along y
  int implx;  // IMPLX: Crank-Nicolson viscous terms along x
  int implcx, implcy;  // IMPLCX, IMPLCY: Crank-Nicolson convective terms along x, y
};

// Poisson plan (src/direct.f SAVE state): eigen-transform of the x operator.
struct PoissonPlan {
  int M, L, N;          // interior sizes along x, y (FFT), z
  int m0;               // index of the null x-mode
  double *Af, *Ab;      // forward/backward transform matrices (M x M, col-major)
  // FP64 tensor-core transforms (k_xform64.cu): matrices [chunk][row][8] for
  // the forward (0) and backward (1) directions, split into even and odd
  // modes when the x operator is mirror-symmetric (dsym); dHp the padded half
  // size (full size when not split); eigenvalues and null mode in that order
  double *dA[2];
  double *dlam;
  int dsym, dHp, dm0;
  double *lam;          // eigenvalues of the x operator (M)
  double *ak;           // modified wavenumber AK(J/2+1) per packed index (L)
  double *an, *bn, *cn; // z operator (N)
  double *wz;           // 1/cp(k): z cell widths for the compatibility projection
  double *twr, *twi;    // FFT twiddles exp(-2 pi i q/L), q < L/2
  double *spec, *spec2; // spectral work arrays, M*L*N each
  double *cprime;       // Thomas scratch, M*L*N
  double *red;          // reduction scratch
};

// kernel categories timed with CUDA events when profiling is enabled
enum {
  PROF_RHS_PRED = 0, PROF_BC, PROF_DIV_FFT, PROF_GEMM_FWD, PROF_TRIDIAG, PROF_GEMM_BWD, PROF_FFT_BWD,
  PROF_CORRECT, PROF_PUPDATE, PROF_DENSITY, PROF_TURVIS, PROF_REFINE, PROF_CONVERT, PROF_IB_REGEN,
  PROF_IB_FORCE, PROF_CN_LINES, PROF_NCAT
};

struct TmaEntry {
  const void *ptr;
  int bx, by;
  alignas(64) CUtensorMap map;
};

struct ProfEvent {
  int cat;
  cudaEvent_t a, b;
};

struct eddy_ctx {
  int device = 0;
  eddy_params prm{};
  Dims d{};
  Scalars sc{};
  cudaStream_t stream = nullptr;
  // immersed-body regeneration overlapped with the predictor: second stream,
  // [0] recorded on the main stream before the predictor, [1] on ib_stream
  // after the regeneration; ib_pending: the main stream has not yet waited [1]
  cudaStream_t ib_stream = nullptr;
  cudaEvent_t ib_ev[2] = {};
  int ib_pending = 0;
  double ib_move_dt = -1.0;  // >= 0: move over this time and regenerate in this substep
  int ib_prefetched = 0;     // the next step's move and regeneration are already queued
  DevMetrics m{};
  // host copies of the 1-D arrays (1-based, size n+2)
  std::vector<double> h[28];
  // fields (device, FP64, Fortran layout)
  double *f[EDDY_NFIELDS] = {};
  double *dens_alt = nullptr;  // ping-pong partner of DENS
  // dynamic procedure: |S| (NX,NY,NZ), Delta^2 (NX,NY,NZ), y averages of
  // max(L.M,0) and M.M ((NX,NZ)); the FP32 procedure of the mixed form uses
  // the same allocations as FP32 storage
  double *gs = nullptr, *dxdydz = nullptr, *ilm2 = nullptr, *imm2 = nullptr;
  double *diag = nullptr;  // diagnostics scratch (k_diag.cu): 2*296 partials + 2 results
  double *scal = nullptr;  // device scalars: [0] pref [1] qin1 [2] qin2 [3] dpm [4] maxdiv; [32, 328) flux partials
  PoissonPlan pp{};
  std::string err;
  std::atomic<int64_t> launches{0};
  // the prefetched immersed-body regeneration runs its host side on a helper
  // thread (its launches go to ib_stream); joined before the body is used
  std::thread ib_thread;
  int ib_thread_rc = 0;
  double dely = 0., delysq = 0.;
  double alfxdt_last = 0.;  // alfxdt of the last CORRECT (the IMPLY pressure correction)
  // hybrid inflow sequence (device-resident): feed_n planes [n][4][NX*NY] of
  // u, v, w, rho in feed order; x indices >= feed_iref take the last plane;
  // icycle is the driver's step counter (src/Eddy6.f:2095)
  double *feed = nullptr;
  int feed_n = 0, feed_iref = 0, icycle = 0;
  double time = 0.;  // TIME: advanced by DTM1 per step in eddy_step
  // time probes (rec_timeprobes_all): probe cells (1-based ijk), and a
  // device buffer of samples [cap][n][5] (time, u, v, w, p), count recorded
  int *probe_ijk = nullptr;
  double *probe_buf = nullptr;
  int nprobe = 0, probe_cap = 0, probe_count = 0;
  double *plane_buf = nullptr;  // staging of eddy_plane (the largest plane of the grid)
  // control-volume body force (k_force.cu): partial sums, and the volume's
  // momentum of the previous call (FB of calcfrc)
  double *cv_buf = nullptr;
  double cv_fb[3] = {0., 0., 0.};
  double *xc_dev = nullptr;     // x cell centres (1-based, NX+2)
  double *kappa = nullptr;      // eddy diffusivity of the learned closure (NX,NY,NZ)
  double *tv_dyn = nullptr;     // last dynamic-model nu_t: closure fallback (NX,NY,NZ)
  void *mlp = nullptr;          // closure network state (k_mlp.cu)
  void *mixed = nullptr;        // FP32 field set of the mixed-precision form (k_mixed.cu)
  void *ib = nullptr;           // immersed body state (k_ib.cu)
  double *ibax[6] = {};         // device xu, xc, yv, yc, zw, zc (1-based) for the body kernels
  long long closure_out = 0, closure_cells = 0, closure_refresh = 0;
  // profiling (CUDA events on the context stream around each category)
  unsigned prof_mask = 0;
  std::vector<ProfEvent> prof_ev;   // recorded in this window
  std::vector<ProfEvent> prof_pool; // reusable events
  std::mutex prof_mu;               // the helper thread records events too
  double prof_ms[PROF_NCAT] = {};
  int *err_flag = nullptr;            // device word set by kernels whose bounded waits expire
  std::vector<TmaEntry> tmaps;        // cached tensor maps per (field pointer, box)
  long long prof_n[PROF_NCAT] = {};
};

// The stream the calling host thread issues work to: the context's main
// stream, or the one a scope set (the immersed-body regeneration's).
extern thread_local cudaStream_t tl_stream;
inline cudaStream_t cur_stream(const eddy_ctx *ctx) { return tl_stream ? tl_stream : ctx->stream; }
struct StreamScope {
  cudaStream_t prev;
  explicit StreamScope(cudaStream_t s) : prev(tl_stream) { tl_stream = s; }
  ~StreamScope() { tl_stream = prev; }
};

// RAII scope: records a start event now and a stop event at scope exit when
// the category is enabled (on the calling thread's stream).
struct ProfScope {
  eddy_ctx *c;
  int cat;
  bool on;
  cudaStream_t st;
  ProfEvent ev{};
  ProfScope(eddy_ctx *ctx, int category)
      : c(ctx), cat(category), on((ctx->prof_mask >> category) & 1u), st(cur_stream(ctx)) {
    if (!on) return;
    {
      std::lock_guard<std::mutex> lk(c->prof_mu);
      if (!c->prof_pool.empty()) {
        ev = c->prof_pool.back();
        c->prof_pool.pop_back();
      }
    }
    if (!ev.a) {
      cudaEventCreate(&ev.a);
      cudaEventCreate(&ev.b);
    }
    ev.cat = cat;
    cudaEventRecord(ev.a, st);
  }
  ~ProfScope() {
    if (!on) return;
    cudaEventRecord(ev.b, st);
    std::lock_guard<std::mutex> lk(c->prof_mu);
    c->prof_ev.push_back(ev);
  }
};

#define EDDY_CUDA(call)                                                     \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);        \
      return EDDY_ECUDA;                                                    \
    }                                                                       \
  } while (0)

#define EDDY_LAUNCHED(ctx)                                                  \
  do {                                                                      \
    cudaError_t e_ = cudaGetLastError();                                    \
    (ctx)->launches++;                                                      \
    if (e_ != cudaSuccess) {                                                \
      (ctx)->err = std::string("kernel launch: ") + cudaGetErrorString(e_); \
      return EDDY_ECUDA;                                                    \
    }                                                                       \
  } while (0)

// Fortran (i,j,k) 1-based -> linear index
__host__ __device__ inline long long fidx(const Dims &d, int i, int j, int k) {
  return (long long)(i - 1) + (long long)d.nx * ((long long)(j - 1) + (long long)d.ny * (long long)(k - 1));
}

// the same for an array with row pitch `pitch` (the mixed form's FP32 arrays)
__host__ __device__ inline long long pidx(const Dims &d, int pitch, int i, int j, int k) {
  return (long long)(i - 1) + (long long)pitch * ((long long)(j - 1) + (long long)d.ny * (long long)(k - 1));
}

// tensor map over an (NX,NY,NZ) FP64 field with a (bx,by,1) box, cached per
// pointer; nullptr on failure (message in ctx->err)
const CUtensorMap *ctx_tensor_map(eddy_ctx *ctx, const double *ptr, int bx, int by);

// kernel drivers (each returns EDDY_* status)
int launch_rhs_predictord(eddy_ctx *ctx, double alfxdt, double gamxdt, double rhoxdt);
int launch_boundary(eddy_ctx *ctx, double *u, double *v, double *w);
int launch_boundinout(eddy_ctx *ctx, double *ubc, double *vbc, double *wbc, const double *uof,
                      const double *vof, const double *wof, double alfxdt, int idiv);
int launch_correct(eddy_ctx *ctx, double alfxdt);
int launch_pressure_update(eddy_ctx *ctx);
int launch_density(eddy_ctx *ctx, double alfxdt, double gamxdt, double rhoxdt);
int launch_boundinoutd_dens(eddy_ctx *ctx, double *dens);
int launch_turvis(eddy_ctx *ctx);
// Crank-Nicolson y lines (k_implicit.cu): INVERSEY on US, VS, WS and
// INVERSEYD on RS (IMPLY = 1)
int launch_inversey(eddy_ctx *ctx, double alfxdt);
int launch_inverseyd(eddy_ctx *ctx, double alfxdt);
int launch_inverseyd_new(eddy_ctx *ctx, double alfxdt);
int launch_inversex(eddy_ctx *ctx, double alfxdt);
int launch_inversexd(eddy_ctx *ctx, double alfxdt);
// FP32 dynamic procedure on FP32 velocities (row pitch px) -> TV (FP64)
int launch_turvis32(eddy_ctx *ctx, int px, const float *u, const float *v, const float *w, float *gs32,
                    float *imm32, float *ilm32);
int launch_filtersize(eddy_ctx *ctx);
int poisson_plan_create(eddy_ctx *ctx);
int poisson_plan_destroy(eddy_ctx *ctx);
// divergence/alfxdt of (us,vs,ws) -> solve -> DP (device), DIRECT semantics
int launch_direct(eddy_ctx *ctx, const double *us, const double *vs, const double *ws,
                  double alfxdt);
// solve from an explicit right-hand side array (interior of rhs) -> dp
int launch_poisson_rhs(eddy_ctx *ctx, const double *rhs, double *dp);
int launch_max_divergence(eddy_ctx *ctx, double *out_host);
// DIRECT's ghost convention on a solution array (z planes zero, x Neumann, y periodic)
int launch_dp_ghost(eddy_ctx *ctx, double *dp);

// immersed boundary (k_ib.cu).  Stencil sets q: 0 u, 1 v, 2 w, 3 p; flag
// arrays fq: 0 u, 1 v, 2 w, 3 tv (taguo), 4 p (flagp)
int ib_set_body(eddy_ctx *ctx, int nb, const double *vert, const double *normals, const double *vel);
int ib_release(eddy_ctx *ctx);
int ib_move(eddy_ctx *ctx, double tmove);
int ib_regen(eddy_ctx *ctx);
// forcing of a by set q, then `interior` where flag fq == 1; mirror (FP32,
// row pitch mpitch) receives every written value when non-null
int ib_force(eddy_ctx *ctx, int q, int fq, double *a, double b0, double interior, float *mirror, int mpitch);
int ib_force32(eddy_ctx *ctx, int q, int fq, float *a, int pitch, double b0, double interior);
// the implicit forcing of the C.N. steps (impl = 1): stencil values from ub
// (the explicit estimate), a + b(1) - ub at the forcing points (ub takes it
// too), a - ub + b0 inside the body
int ib_force_impl(eddy_ctx *ctx, int q, int fq, double *a, double *ub, double b0);
const double *ib_velocity(eddy_ctx *ctx);
int ib_set_cadence(eddy_ctx *ctx, int every_substep);
int ib_every_substep(eddy_ctx *ctx);
int ib_interior(eddy_ctx *ctx, int fq, double *a, double value, float *mirror = nullptr, int mpitch = 0);
// the move and regeneration due in this substep (ctx->ib_move_dt), on
// ctx->ib_stream after ctx->ib_ev[0], overlapping work queued on the main
// stream since; ib_join makes the main stream wait for it
int ib_overlap_regen(eddy_ctx *ctx);
int ib_join(eddy_ctx *ctx);
int ib_prefetch_async(eddy_ctx *ctx, double tmove);
// the tv flag (fq = 3) is double-buffered so the next step's regeneration can
// run while tvinterior still reads the current one: swap before it
int ib_swap_tv_flag(eddy_ctx *ctx);
int ib_download(eddy_ctx *ctx, int which, signed char *out);
int ib_limits(eddy_ctx *ctx, int *lim6);
int ib_stencils(eddy_ctx *ctx, int q, int *n, int *nlev, int *ijk, int *dijk, int *lev, double *xn, double *lu,
                int *indx);
int ib_stencil_kinds(eddy_ctx *ctx, int q, int *mrk, int *dir, double *xe);
// the device flag array fq of the body (nullptr without one)
const signed char *ib_flag_dev(eddy_ctx *ctx, int fq);
int probes_record(eddy_ctx *ctx);

// tensor-core (3xTF32) eigen-transforms of the mixed solve (k_xform.cu).
// sym: mirror-symmetric split form, modes ordered even then odd; lam and m0
// are the eigenvalues and the null mode in the transform's mode order.
struct XformPlan {
  int sym = 0;
  // forward / backward matrices, TF32 hi and lo interleaved in streaming order
  float *fmat = nullptr, *bmat = nullptr;
  double *lam = nullptr;
  int m0 = 0;
};
bool xform_supported(int M);
int xform_prepare(eddy_ctx *ctx, XformPlan *xp);
void xform_release(XformPlan *xp);
// dir 0: x values -> mode coefficients; 1: back
int launch_xform(eddy_ctx *ctx, const XformPlan *xp, int dir, const float *in, float *out);
// FP64 tensor-core transforms over the L*N spectral lines (k_xform64.cu), dir
// 0 forward, 1 backward, in the mode order of pp.dlam / pp.dm0; FP64 or FP32
// storage, FP64 arithmetic
int xform64_prepare(eddy_ctx *ctx, const std::vector<double> &Af, const std::vector<double> &Ab,
                    const std::vector<double> &lam);
int launch_xform64(eddy_ctx *ctx, int dir, const double *in, double *out);
int launch_xform64_f32(eddy_ctx *ctx, int dir, const float *in, float *out);

// mixed-precision form (k_mixed.cu): FP32 stencils and FFTs, FP64 line solves,
// FP64-residual iterative refinement, FP64 projection onto FP64 master velocities
int mixed_create(eddy_ctx *ctx);
void mixed_release(eddy_ctx *ctx);
// refresh the FP32 copy of `field` from its FP64 array (after an upload)
int mixed_from64(eddy_ctx *ctx, int field);
// write the FP64 array of `field` from its FP32 master (before a download)
int mixed_to64(eddy_ctx *ctx, int field);
int mixed_substep(eddy_ctx *ctx, double alfxdt, double gamxdt, double rhoxdt);
// FP32 arrays of the mixed form the learned closure reads and writes
struct MixedViews {
  const float *uo, *vo, *wo, *dens;
  float *tv, *kv;
  int px;
};
int mixed_views(eddy_ctx *ctx, MixedViews *v);
// mixed Poisson solve of L dp = rhs (rhs, dp FP64 device arrays)
int mixed_poisson_rhs(eddy_ctx *ctx, const double *rhs, double *dp);
// max |residual| before each refinement sweep of the last mixed solve (host copy)
int mixed_residuals(eddy_ctx *ctx, double *out, int n);
// around an eddy-viscosity update: FP64 density for the closure features
// before, FP32 copies of nu_t / kappa_t after
int mixed_after_sgs(eddy_ctx *ctx);
// the eddy viscosity of the mixed form: the dynamic procedure in FP32 on the
// FP32 velocities (Smagorinsky stays FP64) -> TV
int mixed_turvis(eddy_ctx *ctx);
int launch_closure(eddy_ctx *ctx, const double *fallback, double *kappa, unsigned long long *out_of_envelope);
void mlp_release(eddy_ctx *ctx);

// host-side symmetric tridiagonal eigensolver (implicit QL with Wilkinson shift)
int tridiag_eigen(int n, std::vector<double> &d, std::vector<double> &e, std::vector<double> &q);
