// k_density.cu -- density equation: RHS_DENSITY (src/rhs_density.f:4-175)
// fused with DENSITY (src/density.f:6-99) and its sponges, plus the
// BOUNDINOUTD / BOUNDARY_DENS ghost fills (src/boundary.f:2001-2281).
// Explicit form: the Crank-Nicolson part RS is zero in the interior and the
// update, its sponges and the ghost copy run in one pass.  With IMPLY = 1
// (IMPLX = 1) the y (x) diffusion is the C.N. part: the predicted density
// goes to RS, INVERSEYD (INVERSEXD) solves its lines, DENS = RS over the whole
// array (density.f:89-104, so the ghost cells take RS's, which only
// BOUNDARY_DENS writes: at slip walls (type 60) the x ghosts become zero, as
// in the reference), then the sponges.
#include "eddy_internal.h"
#include "tma_ring.cuh"
#include "bc_templates.cuh"
#include "stencil_density.cuh"


namespace {


// New density into dn (ping-pong).  Interior: TMA plane ring over
// dens, tv, uo, vo, wo, rha (tma_ring.cuh); the ghost cells of dn are copied
// from the old buffer by k_dens_ghost_copy.
constexpr int DTX = 32, DTY = 8, DKC = 32, DNF = 6;  // dens tv uo vo wo rha

__global__ void __launch_bounds__(DTX *DTY)
    k_density(Dims d, DevMetrics m, Scalars s, const __grid_constant__ TmaMaps<DNF> maps, double *__restrict__ rha,
              double *__restrict__ dn, double repr1, double alfxdt, double gamxdt, double rhoxdt, int *err) {
  tma_march<DNF, DTX, DTY, DKC>(
      d.ix1, d.ix2, d.jy1, d.jy2, d.kz1, d.kz2, maps, err,
      [&](int i, int j, int k, bool active, const RingAcc<DTX, DTY, DNF> &S) {
        if (!active) return;
        double rr = rhs_dens<double>(S, m, repr1, i, j, k);
        double coef = 0.5 * alfxdt;
        double dnew = S.at(0, 0, 0, 0) + gamxdt * rr + rhoxdt * S.at(5, 0, 0, 0) + coef * 0.0;
        long long q = fidx(d, i, j, k);
        rha[q] = rr;
        double bg = m.dens_bg[(i - 1) + d.nx * (j - 1)];
        if (s.idspngl == 1) dnew = dnew + m.dfxdl[k] * (bg - dnew) * alfxdt * 1.0;
        if (i >= d.ix2 - s.dspngx1) dnew = dnew + m.dfxd[i] * (bg - dnew) * alfxdt * 1.0;
        dn[q] = dnew;
      });
}

// any of IMPLX, IMPLY, IMPLCX, IMPLCY = 1: RHS_DENSITY with the terms the flags
// in f name as the C.N. part rt, the DENSITY update with +coef*rt, no sponges
// yet; the predicted density to rs
__global__ void __launch_bounds__(DTX *DTY)
    k_density_cn(Dims d, DevMetrics m, const __grid_constant__ TmaMaps<DNF> maps, double *__restrict__ rha,
                 double *__restrict__ rs, double repr1, double alfxdt, double gamxdt, double rhoxdt, int *err,
                 CnFlags<double> f) {
  tma_march<DNF, DTX, DTY, DKC>(
      d.ix1, d.ix2, d.jy1, d.jy2, d.kz1, d.kz2, maps, err,
      [&](int i, int j, int k, bool active, const RingAcc<DTX, DTY, DNF> &S) {
        if (!active) return;
        double rt = 0.;
        double rr = rhs_dens<double, DevMetrics, RingAcc<DTX, DTY, DNF>, true>(S, m, repr1, i, j, k, &rt, &f);
        double coef = 0.5 * alfxdt;
        double dnew = S.at(0, 0, 0, 0) + gamxdt * rr + rhoxdt * S.at(5, 0, 0, 0) + coef * rt;
        long long q = fidx(d, i, j, k);
        rha[q] = rr;
        rs[q] = dnew;
      });
}

// the density sponges (density.f:103-127) on the interior
__global__ void __launch_bounds__(256) k_dens_sponge(Dims d, DevMetrics m, Scalars s, double *dens, double alfxdt) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int mi = d.ix2 - d.ix1 + 1, mj = d.jy2 - d.jy1 + 1, mk = d.kz2 - d.kz1 + 1;
  if (t >= (long long)mi * mj * mk) return;
  const int i = d.ix1 + (int)(t % mi), j = d.jy1 + (int)((t / mi) % mj), k = d.kz1 + (int)(t / ((long long)mi * mj));
  const long long q = fidx(d, i, j, k);
  const double bg = m.dens_bg[(i - 1) + d.nx * (j - 1)];
  double v = dens[q];
  if (s.idspngl == 1) v = v + m.dfxdl[k] * (bg - v) * alfxdt * 1.0;
  if (i >= d.ix2 - s.dspngx1) v = v + m.dfxd[i] * (bg - v) * alfxdt * 1.0;
  dens[q] = v;
}

__global__ void k_dens_ghost_copy(Dims d, const double *__restrict__ dens, double *__restrict__ dn) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long sxy = (long long)d.nx * d.ny, sxz = (long long)d.nx * d.nz, syz = (long long)d.ny * d.nz;
  int i, j, k;
  if (t < 2 * sxy) {
    long long r = t % sxy;
    i = 1 + (int)(r % d.nx); j = 1 + (int)(r / d.nx); k = (t / sxy) ? d.nz : 1;
  } else if (t < 2 * sxy + 2 * sxz) {
    long long u = t - 2 * sxy, r = u % sxz;
    i = 1 + (int)(r % d.nx); k = 1 + (int)(r / d.nx); j = (u / sxz) ? d.ny : 1;
  } else if (t < 2 * sxy + 2 * sxz + 2 * syz) {
    long long u = t - 2 * sxy - 2 * sxz, r = u % syz;
    j = 1 + (int)(r % d.ny); k = 1 + (int)(r / d.ny); i = (u / syz) ? d.nx : 1;
  } else {
    return;
  }
  long long q = fidx(d, i, j, k);
  dn[q] = dens[q];
}

}  // namespace

// BOUNDINOUTD (src/boundary.f:2241-2281) then BOUNDARY_DENS (:2001-2044)
int launch_boundinoutd_dens(eddy_ctx *ctx, double *dens) {
  return bc_boundinoutd_dens<double>(ctx, ctx->d.nx, dens);
}

int launch_density(eddy_ctx *ctx, double alfxdt, double gamxdt, double rhoxdt) {
  const Dims &d = ctx->d;
  int rc = launch_boundinoutd_dens(ctx, ctx->f[EDDY_DENS]);
  if (rc) return rc;
  double repr1 = ctx->sc.ru1 / ctx->sc.prn;
  TmaMaps<DNF> maps;
  // eddy diffusivity: the dynamic model's nu_t (kappa_t = nu_t, src/Eddy6.f:2959)
  // or the learned closure's kappa_t
  const double *kv = ctx->prm.closure == 1 ? ctx->kappa : ctx->f[EDDY_TV];
  const double *src[DNF] = {ctx->f[EDDY_DENS], kv, ctx->f[EDDY_UO], ctx->f[EDDY_VO], ctx->f[EDDY_WO],
                            ctx->f[EDDY_RHA]};
  for (int q = 0; q < DNF; q++) {
    const CUtensorMap *mp = ctx_tensor_map(ctx, src[q], RingGeom<DTX, DTY>::PX, DTY + 2);
    if (!mp) return EDDY_ECUDA;
    maps.m[q] = *mp;
  }
  size_t smem = ring_smem_bytes<DNF, DTX, DTY>();
  dim3 g((d.ix2 - d.ix1 + DTX) / DTX, (d.jy2 - d.jy1 + DTY) / DTY, (d.kz2 - d.kz1 + DKC) / DKC);
  const Scalars &sc = ctx->sc;
  const CnFlags<double> fl{(double)sc.implx, (double)sc.imply, (double)sc.implcx, (double)sc.implcy};
  if (sc.imply == 1 || sc.implx == 1 || sc.implcx == 1 || sc.implcy == 1) {
    EDDY_CUDA(cudaFuncSetAttribute(k_density_cn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_density_cn<<<g, dim3(DTX, DTY), smem, ctx->stream>>>(d, ctx->m, maps, ctx->f[EDDY_RHA], ctx->f[EDDY_RS], repr1,
                                                          alfxdt, gamxdt, rhoxdt, ctx->err_flag, fl);
    EDDY_LAUNCHED(ctx);
    // INVERSEYD_NEW (IMPLY and IMPLCY) or INVERSEYD (IMPLY), then INVERSEXD
    // (IMPLX or IMPLCX) on RS, each followed by DENS = RS in the reference
    // (density.f:89-104); nothing reads DENS between, so one copy.  With IMPLCY
    // alone the density has no line solve and no whole-array copy: the new
    // interior lands in DENS, which keeps its own ghost cells, as there.
    const bool ysolve = sc.imply == 1, xsolve = sc.implx == 1 || sc.implcx == 1;
    if (ysolve)
      if ((rc = sc.implcy == 1 ? launch_inverseyd_new(ctx, alfxdt) : launch_inverseyd(ctx, alfxdt))) return rc;
    if (xsolve)
      if ((rc = launch_inversexd(ctx, alfxdt))) return rc;
    if (!ysolve && !xsolve) {
      const long long ng = 2LL * d.nx * d.ny + 2LL * d.nx * d.nz + 2LL * d.ny * d.nz;
      k_dens_ghost_copy<<<(unsigned)((ng + 255) / 256), 256, 0, ctx->stream>>>(d, ctx->f[EDDY_DENS],
                                                                               ctx->f[EDDY_RS]);
      EDDY_LAUNCHED(ctx);
    }
    EDDY_CUDA(cudaMemcpyAsync(ctx->f[EDDY_DENS], ctx->f[EDDY_RS], sizeof(double) * (size_t)d.ncell,
                              cudaMemcpyDeviceToDevice, ctx->stream));
    const long long ni = (long long)(d.ix2 - d.ix1 + 1) * (d.jy2 - d.jy1 + 1) * (d.kz2 - d.kz1 + 1);
    k_dens_sponge<<<(unsigned)((ni + 255) / 256), 256, 0, ctx->stream>>>(d, ctx->m, ctx->sc, ctx->f[EDDY_DENS],
                                                                          alfxdt);
    EDDY_LAUNCHED(ctx);
    if ((rc = launch_boundinoutd_dens(ctx, ctx->f[EDDY_DENS]))) return rc;
    // immersed body: correctdens_mod2 + densinterior (src/Eddy6.f:2972-2983)
    if (ctx->ib) return ib_force(ctx, 3, 4, ctx->f[EDDY_DENS], 0.0, 0.0, nullptr, 0);
    return EDDY_OK;
  }
  EDDY_CUDA(cudaFuncSetAttribute(k_density, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_density<<<g, dim3(DTX, DTY), smem, ctx->stream>>>(d, ctx->m, ctx->sc, maps, ctx->f[EDDY_RHA], ctx->dens_alt,
                                                     repr1, alfxdt, gamxdt, rhoxdt, ctx->err_flag);
  EDDY_LAUNCHED(ctx);
  long long nghost = 2LL * d.nx * d.ny + 2LL * d.nx * d.nz + 2LL * d.ny * d.nz;
  k_dens_ghost_copy<<<(unsigned)((nghost + 255) / 256), 256, 0, ctx->stream>>>(d, ctx->f[EDDY_DENS], ctx->dens_alt);
  EDDY_LAUNCHED(ctx);
  double *t = ctx->f[EDDY_DENS];
  ctx->f[EDDY_DENS] = ctx->dens_alt;
  ctx->dens_alt = t;
  if ((rc = launch_boundinoutd_dens(ctx, ctx->f[EDDY_DENS]))) return rc;
  // immersed body: correctdens_mod2 + densinterior (src/Eddy6.f:2972-2983)
  if (ctx->ib) return ib_force(ctx, 3, 4, ctx->f[EDDY_DENS], 0.0, 0.0, nullptr, 0);
  return EDDY_OK;
}
