// k_density.cu -- density equation: RHS_DENSITY (src/rhs_density.f:4-175)
// fused with DENSITY (src/density.f:6-99) and its sponges, plus the
// BOUNDINOUTD / BOUNDARY_DENS ghost fills (src/boundary.f:2001-2281).
// Explicit form: the Crank-Nicolson part RS is zero in the interior.
#include "eddy_internal.h"
#include "tma_ring.cuh"


int launch_fill_plane(eddy_ctx *ctx, double *a, int axis, int dst, int src, double sgn, int zero);

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
        auto dens = [&](int a, int b, int c) { return S.at(0, a, b, c); };
        auto kv = [&](int a, int b, int c) { return S.at(1, a, b, c); };
        double qxp = S.at(2, 0, 0, 0), qxm = S.at(2, -1, 0, 0);
        double rxp = (dens(1, 0, 0) + dens(0, 0, 0)) * 0.5;
        double rxm = (dens(0, 0, 0) + dens(-1, 0, 0)) * 0.5;
        double vyp = S.at(3, 0, 0, 0), vym = S.at(3, 0, -1, 0);
        double ryp = (dens(0, 1, 0) + dens(0, 0, 0)) * 0.5;
        double rym = (dens(0, 0, 0) + dens(0, -1, 0)) * 0.5;
        double wzp = S.at(4, 0, 0, 0), wzm = S.at(4, 0, 0, -1);
        double rzp = (dens(0, 0, 1) + dens(0, 0, 0)) * 0.5;
        double rzm = (dens(0, 0, 0) + dens(0, 0, -1)) * 0.5;
        double drdxp = m.au[i] * (dens(1, 0, 0) - dens(0, 0, 0));
        double drdxm = m.au[i - 1] * (dens(0, 0, 0) - dens(-1, 0, 0));
        double drdyp = m.bv[j] * (dens(0, 1, 0) - dens(0, 0, 0));
        double drdym = m.bv[j - 1] * (dens(0, 0, 0) - dens(0, -1, 0));
        double drdzp = m.cw[k] * (dens(0, 0, 1) - dens(0, 0, 0));
        double drdzm = m.cw[k - 1] * (dens(0, 0, 0) - dens(0, 0, -1));
        double kvip = 0.5 * (kv(1, 0, 0) + kv(0, 0, 0));
        double kvim = 0.5 * (kv(-1, 0, 0) + kv(0, 0, 0));
        double kvjp = 0.5 * (kv(0, 1, 0) + kv(0, 0, 0));
        double kvjm = 0.5 * (kv(0, -1, 0) + kv(0, 0, 0));
        double kvkp = 0.5 * (kv(0, 0, 1) + kv(0, 0, 0));
        double kvkm = 0.5 * (kv(0, 0, -1) + kv(0, 0, 0));
        double txxp = (repr1 + kvip) * drdxp;
        double txxm = (repr1 + kvim) * drdxm;
        double tyyp = (repr1 + kvjp) * drdyp;
        double tyym = (repr1 + kvjm) * drdym;
        double tzzp = (repr1 + kvkp) * drdzp;
        double tzzm = (repr1 + kvkm) * drdzm;
        double h11 = -m.ap[i] * (rxp * qxp - rxm * qxm);
        double h22 = -m.bp[j] * (ryp * vyp - rym * vym);
        double h33 = -m.cp[k] * (rzp * wzp - rzm * wzm);
        double t11 = m.ap[i] * (txxp - txxm);
        double t22 = m.bp[j] * (tyyp - tyym);
        double t33 = m.cp[k] * (tzzp - tzzm);
        double rr = h11 + h22 + h33 + t11 + t22 + t33;
        double coef = 0.5 * alfxdt;
        double dnew = dens(0, 0, 0) + gamxdt * rr + rhoxdt * S.at(5, 0, 0, 0) + coef * 0.0;
        long long q = fidx(d, i, j, k);
        rha[q] = rr;
        double bg = m.dens_bg[(i - 1) + d.nx * (j - 1)];
        if (s.idspngl == 1) dnew = dnew + m.dfxdl[k] * (bg - dnew) * alfxdt * 1.0;
        if (i >= d.ix2 - s.dspngx1) dnew = dnew + m.dfxd[i] * (bg - dnew) * alfxdt * 1.0;
        dn[q] = dnew;
      });
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

__global__ void k_dens_inlet(Dims d, double *dens, const double *plane) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.nx * d.ny) return;
  dens[t] = plane[t];
}

}  // namespace

// BOUNDINOUTD (src/boundary.f:2241-2281) then BOUNDARY_DENS (:2001-2044)
int launch_boundinoutd_dens(eddy_ctx *ctx, double *dens) {
  const Dims &d = ctx->d;
  int rc;
#define F(...) \
  if ((rc = launch_fill_plane(ctx, __VA_ARGS__)) != EDDY_OK) return rc
  if (d.itype[5] == 305) {
    k_dens_inlet<<<(d.nx * d.ny + 255) / 256, 256, 0, ctx->stream>>>(d, dens, ctx->f[EDDY_PLANED]);
    EDDY_LAUNCHED(ctx);
    F(dens, 2, 2, 1, 1., 0);
  }
  if (d.itype[6] == 730) { F(dens, 2, d.kz2, d.kz2 - 1, 1., 0); F(dens, 2, d.nz, d.kz2, 1., 0); }
  if (d.itype[6] == 710) F(dens, 2, d.kz2, d.kz2 - 1, 1., 0);
  // BOUNDARY_DENS
  for (int ib = 1; ib <= 6; ib++) {
    int t = d.itype[ib];
    if (t == 50) {
      ctx->err = "density wall type 50 is not on the restated hot path";
      return EDDY_EINVAL;
    } else if (t == 80 || t == 82) {
      if (ib == 1) F(dens, 0, 1, d.ix1, 1., 0);
      if (ib == 2) { F(dens, 0, d.ix2, d.ix2 - 1, 1., 0); F(dens, 0, d.nx, d.ix2, 1., 0); }
    }
  }
  if (d.itype[1] == 500) { F(dens, 0, 1, d.ix2, 1., 0); F(dens, 0, d.nx, d.ix1, 1., 0); }
  if (d.itype[3] == 500) { F(dens, 1, 1, d.jy2, 1., 0); F(dens, 1, d.ny, d.jy1, 1., 0); }
  if (d.itype[5] == 500) { F(dens, 2, 1, d.kz2, 1., 0); F(dens, 2, d.nz, d.kz1, 1., 0); }
#undef F
  return EDDY_OK;
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
    const CUtensorMap *mp = ctx_tensor_map(ctx, src[q], DTX + 2, DTY + 2);
    if (!mp) return EDDY_ECUDA;
    maps.m[q] = *mp;
  }
  size_t smem = ring_smem_bytes<DNF, DTX, DTY>();
  EDDY_CUDA(cudaFuncSetAttribute(k_density, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 g((d.ix2 - d.ix1 + DTX) / DTX, (d.jy2 - d.jy1 + DTY) / DTY, (d.kz2 - d.kz1 + DKC) / DKC);
  k_density<<<g, dim3(DTX, DTY), smem, ctx->stream>>>(d, ctx->m, ctx->sc, maps, ctx->f[EDDY_RHA], ctx->dens_alt,
                                                     repr1, alfxdt, gamxdt, rhoxdt, ctx->err_flag);
  EDDY_LAUNCHED(ctx);
  long long nghost = 2LL * d.nx * d.ny + 2LL * d.nx * d.nz + 2LL * d.ny * d.nz;
  k_dens_ghost_copy<<<(unsigned)((nghost + 255) / 256), 256, 0, ctx->stream>>>(d, ctx->f[EDDY_DENS], ctx->dens_alt);
  EDDY_LAUNCHED(ctx);
  double *t = ctx->f[EDDY_DENS];
  ctx->f[EDDY_DENS] = ctx->dens_alt;
  ctx->dens_alt = t;
  return launch_boundinoutd_dens(ctx, ctx->f[EDDY_DENS]);
}
