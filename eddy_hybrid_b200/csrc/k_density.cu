// k_density.cu -- density equation: RHS_DENSITY (src/rhs_density.f:4-175)
// fused with DENSITY (src/density.f:6-99) and its sponges, plus the
// BOUNDINOUTD / BOUNDARY_DENS ghost fills (src/boundary.f:2001-2281).
// Explicit form: the Crank-Nicolson part RS is zero in the interior.
#include "eddy_internal.h"

#define A(a, i, j, k) (a)[fidx(d, (i), (j), (k))]

int launch_fill_plane(eddy_ctx *ctx, double *a, int axis, int dst, int src, double sgn, int zero);

namespace {

constexpr int BX = 32, BY = 4, BZ = 2;

// new density into dn (ping-pong; ghost cells copied from the old buffer)
__global__ void __launch_bounds__(BX *BY *BZ)
    k_density(Dims d, DevMetrics m, Scalars s, const double *__restrict__ uo, const double *__restrict__ vo,
              const double *__restrict__ wo, const double *__restrict__ kv, const double *__restrict__ dens,
              double *__restrict__ rha, double *__restrict__ dn, double repr1, double alfxdt, double gamxdt,
              double rhoxdt) {
  int i = 1 + threadIdx.x + blockIdx.x * BX;
  int j = 1 + threadIdx.y + blockIdx.y * BY;
  int k = 1 + threadIdx.z + blockIdx.z * BZ;
  if (i > d.nx || j > d.ny || k > d.nz) return;
  long long q = fidx(d, i, j, k);
  if (!(i >= d.ix1 && i <= d.ix2 && j >= d.jy1 && j <= d.jy2 && k >= d.kz1 && k <= d.kz2)) {
    dn[q] = dens[q];
    return;
  }
  const int sy = d.nx;
  const long long sz = (long long)d.nx * d.ny;
  double qxp = uo[q], qxm = uo[q-1];
  double rxp = (dens[q+1] + dens[q]) * 0.5;
  double rxm = (dens[q] + dens[q-1]) * 0.5;
  double vyp = vo[q], vym = vo[q-sy];
  double ryp = (dens[q+sy] + dens[q]) * 0.5;
  double rym = (dens[q] + dens[q-sy]) * 0.5;
  double wzp = wo[q], wzm = wo[q-sz];
  double rzp = (dens[q+sz] + dens[q]) * 0.5;
  double rzm = (dens[q] + dens[q-sz]) * 0.5;
  double drdxp = m.au[i] * (dens[q+1] - dens[q]);
  double drdxm = m.au[i - 1] * (dens[q] - dens[q-1]);
  double drdyp = m.bv[j] * (dens[q+sy] - dens[q]);
  double drdym = m.bv[j - 1] * (dens[q] - dens[q-sy]);
  double drdzp = m.cw[k] * (dens[q+sz] - dens[q]);
  double drdzm = m.cw[k - 1] * (dens[q] - dens[q-sz]);
  double kvip = 0.5 * (kv[q+1] + kv[q]);
  double kvim = 0.5 * (kv[q-1] + kv[q]);
  double kvjp = 0.5 * (kv[q+sy] + kv[q]);
  double kvjm = 0.5 * (kv[q-sy] + kv[q]);
  double kvkp = 0.5 * (kv[q+sz] + kv[q]);
  double kvkm = 0.5 * (kv[q-sz] + kv[q]);
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
  double dnew = dens[q] + gamxdt * rr + rhoxdt * rha[q] + coef * 0.0;
  rha[q] = rr;
  double bg = m.dens_bg[(i - 1) + d.nx * (j - 1)];
  if (s.idspngl == 1) dnew = dnew + m.dfxdl[k] * (bg - dnew) * alfxdt * 1.0;
  if (i >= d.ix2 - s.dspngx1) dnew = dnew + m.dfxd[i] * (bg - dnew) * alfxdt * 1.0;
  dn[q] = dnew;
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
  dim3 g((d.nx + BX - 1) / BX, (d.ny + BY - 1) / BY, (d.nz + BZ - 1) / BZ);
  double repr1 = ctx->sc.ru1 / ctx->sc.prn;
  k_density<<<g, dim3(BX, BY, BZ), 0, ctx->stream>>>(d, ctx->m, ctx->sc, ctx->f[EDDY_UO], ctx->f[EDDY_VO],
                                                    ctx->f[EDDY_WO], ctx->f[EDDY_TV], ctx->f[EDDY_DENS],
                                                    ctx->f[EDDY_RHA], ctx->dens_alt, repr1, alfxdt, gamxdt,
                                                    rhoxdt);
  EDDY_LAUNCHED(ctx);
  double *t = ctx->f[EDDY_DENS];
  ctx->f[EDDY_DENS] = ctx->dens_alt;
  ctx->dens_alt = t;
  return launch_boundinoutd_dens(ctx, ctx->f[EDDY_DENS]);
}
