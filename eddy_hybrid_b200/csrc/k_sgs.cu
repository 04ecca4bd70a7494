// k_sgs.cu -- dynamic eddy viscosity TURVIS (src/vt.f:16-442), Cartesian,
// y-periodic, y-average branch (vt.f:296-318), z one-sided at both ends.
//
// One fused kernel, k_dynamic_march, replaces the reference's sequence of
// whole-array passes (centring vt.f:64-74, STRAIN vt.f:955-1018, the 22
// test filters filter3d vt.f:1132-1268, M_ij and L_ij vt.f:216-290, the
// clipped y averages vt.f:296-318).  A CTA owns a tile of 30 x-columns by
// KT z-rows and marches along the periodic y axis:
//   * the raw u, v, w tiles of plane j+4 are copied into a 4-plane ring in
//     shared memory by cp.async while plane j is processed; the centred
//     velocities of plane j+2 are computed from that ring into a 4-plane ring
//     of their own (with the x/z halo the strain needs),
//   * the strain and |S| of plane j are computed per thread (one thread per
//     (i,k) column of the tile plus a one-cell halo), the x pass of the filter
//     takes its neighbours by warp shuffles (lanes are x),
//   * the y pass is accumulated progressively in registers:
//       Y(j) = (0.25 X(j-1) + 0.5 X(j)) + 0.25 X(j+1),
//     the reference's operation order, so two partial sums per quantity,
//   * the completed Y(j-1) goes through shared memory for the z pass
//     (warps are z rows), then M_ij M_ij and max(L_ij M_ij, 0) are summed
//     along y in j order and the averages written per (i,k).
// Every product and sum is the reference's, in the reference's order, so the
// FP64 instantiation (compiled with -fmad=false) is bit-identical to the
// separable whole-array passes.  The FP32 instantiation (k_sgs32.cu, with
// FMA contraction) reads the mixed form's FP32 velocities.  Nothing but |S|
// (for nu_t) and the 2-D averages is written to HBM.  The kernels are in
// k_sgs_impl.cuh, shared by both translation units.
#include <cmath>
#include <vector>

#include "eddy_internal.h"

int launch_fill_plane(eddy_ctx *ctx, double *a, int axis, int dst, int src, double sgn, int zero);

namespace {
#include "k_sgs_impl.cuh"
}  // namespace

// FILTERSIZE (vt.f:1096-1127) on the host, same pow as the reference's
// libm, uploaded once.
int launch_filtersize(eddy_ctx *ctx) {
  const Dims &d = ctx->d;
  std::vector<double> dx((size_t)d.ncell);
  const std::vector<double> &ap = ctx->h[2], &bp = ctx->h[8], &cp = ctx->h[14];
  const double ppp = 2. / 3.;
  for (int k = 1; k <= d.nz; k++)
    for (int j = 1; j <= d.ny; j++)
      for (int i = 1; i <= d.nx; i++)
        dx[fidx(d, i, j, k)] = std::pow(std::fabs(1.0) / (ap[i] * bp[j] * cp[k]), ppp);
  if (d.lp == 0)
    for (int k = 1; k <= d.nz; k++)
      for (int i = 1; i <= d.nx; i++) {
        dx[fidx(d, i, 1, k)] = dx[fidx(d, i, d.ny - 1, k)];
        dx[fidx(d, i, d.ny, k)] = dx[fidx(d, i, 2, k)];
      }
  EDDY_CUDA(cudaMemcpy(ctx->dxdydz, dx.data(), sizeof(double) * dx.size(), cudaMemcpyHostToDevice));
  return EDDY_OK;
}

// FP64 TURVIS on (UO, VO, WO) -> TV
int launch_turvis(eddy_ctx *ctx) {
  const Dims &d = ctx->d;
  double **f = ctx->f;
  if (ctx->prm.isgs == 1) {
    long long nb = (d.ncell + 255) / 256;
    k_smag<<<(unsigned)nb, 256, 0, ctx->stream>>>(d, ctx->m, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], ctx->dxdydz,
                                                   f[EDDY_TV], ctx->sc.css);
    EDDY_LAUNCHED(ctx);
  } else {
    int rc = turvis_dynamic<double>(ctx, d.nx, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], ctx->gs, ctx->imm2, ctx->ilm2);
    if (rc) return rc;
  }
  return boundturb_tv(ctx);
}
