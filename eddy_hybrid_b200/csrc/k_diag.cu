// k_diag.cu -- per-step diagnostics on the device: the CFL number of CALCFL
// (src/timestep.f:2-78) behind the reference's constant-CFL time step
// DTM1 = CFLC/CFLM (src/Eddy6.f:2114-2128), and the field extrema of SCRINFO
// (src/info.f:5-164).  Two-stage reductions; max and min are exact, so the
// result does not depend on the reduction order.
#include <cfloat>

#include "eddy_internal.h"

namespace {

constexpr int NB = 296;  // blocks of the first stage (2 per SM)

// CALCFL (Cartesian: CONST = 2, rp = 1; RVIMPLX = RVIMPLY = 1): per interior
// cell the largest of the three convective and three viscous constraints
__global__ void __launch_bounds__(256)
    k_cfl_partial(Dims d, DevMetrics m, const double *__restrict__ uo, const double *__restrict__ vo,
                  const double *__restrict__ wo, const double *__restrict__ tv, double ru1, double rflagy,
                  double *part) {
  __shared__ double sh[256];
  const double cst = 2., rflagx = 0., rflagcx = 0., rflagcy = 0.;
  const long long mi = d.ix2 - d.ix1 + 1, mj = d.jy2 - d.jy1 + 1, mk = d.kz2 - d.kz1 + 1, n = mi * mj * mk;
  double mx = 0.;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = d.ix1 + (int)(t % mi), j = d.jy1 + (int)((t / mi) % mj), k = d.kz1 + (int)(t / (mi * mj));
    const long long q = fidx(d, i, j, k);
    const double cflx = (1. - rflagcx * 1.) * 0.5 * fabs(uo[q - 1] + uo[q]) * m.ap[i];
    const double cfly = (1. - rflagcy * 1.) * 0.5 * fabs(vo[q - d.nx] + vo[q]) * m.bp[j] / 1.0;
    const double cflz = 0.5 * fabs(wo[q - (long long)d.nx * d.ny] + wo[q]) * m.cp[k];
    const double totvx = ru1 + tv[q];
    const double cflvx = (1. - rflagx * 1.) * (m.ap[i] * m.ap[i]);
    const double by = m.bp[j] / 1.0;
    const double cflvy = (1. - rflagy * 1.) * (by * by);
    const double cflvz = m.cp[k] * m.cp[k];
    double c = fmax(fmax(fmax(cflx, cfly), fmax(cflz, cst * totvx * cflvx)),
                    fmax(cst * totvx * cflvy, cst * totvx * cflvz));
    mx = fmax(mx, c);
  }
  sh[threadIdx.x] = mx;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// min and max over the interior of one field
__global__ void __launch_bounds__(256) k_extrema_partial(Dims d, const double *__restrict__ a, double *part) {
  __shared__ double smin[256], smax[256];
  const long long mi = d.ix2 - d.ix1 + 1, mj = d.jy2 - d.jy1 + 1, mk = d.kz2 - d.kz1 + 1, n = mi * mj * mk;
  double lo = DBL_MAX, hi = -DBL_MAX;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = d.ix1 + (int)(t % mi), j = d.jy1 + (int)((t / mi) % mj), k = d.kz1 + (int)(t / (mi * mj));
    const double v = a[fidx(d, i, j, k)];
    lo = fmin(lo, v);
    hi = fmax(hi, v);
  }
  smin[threadIdx.x] = lo;
  smax[threadIdx.x] = hi;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[blockIdx.x] = smin[0];
    part[NB + blockIdx.x] = smax[0];
  }
}

__global__ void k_final(int np, const double *part, double *out, int with_min) {
  if (threadIdx.x != 0) return;
  double lo = DBL_MAX, hi = -DBL_MAX;
  for (int b = 0; b < np; b++) {
    if (with_min) lo = fmin(lo, part[b]);
    hi = fmax(hi, part[(with_min ? NB : 0) + b]);
  }
  out[0] = with_min ? lo : hi;
  out[1] = hi;
}

}  // namespace

extern "C" int eddy_cfl(eddy_ctx *ctx, double *cflm) {
  if (!ctx || !cflm) return EDDY_EINVAL;
  const Dims &d = ctx->d;
  double **f = ctx->f;
  double *part = ctx->diag, *out = ctx->diag + 2 * NB;
  k_cfl_partial<<<NB, 256, 0, ctx->stream>>>(d, ctx->m, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], f[EDDY_TV], ctx->sc.ru1,
                                              (double)ctx->sc.imply, part);
  EDDY_LAUNCHED(ctx);
  k_final<<<1, 32, 0, ctx->stream>>>(NB, part, out, 0);
  EDDY_LAUNCHED(ctx);
  double h[2];
  EDDY_CUDA(cudaMemcpyAsync(h, out, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  *cflm = h[1];
  return EDDY_OK;
}

extern "C" int eddy_field_extrema(eddy_ctx *ctx, int field, double *vmin, double *vmax) {
  if (!ctx || field < 0 || field >= EDDY_PLANEU || !vmin || !vmax) return EDDY_EINVAL;
  int rc = mixed_to64(ctx, field);
  if (rc) return rc;
  double *part = ctx->diag, *out = ctx->diag + 2 * NB;
  k_extrema_partial<<<NB, 256, 0, ctx->stream>>>(ctx->d, ctx->f[field], part);
  EDDY_LAUNCHED(ctx);
  k_final<<<1, 32, 0, ctx->stream>>>(NB, part, out, 1);
  EDDY_LAUNCHED(ctx);
  double h[2];
  EDDY_CUDA(cudaMemcpyAsync(h, out, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  *vmin = h[0];
  *vmax = h[1];
  return EDDY_OK;
}
