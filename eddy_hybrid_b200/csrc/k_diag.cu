// k_diag.cu -- per-step diagnostics on the device: the CFL number of CALCFL
// (src/timestep.f:2-78) behind the reference's constant-CFL time step
// DTM1 = CFLC/CFLM (src/Eddy6.f:2114-2128), and the field extrema of SCRINFO
// (src/info.f:5-164).  Two-stage reductions; max and min are exact, so the
// result does not depend on the reduction order.
#include <algorithm>
#include <cfloat>

#include "eddy_internal.h"

namespace {

constexpr int NB = 296;  // blocks of the first stage (2 per SM)

// CALCFL (Cartesian: CONST = 2, rp = 1; RVIMPLX = RVIMPLY = 1): per interior
// cell the largest of the three convective and three viscous constraints
__global__ void __launch_bounds__(256)
    k_cfl_partial(Dims d, DevMetrics m, const double *__restrict__ uo, const double *__restrict__ vo,
                  const double *__restrict__ wo, const double *__restrict__ tv, double ru1, double rflagx,
                  double rflagy, double rflagcx, double rflagcy, double *part) {
  __shared__ double sh[256];
  const double cst = 2.;
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

// rec_timeprobes_all (src/stats.f:132-185): the cell values of UO, VO, WO, P
// at each probe, with TIME, into sample slot `slot`
__global__ void k_probe_record(Dims d, int n, const int *ijk, const double *uo, const double *vo, const double *wo,
                               const double *p, double time, double *buf, int slot) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const long long q = fidx(d, ijk[3 * t], ijk[3 * t + 1], ijk[3 * t + 2]);
  double *o = buf + ((long long)slot * n + t) * 5;
  o[0] = time;
  o[1] = uo[q];
  o[2] = vo[q];
  o[3] = wo[q];
  o[4] = p[q];
}

// the value at (i, j, k) of yface_velocity (src/Planes.f:481-543) in mode
// center: 0 or 2 the cell value; 1 the x face average over i-1, i and j,
// j+1 (i = 2..NX-1, j = 1..NY-1, k = 2..NZ-1, else 0); 3 the same over k-1,
// k and j, j+1; 4 the average over j, j+1 (j = 1..NY-1, else 0)
__device__ double yface_value(const Dims &d, const double *a, int center, int i, int j, int k) {
  if (center == 1) {
    if (i < 2 || i > d.nx - 1 || j > d.ny - 1 || k < 2 || k > d.nz - 1) return 0.;
    return 0.250 * (((a[fidx(d, i, j, k)] + a[fidx(d, i - 1, j, k)]) + a[fidx(d, i, j + 1, k)]) +
                    a[fidx(d, i - 1, j + 1, k)]);
  }
  if (center == 3) {
    if (i < 2 || i > d.nx - 1 || j > d.ny - 1 || k < 2 || k > d.nz - 1) return 0.;
    return 0.250 * (((a[fidx(d, i, j, k)] + a[fidx(d, i, j, k - 1)]) + a[fidx(d, i, j + 1, k)]) +
                    a[fidx(d, i, j + 1, k - 1)]);
  }
  if (center == 4) {
    if (j > d.ny - 1) return 0.;
    return 0.50 * (a[fidx(d, i, j, k)] + a[fidx(d, i, j + 1, k)]);
  }
  return a[fidx(d, i, j, k)];
}

// one plane of a field: axis 1 the (j, k) plane at i = index, 2 the (i, k)
// plane at j = index, 3 the (i, j) plane at k = index; out Fortran-ordered
__global__ void k_plane(Dims d, const double *a, int center, int axis, int index, double *out) {
  const int n1 = axis == 1 ? d.ny : d.nx, n2 = axis == 3 ? d.ny : d.nz;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n1 * n2) return;
  const int u = 1 + t % n1, v = 1 + t / n1;
  const int i = axis == 1 ? index : u, j = axis == 1 ? u : (axis == 2 ? index : v), k = axis == 3 ? index : v;
  out[t] = yface_value(d, a, center, i, j, k);
}

}  // namespace

int probes_record(eddy_ctx *ctx) {
  if (ctx->nprobe <= 0 || ctx->probe_count >= ctx->probe_cap) return EDDY_OK;
  double **f = ctx->f;
  k_probe_record<<<(ctx->nprobe + 127) / 128, 128, 0, ctx->stream>>>(ctx->d, ctx->nprobe, ctx->probe_ijk,
                                                                     f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], f[EDDY_P],
                                                                     ctx->time, ctx->probe_buf, ctx->probe_count);
  EDDY_LAUNCHED(ctx);
  ctx->probe_count++;
  return EDDY_OK;
}

extern "C" int eddy_probes_set(eddy_ctx *ctx, int n, const int *ijk, int capacity) {
  if (!ctx || n < 0 || (n > 0 && (!ijk || capacity < 1))) return EDDY_EINVAL;
  const Dims &d = ctx->d;
  for (int t = 0; t < n; t++)
    if (ijk[3 * t] < 1 || ijk[3 * t] > d.nx || ijk[3 * t + 1] < 1 || ijk[3 * t + 1] > d.ny || ijk[3 * t + 2] < 1 ||
        ijk[3 * t + 2] > d.nz)
      return EDDY_EINVAL;
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  if (ctx->probe_ijk) cudaFree(ctx->probe_ijk);
  if (ctx->probe_buf) cudaFree(ctx->probe_buf);
  ctx->probe_ijk = nullptr;
  ctx->probe_buf = nullptr;
  ctx->nprobe = ctx->probe_cap = ctx->probe_count = 0;
  if (n == 0) return EDDY_OK;
  EDDY_CUDA(cudaMalloc(&ctx->probe_ijk, sizeof(int) * 3 * n));
  EDDY_CUDA(cudaMalloc(&ctx->probe_buf, sizeof(double) * 5 * (size_t)n * capacity));
  EDDY_CUDA(cudaMemcpy(ctx->probe_ijk, ijk, sizeof(int) * 3 * n, cudaMemcpyHostToDevice));
  ctx->nprobe = n;
  ctx->probe_cap = capacity;
  return EDDY_OK;
}

extern "C" int eddy_probes_read(eddy_ctx *ctx, double *out, int max_samples, int *nsamples) {
  if (!ctx || !nsamples || max_samples < 0 || (max_samples > 0 && !out)) return EDDY_EINVAL;
  const int m = ctx->probe_count < max_samples ? ctx->probe_count : max_samples;
  if (m > 0)
    EDDY_CUDA(cudaMemcpyAsync(out, ctx->probe_buf, sizeof(double) * 5 * (size_t)ctx->nprobe * m,
                              cudaMemcpyDeviceToHost, ctx->stream));
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  *nsamples = ctx->probe_count;
  // the samples read are consumed; later ones move to the front
  if (m > 0) {
    const size_t per = 5 * (size_t)ctx->nprobe;
    if (ctx->probe_count > m)
      EDDY_CUDA(cudaMemcpy(ctx->probe_buf, ctx->probe_buf + per * m, sizeof(double) * per * (ctx->probe_count - m),
                           cudaMemcpyDeviceToDevice));
    ctx->probe_count -= m;
  }
  return EDDY_OK;
}

extern "C" int eddy_plane(eddy_ctx *ctx, int field, int center, int axis, int index, double *out) {
  if (!ctx || field < 0 || field >= EDDY_PLANEU || !out || center < 0 || center > 4 || axis < 1 || axis > 3)
    return EDDY_EINVAL;
  const Dims &d = ctx->d;
  const int lim = axis == 1 ? d.nx : (axis == 2 ? d.ny : d.nz);
  if (index < 1 || index > lim) return EDDY_EINVAL;
  int rc = mixed_to64(ctx, field);
  if (rc) return rc;
  const int n1 = axis == 1 ? d.ny : d.nx, n2 = axis == 3 ? d.ny : d.nz;
  const size_t np = (size_t)n1 * n2;
  if (np > (size_t)(1 << 30)) return EDDY_EINVAL;
  if (!ctx->plane_buf) {
    const size_t big = std::max({(size_t)d.nx * d.ny, (size_t)d.nx * d.nz, (size_t)d.ny * d.nz});
    EDDY_CUDA(cudaMalloc(&ctx->plane_buf, sizeof(double) * big));
  }
  double *tmp = ctx->plane_buf;
  k_plane<<<(unsigned)((np + 255) / 256), 256, 0, ctx->stream>>>(d, ctx->f[field], center, axis, index, tmp);
  EDDY_LAUNCHED(ctx);
  EDDY_CUDA(cudaMemcpyAsync(out, tmp, sizeof(double) * np, cudaMemcpyDeviceToHost, ctx->stream));
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  return EDDY_OK;
}

extern "C" int eddy_cfl(eddy_ctx *ctx, double *cflm) {
  if (!ctx || !cflm) return EDDY_EINVAL;
  const Dims &d = ctx->d;
  double **f = ctx->f;
  double *part = ctx->diag, *out = ctx->diag + 2 * NB;
  k_cfl_partial<<<NB, 256, 0, ctx->stream>>>(d, ctx->m, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], f[EDDY_TV], ctx->sc.ru1,
                                              (double)ctx->sc.implx, (double)ctx->sc.imply,
                                              (double)ctx->sc.implcx, (double)ctx->sc.implcy, part);
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
