// eddy_ctx.cu -- context, metrics, field storage, and the C ABI entry points
// (include/eddy_b200.h).  The driver sequence in eddy_substep/eddy_step is
// the time loop of src/Eddy6.f:2095-3049 (ibm=0, explicit viscous terms).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "eddy_internal.h"
#include "tma_ring.cuh"

int launch_fill_plane(eddy_ctx *ctx, double *a, int axis, int dst, int src, double sgn, int zero);

namespace {

// Metric arrays from face coordinates, src/grid.f:21-173 (igrid=1, uniform y,
// kgrid=1); index bounds src/setup.f:2-75; sponge src/Initialize.f:129-271.
void build_metrics(eddy_ctx *ctx, const double *xf, double ymin, double ymax, const double *zf) {
  const eddy_params &p = ctx->prm;
  int nx = p.nx, ny = p.ny, nz = p.nz;
  for (int a = 0; a < 28; a++) ctx->h[a].clear();
  auto arr = [&](int id, int n) -> std::vector<double> & {
    ctx->h[id].assign((size_t)n + 2, 0.0);
    return ctx->h[id];
  };
  auto &xu = arr(0, nx), &xc = arr(1, nx), &ap = arr(2, nx), &au = arr(3, nx), &av = arr(4, nx), &aw = arr(5, nx);
  auto &yv = arr(6, ny), &yc = arr(7, ny), &bp = arr(8, ny), &bu = arr(9, ny), &bv = arr(10, ny), &bw = arr(11, ny);
  auto &zw = arr(12, nz), &zc = arr(13, nz), &cp = arr(14, nz), &cu = arr(15, nz), &cv = arr(16, nz),
       &cw = arr(17, nz);
  int ix1 = 2, ix2 = nx - 1;
  for (int i = 1; i <= ix2; i++) xu[i] = xf[i - 1];
  xu[nx] = 2. * xu[ix2] - xu[ix2 - 1];
  for (int i = ix1; i <= ix2; i++) xc[i] = .5 * (xu[i - 1] + xu[i]);
  xc[1] = 2. * xu[1] - xc[2];
  xc[nx] = 2. * xu[ix2] - xc[ix2];
  for (int i = ix1; i <= ix2; i++) au[i] = 2. / (xu[i + 1] - xu[i - 1]);
  au[1] = 2. / (-3. * xu[1] + 4. * xu[2] - xu[3]);
  au[ix2] = 2. / (3. * xu[ix2] - 4. * xu[ix2 - 1] + xu[ix2 - 2]);
  au[nx] = au[ix2];
  for (int i = ix1; i <= ix2; i++) ap[i] = 1. / (xu[i] - xu[i - 1]);
  ap[1] = ap[ix1];
  ap[nx] = ap[ix2];
  for (int i = ix1; i <= ix2; i++) av[i] = 2. / (xc[i + 1] - xc[i - 1]);
  av[1] = 2. / (-3. * xc[1] + 4. * xc[2] - xc[3]);
  av[nx] = 2. / (3. * xc[nx] - 4. * xc[nx - 1] + xc[nx - 2]);
  for (int i = 1; i <= nx; i++) aw[i] = av[i];
  int jy1 = 2, jy2 = ny - 1;
  double dely = (ymax - ymin) / (double)(ny - 2), rdely = 1. / dely;
  for (int j = 1; j <= ny; j++) {
    yv[j] = (double)(j - 1) * dely + ymin;
    bp[j] = bu[j] = bv[j] = bw[j] = rdely;
  }
  ctx->dely = dely;
  ctx->delysq = dely * dely;
  for (int j = jy1; j <= jy2; j++) yc[j] = 0.5 * (yv[j] + yv[j - 1]);
  yc[1] = 2. * yv[1] - yc[jy1];
  yc[jy2 + 1] = 2. * yv[jy2] - yc[jy2];
  int kz1 = 2, kz2 = nz - 1;
  for (int k = 1; k <= kz2; k++) zw[k] = zf[k - 1];
  zw[nz] = 2. * zw[kz2] - zw[kz2 - 1];
  for (int k = kz1; k <= kz2; k++) zc[k] = .5 * (zw[k - 1] + zw[k]);
  zc[1] = 2. * zw[1] - zc[2];
  zc[nz] = 2. * zw[kz2] - zc[kz2];
  for (int k = kz1; k <= kz2; k++) cw[k] = 2. / (zw[k + 1] - zw[k - 1]);
  cw[1] = 2. / (-3. * zw[1] + 4. * zw[2] - zw[3]);
  cw[kz2] = 2. / (3. * zw[kz2] - 4. * zw[kz2 - 1] + zw[kz2 - 2]);
  cw[nz] = 0.;  // grid.f:112 copies the not yet filled COMMON cw(kz2)
  for (int k = kz1; k <= kz2; k++) cp[k] = 1. / (zw[k] - zw[k - 1]);
  cp[1] = cp[kz1];
  cp[nz] = cp[kz2];
  for (int k = kz1; k <= kz2; k++) cv[k] = 2. / (zc[k + 1] - zc[k - 1]);
  cv[1] = 2. / (-3. * zc[1] + 4. * zc[2] - zc[3]);
  cv[nz] = 2. / (3. * zc[nz] - 4. * zc[nz - 1] + zc[nz - 2]);
  for (int k = 1; k <= nz; k++) cu[k] = cv[k];

  Dims &d = ctx->d;
  d.nx = nx; d.ny = ny; d.nz = nz;
  d.ix1 = ix1; d.ix2 = ix2; d.jy1 = jy1; d.jy2 = jy2; d.kz1 = kz1; d.kz2 = kz2;
  for (int b = 0; b < 7; b++) d.itype[b] = p.itype[b];
  d.ibu = ix1;
  d.ieu = p.itype[2] == 500 ? ix2 : ix2 - 1;
  d.jbv = jy1;
  d.jev = p.itype[4] == 500 ? jy2 : jy2 - 1;
  d.kbw = kz1;
  d.kew = (p.itype[6] == 500 || p.itype[6] == 0) ? kz2 : kz2 - 1;
  d.mp = p.itype[2] == 500 ? 0 : 1;
  d.lp = p.itype[4] == 500 ? 0 : 1;
  d.np = p.itype[6] == 500 ? 0 : 1;
  d.ncell = (long long)nx * ny * nz;

  // filter weights (vt.f:1374-1434)
  auto &whx = ctx->h[18], &why = ctx->h[19], &whz = ctx->h[20];
  whx.assign((size_t)3 * (nx + 1), 0.0);
  why.assign((size_t)3 * (ny + 1), 0.0);
  whz.assign((size_t)3 * (nz + 1), 0.0);
#define WH(a, i, dd) a[(size_t)((i)*3 + (dd) + 1)]
  for (int i = ix1; i <= ix2; i++) WH(whx, i, 0) = 0.50;
  for (int i = ix1 + 1; i <= ix2 - 1; i++) {
    WH(whx, i, -1) = 0.25 * av[i] / au[i];
    WH(whx, i, 1) = 0.25 * av[i] / au[i - 1];
  }
  WH(whx, ix1, -1) = 0.50 * av[ix1 + 1] / au[ix1] + 0.25 * av[ix1 + 1] / au[ix1 + 1];
  WH(whx, ix1, 1) = -0.25 * av[ix1 + 1] / au[ix1];
  WH(whx, ix2, -1) = 0.50 * av[ix2 - 1] / au[ix2 - 1] + 0.25 * av[ix2 - 1] / au[ix2 - 2];
  WH(whx, ix2, 1) = -0.25 * av[ix2 - 1] / au[ix2 - 1];
  for (int j = jy1; j <= jy2; j++) WH(why, j, 0) = 0.50;
  for (int j = jy1 + 1; j <= jy2 - 1; j++) {
    WH(why, j, -1) = 0.25 * bw[j] / bv[j];
    WH(why, j, 1) = 0.25 * bw[j] / bv[j - 1];
  }
  WH(why, jy1, -1) = 0.50 * bw[jy1 + 1] / bv[jy1] + 0.25 * bw[jy1 + 1] / bv[jy1 + 1];
  WH(why, jy1, 1) = -0.25 * bw[jy1 + 1] / bv[jy1];
  WH(why, jy2, -1) = 0.50 * bw[jy2 - 1] / bv[jy2 - 1] + 0.25 * bw[jy2 - 1] / bv[jy2 - 2];
  WH(why, jy2, 1) = -0.25 * bw[jy2 - 1] / bv[jy2 - 1];
  for (int k = kz1; k <= kz2; k++) {
    WH(whz, k, 0) = 0.50;
    WH(whz, k, -1) = 0.25 * cu[k] / cw[k];
    WH(whz, k, 1) = 0.25 * cu[k] / cw[k - 1];
  }
  if (p.itype[5] != 0) {
    WH(whz, kz1, -1) = 0.50 * cu[kz1 + 1] / cw[kz1] + 0.25 * cu[kz1 + 1] / cw[kz1 + 1];
    WH(whz, kz1, 1) = -0.25 * cu[kz1 + 1] / cw[kz1];
  }
  if (p.itype[6] != 0) {
    WH(whz, kz2, -1) = 0.50 * cu[kz2 - 1] / cw[kz2 - 1] + 0.25 * cu[kz2 - 1] / cw[kz2 - 2];
    WH(whz, kz2, 1) = -0.25 * cu[kz2 - 1] / cw[kz2 - 1];
  }
#undef WH
  // sponges
  auto &dfxu = arr(21, nx), &dfxw = arr(22, nx), &dfxul = arr(23, nz), &dfxwl = arr(24, nz), &dfxd = arr(25, nx),
       &dfxdl = arr(26, nz);
  int ibu = d.ibu, ieu = d.ieu, nzg = nz;
  int vx1 = p.vspngx1, vin = p.vspngx3in, vout = p.vspngx3out, dx1 = p.dspngx1, din = p.dspngx3in,
      dout = p.dspngx3out;
  for (int i = ibu; i <= ieu; i++) {
    dfxu[i] = 0.0;
    if (i >= ieu - vx1 && vx1 > 0) {
      double r = (xu[i] - xu[ieu - vx1]) / (xu[ieu] - xu[ieu - vx1]);
      dfxu[i] = 5.0 * (r * r);
    }
  }
  for (int i = ix1; i <= ix2; i++) {
    dfxw[i] = 0.0;
    if (i >= ix2 - vx1 && vx1 > 0) {
      double r = (xc[i] - xc[ix2 - vx1]) / (xc[ix2] - xc[ix2 - vx1]);
      dfxw[i] = 5.0 * (r * r);
    }
  }
  std::vector<double> dfxug(nzg + 2, 0.), dfxwg(nzg + 2, 0.), dfxdg(nzg + 2, 0.);
  for (int k = nzg; k >= 1; k--) {
    if (k <= vin + 1 && vin > 0) {
      double r = (zc[k] - zc[vin + 1]) / (zc[2] - zc[vin + 1]);
      dfxug[k] = 20.0 * (r * r);
      double r2 = (zw[k] - zw[vin + 1]) / (zw[2] - zw[vin + 1]);
      dfxwg[k] = 20.0 * (r2 * r2);
    }
  }
  for (int k = 1; k <= nzg; k++) {
    if (k >= nzg - vout && vout > 0) {
      double r = (zc[k - 2] - zc[nzg - vout]) / (zc[nzg - 2] - zc[nzg - dout]);
      dfxug[k] = 10.0 * (r * r);
      double r2 = (zw[k - 2] - zw[nzg - dout]) / (zw[nzg - 2] - zw[nzg - dout]);
      dfxwg[k] = 10.0 * (r2 * r2);
    }
  }
  int ivs = 0;
  for (int k = kz1; k <= kz2; k++) {
    dfxul[k] = dfxug[k];
    dfxwl[k] = dfxwg[k];
    if (dfxwl[k] > 0.0) ivs = 1;
  }
  for (int k = 1; k <= nzg; k++)
    if (k >= nzg - dout && dout > 0) {
      double r = (zc[k - 2] - zc[nzg - dout]) / (zc[nzg - 2] - zc[nzg - dout]);
      dfxdg[k] = 100.0 * (r * r);
    }
  for (int k = nzg; k >= 1; k--)
    if (k <= din + 1 && din > 0) {
      double r = (zc[k] - zc[din + 1]) / (zc[2] - zc[din + 1]);
      dfxdg[k] = 100.0 * (r * r);
    }
  int ids = 0;
  for (int k = kz1; k <= kz2; k++) {
    dfxdl[k] = dfxdg[k];
    if (dfxdl[k] > 0.0) ids = 1;
  }
  for (int i = ibu; i <= ieu; i++)
    if (i >= ieu - dx1 && dx1 > 0) {
      double r = (xc[i] - xc[ieu - dx1]) / (xc[ieu] - xc[ieu - dx1]);
      dfxd[i] = 5.0 * (r * r);
    }
  // background density (Cartesian vertical = x)
  auto &dbg = ctx->h[27];
  dbg.assign((size_t)nx * ny, 0.0);
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++) dbg[(size_t)(i - 1) + (size_t)nx * (j - 1)] = p.denP1 * xc[i];

  Scalars &s = ctx->sc;
  s.ru1 = p.ru1; s.prn = p.prn; s.grav = p.grav; s.dpdx = p.dpdx; s.dpdy = p.dpdy; s.dpdz = p.dpdz;
  s.eps = p.eps; s.css = p.css; s.vspngx1 = p.vspngx1; s.dspngx1 = p.dspngx1;
  s.ivspngl = ivs; s.idspngl = ids; s.idens = p.idens; s.isgs = p.isgs; s.imply = p.imply;
  s.implx = p.implx; s.implcx = p.implcx; s.implcy = p.implcy;
}

int upload_metrics(eddy_ctx *ctx) {
  double **dst[] = {nullptr, nullptr, &ctx->m.ap, &ctx->m.au, &ctx->m.av, &ctx->m.aw, nullptr, nullptr,
                    &ctx->m.bp, &ctx->m.bu, &ctx->m.bv, &ctx->m.bw, nullptr, nullptr, &ctx->m.cp, &ctx->m.cu,
                    &ctx->m.cv, &ctx->m.cw, &ctx->m.whx, &ctx->m.why, &ctx->m.whz, &ctx->m.dfxu, &ctx->m.dfxw,
                    &ctx->m.dfxul, &ctx->m.dfxwl, &ctx->m.dfxd, &ctx->m.dfxdl, &ctx->m.dens_bg};
  for (int a = 0; a < 28; a++) {
    if (!dst[a]) continue;
    size_t b = sizeof(double) * ctx->h[a].size();
    EDDY_CUDA(cudaMalloc(dst[a], b));
    EDDY_CUDA(cudaMemcpy(*dst[a], ctx->h[a].data(), b, cudaMemcpyHostToDevice));
  }
  return EDDY_OK;
}

void free_all(eddy_ctx *ctx) {
  DevMetrics &m = ctx->m;
  double *mp[] = {m.ap, m.au, m.av, m.aw, m.bp, m.bu, m.bv, m.bw, m.cp, m.cu, m.cv, m.cw, m.whx, m.why, m.whz,
                  m.dfxu, m.dfxw, m.dfxul, m.dfxwl, m.dfxd, m.dfxdl, m.dens_bg};
  for (double *p : mp) if (p) cudaFree(p);
  for (int f = 0; f < EDDY_NFIELDS; f++) if (ctx->f[f]) cudaFree(ctx->f[f]);
  double *o[] = {ctx->dens_alt, ctx->gs, ctx->dxdydz, ctx->ilm2, ctx->imm2, ctx->scal, ctx->diag, ctx->feed,
                 ctx->probe_buf, ctx->plane_buf, ctx->cv_buf};
  if (ctx->probe_ijk) cudaFree(ctx->probe_ijk);
  for (double *p : o) if (p) cudaFree(p);
  if (ctx->err_flag) cudaFree(ctx->err_flag);
  poisson_plan_destroy(ctx);
  mlp_release(ctx);
  mixed_release(ctx);
  ib_release(ctx);
  double *o2[] = {ctx->xc_dev, ctx->kappa, ctx->tv_dyn};
  for (double *p : o2) if (p) cudaFree(p);
  for (ProfEvent &e : ctx->prof_ev) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
  for (ProfEvent &e : ctx->prof_pool) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
  if (ctx->ib_stream) cudaStreamSynchronize(ctx->ib_stream);
  for (cudaEvent_t e : ctx->ib_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->ib_stream) cudaStreamDestroy(ctx->ib_stream);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
}

int check_ctx(eddy_ctx *ctx) { return ctx ? EDDY_OK : EDDY_EINVAL; }

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

void scheme(int ischm, double gam[3], double rho[3], double alf[3]) {
  if (ischm == 1) {
    gam[0] = 1.5; gam[1] = 0.; gam[2] = 0.;
    rho[0] = -0.5; rho[1] = 0.; rho[2] = 0.;
  } else {
    gam[0] = 8. / 15.; gam[1] = 5. / 12.; gam[2] = 3. / 4.;
    rho[0] = 0.; rho[1] = -17. / 60.; rho[2] = -5. / 12.;
  }
  for (int q = 0; q < 3; q++) alf[q] = gam[q] + rho[q];
}

}  // namespace

int make_tensor_map_3d(CUtensorMap *map, const void *base, int nx, int ny, int nz, int bx, int by, int esize,
                       int pitch) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return -1;
  if (pitch <= 0) pitch = nx;
  cuuint64_t gdim[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
  cuuint64_t gstr[2] = {(cuuint64_t)pitch * esize, (cuuint64_t)pitch * ny * esize};
  cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  cuuint32_t est[3] = {1, 1, 1};
  CUtensorMapDataType dt = esize == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  CUresult r = fn(map, dt, 3, const_cast<void *>(base), gdim, gstr, box, est, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : (int)r;
}

int make_tensor_map_2d(CUtensorMap *map, const void *base, long long w, long long h, int bx, int by, int swizzle32) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return -1;
  cuuint64_t gdim[2] = {(cuuint64_t)w, (cuuint64_t)h};
  cuuint64_t gstr[1] = {(cuuint64_t)w * 4};
  cuuint32_t box[2] = {(cuuint32_t)bx, (cuuint32_t)by};
  cuuint32_t est[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base), gdim, gstr, box, est,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle32 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : (int)r;
}

const CUtensorMap *ctx_tensor_map(eddy_ctx *ctx, const double *ptr, int bx, int by) {
  for (TmaEntry &e : ctx->tmaps)
    if (e.ptr == ptr && e.bx == bx && e.by == by) return &e.map;
  TmaEntry e;
  e.ptr = ptr;
  e.bx = bx;
  e.by = by;
  int r = make_tensor_map_3d(&e.map, ptr, ctx->d.nx, ctx->d.ny, ctx->d.nz, bx, by, 8);
  if (r != 0) {
    ctx->err = "cuTensorMapEncodeTiled failed (" + std::to_string(r) + ")";
    return nullptr;
  }
  ctx->tmaps.push_back(e);
  return &ctx->tmaps.back().map;
}

thread_local cudaStream_t tl_stream = nullptr;

extern "C" {

int eddy_create(eddy_ctx **out, const eddy_params *prm, const double *xu_faces, double ymin, double ymax,
                const double *zw_faces, int device) {
  if (!out || !prm || !xu_faces || !zw_faces) return EDDY_EINVAL;
  *out = nullptr;
  eddy_ctx *ctx = new (std::nothrow) eddy_ctx();
  if (!ctx) return EDDY_ENOMEM;
  ctx->prm = *prm;
  const eddy_params &p = *prm;
  auto fail = [&](int rc, const char *msg) {
    if (msg) ctx->err = msg;
    *out = ctx;  // keep the context so the caller can read the message
    return rc;
  };
  if (p.nx < 6 || p.ny < 4 || p.nz < 6) return fail(EDDY_EINVAL, "grid too small (need NX,NZ >= 6, NY >= 4)");
  if (p.nx % 2 != 0)
    return fail(EDDY_EINVAL, "NX must be even (TMA rows of FP64 need 16-byte strides)");
  if (p.ischm != 3 && p.ischm != 1) return fail(EDDY_EINVAL, "ischm must be 1 or 3");
  if (p.isgs != 0 && p.isgs != 1 && p.isgs != 2)
    return fail(EDDY_EINVAL, "only isgs 0 (none), 1 (Smagorinsky), 2 (dynamic, y average) are supported");
  if (p.itype[3] != 500 || p.itype[4] != 500) return fail(EDDY_EINVAL, "y (ITYPE 3/4) must be periodic (500)");
  for (int b = 1; b <= 2; b++)
    if (p.itype[b] != 60 && p.itype[b] != 82) return fail(EDDY_EINVAL, "x boundaries must be type 60 or 82");
  if (p.itype[5] != 305 || (p.itype[6] != 730))
    return fail(EDDY_EINVAL, "z boundaries must be the hybrid inlet 305 and the convective outlet 730");
  if (p.precision != EDDY_PLAIN_FP64 && p.precision != EDDY_MIXED)
    return fail(EDDY_EINVAL, "precision must be EDDY_PLAIN_FP64 or EDDY_MIXED");
  if (p.closure != 0 && p.closure != 1) return fail(EDDY_EINVAL, "closure must be 0 (dynamic) or 1 (learned)");
  if (p.imply != 0 && p.imply != 1) return fail(EDDY_EINVAL, "imply must be 0 or 1");
  if (p.imply == 1 && (p.precision != EDDY_PLAIN_FP64 || p.closure != 0))
    return fail(EDDY_EINVAL, "the implicit y terms (imply = 1) are built for the plain FP64 form with the dynamic model");
  if (p.imply == 1 && p.ny - 2 < 3) return fail(EDDY_EINVAL, "imply = 1 needs at least 3 cells along y");
  if (p.implx != 0 && p.implx != 1) return fail(EDDY_EINVAL, "implx must be 0 or 1");
  if (p.implx == 1 && (p.precision != EDDY_PLAIN_FP64 || p.closure != 0))
    return fail(EDDY_EINVAL, "the implicit x terms (implx = 1) are built for the plain FP64 form with the dynamic model");
  if (p.implx == 1 && (p.itype[1] != 60 || p.itype[2] != 60))
    return fail(EDDY_EINVAL, "implx = 1 is built for slip walls (type 60) on both x boundaries");
  if (p.implcx != 0 && p.implcx != 1) return fail(EDDY_EINVAL, "implcx must be 0 or 1");
  if (p.implcy != 0 && p.implcy != 1) return fail(EDDY_EINVAL, "implcy must be 0 or 1");
  if ((p.implcx == 1 || p.implcy == 1) && (p.precision != EDDY_PLAIN_FP64 || p.closure != 0))
    return fail(EDDY_EINVAL,
                "the implicit convective terms (implcx, implcy = 1) are built for the plain FP64 form with the dynamic model");
  if (p.implcx == 1 && (p.itype[1] != 60 || p.itype[2] != 60))
    return fail(EDDY_EINVAL, "implcx = 1 is built for slip walls (type 60) on both x boundaries");
  if (p.implcy == 1 && p.ny - 2 < 3) return fail(EDDY_EINVAL, "implcy = 1 needs at least 3 cells along y");
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess) return fail(EDDY_ECUDA, "cudaSetDevice failed");
  // the regeneration's stream has the highest priority: its short kernels
  // (and the host waits between them) must not queue behind the blocks of a
  // long kernel on the main stream
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithPriority(&ctx->ib_stream, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ib_ev[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ib_ev[1], cudaEventDisableTiming) != cudaSuccess)
    return fail(EDDY_ECUDA, "cudaStreamCreate failed");
  build_metrics(ctx, xu_faces, ymin, ymax, zw_faces);
  int rc = upload_metrics(ctx);
  if (rc) return fail(rc, nullptr);
  size_t n3 = sizeof(double) * (size_t)ctx->d.ncell, n2 = sizeof(double) * (size_t)p.nx * p.ny;
  for (int f = 0; f < EDDY_NFIELDS; f++) {
    size_t b = (f >= EDDY_PLANEU) ? n2 : n3;
    if (cudaMalloc(&ctx->f[f], b) != cudaSuccess) return fail(EDDY_ENOMEM, "device allocation failed");
    cudaMemset(ctx->f[f], 0, b);
  }
  double **o[] = {&ctx->dens_alt, &ctx->gs, &ctx->dxdydz};
  for (double **pp : o) {
    if (cudaMalloc(pp, n3) != cudaSuccess) return fail(EDDY_ENOMEM, "device allocation failed");
    cudaMemset(*pp, 0, n3);
  }
  size_t n2xz = sizeof(double) * (size_t)p.nx * p.nz;
  if (cudaMalloc(&ctx->ilm2, n2xz) != cudaSuccess || cudaMalloc(&ctx->imm2, n2xz) != cudaSuccess)
    return fail(EDDY_ENOMEM, "device allocation failed");
  cudaMemset(ctx->ilm2, 0, n2xz);
  cudaMemset(ctx->imm2, 0, n2xz);
  // scalars [0, 32) and the plane-flux partial sums [32, 32 + 2 * 148)
  if (cudaMalloc(&ctx->scal, sizeof(double) * 640) != cudaSuccess) return fail(EDDY_ENOMEM, "allocation failed");
  cudaMemset(ctx->scal, 0, sizeof(double) * 640);
  if (cudaMalloc(&ctx->diag, sizeof(double) * 600) != cudaSuccess) return fail(EDDY_ENOMEM, "allocation failed");
  if (cudaMalloc(&ctx->err_flag, sizeof(int)) != cudaSuccess) return fail(EDDY_ENOMEM, "allocation failed");
  cudaMemset(ctx->err_flag, 0, sizeof(int));
  rc = poisson_plan_create(ctx);
  if (rc) return fail(rc, nullptr);
  if (p.precision == EDDY_MIXED && (rc = mixed_create(ctx))) return fail(rc, nullptr);
  {
    size_t bx = sizeof(double) * ctx->h[1].size();
    if (cudaMalloc(&ctx->xc_dev, bx) != cudaSuccess) return fail(EDDY_ENOMEM, "allocation failed");
    cudaMemcpy(ctx->xc_dev, ctx->h[1].data(), bx, cudaMemcpyHostToDevice);
    if (cudaMalloc(&ctx->kappa, n3) != cudaSuccess || cudaMalloc(&ctx->tv_dyn, n3) != cudaSuccess)
      return fail(EDDY_ENOMEM, "allocation failed");
    cudaMemset(ctx->kappa, 0, n3);
    cudaMemset(ctx->tv_dyn, 0, n3);
  }
  if (p.isgs != 0) {
    rc = launch_filtersize(ctx);
    if (rc) return fail(rc, nullptr);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(EDDY_ECUDA, "device error during set-up");
  *out = ctx;
  return EDDY_OK;
}

int eddy_destroy(eddy_ctx *ctx) {
  if (!ctx) return EDDY_OK;
  if (ctx->ib_thread.joinable()) ctx->ib_thread.join();
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_all(ctx);
  delete ctx;
  return EDDY_OK;
}

int eddy_upload(eddy_ctx *ctx, int field, const double *host) {
  if (check_ctx(ctx) || field < 0 || field >= EDDY_NFIELDS || !host) return EDDY_EINVAL;
  size_t b = sizeof(double) * (field >= EDDY_PLANEU ? (size_t)ctx->d.nx * ctx->d.ny : (size_t)ctx->d.ncell);
  EDDY_CUDA(cudaMemcpyAsync(ctx->f[field], host, b, cudaMemcpyHostToDevice, ctx->stream));
  if (field == EDDY_DENS) EDDY_CUDA(cudaMemcpyAsync(ctx->dens_alt, host, b, cudaMemcpyHostToDevice, ctx->stream));
  int rc = mixed_from64(ctx, field);
  if (rc) return rc;
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  return EDDY_OK;
}

int eddy_download(eddy_ctx *ctx, int field, double *host) {
  if (check_ctx(ctx) || field < 0 || field >= EDDY_NFIELDS || !host) return EDDY_EINVAL;
  size_t b = sizeof(double) * (field >= EDDY_PLANEU ? (size_t)ctx->d.nx * ctx->d.ny : (size_t)ctx->d.ncell);
  int rc = mixed_to64(ctx, field);
  if (rc) return rc;
  EDDY_CUDA(cudaMemcpyAsync(host, ctx->f[field], b, cudaMemcpyDeviceToHost, ctx->stream));
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  return EDDY_OK;
}

int eddy_save_field(eddy_ctx *ctx, int field, const char *path, int nstep, double time, double dtm1) {
  if (check_ctx(ctx) || field < 0 || field >= EDDY_PLANEU || !path) return EDDY_EINVAL;
  std::vector<double> h((size_t)ctx->d.ncell);
  int rc = eddy_download(ctx, field, h.data());
  if (rc) return rc;
  rc = eddy_ioscalar_write(path, ctx->d.nx, ctx->d.ny, ctx->d.nz, h.data(), nstep, time, dtm1, ctx->sc.grav);
  if (rc) ctx->err = std::string("cannot write the restart file ") + path;
  return rc;
}

int eddy_load_field(eddy_ctx *ctx, int field, const char *path, int *nstep, double *time, double *dtm1,
                    double *grav) {
  if (check_ctx(ctx) || field < 0 || field >= EDDY_PLANEU || !path) return EDDY_EINVAL;
  std::vector<double> h((size_t)ctx->d.ncell);
  int rc = eddy_ioscalar_read(path, ctx->d.nx, ctx->d.ny, ctx->d.nz, h.data(), nstep, time, dtm1, grav);
  if (rc) {
    ctx->err = std::string("cannot read the restart file ") + path + " (missing, truncated or another grid)";
    return rc;
  }
  return eddy_upload(ctx, field, h.data());
}

int eddy_get_metric(eddy_ctx *ctx, int which, double *out, int n) {
  if (check_ctx(ctx) || which < 0 || which >= 28 || !out) return -1;
  const std::vector<double> &h = ctx->h[which];
  int off = (which >= 18 && which <= 20) || which == 27 ? 0 : 1;
  int len = (int)h.size() - (off ? 2 : 0);
  if (which >= 18 && which <= 20) len = (int)h.size();
  if (n < len) return -2;
  std::memcpy(out, h.data() + off, sizeof(double) * (size_t)len);
  return len;
}

int eddy_grid_metric(const eddy_params *prm, const double *xu_faces, double ymin, double ymax,
                     const double *zw_faces, int which, double *out, int n) {
  if (!prm || !xu_faces || !zw_faces || !out || which < 0 || which >= 28) return -1;
  if (prm->nx < 6 || prm->ny < 4 || prm->nz < 6) return -1;
  eddy_ctx tmp;
  tmp.prm = *prm;
  build_metrics(&tmp, xu_faces, ymin, ymax, zw_faces);
  return eddy_get_metric(&tmp, which, out, n);
}

int eddy_rhs_predictord(eddy_ctx *ctx, double alfxdt, double gamxdt, double rhoxdt) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  return launch_rhs_predictord(ctx, alfxdt, gamxdt, rhoxdt);
}

int eddy_inversey(eddy_ctx *ctx, double alfxdt) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  if (ctx->prm.imply != 1 && ctx->prm.implcy != 1) {
    ctx->err = "eddy_inversey needs imply = 1 or implcy = 1";
    return EDDY_EINVAL;
  }
  return launch_inversey(ctx, alfxdt);
}

int eddy_inversex(eddy_ctx *ctx, double alfxdt) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  if (ctx->prm.implx != 1 && ctx->prm.implcx != 1) {
    ctx->err = "eddy_inversex needs implx = 1 or implcx = 1";
    return EDDY_EINVAL;
  }
  return launch_inversex(ctx, alfxdt);
}

int eddy_boundary(eddy_ctx *ctx, int set) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  double **f = ctx->f;
  if (set == 0) return launch_boundary(ctx, f[EDDY_US], f[EDDY_VS], f[EDDY_WS]);
  return launch_boundary(ctx, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO]);
}

int eddy_boundinout(eddy_ctx *ctx, int idiv, double alfxdt) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  double **f = ctx->f;
  if (idiv == 1)
    return launch_boundinout(ctx, f[EDDY_US], f[EDDY_VS], f[EDDY_WS], f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], alfxdt, 1);
  return launch_boundinout(ctx, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], f[EDDY_US], f[EDDY_VS], f[EDDY_WS], alfxdt, 0);
}

int eddy_direct(eddy_ctx *ctx, double alfxdt) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  return launch_direct(ctx, ctx->f[EDDY_US], ctx->f[EDDY_VS], ctx->f[EDDY_WS], alfxdt);
}

int eddy_correct(eddy_ctx *ctx, double alfxdt) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  return launch_correct(ctx, alfxdt);
}

int eddy_pressure_update(eddy_ctx *ctx) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  return launch_pressure_update(ctx);
}

int eddy_density(eddy_ctx *ctx, double alfxdt, double gamxdt, double rhoxdt) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  if (ctx->prm.idens != 1) return EDDY_OK;
  return launch_density(ctx, alfxdt, gamxdt, rhoxdt);
}

int eddy_turvis(eddy_ctx *ctx) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  if (ctx->prm.isgs == 0) return EDDY_OK;
  int rc = ctx->mixed ? mixed_turvis(ctx) : launch_turvis(ctx);
  if (rc == EDDY_OK && ctx->mixed) rc = mixed_after_sgs(ctx);
  return rc;
}

int eddy_ib_set_body(eddy_ctx *ctx, int nb, const double *vertices, const double *normals,
                     const double *velocity) {
  if (check_ctx(ctx) || nb < 0 || (nb > 0 && (!vertices || !normals))) return EDDY_EINVAL;
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  return ib_set_body(ctx, nb, vertices, normals, velocity);
}

int eddy_ib_set_cadence(eddy_ctx *ctx, int every_substep) {
  if (check_ctx(ctx) || !ctx->ib) return EDDY_EINVAL;
  return ib_set_cadence(ctx, every_substep);
}

int eddy_ib_move(eddy_ctx *ctx, double tmove) {
  if (check_ctx(ctx) || !ctx->ib) return EDDY_EINVAL;
  return ib_move(ctx, tmove);
}

int eddy_ib_regen(eddy_ctx *ctx) {
  if (check_ctx(ctx) || !ctx->ib) return EDDY_EINVAL;
  return ib_regen(ctx);
}

int eddy_ib_momforc(eddy_ctx *ctx) {
  if (check_ctx(ctx) || !ctx->ib) return EDDY_EINVAL;
  const double *vb = ib_velocity(ctx);
  double **f = ctx->f;
  int rc;
  if ((rc = ib_force(ctx, 0, 0, f[EDDY_US], vb[0], vb[0], nullptr, 0))) return rc;
  if ((rc = ib_force(ctx, 1, 1, f[EDDY_VS], vb[1], vb[1], nullptr, 0))) return rc;
  return ib_force(ctx, 2, 2, f[EDDY_WS], vb[2], vb[2], nullptr, 0);
}

int eddy_ib_correct(eddy_ctx *ctx, int field) {
  if (check_ctx(ctx) || !ctx->ib || (field != EDDY_P && field != EDDY_DENS)) return EDDY_EINVAL;
  return ib_force(ctx, 3, 4, ctx->f[field], 0.0, 0.0, nullptr, 0);
}

int eddy_ib_flags(eddy_ctx *ctx, int which, signed char *out) {
  if (check_ctx(ctx) || !ctx->ib || !out) return EDDY_EINVAL;
  return ib_download(ctx, which, out);
}

int eddy_ib_limits(eddy_ctx *ctx, int *lim6) {
  if (check_ctx(ctx) || !ctx->ib || !lim6) return EDDY_EINVAL;
  return ib_limits(ctx, lim6);
}

int eddy_ib_stencils(eddy_ctx *ctx, int q, int *n, int *nlev, int *ijk, int *dijk, int *lev, double *xn,
                     double *lu, int *indx) {
  if (check_ctx(ctx) || !ctx->ib) return EDDY_EINVAL;
  return ib_stencils(ctx, q, n, nlev, ijk, dijk, lev, xn, lu, indx);
}

int eddy_ib_stencil_kinds(eddy_ctx *ctx, int q, int *mrk, int *dir, double *xe) {
  if (check_ctx(ctx) || !ctx->ib) return EDDY_EINVAL;
  return ib_stencil_kinds(ctx, q, mrk, dir, xe);
}

int eddy_refine_residuals(eddy_ctx *ctx, double *out, int n) {
  if (check_ctx(ctx) || !out || n < 1) return EDDY_EINVAL;
  if (!ctx->mixed) {
    ctx->err = "refinement residuals exist only in the mixed-precision form";
    return EDDY_EINVAL;
  }
  return mixed_residuals(ctx, out, n);
}

int eddy_initialize(eddy_ctx *ctx, double dt) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  const Dims &d = ctx->d;
  double **f = ctx->f;
  int rc;
  if ((rc = launch_boundary(ctx, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO]))) return rc;
  // BOUNDARY_DENS alone (the inlet plane is applied after BOUNDINOUT below)
  double *dn = f[EDDY_DENS];
  if (d.itype[3] == 500) {
    if ((rc = launch_fill_plane(ctx, dn, 1, 1, d.jy2, 1., 0))) return rc;
    if ((rc = launch_fill_plane(ctx, dn, 1, d.ny, d.jy1, 1., 0))) return rc;
  }
  // pressure ghosts (src/Eddy6.f:585-617)
  double *p = f[EDDY_P];
  double sx = d.mp == 0 ? 1. : -1.;
  if ((rc = launch_fill_plane(ctx, p, 0, 1, d.mp == 0 ? d.ix2 : d.ix1, sx, 0))) return rc;
  if ((rc = launch_fill_plane(ctx, p, 0, d.nx, d.mp == 0 ? d.ix1 : d.ix2, sx, 0))) return rc;
  if ((rc = launch_fill_plane(ctx, p, 1, 1, d.lp == 0 ? d.jy2 : d.jy1, 1., 0))) return rc;
  if ((rc = launch_fill_plane(ctx, p, 1, d.ny, d.lp == 0 ? d.jy1 : d.jy2, 1., 0))) return rc;
  if ((rc = launch_fill_plane(ctx, p, 2, 1, d.kz1, 1., 0))) return rc;
  if ((rc = launch_fill_plane(ctx, p, 2, d.nz, d.kz2, 1., 0))) return rc;
  double gam[3], rho[3], alf[3];
  scheme(ctx->prm.ischm, gam, rho, alf);
  if ((rc = launch_boundinout(ctx, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], f[EDDY_UO], f[EDDY_VO], f[EDDY_WO],
                              alf[0] * dt, 1)))
    return rc;
  if ((rc = launch_boundary(ctx, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO]))) return rc;
  if (ctx->prm.idens == 1) {
    // BOUNDINOUTD only (src/Eddy6.f:757)
    if (d.itype[5] == 305) {
      EDDY_CUDA(cudaMemcpyAsync(dn, f[EDDY_PLANED], sizeof(double) * d.nx * d.ny, cudaMemcpyDeviceToDevice,
                                ctx->stream));
      if ((rc = launch_fill_plane(ctx, dn, 2, 2, 1, 1., 0))) return rc;
    }
    if (d.itype[6] == 730) {
      if ((rc = launch_fill_plane(ctx, dn, 2, d.kz2, d.kz2 - 1, 1., 0))) return rc;
      if ((rc = launch_fill_plane(ctx, dn, 2, d.nz, d.kz2, 1., 0))) return rc;
    }
    EDDY_CUDA(cudaMemcpyAsync(ctx->dens_alt, dn, sizeof(double) * d.ncell, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  if (ctx->prm.isgs != 0 && (rc = launch_turvis(ctx))) return rc;
  EDDY_CUDA(cudaMemcpyAsync(ctx->tv_dyn, f[EDDY_TV], sizeof(double) * d.ncell, cudaMemcpyDeviceToDevice, ctx->stream));
  EDDY_CUDA(cudaMemcpyAsync(ctx->kappa, f[EDDY_TV], sizeof(double) * d.ncell, cudaMemcpyDeviceToDevice, ctx->stream));
  if (ctx->mixed) {
    // FP32 copies of every field the mixed form reads
    const int fl[] = {EDDY_UO, EDDY_VO, EDDY_WO, EDDY_P, EDDY_DENS, EDDY_TV, EDDY_UA, EDDY_VA, EDDY_WA, EDDY_RHA};
    for (int q : fl)
      if ((rc = mixed_from64(ctx, q))) return rc;
  }
  return EDDY_OK;
}

// sequence_hybrid (src/hybrid.f:213-260): the inflow planes of sequence
// position pos, the cells i >= iref from the last (reference) plane; one
// thread per (i, j)
__global__ void k_feed_load(int nx, int ny, const double *feed, int pos, int last, int iref, double *pu, double *pv,
                            double *pw, double *pd) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const long long n2 = (long long)nx * ny;
  if (t >= n2) return;
  const int i = 1 + t % nx;
  const double *src = feed + (long long)(i >= iref ? last : pos) * 4 * n2;
  pu[t] = src[t];
  pv[t] = src[n2 + t];
  pw[t] = src[2 * n2 + t];
  pd[t] = src[3 * n2 + t];
}

// the plane of cycle c into the inlet planes: position c - n floor(c / n) of
// the feed (icycle_feed, src/hybrid.f:224-232)
static int feed_load(eddy_ctx *ctx, int c) {
  if (!ctx->feed || ctx->feed_n <= 0) return EDDY_OK;
  const int n = ctx->feed_n;
  const int pos = c - (int)std::floor((double)c / (double)n) * n;
  const long long n2 = (long long)ctx->d.nx * ctx->d.ny;
  double **f = ctx->f;
  k_feed_load<<<(unsigned)((n2 + 255) / 256), 256, 0, ctx->stream>>>(ctx->d.nx, ctx->d.ny, ctx->feed, pos, n - 1,
                                                                     ctx->feed_iref, f[EDDY_PLANEU], f[EDDY_PLANEV],
                                                                     f[EDDY_PLANEW], f[EDDY_PLANED]);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

int eddy_inflow_sequence(eddy_ctx *ctx, int n, const double *planes, int iref, int nstep) {
  if (check_ctx(ctx) || n < 0 || (n > 0 && !planes)) return EDDY_EINVAL;
  if (ctx->feed) {
    EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->feed);
    ctx->feed = nullptr;
  }
  ctx->feed_n = 0;
  if (n == 0) return EDDY_OK;
  const size_t b = sizeof(double) * 4 * (size_t)ctx->d.nx * ctx->d.ny * (size_t)n;
  EDDY_CUDA(cudaMalloc(&ctx->feed, b));
  EDDY_CUDA(cudaMemcpyAsync(ctx->feed, planes, b, cudaMemcpyHostToDevice, ctx->stream));
  ctx->feed_n = n;
  ctx->feed_iref = iref;
  ctx->icycle = nstep;
  // the start-up read of cycle nstep - 1 (src/Eddy6.f:806-814)
  int rc = feed_load(ctx, nstep - 1);
  if (rc) return rc;
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  return EDDY_OK;
}

int eddy_inflow_cycle(eddy_ctx *ctx, int icycle) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  ctx->icycle = icycle;
  return EDDY_OK;
}

static int substep_core(eddy_ctx *ctx, int is, double dt);

// one substep, then the inflow plane of the current cycle (sequence_hybrid
// after each substep, src/Eddy6.f:2985-2991)
int eddy_substep(eddy_ctx *ctx, int is, double dt) {
  int rc = substep_core(ctx, is, dt);
  if (rc) return rc;
  return feed_load(ctx, ctx->icycle);
}

static int substep_core(eddy_ctx *ctx, int is, double dt) {
  if (check_ctx(ctx) || is < 0 || is > 2) return EDDY_EINVAL;
  double gam[3], rho[3], alf[3];
  scheme(ctx->prm.ischm, gam, rho, alf);
  double alfxdt = alf[is] * dt, gamxdt = gam[is] * dt, rhoxdt = rho[is] * dt;
  int rc;
  // moving body: RBM, then new tags and stencils (src/Eddy6.f:2163-2380), every
  // substep over alfxdt, or at the first substep over the whole step.  They
  // run on the second stream while the predictor runs on the main stream
  // (the predictor does not read the body's data; the forcing after it waits)
  if (ctx->ib && (ib_every_substep(ctx) || is == 0)) {
    if (is == 0 && ctx->ib_prefetched) {
      ctx->ib_prefetched = 0;  // queued at the end of the previous step (eddy_step)
    } else {
      if ((rc = ib_join(ctx))) return rc;
      EDDY_CUDA(cudaEventRecord(ctx->ib_ev[0], ctx->stream));
      ctx->ib_move_dt = ib_every_substep(ctx) ? alfxdt : dt;
    }
  }
  if (ctx->mixed) return mixed_substep(ctx, alfxdt, gamxdt, rhoxdt);
  double **f = ctx->f;
  {
    ProfScope ps(ctx, PROF_RHS_PRED);
    if ((rc = launch_rhs_predictord(ctx, alfxdt, gamxdt, rhoxdt))) return rc;
  }
  const bool implicit = ctx->sc.imply == 1 || ctx->sc.implx == 1;
  // with a body and the C.N. steps the forcing comes first, from the explicit
  // estimate UB the predictor wrote (src/Eddy6.f:2495-2575, impl = 1)
  if (ctx->ib && implicit) {
    if ((rc = ib_overlap_regen(ctx))) return rc;
    {
      ProfScope ps(ctx, PROF_BC);
      if ((rc = launch_boundary(ctx, f[EDDY_UB], f[EDDY_VB], f[EDDY_WB]))) return rc;
      if ((rc = launch_boundinout(ctx, f[EDDY_UB], f[EDDY_VB], f[EDDY_WB], f[EDDY_UO], f[EDDY_VO], f[EDDY_WO],
                                  alfxdt, 1)))
        return rc;
      if ((rc = launch_boundary(ctx, f[EDDY_UB], f[EDDY_VB], f[EDDY_WB]))) return rc;
    }
    ProfScope ps(ctx, PROF_IB_FORCE);
    const double *vb = ib_velocity(ctx);
    if ((rc = ib_force_impl(ctx, 0, 0, f[EDDY_US], f[EDDY_UB], vb[0]))) return rc;
    if ((rc = ib_force_impl(ctx, 1, 1, f[EDDY_VS], f[EDDY_VB], vb[1]))) return rc;
    if ((rc = ib_force_impl(ctx, 2, 2, f[EDDY_WS], f[EDDY_WB], vb[2]))) return rc;
  }
  if (!implicit && (rc = ib_overlap_regen(ctx))) return rc;
  // momforc_mod2 + velinterior (src/Eddy6.f:2526-2575), before any line
  // solve of the convective terms alone (impl = 0)
  if (ctx->ib && !implicit) {
    ProfScope ps(ctx, PROF_IB_FORCE);
    const double *vb = ib_velocity(ctx);
    if ((rc = ib_force(ctx, 0, 0, f[EDDY_US], vb[0], vb[0], nullptr, 0))) return rc;
    if ((rc = ib_force(ctx, 1, 1, f[EDDY_VS], vb[1], vb[1], nullptr, 0))) return rc;
    if ((rc = ib_force(ctx, 2, 2, f[EDDY_WS], vb[2], vb[2], nullptr, 0))) return rc;
  }
  // Crank-Nicolson y, then x lines (src/Eddy6.f:2596-2607)
  if (ctx->sc.imply == 1 || ctx->sc.implcy == 1) {
    ProfScope ps(ctx, PROF_CN_LINES);
    if ((rc = launch_inversey(ctx, alfxdt))) return rc;
  }
  if (ctx->sc.implx == 1 || ctx->sc.implcx == 1) {
    ProfScope ps(ctx, PROF_CN_LINES);
    if ((rc = launch_inversex(ctx, alfxdt))) return rc;
  }
  {
    ProfScope ps(ctx, PROF_BC);
    if ((rc = launch_boundary(ctx, f[EDDY_US], f[EDDY_VS], f[EDDY_WS]))) return rc;
    if ((rc = launch_boundinout(ctx, f[EDDY_US], f[EDDY_VS], f[EDDY_WS], f[EDDY_UO], f[EDDY_VO], f[EDDY_WO],
                                alfxdt, 1)))
      return rc;
    if ((rc = launch_boundary(ctx, f[EDDY_US], f[EDDY_VS], f[EDDY_WS]))) return rc;
  }
  if ((rc = launch_direct(ctx, f[EDDY_US], f[EDDY_VS], f[EDDY_WS], alfxdt))) return rc;
  {
    ProfScope ps(ctx, PROF_CORRECT);
    if ((rc = launch_correct(ctx, alfxdt))) return rc;
  }
  {
    ProfScope ps(ctx, PROF_BC);
    if ((rc = launch_boundary(ctx, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO]))) return rc;
    if ((rc = launch_boundinout(ctx, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], f[EDDY_US], f[EDDY_VS], f[EDDY_WS],
                                alfxdt, 0)))
      return rc;
    if ((rc = launch_boundary(ctx, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO]))) return rc;
  }
  {
    ProfScope ps(ctx, PROF_PUPDATE);
    if ((rc = launch_pressure_update(ctx))) return rc;
  }
  if (ctx->prm.idens == 1) {
    ProfScope ps(ctx, PROF_DENSITY);
    if ((rc = launch_density(ctx, alfxdt, gamxdt, rhoxdt))) return rc;
  }
  return EDDY_OK;
}

int eddy_step(eddy_ctx *ctx, double dt, int nsteps) {
  if (check_ctx(ctx) || nsteps < 0) return EDDY_EINVAL;
  int nsub = ctx->prm.ischm == 1 ? 1 : 3;
  for (int n = 0; n < nsteps; n++) {
    ctx->icycle++;  // do icycle=1+nstep,... (src/Eddy6.f:2095)
    for (int is = 0; is < nsub; is++) {
      int rc = eddy_substep(ctx, is, dt);
      if (rc) return rc;
    }
    // within one call the next step's move (same dt) and regeneration run on
    // the second stream during this step's eddy viscosity update; they only
    // need this step's forcing to be done (the event), and tvinterior below
    // keeps reading the current tv flag (double-buffered)
    const bool prefetch = ctx->ib && !ib_every_substep(ctx) && n + 1 < nsteps && ctx->prm.isgs != 0;
    if (prefetch) {
      int rc = ib_join(ctx);
      if (rc) return rc;
      EDDY_CUDA(cudaEventRecord(ctx->ib_ev[0], ctx->stream));
    }
    if (ctx->prm.isgs != 0) {
      int rc;
      // the learned closure writes the mixed form's FP32 copies itself
      const bool closure = ctx->prm.closure == 1;
      {
        ProfScope ps(ctx, PROF_TURVIS);
        if (closure) {
          rc = launch_closure(ctx, ctx->tv_dyn, ctx->kappa, nullptr);
        } else {
          rc = ctx->mixed ? mixed_turvis(ctx) : launch_turvis(ctx);
        }
        if (rc) return rc;
      }
      // tvinterior (src/Eddy6.f:3040-3042)
      MixedViews mv{};
      const bool mirror = ctx->mixed && closure && mixed_views(ctx, &mv) == EDDY_OK;
      if (ctx->ib && (rc = ib_interior(ctx, 3, ctx->f[EDDY_TV], 0.0, mirror ? mv.tv : nullptr, mv.px))) return rc;
      if (ctx->mixed && !closure && (rc = mixed_after_sgs(ctx))) return rc;
    }
    if (prefetch) {
      int rc;
      if ((rc = ib_swap_tv_flag(ctx))) return rc;
      if ((rc = ib_prefetch_async(ctx, dt))) return rc;
      ctx->ib_prefetched = 1;
    }
    // TIME after the step (the RK3 / AB2 alphas sum to one), then the time
    // probes (rec_timeprobes_all, src/Eddy6.f:3640)
    ctx->time += dt;
    if (ctx->nprobe > 0) {
      int rc = probes_record(ctx);
      if (rc) return rc;
    }
  }
  return EDDY_OK;
}

int eddy_set_time(eddy_ctx *ctx, double time) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  ctx->time = time;
  return EDDY_OK;
}

int eddy_get_time(eddy_ctx *ctx, double *time) {
  if (check_ctx(ctx) || !time) return EDDY_EINVAL;
  *time = ctx->time;
  return EDDY_OK;
}

// the learned closure's fallback bookkeeping: fraction of cells outside the
// training envelope in the last closure evaluation
int closure_envelope_check(eddy_ctx *ctx, unsigned long long *nout) {
  return launch_closure(ctx, ctx->tv_dyn, ctx->kappa, nout);
}

int eddy_poisson_solve(eddy_ctx *ctx, const double *rhs, double *sol, int on_device) {
  if (check_ctx(ctx) || !rhs || !sol) return EDDY_EINVAL;
  size_t b = sizeof(double) * (size_t)ctx->d.ncell;
  if (on_device) return ctx->mixed ? mixed_poisson_rhs(ctx, rhs, sol) : launch_poisson_rhs(ctx, rhs, sol);
  // host arrays: stage through DP / US on the device
  EDDY_CUDA(cudaMemcpyAsync(ctx->f[EDDY_US], rhs, b, cudaMemcpyHostToDevice, ctx->stream));
  int rc = ctx->mixed ? mixed_poisson_rhs(ctx, ctx->f[EDDY_US], ctx->f[EDDY_DP])
                      : launch_poisson_rhs(ctx, ctx->f[EDDY_US], ctx->f[EDDY_DP]);
  if (rc) return rc;
  EDDY_CUDA(cudaMemcpyAsync(sol, ctx->f[EDDY_DP], b, cudaMemcpyDeviceToHost, ctx->stream));
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  return EDDY_OK;
}

int eddy_closure_apply(eddy_ctx *ctx, long long *out_of_envelope) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  unsigned long long n = 0;
  int rc;
  if ((rc = launch_closure(ctx, ctx->tv_dyn, ctx->kappa, &n))) return rc;
  if (ctx->mixed && (rc = mixed_after_sgs(ctx))) return rc;
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  if (out_of_envelope) *out_of_envelope = (long long)n;
  return EDDY_OK;
}

int eddy_closure_refresh_fallback(eddy_ctx *ctx) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  int rc = launch_turvis(ctx);
  if (rc) return rc;
  if (ctx->mixed && (rc = mixed_after_sgs(ctx))) return rc;
  EDDY_CUDA(cudaMemcpyAsync(ctx->tv_dyn, ctx->f[EDDY_TV], sizeof(double) * ctx->d.ncell, cudaMemcpyDeviceToDevice,
                            ctx->stream));
  ctx->closure_refresh++;
  return EDDY_OK;
}

int eddy_download_kappa(eddy_ctx *ctx, double *host) {
  if (check_ctx(ctx) || !host) return EDDY_EINVAL;
  EDDY_CUDA(cudaMemcpyAsync(host, ctx->kappa, sizeof(double) * ctx->d.ncell, cudaMemcpyDeviceToHost, ctx->stream));
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  return EDDY_OK;
}

int eddy_max_divergence(eddy_ctx *ctx, double *out) {
  if (check_ctx(ctx) || !out) return EDDY_EINVAL;
  return launch_max_divergence(ctx, out);
}

int eddy_profile_enable(eddy_ctx *ctx, unsigned mask) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  for (ProfEvent &e : ctx->prof_ev) ctx->prof_pool.push_back(e);
  ctx->prof_ev.clear();
  ctx->prof_mask = mask;
  for (int c = 0; c < PROF_NCAT; c++) { ctx->prof_ms[c] = 0.; ctx->prof_n[c] = 0; }
  return EDDY_OK;
}

int eddy_profile_read(eddy_ctx *ctx, double *ms, long long *counts) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  if (int rcj = ib_join(ctx)) return rcj;
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  if (ctx->ib) EDDY_CUDA(cudaStreamSynchronize(ctx->ib_stream));
  std::lock_guard<std::mutex> lk(ctx->prof_mu);
  for (ProfEvent &e : ctx->prof_ev) {
    float t = 0.f;
    EDDY_CUDA(cudaEventElapsedTime(&t, e.a, e.b));
    ctx->prof_ms[e.cat] += t;
    ctx->prof_n[e.cat] += 1;
    ctx->prof_pool.push_back(e);
  }
  ctx->prof_ev.clear();
  for (int c = 0; c < PROF_NCAT; c++) {
    if (ms) ms[c] = ctx->prof_ms[c];
    if (counts) counts[c] = ctx->prof_n[c];
  }
  return EDDY_OK;
}

int eddy_sync(eddy_ctx *ctx) {
  if (check_ctx(ctx)) return EDDY_EINVAL;
  if (int rcj = ib_join(ctx)) return rcj;
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  int e = 0;
  EDDY_CUDA(cudaMemcpy(&e, ctx->err_flag, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    cudaMemset(ctx->err_flag, 0, sizeof(int));
    ctx->err = "a device-side bounded wait expired (a kernel's barrier wait gave up)";
    return EDDY_ETIMEOUT;
  }
  return EDDY_OK;
}

int eddy_last_error(eddy_ctx *ctx, char *buf, int len) {
  if (!ctx || !buf || len <= 0) return EDDY_EINVAL;
  std::snprintf(buf, (size_t)len, "%s", ctx->err.c_str());
  return EDDY_OK;
}

int64_t eddy_launch_count(eddy_ctx *ctx) { return ctx ? ctx->launches.load() : -1; }

void *eddy_stream(eddy_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

}  // extern "C"
