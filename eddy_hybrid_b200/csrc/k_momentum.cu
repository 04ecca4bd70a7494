// k_momentum.cu -- momentum right-hand side fused with the RK predictor,
// boundary-condition plane fills, BOUNDINOUT, CORRECT and the pressure update.
//
// Plain FP64 form: compiled with -fmad=false so every expression rounds in the
// reference's operation order (src/rhs.f, src/timeindeg.f); the explicit
// (non Crank-Nicolson) branch of the Cartesian equations.
#include "eddy_internal.h"
#include "tma_ring.cuh"
#include "bc_templates.cuh"

#define A(a, i, j, k) (a)[fidx(d, (i), (j), (k))]

namespace {

constexpr int BX = 32, BY = 4, BZ = 2;

#include "stencil_rhs.cuh"

// RHS + PREDICTORD + sponges (src/rhs.f:4-438, src/timeindeg.f:1041-1265).
// A block owns a 32x8 tile of (i,j) columns and marches along k over a chunk
// of planes; planes of uo,vo,wo,tv,p,dens,ua,va,wa (one-cell halo in i and j)
// stream into the shared-memory ring of tma_ring.cuh.
constexpr int TX = 32, TY = 8, NFLD = 9, KCHUNK = 32;  // uo vo wo tv p dens ua va wa
using Acc9 = RingAcc<TX, TY, NFLD>;

struct MomAcc {
  const Acc9 &r;
  __device__ __forceinline__ double u(int di, int dj, int dk) const { return r.at(0, di, dj, dk); }
  __device__ __forceinline__ double v(int di, int dj, int dk) const { return r.at(1, di, dj, dk); }
  __device__ __forceinline__ double w(int di, int dj, int dk) const { return r.at(2, di, dj, dk); }
  __device__ __forceinline__ double t(int di, int dj, int dk) const { return r.at(3, di, dj, dk); }
};

// CN: any implicit flag on, f the terms that form the C.N. part; ub, vb, wb
// (viscous C.N. steps with an immersed body, else null): the explicit estimate u* +
// alfxdt/2 (C.N. part) the implicit forcing reads (UB = US + 0.5*ALFXDT*UB,
// src/Eddy6.f:2499-2501)
template <bool CN>
__global__ void __launch_bounds__(TX *TY)
    k_rhs_predictord(Dims d, DevMetrics m, Scalars s, const __grid_constant__ TmaMaps<NFLD> maps,
                     double *__restrict__ us, double *__restrict__ vs, double *__restrict__ ws,
                     double *__restrict__ ua, double *__restrict__ va, double *__restrict__ wa, double alfxdt,
                     double gamxdt, double rhoxdt, int *err, double *__restrict__ ub, double *__restrict__ vb,
                     double *__restrict__ wb, CnFlags<double> f) {
  const double coef = 0.5 * alfxdt, coefd = alfxdt;
  tma_march<NFLD, TX, TY, KCHUNK>(
      d.ix1, d.ix2, d.jy1, d.jy2, d.kz1, d.kz2, maps, err, [&](int i, int j, int k, bool active, const Acc9 &R) {
        if (!active) return;
        MomAcc S{R};
        long long q = fidx(d, i, j, k);
        const bool jin = j >= d.jy1 && j <= d.jy2;
        const bool kin = (k >= d.kz1 && k <= d.kz2);
        // ---- u ----
        double uval = 0.0, ubv = 0.0;
        if (kin && jin && i >= d.ibu && i <= d.ieu) {
          double ucn = 0.0;  // the C.N. part (IMPLY / IMPLX), else 0
          double ur = rhs_u<double, DevMetrics, MomAcc, CN>(S, m, s.ru1, i, j, k, &ucn, &f);
          double ustar = R.at(0, 0, 0, 0) + gamxdt * ur + rhoxdt * R.at(6, 0, 0, 0) -
                         alfxdt * m.au[i] * (R.at(4, 1, 0, 0) - R.at(4, 0, 0, 0)) + coef * ucn - alfxdt * s.dpdx;
          if (s.idens == 1)
            ustar = ustar - coefd * 0.50 * s.grav *
                                ((R.at(5, 1, 0, 0) - m.dens_bg[i + d.nx * (j - 1)]) +
                                 (R.at(5, 0, 0, 0) - m.dens_bg[(i - 1) + d.nx * (j - 1)]));
          ua[q] = ur;
          if (i >= d.ieu - s.vspngx1) ustar = ustar + m.dfxu[i] * (0. - ustar) * alfxdt * 1.0;
          if (s.ivspngl == 1) ustar = ustar + m.dfxul[k] * (0. - ustar) * alfxdt * 1.0;
          uval = ustar;
          ubv = ustar + coef * ucn;
        }
        us[q] = uval;
        if (ub) ub[q] = ubv;
        // ---- v ----
        double vval = 0.0, vbv = 0.0;
        if (kin && j >= d.jbv && j <= d.jev && i >= d.ix1 && i <= d.ix2) {
          double vcn = 0.0;
          double vr = rhs_v<double, DevMetrics, MomAcc, CN>(S, m, s.ru1, i, j, k, &vcn, &f);
          double vstar = R.at(1, 0, 0, 0) + gamxdt * vr + rhoxdt * R.at(7, 0, 0, 0) -
                         alfxdt * m.bv[j] * (R.at(4, 0, 1, 0) - R.at(4, 0, 0, 0)) + coef * vcn - alfxdt * s.dpdy;
          va[q] = vr;
          if (i >= d.ix2 - s.vspngx1) vstar = vstar + m.dfxw[i] * (0. - vstar) * alfxdt * 1.0;
          if (s.ivspngl == 1 && i >= d.ibu && i <= d.ieu && jin)
            vstar = vstar + m.dfxwl[k] * (0. - vstar) * alfxdt * 1.0;
          vval = vstar;
          vbv = vstar + coef * vcn;
        }
        vs[q] = vval;
        if (vb) vb[q] = vbv;
        // ---- w ----
        double wval = 0.0, wbv = 0.0;
        if (k >= d.kbw && k <= d.kew && jin && i >= d.ix1 && i <= d.ix2) {
          double wcn = 0.0;
          double wr = rhs_w<double, DevMetrics, MomAcc, CN>(S, m, s.ru1, i, j, k, &wcn, &f);
          double wstar = R.at(2, 0, 0, 0) + gamxdt * wr + rhoxdt * R.at(8, 0, 0, 0) -
                         alfxdt * m.cw[k] * (R.at(4, 0, 0, 1) - R.at(4, 0, 0, 0)) + coef * wcn - alfxdt * s.dpdz;
          wa[q] = wr;
          if (i >= d.ix2 - s.vspngx1) wstar = wstar + m.dfxw[i] * (1. - wstar) * alfxdt * 1.0;
          if (s.ivspngl == 1) wstar = wstar + m.dfxwl[k] * (1. - wstar) * alfxdt * 1.0;
          wval = wstar;
          wbv = wstar + coef * wcn;
        }
        ws[q] = wval;
        if (wb) wb[q] = wbv;
      });
}

// ghost faces of u*,v*,w* are zero (RHS zeroes the whole arrays, src/rhs.f:65-70)
__global__ void k_zero_faces3(Dims d, double *a, double *b, double *c3) {
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
  a[q] = 0.;
  b[q] = 0.;
  c3[q] = 0.;
}

// CORRECT (src/timeindeg.f:981-1028)
__global__ void __launch_bounds__(BX *BY *BZ)
    k_correct(Dims d, DevMetrics m, const double *__restrict__ us, const double *__restrict__ vs,
              const double *__restrict__ ws, const double *__restrict__ dp, double *__restrict__ uo,
              double *__restrict__ vo, double *__restrict__ wo, double alfxdt) {
  int i = 1 + threadIdx.x + blockIdx.x * BX;
  int j = 1 + threadIdx.y + blockIdx.y * BY;
  int k = 1 + threadIdx.z + blockIdx.z * BZ;
  if (i > d.nx || j > d.ny || k > d.nz) return;
  long long q = fidx(d, i, j, k);
  const int sy = d.nx;
  const long long sz = (long long)d.nx * d.ny;
  bool kin = k >= d.kz1 && k <= d.kz2, jin = j >= d.jy1 && j <= d.jy2;
  if (kin && jin && i >= d.ibu && i <= d.ieu)
    uo[q] = us[q] - m.au[i] * (dp[q + 1] - dp[q]) * alfxdt;
  if (kin && j >= d.jbv && j <= d.jev && i >= d.ix1 && i <= d.ix2)
    vo[q] = vs[q] - m.bv[j] * (dp[q + sy] - dp[q]) * alfxdt;
  if (k >= d.kbw && k <= d.kew && jin && i >= d.ix1 && i <= d.ix2)
    wo[q] = ws[q] - m.cw[k] * (dp[q + sz] - dp[q]) * alfxdt;
}

// pref = sum_j (p+dp)(ix1,j,2) / (NY-2), summed in order (src/Eddy6.f:2802)
// P + DP, then with IMPLY the correction of src/Eddy6.f:2775-2785 (rp = 1,
// RVIMPLY = 1) and with IMPLX that of :2787-2795 (rp = ru = 1, RVIMPLX = 1),
// both on i in [2, ix2], j in [2, jy2], k in [2, kz2]; cimp = 0.5 alfxdt ru1 /
// dely^2, 0 without IMPLY; cimpx = 0.5 alfxdt ru1, 0 without IMPLX
__device__ __forceinline__ double p_plus_dp(const Dims &d, const DevMetrics &m, const double *p, const double *dp,
                                            long long q, int i, int j, int k, double cimp, double cimpx) {
  double v = p[q] + dp[q];
  const bool in = i >= 2 && i <= d.ix2 && j >= 2 && j <= d.jy2 && k >= 2 && k <= d.kz2;
  if (cimp != 0.0 && in) v = v - cimp * ((dp[q - d.nx] - 2. * dp[q]) + dp[q + d.nx]) * 1.0;
  if (cimpx != 0.0 && in)
    v = v - cimpx * m.ap[i] / 1.0 *
                ((dp[q + 1] - dp[q]) * m.au[i] * 1.0 - (dp[q] - dp[q - 1]) * m.au[i - 1] * 1.0) * 1.0;
  return v;
}

__global__ void k_pref(Dims d, DevMetrics m, const double *p, const double *dp, double *out, double cimp,
                       double cimpx) {
  double s = 0.;
  for (int j = d.jy1; j <= d.jy2; j++) {
    long long q = fidx(d, d.ix1, j, 2);
    s += p_plus_dp(d, m, p, dp, q, d.ix1, j, 2, cimp, cimpx);
  }
  out[0] = s / (double)(d.ny - 2);
}

__global__ void __launch_bounds__(256)
    k_pupdate(Dims d, DevMetrics m, double *p, const double *dp, const double *pref, double cimp, double cimpx) {
  // blockIdx.y is the plane k; 32-bit index arithmetic inside the plane
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int n2 = d.nx * d.ny;
  if (t >= n2) return;
  const int k = 1 + blockIdx.y, j = 1 + t / d.nx, i = 1 + (t - (j - 1) * d.nx);
  const long long q = (long long)blockIdx.y * n2 + t;
  p[q] = p_plus_dp(d, m, p, dp, q, i, j, k, cimp, cimpx) - pref[0];
}

// final pressure ghosts: value of the mapped interior cell (the composition
// of the z, x, y fills of src/Eddy6.f:2911-2953)
__device__ __forceinline__ int map_axis(int a, int n, int lo, int hi, int periodic, int active) {
  if (!active) return a;
  if (a == 1) return periodic ? hi : lo;
  if (a == n) return periodic ? lo : hi;
  return a;
}

__global__ void k_pghost(Dims d, double *p) {
  // threads over all ghost cells of the 6 faces (grid-stride over the volume
  // surface via three plane sets)
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long sxy = (long long)d.nx * d.ny, sxz = (long long)d.nx * d.nz, syz = (long long)d.ny * d.nz;
  int i, j, k;
  if (t < 2 * sxy) {
    int f = (int)(t / sxy);
    long long r = t % sxy;
    i = 1 + (int)(r % d.nx); j = 1 + (int)(r / d.nx); k = f ? d.nz : 1;
  } else if (t < 2 * sxy + 2 * sxz) {
    long long u = t - 2 * sxy;
    int f = (int)(u / sxz);
    long long r = u % sxz;
    i = 1 + (int)(r % d.nx); k = 1 + (int)(r / d.nx); j = f ? d.ny : 1;
  } else if (t < 2 * sxy + 2 * sxz + 2 * syz) {
    long long u = t - 2 * sxy - 2 * sxz;
    int f = (int)(u / syz);
    long long r = u % syz;
    j = 1 + (int)(r % d.ny); k = 1 + (int)(r / d.ny); i = f ? d.nx : 1;
  } else {
    return;
  }
  int zact = d.itype[5] != 0 || d.itype[6] != 0;
  int zper = d.itype[5] == 500;
  int si = map_axis(i, d.nx, d.ix1, d.ix2, d.mp == 0, 1);
  int sj = map_axis(j, d.ny, d.jy1, d.jy2, d.lp == 0, 1);
  int sk = map_axis(k, d.nz, d.kz1, d.kz2, zper, zact);
  if (si == i && sj == j && sk == k) return;
  p[fidx(d, i, j, k)] = p[fidx(d, si, sj, sk)];
}

inline dim3 grid3(const Dims &d) {
  return dim3((d.nx + BX - 1) / BX, (d.ny + BY - 1) / BY, (d.nz + BZ - 1) / BZ);
}

}  // namespace

int launch_fill_plane(eddy_ctx *ctx, double *a, int axis, int dst, int src, double sgn, int zero) {
  return bc_fill<double>(ctx, ctx->d.nx, a, axis, dst, src, sgn, zero);
}

int launch_rhs_predictord(eddy_ctx *ctx, double alfxdt, double gamxdt, double rhoxdt) {
  const Dims &d = ctx->d;
  double **f = ctx->f;
  TmaMaps<NFLD> maps;
  const double *src[NFLD] = {f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], f[EDDY_TV], f[EDDY_P], f[EDDY_DENS],
                             f[EDDY_UA], f[EDDY_VA], f[EDDY_WA]};
  for (int q = 0; q < NFLD; q++) {
    const CUtensorMap *mp = ctx_tensor_map(ctx, src[q], RingGeom<TX, TY>::PX, TY + 2);
    if (!mp) return EDDY_ECUDA;
    maps.m[q] = *mp;
  }
  size_t smem = ring_smem_bytes<NFLD, TX, TY>();
  dim3 g((d.ix2 - d.ix1 + TX) / TX, (d.jy2 - d.jy1 + TY) / TY, (d.kz2 - d.kz1 + KCHUNK) / KCHUNK);
  const CnFlags<double> fl{(double)ctx->sc.implx, (double)ctx->sc.imply, (double)ctx->sc.implcx,
                           (double)ctx->sc.implcy};
  const bool cn = ctx->sc.imply == 1 || ctx->sc.implx == 1 || ctx->sc.implcx == 1 || ctx->sc.implcy == 1;
  auto kern = cn ? k_rhs_predictord<true> : k_rhs_predictord<false>;
  EDDY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // the implicit forcing's explicit estimate (impl = 1: viscous C.N. steps with a body)
  const bool est = (ctx->sc.imply == 1 || ctx->sc.implx == 1) && ctx->ib;
  double *ub = est ? f[EDDY_UB] : nullptr, *vb = est ? f[EDDY_VB] : nullptr, *wb = est ? f[EDDY_WB] : nullptr;
  kern<<<g, dim3(TX, TY), smem, ctx->stream>>>(d, ctx->m, ctx->sc, maps, f[EDDY_US], f[EDDY_VS], f[EDDY_WS],
                                              f[EDDY_UA], f[EDDY_VA], f[EDDY_WA], alfxdt, gamxdt, rhoxdt,
                                              ctx->err_flag, ub, vb, wb, fl);
  EDDY_LAUNCHED(ctx);
  long long nghost = 2LL * d.nx * d.ny + 2LL * d.nx * d.nz + 2LL * d.ny * d.nz;
  k_zero_faces3<<<(unsigned)((nghost + 255) / 256), 256, 0, ctx->stream>>>(d, f[EDDY_US], f[EDDY_VS],
                                                                            f[EDDY_WS]);
  EDDY_LAUNCHED(ctx);
  if (est) {
    k_zero_faces3<<<(unsigned)((nghost + 255) / 256), 256, 0, ctx->stream>>>(d, ub, vb, wb);
    EDDY_LAUNCHED(ctx);
  }
  return EDDY_OK;
}

// BOUNDARY (src/boundary.f:7-66)
int launch_boundary(eddy_ctx *ctx, double *u, double *v, double *w) {
  return bc_boundary<double>(ctx, ctx->d.nx, u, v, w);
}

// BOUNDINOUT (src/boundary.f:505-994)
int launch_boundinout(eddy_ctx *ctx, double *ubc, double *vbc, double *wbc, const double *uof,
                      const double *vof, const double *wof, double alfxdt, int idiv) {
  return bc_boundinout<double, double>(ctx, ctx->d.nx, ctx->d.nx, ubc, vbc, wbc, uof, vof, wof, alfxdt, idiv);
}

int launch_correct(eddy_ctx *ctx, double alfxdt) {
  const Dims &d = ctx->d;
  ctx->alfxdt_last = alfxdt;
  double **f = ctx->f;
  k_correct<<<grid3(d), dim3(BX, BY, BZ), 0, ctx->stream>>>(d, ctx->m, f[EDDY_US], f[EDDY_VS], f[EDDY_WS],
                                                            f[EDDY_DP], f[EDDY_UO], f[EDDY_VO], f[EDDY_WO],
                                                            alfxdt);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

int launch_pressure_update(eddy_ctx *ctx) {
  const Dims &d = ctx->d;
  double *p = ctx->f[EDDY_P], *dp = ctx->f[EDDY_DP];
  const double cimp = ctx->sc.imply == 1 ? 0.5 * ctx->alfxdt_last * ctx->sc.ru1 / ((ctx->dely * 1.0) * (ctx->dely * 1.0))
                                         : 0.0;
  const double cimpx = ctx->sc.implx == 1 ? 0.5 * ctx->alfxdt_last * ctx->sc.ru1 : 0.0;
  k_pref<<<1, 1, 0, ctx->stream>>>(d, ctx->m, p, dp, ctx->scal, cimp, cimpx);
  EDDY_LAUNCHED(ctx);
  k_pupdate<<<dim3((unsigned)((d.nx * d.ny + 255) / 256), (unsigned)d.nz), 256, 0, ctx->stream>>>(
      d, ctx->m, p, dp, ctx->scal, cimp, cimpx);
  EDDY_LAUNCHED(ctx);
  // immersed body: correctpres_mod2 + presinterior (src/Eddy6.f:2881-2897)
  if (ctx->ib) {
    int rc = ib_force(ctx, 3, 4, p, 0.0, 0.0, nullptr, 0);
    if (rc) return rc;
  }
  long long nghost = 2LL * d.nx * d.ny + 2LL * d.nx * d.nz + 2LL * d.ny * d.nz;
  k_pghost<<<(unsigned)((nghost + 255) / 256), 256, 0, ctx->stream>>>(d, p);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}
