// k_sgs.cu -- dynamic eddy viscosity TURVIS (src/vt.f:16-442), Cartesian,
// y-periodic, y-average branch (vt.f:296-318).
//
//   T0 centred velocities UC,VC,WC over the whole array (vt.f:64-74)
//   T1 strain S_ij and |S| at interior cells plus the periodic y-ghost rows
//      (STRAIN vt.f:955-1018, copies vt.f:176-191)
//   T2 one pass per cell: the 22 test filters (filter3d vt.f:1132-1268, the
//      x, y, z passes evaluated in the reference's order so the rounding is
//      the same), M_ij, M_ij M_ij and L_ij M_ij (vt.f:216-290)
//   T3 clip LM<0 and average MM, LM along y per (i,k) (vt.f:305-316),
//      BOUNDTURB on the 2-D averages
//   T4 TV = (ILM/IMM) Delta^2 |S| where IMM > sqrt(eps), >= 0 (vt.f:416-427)
//      and BOUNDTURB(TV) ghosts.
#include <cmath>
#include <vector>

#include "eddy_internal.h"

#define A(a, i, j, k) (a)[fidx(d, (i), (j), (k))]

int launch_fill_plane(eddy_ctx *ctx, double *a, int axis, int dst, int src, double sgn, int zero);

namespace {

constexpr int BX = 32, BY = 4, BZ = 2;

__global__ void __launch_bounds__(BX *BY *BZ)
    k_center(Dims d, const double *__restrict__ uo, const double *__restrict__ vo, const double *__restrict__ wo,
             double *__restrict__ uc, double *__restrict__ vc, double *__restrict__ wc) {
  int i = 1 + threadIdx.x + blockIdx.x * BX;
  int j = 1 + threadIdx.y + blockIdx.y * BY;
  int k = 1 + threadIdx.z + blockIdx.z * BZ;
  if (i > d.nx || j > d.ny || k > d.nz) return;
  long long q = fidx(d, i, j, k);
  // UC
  if (i >= d.ix1 && i <= d.ix2) uc[q] = 0.5 * (A(uo, i - 1, j, k) + uo[q]);
  else if (i == 1) uc[q] = 2. * uo[q] - 0.5 * (A(uo, d.ix1 - 1, j, k) + A(uo, d.ix1, j, k));
  else uc[q] = 2. * A(uo, d.ix2, j, k) - 0.5 * (A(uo, d.ix2 - 1, j, k) + A(uo, d.ix2, j, k));
  // VC
  if (j >= d.jy1 && j <= d.jy2) vc[q] = 0.5 * (A(vo, i, j - 1, k) + vo[q]);
  else if (j == 1) vc[q] = 2. * vo[q] - 0.5 * (A(vo, i, d.jy1 - 1, k) + A(vo, i, d.jy1, k));
  else vc[q] = 2. * A(vo, i, d.jy2, k) - 0.5 * (A(vo, i, d.jy2 - 1, k) + A(vo, i, d.jy2, k));
  // WC
  if (k >= d.kz1 && k <= d.kz2) wc[q] = 0.5 * (A(wo, i, j, k - 1) + wo[q]);
  else if (k == 1) wc[q] = 2. * wo[q] - 0.5 * (A(wo, i, j, d.kz1 - 1) + A(wo, i, j, d.kz1));
  else wc[q] = 2. * A(wo, i, j, d.kz2) - 0.5 * (A(wo, i, j, d.kz2 - 1) + A(wo, i, j, d.kz2));
}

// strain at (i,j,k) interior; sij layout: 6 fields of ncell (xx,yy,zz,xy,xz,yz)
__global__ void __launch_bounds__(BX *BY *BZ)
    k_strain(Dims d, DevMetrics m, const double *__restrict__ uc, const double *__restrict__ vc,
             const double *__restrict__ wc, double *__restrict__ sij, double *__restrict__ gs) {
  int i = 1 + threadIdx.x + blockIdx.x * BX;
  int jj = 1 + threadIdx.y + blockIdx.y * BY;
  int k = 1 + threadIdx.z + blockIdx.z * BZ;
  if (i < d.ix1 || i > d.ix2 || jj > d.ny || k < d.kz1 || k > d.kz2) return;
  // periodic y-ghost rows take the value of the mapped interior row
  int j = jj == 1 ? d.jy2 : (jj == d.ny ? 2 : jj);
  const int sy = d.nx;
  const long long sz = (long long)d.nx * d.ny;
  long long q = fidx(d, i, j, k);
  const double *au = m.au, *bv = m.bv, *cw = m.cw;
  double dudxp = au[i] * (uc[q+1] - uc[q]);
  double dudxm = au[i - 1] * (uc[q] - uc[q-1]);
  double dudyp = bv[j] * (uc[q+sy] - uc[q]);
  double dudym = bv[j - 1] * (uc[q] - uc[q-sy]);
  double dudzp = cw[k] * (uc[q+sz] - uc[q]);
  double dudzm = cw[k - 1] * (uc[q] - uc[q-sz]);
  double dvdxp = au[i] * (vc[q+1] - vc[q]);
  double dvdxm = au[i - 1] * (vc[q] - vc[q-1]);
  double dvdyp = bv[j] * (vc[q+sy] - vc[q]);
  double dvdym = bv[j - 1] * (vc[q] - vc[q-sy]);
  double dvdzp = cw[k] * (vc[q+sz] - vc[q]);
  double dvdzm = cw[k - 1] * (vc[q] - vc[q-sz]);
  double dwdxp = au[i] * (wc[q+1] - wc[q]);
  double dwdxm = au[i - 1] * (wc[q] - wc[q-1]);
  double dwdyp = bv[j] * (wc[q+sy] - wc[q]);
  double dwdym = bv[j - 1] * (wc[q] - wc[q-sy]);
  double dwdzp = cw[k] * (wc[q+sz] - wc[q]);
  double dwdzm = cw[k - 1] * (wc[q] - wc[q-sz]);
  double sxx = 0.5 * (dudxp + dudxm);
  double syy = 0.5 * (dvdyp + dvdym);
  double szz = 0.5 * (dwdzp + dwdzm);
  double sxy = 0.25 * (dudyp + dudym + dvdxp + dvdxm);
  double sxz = 0.25 * (dudzp + dudzm + dwdxp + dwdxm);
  double syz = 0.25 * (dwdyp + dwdym + dvdzp + dvdzm);
  long long qo = fidx(d, i, jj, k), n = d.ncell;
  sij[qo] = sxx; sij[qo + n] = syy; sij[qo + 2 * n] = szz;
  sij[qo + 3 * n] = sxy; sij[qo + 4 * n] = sxz; sij[qo + 5 * n] = syz;
  gs[qo] = sqrt(2. * (sxx * sxx + syy * syy + szz * szz) + 4. * (sxy * sxy + syz * syz + sxz * sxz));
}

// the 22 filtered quantities at one point from the base fields
struct Base {
  double uc, vc, wc, g, s[6];
};

__device__ __forceinline__ void load_base(const Dims &d, long long q, const double *__restrict__ uc,
                                          const double *__restrict__ vc, const double *__restrict__ wc,
                                          const double *__restrict__ gs, const double *__restrict__ sij,
                                          Base &b) {
  long long n = d.ncell;
  b.uc = uc[q]; b.vc = vc[q]; b.wc = wc[q]; b.g = gs[q];
#pragma unroll
  for (int c = 0; c < 6; c++) b.s[c] = sij[q + c * n];
}

// order: 0-5 G*S(xx,yy,zz,xy,yz,xz), 6-11 S(xx,yy,zz,xy,yz,xz), 12 G,
// 13-15 uc,vc,wc, 16-21 uc*uc, vc*vc, wc*wc, uc*vc, vc*wc, uc*wc
__device__ __forceinline__ double quant(const Base &b, int c) {
  // S storage order is xx,yy,zz,xy,xz,yz; the reference filters xx,yy,zz,xy,yz,xz
  const int sidx[6] = {0, 1, 2, 3, 5, 4};
  if (c < 6) return b.g * b.s[sidx[c]];
  if (c < 12) return b.s[sidx[c - 6]];
  if (c == 12) return b.g;
  if (c == 13) return b.uc;
  if (c == 14) return b.vc;
  if (c == 15) return b.wc;
  if (c == 16) return b.uc * b.uc;
  if (c == 17) return b.vc * b.vc;
  if (c == 18) return b.wc * b.wc;
  if (c == 19) return b.uc * b.vc;
  if (c == 20) return b.vc * b.wc;
  return b.uc * b.wc;
}

constexpr int NQ = 22;

__global__ void __launch_bounds__(128)
    k_dynamic(Dims d, DevMetrics m, const double *__restrict__ uc, const double *__restrict__ vc,
              const double *__restrict__ wc, const double *__restrict__ gs, const double *__restrict__ sij,
              const double *__restrict__ dxdydz, double *__restrict__ mm, double *__restrict__ lm,
              int top_onesided, int bot_onesided) {
  int i = d.ix1 + threadIdx.x + blockIdx.x * 32;
  int j = d.jy1 + threadIdx.y + blockIdx.y * 4;
  int k = d.kz1 + blockIdx.z;
  if (i > d.ix2 || j > d.jy2) return;
  // x-pass stencil (vt.f:1156-1169)
  int xi[3];
  double wx[3];
  const double *whx = m.whx, *whz = m.whz;
  if (i == d.ix1) { xi[0] = d.ix1; xi[1] = d.ix1 + 1; xi[2] = d.ix1 + 2; }
  else if (i == d.ix2) { xi[0] = d.ix2; xi[1] = d.ix2 - 1; xi[2] = d.ix2 - 2; }
  else { xi[0] = i - 1; xi[1] = i; xi[2] = i + 1; }
  wx[0] = whx[i * 3 + 0]; wx[1] = whx[i * 3 + 1]; wx[2] = whx[i * 3 + 2];
  // z-pass stencil (vt.f:1216-1264)
  int zk[3];
  double wz[3] = {whz[k * 3 + 0], whz[k * 3 + 1], whz[k * 3 + 2]};
  if (k == d.kz1 && bot_onesided) { zk[0] = d.kz1; zk[1] = d.kz1 + 1; zk[2] = d.kz1 + 2; }
  else if (k == d.kz2 && top_onesided) { zk[0] = d.kz2; zk[1] = d.kz2 - 1; zk[2] = d.kz2 - 2; }
  else { zk[0] = k - 1; zk[1] = k; zk[2] = k + 1; }
  const double wy[3] = {0.25, 0.50, 0.25};
  const long long q0 = fidx(d, i, j, k), nxy = (long long)d.nx * d.ny;
  double Z[NQ];
#pragma unroll
  for (int c = 0; c < NQ; c++) Z[c] = 0.;
  for (int a = 0; a < 3; a++) {
    double Y[NQ];
#pragma unroll
    for (int c = 0; c < NQ; c++) Y[c] = 0.;
    for (int b = 0; b < 3; b++) {
      int jj = j - 1 + b;
      double X[NQ];
#pragma unroll
      for (int c = 0; c < NQ; c++) X[c] = 0.;
      for (int e = 0; e < 3; e++) {
        Base bs;
        load_base(d, q0 + (xi[e] - i) + (long long)(jj - j) * d.nx + (long long)(zk[a] - k) * nxy, uc, vc, wc, gs,
                  sij, bs);
#pragma unroll
        for (int c = 0; c < NQ; c++) {
          double t = wx[e] * quant(bs, c);
          X[c] = (e == 0) ? t : X[c] + t;
        }
      }
#pragma unroll
      for (int c = 0; c < NQ; c++) {
        double t = wy[b] * X[c];
        Y[c] = (b == 0) ? t : Y[c] + t;
      }
    }
#pragma unroll
    for (int c = 0; c < NQ; c++) {
      double t = wz[a] * Y[c];
      Z[c] = (a == 0) ? t : Z[c] + t;
    }
  }
  long long q = fidx(d, i, j, k);
  const double C = 1.0, R = 6.;
  double dx = dxdydz[q];
  double gb = Z[12];
  double mxx = C * dx * (R * gb * Z[6] - Z[0]);
  double myy = C * dx * (R * gb * Z[7] - Z[1]);
  double mzz = C * dx * (R * gb * Z[8] - Z[2]);
  double mxy = C * dx * (R * gb * Z[9] - Z[3]);
  double myz = C * dx * (R * gb * Z[10] - Z[4]);
  double mxz = C * dx * (R * gb * Z[11] - Z[5]);
  mm[q] = mxx * mxx + myy * myy + mzz * mzz + 2. * (mxy * mxy + myz * myz + mxz * mxz);
  double uh = Z[13], vh = Z[14], wh = Z[15];
  double lxx = (Z[16] - uh * uh) * mxx;
  double lyy = (Z[17] - vh * vh) * myy;
  double lzz = (Z[18] - wh * wh) * mzz;
  double lxy = (Z[19] - uh * vh) * mxy;
  double lyz = (Z[20] - vh * wh) * myz;
  double lxz = (Z[21] - uh * wh) * mxz;
  lm[q] = lxx + lyy + lzz + 2. * (lxy + lyz + lxz);
}

// y averages per (i,k) into 2-D arrays (NX,NZ), summed in j order
__global__ void k_yavg(Dims d, const double *__restrict__ mm, const double *__restrict__ lm, double *imm2,
                       double *ilm2) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int mi = d.ix2 - d.ix1 + 1, mk = d.kz2 - d.kz1 + 1;
  if (t >= mi * mk) return;
  int i = d.ix1 + t % mi, k = d.kz1 + t / mi;
  double sm = 0., sl = 0.;
  for (int j = d.jy1; j <= d.jy2; j++) {
    long long q = fidx(d, i, j, k);
    sm += mm[q];
    double l = lm[q];
    if (l < 0.) l = 0.;
    sl += l;
  }
  imm2[(i - 1) + d.nx * (k - 1)] = sm / (double)(d.ny - 2);
  ilm2[(i - 1) + d.nx * (k - 1)] = sl / (double)(d.ny - 2);
}

// BOUNDTURB on a j-independent (NX,NZ) array: x sides then z sides
__global__ void k_boundturb2(Dims d, double *a, int iflg) {
  // single block: the x-side fills, then the z-side fills, in order
  for (int ib = 1; ib <= 6; ib++) {
    int t = d.itype[ib];
    int mode = 0;
    if (iflg == 0) {
      if (t > 700) mode = 2;
      else if (t != 0 && t != 500 && t != 300) mode = 1;
    } else {
      if (t != 0 && t != 500 && t != 300) mode = 2;
    }
    if (!mode || ib == 3 || ib == 4) continue;
    double sg = mode == 1 ? -1. : 1.;
    if (ib <= 2) {
      int dst = ib == 1 ? 1 : d.nx, src = ib == 1 ? 2 : d.ix2;
      for (int k = 1 + threadIdx.x; k <= d.nz; k += blockDim.x)
        a[(dst - 1) + d.nx * (k - 1)] = sg * a[(src - 1) + d.nx * (k - 1)];
    } else {
      int dst = ib == 5 ? 1 : d.nz, src = ib == 5 ? 2 : d.kz2;
      for (int i = 1 + threadIdx.x; i <= d.nx; i += blockDim.x)
        a[(i - 1) + d.nx * (dst - 1)] = sg * a[(i - 1) + d.nx * (src - 1)];
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256)
    k_tv(Dims d, const double *__restrict__ ilm2, const double *__restrict__ imm2,
         const double *__restrict__ dxdydz, const double *__restrict__ gs, double *__restrict__ tv, double seps) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= d.ncell) return;
  int i = 1 + (int)(q % d.nx);
  int k = 1 + (int)(q / ((long long)d.nx * d.ny));
  int j = 1 + (int)((q / d.nx) % d.ny);
  if (i < d.ix1 || i > d.ix2 || j < d.jy1 || j > d.jy2 || k < d.kz1 || k > d.kz2) return;
  double il = ilm2[(i - 1) + d.nx * (k - 1)], im = imm2[(i - 1) + d.nx * (k - 1)];
  if (il < 0) il = 0.;
  double v = 0.;
  if (im > seps) v = (il / im) * dxdydz[q] * gs[q];
  if (v < 0.0) v = 0.0;
  tv[q] = v;
}

__global__ void __launch_bounds__(256)
    k_smag(Dims d, const double *__restrict__ dxdydz, const double *__restrict__ gs, double *__restrict__ tv,
           double css) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= d.ncell) return;
  tv[q] = css * css * 1.0 * dxdydz[q] * gs[q];
}

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

int launch_turvis(eddy_ctx *ctx) {
  const Dims &d = ctx->d;
  cudaStream_t st = ctx->stream;
  dim3 blk(BX, BY, BZ), g((d.nx + BX - 1) / BX, (d.ny + BY - 1) / BY, (d.nz + BZ - 1) / BZ);
  double **f = ctx->f;
  k_center<<<g, blk, 0, st>>>(d, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], ctx->uc, ctx->vc, ctx->wc);
  EDDY_LAUNCHED(ctx);
  k_strain<<<g, blk, 0, st>>>(d, ctx->m, ctx->uc, ctx->vc, ctx->wc, ctx->sij, ctx->gs);
  EDDY_LAUNCHED(ctx);
  double *tv = f[EDDY_TV];
  long long nb = (d.ncell + 255) / 256;
  if (ctx->prm.isgs == 1) {
    k_smag<<<(unsigned)nb, 256, 0, st>>>(d, ctx->dxdydz, ctx->gs, tv, ctx->sc.css);
    EDDY_LAUNCHED(ctx);
  } else {
    int mi = d.ix2 - d.ix1 + 1, mj = d.jy2 - d.jy1 + 1, mk = d.kz2 - d.kz1 + 1;
    dim3 g2((mi + 31) / 32, (mj + 3) / 4, mk);
    k_dynamic<<<g2, dim3(32, 4, 1), 0, st>>>(d, ctx->m, ctx->uc, ctx->vc, ctx->wc, ctx->gs, ctx->sij, ctx->dxdydz,
                                             ctx->mm, ctx->lm, d.itype[6] > 0, d.itype[5] > 0);
    EDDY_LAUNCHED(ctx);
    k_yavg<<<(mi * mk + 255) / 256, 256, 0, st>>>(d, ctx->mm, ctx->lm, ctx->imm2, ctx->ilm2);
    EDDY_LAUNCHED(ctx);
    k_boundturb2<<<1, 256, 0, st>>>(d, ctx->ilm2, 0);
    EDDY_LAUNCHED(ctx);
    k_boundturb2<<<1, 256, 0, st>>>(d, ctx->imm2, 1);
    EDDY_LAUNCHED(ctx);
    k_tv<<<(unsigned)nb, 256, 0, st>>>(d, ctx->ilm2, ctx->imm2, ctx->dxdydz, ctx->gs, tv, std::sqrt(ctx->sc.eps));
    EDDY_LAUNCHED(ctx);
  }
  // BOUNDTURB(TV,0) (vt.f:700-757)
  int rc;
#define F(...) \
  if ((rc = launch_fill_plane(ctx, __VA_ARGS__)) != EDDY_OK) return rc
  for (int ib = 1; ib <= 6; ib++) {
    int t = d.itype[ib];
    int mode = 0;
    if (t > 700) mode = 2;
    else if (t != 0 && t != 500 && t != 300) mode = 1;
    if (!mode) continue;
    double sg = mode == 1 ? -1. : 1.;
    switch (ib) {
      case 1: F(tv, 0, 1, 2, sg, 0); break;
      case 2: F(tv, 0, d.nx, d.ix2, sg, 0); break;
      case 3: F(tv, 1, 1, 2, sg, 0); break;
      case 4: F(tv, 1, d.ny, d.jy2, sg, 0); break;
      case 5: F(tv, 2, 1, 2, sg, 0); break;
      case 6: F(tv, 2, d.nz, d.kz2, sg, 0); break;
    }
  }
  for (int ib = 1; ib <= 4; ib++) {
    if (d.itype[ib] != 500) continue;
    switch (ib) {
      case 1: F(tv, 0, 1, d.ix2, 1., 0); break;
      case 2: F(tv, 0, d.nx, 2, 1., 0); break;
      case 3: F(tv, 1, 1, d.jy2, 1., 0); break;
      case 4: F(tv, 1, d.ny, 2, 1., 0); break;
    }
  }
#undef F
  return EDDY_OK;
}
