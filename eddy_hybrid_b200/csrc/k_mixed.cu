// k_mixed.cu -- the mixed-precision form of the time advance.
//
// Storage: FP32 copies of u, v, w, p, nu_t, kappa_t feed the stencils; the
// predictor outputs u*, v*, w*, the RHS history and the density live in FP32
// only.  FP64 is kept for
//   * the master velocities written by the projection (max|div u| is a
//     difference of nearly equal face fluxes and needs FP64 storage),
//   * the pressure and the Poisson solution,
//   * the per-wavenumber z-line elimination, the residual and the divergence.
// FP32 arrays are (NX,NY,NZ) with the row pitch rounded up to 4 elements so
// every row starts on a 16-byte boundary (TMA row strides).
//
// Poisson solve (src/direct.f:2-1118 semantics): the FP32 path (divergence in
// FP64 -> FP32 FFT along y -> FP32 eigen-transform GEMM -> FP64 Thomas along z
// on FP32 storage -> FP32 GEMM -> FP32 inverse FFT) is wrapped in FP64-residual
// iterative refinement: phi_0 = S(d); r_s = d - L phi_s (FP64); phi_{s+1} =
// phi_s + S(r_s).
#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "bc_templates.cuh"
#include "eddy_internal.h"
#include "tma_ring.cuh"

namespace {

#include "stencil_density.cuh"
#include "stencil_rhs.cuh"

// 1-D metric arrays in FP32 (same indexing as DevMetrics)
struct DevMetrics32 {
  float *ap, *au, *av, *aw;
  float *bp, *bu, *bv, *bw;
  float *cp, *cu, *cv, *cw;
  float *whx, *why, *whz;
  float *dfxu, *dfxw, *dfxul, *dfxwl, *dfxd, *dfxdl;
  float *dens_bg;
};

struct MixedState {
  int px = 0;      // row pitch (elements) of the FP32 arrays
  size_t n32 = 0;  // px * ny * nz
  float *uo = nullptr, *vo = nullptr, *wo = nullptr, *p = nullptr, *tv = nullptr, *kv = nullptr;
  float *us = nullptr, *vs = nullptr, *ws = nullptr, *ua = nullptr, *va = nullptr, *wa = nullptr;
  float *dens = nullptr, *dens_alt = nullptr, *rha = nullptr;
  float *mbuf = nullptr;
  DevMetrics32 m{};
  float *twr = nullptr, *twi = nullptr;  // FFT twiddles: forward table then backward table
  double *resid = nullptr;               // max |r| before each sweep (device, 4 entries)
  double *wout = nullptr;                // outlet-face w (NX,NY) in FP64: exact mass balance
  // 3xTF32 tensor-core transforms (null fmat: the FP64 tensor-core transforms of k_xform64.cu)
  XformPlan xp;
  float *cpz = nullptr;  // z-line c' of every (m, J) line (M*L*N, FP32), computed once per plan
};

MixedState *ms(eddy_ctx *ctx) { return static_cast<MixedState *>(ctx->mixed); }

// ---------------------------------------------------------------------------
// precision copies over the whole (NX,NY,NZ) array: blockIdx.y is the plane k,
// x runs over the NX*NY cells of the plane (32-bit index arithmetic)
struct PlaneCell {
  int i, j, k;
  long long t;  // the FP64 (unpadded) index
};

__device__ __forceinline__ bool plane_cell(const Dims &d, PlaneCell &c) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int n2 = d.nx * d.ny;
  if (q >= n2) return false;
  c.k = 1 + blockIdx.y;
  c.j = 1 + q / d.nx;
  c.i = 1 + (q - (c.j - 1) * d.nx);
  c.t = (long long)blockIdx.y * n2 + q;
  return true;
}

__global__ void k_to32(Dims d, int px, const double *__restrict__ a, float *__restrict__ b) {
  PlaneCell c;
  if (!plane_cell(d, c)) return;
  b[pidx(d, px, c.i, c.j, c.k)] = (float)a[c.t];
}

// one FP64 array to two FP32 copies (read once)
__global__ void k_to32x2(Dims d, int px, const double *__restrict__ a, float *__restrict__ b,
                         float *__restrict__ cc) {
  PlaneCell c;
  if (!plane_cell(d, c)) return;
  const float v = (float)a[c.t];
  const long long q = pidx(d, px, c.i, c.j, c.k);
  b[q] = v;
  cc[q] = v;
}

__global__ void k_to64(Dims d, int px, const float *__restrict__ b, double *__restrict__ a) {
  PlaneCell c;
  if (!plane_cell(d, c)) return;
  a[c.t] = (double)b[pidx(d, px, c.i, c.j, c.k)];
}

// ---------------------------------------------------------------------------
// RHS + PREDICTORD in FP32 (src/rhs.f:4-438, src/timeindeg.f:1041-1265) on the
// TMA plane ring; same structure as the FP64 kernel.
constexpr int TX = 32, TY = 8, NFLD = 9, KCHUNK = 64;  // uo vo wo tv p dens ua va wa
using Acc9 = RingAcc<TX, TY, NFLD, float>;

struct MomAcc32 {
  const Acc9 &r;
  __device__ __forceinline__ float u(int di, int dj, int dk) const { return r.at(0, di, dj, dk); }
  __device__ __forceinline__ float v(int di, int dj, int dk) const { return r.at(1, di, dj, dk); }
  __device__ __forceinline__ float w(int di, int dj, int dk) const { return r.at(2, di, dj, dk); }
  __device__ __forceinline__ float t(int di, int dj, int dk) const { return r.at(3, di, dj, dk); }
};

// metric values around one (i, j) column and one k plane, in registers: the
// stencil templates read m.xx[i + o], m.xx[j + o], m.xx[k + o] with o in
// {-1, 0, 1}, which fold to one of the three fields after inlining
struct Reg3 {
  float lo, mid, hi;
  int base;
  __device__ __forceinline__ float operator[](int idx) const {
    const int o = idx - base;
    return o < 0 ? lo : (o == 0 ? mid : hi);
  }
};

__device__ __forceinline__ Reg3 reg3(const float *a, int c) { return Reg3{a[c - 1], a[c], a[c + 1], c}; }

struct MetricCol32 {
  Reg3 ap, au, av, aw, bp, bu, bv, bw, cp, cu, cv, cw;
};

__global__ void __launch_bounds__(TX *TY)
    k_rhs32(Dims d, DevMetrics32 m, Scalars s, int px, const __grid_constant__ TmaMaps<NFLD> maps,
            float *__restrict__ us, float *__restrict__ vs, float *__restrict__ ws, float *__restrict__ ua,
            float *__restrict__ va, float *__restrict__ wa, float alfxdt, float gamxdt, float rhoxdt, int *err) {
  const float ru1 = (float)s.ru1, grav = (float)s.grav;
  const float dpdx = (float)s.dpdx, dpdy = (float)s.dpdy, dpdz = (float)s.dpdz;
  // this thread's column (the mapping of tma_march), clamped for idle threads
  const int ic = min(d.ix1 + (int)(blockIdx.x * TX + threadIdx.x), d.ix2);
  const int jc = min(d.jy1 + (int)(blockIdx.y * TY + threadIdx.y), d.jy2);
  MetricCol32 mc;
  mc.ap = reg3(m.ap, ic); mc.au = reg3(m.au, ic); mc.av = reg3(m.av, ic); mc.aw = reg3(m.aw, ic);
  mc.bp = reg3(m.bp, jc); mc.bu = reg3(m.bu, jc); mc.bv = reg3(m.bv, jc); mc.bw = reg3(m.bw, jc);
  const float dfxu_i = m.dfxu[ic], dfxw_i = m.dfxw[ic];
  const float bg1 = m.dens_bg[ic + d.nx * (jc - 1)], bg0 = m.dens_bg[(ic - 1) + d.nx * (jc - 1)];
  tma_march<NFLD, TX, TY, KCHUNK, float>(
      d.ix1, d.ix2, d.jy1, d.jy2, d.kz1, d.kz2, maps, err, [&](int i, int j, int k, bool active, const Acc9 &R) {
        if (!active) return;
        mc.cp = reg3(m.cp, k); mc.cu = reg3(m.cu, k); mc.cv = reg3(m.cv, k); mc.cw = reg3(m.cw, k);
        MomAcc32 S{R};
        long long q = pidx(d, px, i, j, k);
        const bool jin = j >= d.jy1 && j <= d.jy2;
        const bool kin = (k >= d.kz1 && k <= d.kz2);
        float uval = 0.f;
        if (kin && jin && i >= d.ibu && i <= d.ieu) {
          float ur = rhs_u<float>(S, mc, ru1, i, j, k);
          float ustar = R.at(0, 0, 0, 0) + gamxdt * ur + rhoxdt * R.at(6, 0, 0, 0) -
                        alfxdt * mc.au[i] * (R.at(4, 1, 0, 0) - R.at(4, 0, 0, 0)) - alfxdt * dpdx;
          if (s.idens == 1)
            ustar = ustar - alfxdt * 0.5f * grav * ((R.at(5, 1, 0, 0) - bg1) + (R.at(5, 0, 0, 0) - bg0));
          ua[q] = ur;
          if (i >= d.ieu - s.vspngx1) ustar = ustar + dfxu_i * (0.f - ustar) * alfxdt;
          if (s.ivspngl == 1) ustar = ustar + m.dfxul[k] * (0.f - ustar) * alfxdt;
          uval = ustar;
        }
        us[q] = uval;
        float vval = 0.f;
        if (kin && j >= d.jbv && j <= d.jev && i >= d.ix1 && i <= d.ix2) {
          float vr = rhs_v<float>(S, mc, ru1, i, j, k);
          float vstar = R.at(1, 0, 0, 0) + gamxdt * vr + rhoxdt * R.at(7, 0, 0, 0) -
                        alfxdt * mc.bv[j] * (R.at(4, 0, 1, 0) - R.at(4, 0, 0, 0)) - alfxdt * dpdy;
          va[q] = vr;
          if (i >= d.ix2 - s.vspngx1) vstar = vstar + dfxw_i * (0.f - vstar) * alfxdt;
          if (s.ivspngl == 1 && i >= d.ibu && i <= d.ieu && jin) vstar = vstar + m.dfxwl[k] * (0.f - vstar) * alfxdt;
          vval = vstar;
        }
        vs[q] = vval;
        float wval = 0.f;
        if (k >= d.kbw && k <= d.kew && jin && i >= d.ix1 && i <= d.ix2) {
          float wr = rhs_w<float>(S, mc, ru1, i, j, k);
          float wstar = R.at(2, 0, 0, 0) + gamxdt * wr + rhoxdt * R.at(8, 0, 0, 0) -
                        alfxdt * mc.cw[k] * (R.at(4, 0, 0, 1) - R.at(4, 0, 0, 0)) - alfxdt * dpdz;
          wa[q] = wr;
          if (i >= d.ix2 - s.vspngx1) wstar = wstar + dfxw_i * (1.f - wstar) * alfxdt;
          if (s.ivspngl == 1) wstar = wstar + m.dfxwl[k] * (1.f - wstar) * alfxdt;
          wval = wstar;
        }
        ws[q] = wval;
      });
}

// ghost faces of u*,v*,w* are zero (src/rhs.f:65-70)
__global__ void k_zero_faces32(Dims d, int px, float *a, float *b, float *c3) {
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
  long long q = pidx(d, px, i, j, k);
  a[q] = 0.f;
  b[q] = 0.f;
  c3[q] = 0.f;
}

// ---------------------------------------------------------------------------
// FP32 FFT along y on TI32 consecutive x lines per block (one k plane).
// Lane l of every warp owns line i0 + l for the whole block, warp w owns a
// contiguous run of JW = L/8 rows; lines l and l + 16 share one complex FFT
// (re, im).  Neighbours along y come from the previous/next iteration's
// registers and along x from the adjacent lanes (shuffles), so each element
// is loaded once; offsets within a k plane are 32-bit.
constexpr int TI32 = 32, FT32 = 256, HL32 = TI32 / 2;

inline size_t fft32_smem(int L) { return sizeof(float) * (2 * (size_t)L * HL32 + HL32 + L); }


#include "fft_lines.cuh"

// shared-memory slot of line `lane` at row r (the second half of the lines is
// the imaginary part; the im array is offset by 16 words so the two halves of
// a warp hit different banks)
__device__ __forceinline__ float &slot32(float *re, float *im, int r, int lane) {
  return lane < HL32 ? re[r * HL32 + lane] : im[r * HL32 + lane - HL32];
}

// Forward transform of the right-hand side.  MODE 0: d = div(u*)/alfxdt in
// FP64 from the FP32 predictor velocities (src/timeindeg.f:941-949), stored
// to dvec; MODE 1: d = dvec; MODE 2: r = dvec - L phi (FP64 residual of the
// DIRECT operator: Neumann x and z, periodic y), max|r| -> rmax.
template <int MODE>
__global__ void __launch_bounds__(FT32, 4)
    k_fwd32(Dims d, DevMetrics m, int px, const float *__restrict__ us, const float *__restrict__ vs,
            const float *__restrict__ ws, const double *__restrict__ win, const double *__restrict__ wout,
            const double *__restrict__ phi, double *__restrict__ dvec, double ralf, double rdy2, int code,
            const float *__restrict__ twr, const float *__restrict__ twi, float *__restrict__ spec,
            unsigned long long *rmax) {
  constexpr int U = 8;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ float smf[];
  __shared__ double red[FT32 / 32];
  const int L = fft_len(code), M = d.nx - 2;
  float *re = smf, *im = smf + L * HL32 + HL32;
  float *tsr = im + L * HL32, *tsi = tsr + L / 2;
  load_twiddles(tsr, tsi, twr, twi, L / 2);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i = d.ix1 + blockIdx.x * TI32 + lane;
  const bool act = i <= d.ix2;
  const int ic = act ? i : d.ix2;  // loads of idle lanes stay in bounds
  const int k = d.kz1 + blockIdx.y;
  const int JW = (L + 7) / 8, jb = min(L, warp * JW), je = min(L, jb + JW);
  const int nx = d.nx;
  double *D = dvec + fidx(d, ic, d.jy1, k);
  double amax = 0.;
  if (MODE == 0) {
    constexpr int U0 = 3;
    const long long pb = pidx(d, px, ic, d.jy1, k);
    const float *Us = us + pb, *Vs = vs + pb, *Ws = ws + pb;
    const int pz = px * d.ny;
    const bool top = k == d.kz2, bot = k == d.kz1;
    const double *Wo = wout + (ic - 1) + (long long)nx * (d.jy1 - 1);
    const double *Wi = win + (ic - 1) + (long long)nx * (d.jy1 - 1);
    const double api = m.ap[ic], cpk = m.cp[k];
    const double *bp = m.bp + d.jy1;
    double vprev = jb < je ? (double)Vs[(jb - 1) * px] : 0.;
    for (int j0 = jb; j0 < je; j0 += U0) {
      float uu[U0], ul[U0], vv[U0];
      double wk[U0], wm[U0];
#pragma unroll
      for (int u = 0; u < U0; u++) {
        const int jj = j0 + u;
        if (jj < je) {
          const int o = jj * px;
          uu[u] = Us[o];
          vv[u] = Vs[o];
          ul[u] = lane == 0 ? Us[o - 1] : 0.f;
          wk[u] = top ? Wo[jj * nx] : (double)Ws[o];
          wm[u] = bot ? Wi[jj * nx] : (double)Ws[o - pz];
        }
      }
#pragma unroll
      for (int u = 0; u < U0; u++) {
        const int jj = j0 + u;
        if (jj < je) {
          float w = __shfl_up_sync(FULL, uu[u], 1);
          if (lane == 0) w = ul[u];
          const double vc = (double)vv[u];
          double x = api * ((double)uu[u] - (double)w) + bp[jj] * (vc - vprev) + cpk * (wk[u] - wm[u]);
          x = act ? x * ralf : 0.;
          vprev = vc;
          if (act) D[jj * nx] = x;
          slot32(re, im, fft_slot(jj, code), lane) = (float)x;
        }
      }
    }
  } else if (MODE == 1) {
    for (int j0 = jb; j0 < je; j0 += U) {
      double v[U];
#pragma unroll
      for (int u = 0; u < U; u++) v[u] = (j0 + u < je) ? D[(j0 + u) * nx] : 0.;
#pragma unroll
      for (int u = 0; u < U; u++)
        if (j0 + u < je) slot32(re, im, fft_slot(j0 + u, code), lane) = act ? (float)v[u] : 0.f;
    }
  } else {
    constexpr int U2 = 2;
    const double *P = phi + fidx(d, ic, d.jy1, k);
    const int sz = nx * d.ny;
    const bool has_e = act && i < d.ix2, has_w = act && i > d.ix1;
    const bool kt = k < d.kz2, kb = k > d.kz1;
    const double ae = m.ap[ic] * m.au[ic], aw = m.ap[ic] * m.au[ic - 1];
    const double ct = m.cp[k] * m.cw[k], cb = m.cp[k] * m.cw[k - 1];
    double cprev = 0., ccur = 0.;
    if (jb < je) {
      cprev = P[((jb - 1 + L) % L) * nx];
      ccur = P[jb * nx];
    }
    for (int j0 = jb; j0 < je; j0 += U2) {
      // edge[u]: the east neighbour for lane 31, the west one for lane 0
      double cn[U2], tt[U2], bb[U2], dd[U2], edge[U2];
#pragma unroll
      for (int u = 0; u < U2; u++) {
        const int jj = j0 + u;
        if (jj < je) {
          const int o = jj * nx;
          cn[u] = P[(jj + 1 == L ? 0 : jj + 1) * nx];
          tt[u] = kt ? P[o + sz] : 0.;
          bb[u] = kb ? P[o - sz] : 0.;
          dd[u] = D[o];
          edge[u] = (lane == 31 && has_e) ? P[o + 1] : ((lane == 0 && has_w) ? P[o - 1] : 0.);
        }
      }
#pragma unroll
      for (int u = 0; u < U2; u++) {
        const int jj = j0 + u;
        if (jj < je) {
          const double c = ccur;
          double pe = __shfl_down_sync(FULL, c, 1), pw = __shfl_up_sync(FULL, c, 1);
          if (lane == 31) pe = edge[u];
          if (lane == 0) pw = edge[u];
          if (!has_e) pe = c;
          if (!has_w) pw = c;
          const double pt = kt ? tt[u] : c, pbm = kb ? bb[u] : c;
          const double lap = ae * (pe - c) + aw * (pw - c) + (cn[u] - 2. * c + cprev) * rdy2 + ct * (pt - c) +
                             cb * (pbm - c);
          const double x = act ? dd[u] - lap : 0.;
          amax = fmax(amax, fabs(x));
          slot32(re, im, fft_slot(jj, code), lane) = (float)x;
          cprev = c;
          ccur = cn[u];
        }
      }
    }
    for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(FULL, amax, o));
    if (lane == 0) red[warp] = amax;
  }
  __syncthreads();
  if (MODE == 2 && threadIdx.x == 0) {
    double b = 0.;
    for (int w = 0; w < FT32 / 32; w++) b = fmax(b, red[w]);
    atomicMax(rmax, (unsigned long long)__double_as_longlong(b));
  }
  fft_lines_any<float, HL32>(re, im, code, tsr, tsi);
  // separate the two real transforms: A_q = (Z_q + conj Z_{L-q}) / 2,
  // B_q = (Z_q - conj Z_{L-q}) / 2i; packed order [a0, a1, b1, ..., a_{L/2}]
  const int pl = lane & (HL32 - 1);
  const bool second = lane >= HL32;
  float *S = spec + (long long)(ic - d.ix1) + (long long)M * L * (k - d.kz1);
  for (int q = warp; q <= L / 2; q += FT32 / 32) {
    const int qm = q == 0 ? 0 : L - q;
    const float zr = re[q * HL32 + pl], zi = im[q * HL32 + pl];
    const float wr = re[qm * HL32 + pl], wi = im[qm * HL32 + pl];
    const float vr = second ? 0.5f * (zi + wi) : 0.5f * (zr + wr);
    const float vi = second ? 0.5f * (wr - zr) : 0.5f * (zi - wi);
    if (act) {
      if (q == 0) {
        S[0] = vr;
      } else if (q == L / 2) {
        S[(long long)M * (L - 1)] = vr;
      } else {
        S[(long long)M * (2 * q - 1)] = vr;
        S[(long long)M * (2 * q)] = vi;
      }
    }
  }
}

// (S - mean[J==0]) / L, Hermitian extension, inverse FFT; phi = (ACC ? phi +
// : ) result.  Lanes l < 16 hold A_q of line l, lanes l + 16 B_q of line
// l + 16; one shuffle gives each half the other's values to form Z_q (low
// half) and Z_{L-q} (high half).
template <int ACC>
__global__ void __launch_bounds__(FT32, 4)
    k_bwd32(Dims d, const float *__restrict__ spec, const double *__restrict__ dpm, int code,
            const float *__restrict__ twr, const float *__restrict__ twi, double *__restrict__ phi) {
  constexpr int U = 8;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ float smf[];
  const int L = fft_len(code), M = d.nx - 2;
  float *re = smf, *im = smf + L * HL32 + HL32;
  float *tsr = im + L * HL32, *tsi = tsr + L / 2;
  load_twiddles(tsr, tsi, twr, twi, L / 2);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i = d.ix1 + blockIdx.x * TI32 + lane;
  const bool act = i <= d.ix2;
  const int ic = act ? i : d.ix2;
  const int k = d.kz1 + blockIdx.y;
  const int pl = lane & (HL32 - 1);
  const bool low = lane < HL32;
  const float *S = spec + (long long)(ic - d.ix1) + (long long)M * L * (k - d.kz1);
  const float mean = (float)dpm[0], rl = 1.f / (float)L;
  for (int q0 = warp; q0 <= L / 2; q0 += U * (FT32 / 32)) {
    float a[U], b[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int q = q0 + u * (FT32 / 32);
      a[u] = 0.f;
      b[u] = 0.f;
      if (q <= L / 2 && act) {
        if (q == 0) {
          a[u] = S[0] - mean;
        } else if (q == L / 2) {
          a[u] = S[(long long)M * (L - 1)];
        } else {
          a[u] = S[(long long)M * (2 * q - 1)];
          b[u] = S[(long long)M * (2 * q)];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int q = q0 + u * (FT32 / 32);
      if (q <= L / 2) {
        const float ar = a[u] * rl, ai = b[u] * rl;
        const float orr = __shfl_xor_sync(FULL, ar, HL32), oi = __shfl_xor_sync(FULL, ai, HL32);
        if (low) {  // own A_q, other B_q: Z_q = (Ar - Bi) + i (Ai + Br)
          const int r = fft_slot(q, code);
          re[r * HL32 + pl] = ar - oi;
          im[r * HL32 + pl] = ai + orr;
        } else if (q != 0 && q != L / 2) {  // own B_q, other A_q: Z_{L-q} = (Ar + Bi) + i (Br - Ai)
          const int r = fft_slot(L - q, code);
          re[r * HL32 + pl] = orr + ai;
          im[r * HL32 + pl] = ar - oi;
        }
      }
    }
  }
  __syncthreads();
  fft_lines_any<float, HL32>(re, im, code, tsr, tsi);
  // real part -> line pl, imaginary part -> line pl + 16
  const int JW = (L + 7) / 8, jb = min(L, warp * JW), je = min(L, jb + JW);
  const int nx = d.nx;
  double *P = phi + fidx(d, ic, d.jy1, k);
  for (int j0 = jb; j0 < je; j0 += 8) {
    double old[8];
#pragma unroll
    for (int u = 0; u < 8; u++) old[u] = (ACC && act && j0 + u < je) ? P[(j0 + u) * nx] : 0.;
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int jj = j0 + u;
      if (jj < je && act) P[jj * nx] = old[u] + (double)slot32(re, im, jj, lane);
    }
  }
}
#include "tridiag_z.cuh"

__global__ void k_plane_sum32(int M, int L, int N, const float *__restrict__ s, double *part) {
  __shared__ double sh[256];
  double acc = 0.;
  long long n = (long long)M * N;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    long long k = t / M, i = t % M;
    acc += (double)s[i + (long long)M * L * k];
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_sum_final(int nparts, long long count, const double *part, double *out) {
  if (threadIdx.x != 0) return;
  double s = 0.;
  for (int b = 0; b < nparts; b++) s += part[b];
  out[0] = s / (double)count;
}

// ---------------------------------------------------------------------------
// CORRECT (src/timeindeg.f:981-1028) in FP64 onto the FP64 masters, with the
// FP32 copies written alongside
constexpr int BX = 32, BY = 4, BZ = 2;

__global__ void __launch_bounds__(BX *BY *BZ)
    k_correct_mixed(Dims d, DevMetrics m, int px, const float *__restrict__ us, const float *__restrict__ vs,
                    const float *__restrict__ ws, const double *__restrict__ dp, double *__restrict__ uo,
                    double *__restrict__ vo, double *__restrict__ wo, float *__restrict__ uo32,
                    float *__restrict__ vo32, float *__restrict__ wo32, double alfxdt) {
  int i = 1 + threadIdx.x + blockIdx.x * BX;
  int j = 1 + threadIdx.y + blockIdx.y * BY;
  int k = 1 + threadIdx.z + blockIdx.z * BZ;
  if (i > d.nx || j > d.ny || k > d.nz) return;
  long long q = fidx(d, i, j, k), p = pidx(d, px, i, j, k);
  const int sy = d.nx;
  const long long sz = (long long)d.nx * d.ny;
  bool kin = k >= d.kz1 && k <= d.kz2, jin = j >= d.jy1 && j <= d.jy2;
  if (kin && jin && i >= d.ibu && i <= d.ieu) {
    double u = (double)us[p] - m.au[i] * (dp[q + 1] - dp[q]) * alfxdt;
    uo[q] = u;
    uo32[p] = (float)u;
  }
  if (kin && j >= d.jbv && j <= d.jev && i >= d.ix1 && i <= d.ix2) {
    double v = (double)vs[p] - m.bv[j] * (dp[q + sy] - dp[q]) * alfxdt;
    vo[q] = v;
    vo32[p] = (float)v;
  }
  if (k >= d.kbw && k <= d.kew && jin && i >= d.ix1 && i <= d.ix2) {
    double w = (double)ws[p] - m.cw[k] * (dp[q + sz] - dp[q]) * alfxdt;
    wo[q] = w;
    wo32[p] = (float)w;
  }
}

// FP32 copies of the planes the velocity boundary conditions write:
// x planes 1, IX2, NX; y planes 1, NY; z planes 1, KZ2, NZ
__global__ void k_sync_planes(Dims d, int px, const double *__restrict__ u, const double *__restrict__ v,
                              const double *__restrict__ w, float *__restrict__ u32, float *__restrict__ v32,
                              float *__restrict__ w32) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long syz = (long long)d.ny * d.nz, sxz = (long long)d.nx * d.nz, sxy = (long long)d.nx * d.ny;
  int i, j, k;
  if (t < 3 * syz) {
    int f = (int)(t / syz);
    long long r = t % syz;
    j = 1 + (int)(r % d.ny); k = 1 + (int)(r / d.ny);
    i = f == 0 ? 1 : (f == 1 ? d.ix2 : d.nx);
  } else if (t < 3 * syz + 2 * sxz) {
    long long u2 = t - 3 * syz, r = u2 % sxz;
    i = 1 + (int)(r % d.nx); k = 1 + (int)(r / d.nx);
    j = (u2 / sxz) ? d.ny : 1;
  } else if (t < 3 * syz + 2 * sxz + 3 * sxy) {
    long long u2 = t - 3 * syz - 2 * sxz;
    int f = (int)(u2 / sxy);
    long long r = u2 % sxy;
    i = 1 + (int)(r % d.nx); j = 1 + (int)(r / d.nx);
    k = f == 0 ? 1 : (f == 1 ? d.kz2 : d.nz);
  } else {
    return;
  }
  long long q = fidx(d, i, j, k), p = pidx(d, px, i, j, k);
  u32[p] = (float)u[q];
  v32[p] = (float)v[q];
  w32[p] = (float)w[q];
}

// pressure update (src/Eddy6.f:2772-2806, 2911-2953) in FP64, FP32 copy alongside
// reference pressure: mean of p + dp over the row (ix1, :, 2); one warp
__global__ void k_pref_m(Dims d, const double *p, const double *dp, double *out) {
  double s = 0.;
  for (int j = d.jy1 + (int)threadIdx.x; j <= d.jy2; j += 32) {
    long long q = fidx(d, d.ix1, j, 2);
    s += p[q] + dp[q];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) out[0] = s / (double)(d.ny - 2);
}

__global__ void __launch_bounds__(256)
    k_pupdate_m(Dims d, int px, double *__restrict__ p, const double *__restrict__ dp,
                const double *__restrict__ pref, float *__restrict__ p32) {
  PlaneCell c;
  if (!plane_cell(d, c)) return;
  const double v = (p[c.t] + dp[c.t]) - pref[0];
  p[c.t] = v;
  p32[pidx(d, px, c.i, c.j, c.k)] = (float)v;
}

__device__ __forceinline__ int map_axis(int a, int n, int lo, int hi, int periodic, int active) {
  if (!active) return a;
  if (a == 1) return periodic ? hi : lo;
  if (a == n) return periodic ? lo : hi;
  return a;
}

__global__ void k_pghost_m(Dims d, int px, double *p, float *p32) {
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
  int zact = d.itype[5] != 0 || d.itype[6] != 0;
  int zper = d.itype[5] == 500;
  int si = map_axis(i, d.nx, d.ix1, d.ix2, d.mp == 0, 1);
  int sj = map_axis(j, d.ny, d.jy1, d.jy2, d.lp == 0, 1);
  int sk = map_axis(k, d.nz, d.kz1, d.kz2, zper, zact);
  if (si == i && sj == j && sk == k) return;
  double v = p[fidx(d, si, sj, sk)];
  p[fidx(d, i, j, k)] = v;
  p32[pidx(d, px, i, j, k)] = (float)v;
}

// ---------------------------------------------------------------------------
// density in FP32 (src/rhs_density.f + src/density.f:6-99) on the plane ring
constexpr int DTX = 32, DTY = 8, DKC = 32, DNF = 6;  // dens kv uo vo wo rha
using Acc6 = RingAcc<DTX, DTY, DNF, float>;

__global__ void __launch_bounds__(DTX *DTY)
    k_density32(Dims d, DevMetrics32 m, Scalars s, int px, const __grid_constant__ TmaMaps<DNF> maps,
                float *__restrict__ rha, float *__restrict__ dn, float repr1, float alfxdt, float gamxdt,
                float rhoxdt, int *err) {
  // per-column metric values in registers (the tma_march column of this thread)
  const int ic = min(d.ix1 + (int)(blockIdx.x * DTX + threadIdx.x), d.ix2);
  const int jc = min(d.jy1 + (int)(blockIdx.y * DTY + threadIdx.y), d.jy2);
  MetricCol32 mc;
  mc.ap = reg3(m.ap, ic); mc.au = reg3(m.au, ic);
  mc.bp = reg3(m.bp, jc); mc.bv = reg3(m.bv, jc);
  const float bg = m.dens_bg[(ic - 1) + d.nx * (jc - 1)], dfxd_i = m.dfxd[ic];
  tma_march<DNF, DTX, DTY, DKC, float>(d.ix1, d.ix2, d.jy1, d.jy2, d.kz1, d.kz2, maps, err,
                                       [&](int i, int j, int k, bool active, const Acc6 &S) {
                                         if (!active) return;
                                         mc.cp = reg3(m.cp, k); mc.cw = reg3(m.cw, k);
                                         float rr = rhs_dens<float>(S, mc, repr1, i, j, k);
                                         float dnew = S.at(0, 0, 0, 0) + gamxdt * rr + rhoxdt * S.at(5, 0, 0, 0);
                                         long long q = pidx(d, px, i, j, k);
                                         rha[q] = rr;
                                         if (s.idspngl == 1) dnew = dnew + m.dfxdl[k] * (bg - dnew) * alfxdt;
                                         if (i >= d.ix2 - s.dspngx1) dnew = dnew + dfxd_i * (bg - dnew) * alfxdt;
                                         dn[q] = dnew;
                                       });
}

__global__ void k_dens_ghost32(Dims d, int px, const float *__restrict__ dens, float *__restrict__ dn) {
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
  long long q = pidx(d, px, i, j, k);
  dn[q] = dens[q];
}

// ---------------------------------------------------------------------------
// outlet-face plane in FP64 (BOUNDINOUT 730 mass balance, src/boundary.f:920-944)
__global__ void k_plane_from32(Dims d, int px, const float *__restrict__ w32, int k, double *__restrict__ plane) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.nx * d.ny) return;
  int i = 1 + t % d.nx, j = 1 + t / d.nx;
  plane[t] = (double)w32[pidx(d, px, i, j, k)];
}

__global__ void k_rescale_plane(Dims d, int px, double *__restrict__ plane, float *__restrict__ w32,
                                const double *flux_in, const double *flux_out) {
  int mi = d.ix2 - d.ix1 + 1, mj = d.jy2 - d.jy1 + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= mi * mj) return;
  int i = d.ix1 + t % mi, j = d.jy1 + t / mi;
  int q = (i - 1) + d.nx * (j - 1);
  double qin1 = flux_in[0], qout = flux_out[0];
  double v = qout != 0. ? plane[q] * (qin1 / qout) : qin1 / flux_out[1];
  plane[q] = v;
  w32[pidx(d, px, i, j, d.kz2)] = (float)v;
}

__global__ void k_plane_to64(Dims d, const double *__restrict__ plane, double *__restrict__ w, int k) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.nx * d.ny) return;
  w[(long long)t + (long long)d.nx * d.ny * (k - 1)] = plane[t];
}

// ---------------------------------------------------------------------------
const CUtensorMap *tmap32(eddy_ctx *ctx, const float *ptr, int bx, int by) {
  for (TmaEntry &e : ctx->tmaps)
    if (e.ptr == ptr && e.bx == bx && e.by == by) return &e.map;
  TmaEntry e;
  e.ptr = ptr;
  e.bx = bx;
  e.by = by;
  int r = make_tensor_map_3d(&e.map, ptr, ctx->d.nx, ctx->d.ny, ctx->d.nz, bx, by, 4, ms(ctx)->px);
  if (r != 0) {
    ctx->err = "cuTensorMapEncodeTiled failed (" + std::to_string(r) + ")";
    return nullptr;
  }
  ctx->tmaps.push_back(e);
  return &ctx->tmaps.back().map;
}

constexpr int NPART = 296;

inline unsigned nblk(long long n) { return (unsigned)((n + 255) / 256); }
inline dim3 plane_grid(const Dims &d) { return dim3((unsigned)((d.nx * d.ny + 255) / 256), (unsigned)d.nz); }

int to32(eddy_ctx *ctx, const double *a, float *b) {
  k_to32<<<plane_grid(ctx->d), 256, 0, ctx->stream>>>(ctx->d, ms(ctx)->px, a, b);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

int to64(eddy_ctx *ctx, const float *b, double *a) {
  k_to64<<<plane_grid(ctx->d), 256, 0, ctx->stream>>>(ctx->d, ms(ctx)->px, b, a);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}


// FP32 spectral solve of the transformed right-hand side in pp.spec (as
// float) -> phi (set or accumulate)
int solve32(eddy_ctx *ctx, double *phi, int accumulate) {
  MixedState *x = ms(ctx);
  PoissonPlan &pp = ctx->pp;
  const Dims &d = ctx->d;
  int M = pp.M, L = pp.L, N = pp.N;
  float *s1 = reinterpret_cast<float *>(pp.spec), *s2 = reinterpret_cast<float *>(pp.spec2);
  int rc;
  {
    ProfScope ps(ctx, PROF_GEMM_FWD);
    if (x->xp.fmat) {
      if ((rc = launch_xform(ctx, &x->xp, 0, s1, s2))) return rc;
    } else {
      if ((rc = launch_xform64_f32(ctx, 0, s1, s2))) return rc;
    }
  }
  {
    ProfScope ps(ctx, PROF_TRIDIAG);
    long long nl = (long long)M * L;
    // mode order of the transforms: the split form orders even modes first
    const double *lam = x->xp.fmat ? x->xp.lam : pp.dlam;
    const int m0 = x->xp.fmat ? x->xp.m0 : pp.dm0;
    k_line_mean<float><<<1, 256, 0, ctx->stream>>>(M, L, N, m0, pp.wz, s2, ctx->scal + 5);
    EDDY_LAUNCHED(ctx);
    float *e32 = reinterpret_cast<float *>(pp.cprime);
    k_tridiag_lines<float, float, 8, true, true, 16><<<(unsigned)((nl + 127) / 128), 128, 0, ctx->stream>>>(
        M, L, N, m0, lam, pp.ak, pp.an, pp.bn, pp.cn, ctx->scal + 5, s2, x->cpz, e32);
    EDDY_LAUNCHED(ctx);
  }
  {
    ProfScope ps(ctx, PROF_GEMM_BWD);
    if (x->xp.bmat) {
      if ((rc = launch_xform(ctx, &x->xp, 1, s2, s1))) return rc;
    } else {
      if ((rc = launch_xform64_f32(ctx, 1, s2, s1))) return rc;
    }
  }
  ProfScope ps(ctx, PROF_FFT_BWD);
  k_plane_sum32<<<NPART, 256, 0, ctx->stream>>>(M, L, N, s1, pp.red);
  EDDY_LAUNCHED(ctx);
  k_sum_final<<<1, 32, 0, ctx->stream>>>(NPART, (long long)M * N, pp.red, ctx->scal + 3);
  EDDY_LAUNCHED(ctx);
  size_t smem = fft32_smem(L);
  dim3 g((M + TI32 - 1) / TI32, N);
  if (accumulate)
    k_bwd32<1><<<g, FT32, smem, ctx->stream>>>(d, s1, ctx->scal + 3, fft_code(L), x->twr + L / 2, x->twi + L / 2, phi);
  else
    k_bwd32<0><<<g, FT32, smem, ctx->stream>>>(d, s1, ctx->scal + 3, fft_code(L), x->twr + L / 2, x->twi + L / 2, phi);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

// forward pass (mode as in k_fwd32) into pp.spec (as float)
int fwd32(eddy_ctx *ctx, int mode, double alfxdt, const double *phi, double *dvec, int sweep) {
  MixedState *x = ms(ctx);
  PoissonPlan &pp = ctx->pp;
  const Dims &d = ctx->d;
  size_t smem = fft32_smem(pp.L);
  dim3 g((pp.M + TI32 - 1) / TI32, pp.N);
  const double ralf = 1.0 / alfxdt;
  ProfScope ps(ctx, mode == 2 ? PROF_REFINE : PROF_DIV_FFT);
  auto *rm = reinterpret_cast<unsigned long long *>(x->resid + sweep);
  float *sp = reinterpret_cast<float *>(pp.spec);
  const int lg = fft_code(pp.L);
  const double rdy2 = 1.0 / ctx->delysq;
  if (mode == 0)
    k_fwd32<0><<<g, FT32, smem, ctx->stream>>>(d, ctx->m, x->px, x->us, x->vs, x->ws, ctx->f[EDDY_PLANEW], x->wout,
                                               phi, dvec, ralf, rdy2, lg, x->twr, x->twi, sp, rm);
  else if (mode == 1)
    k_fwd32<1><<<g, FT32, smem, ctx->stream>>>(d, ctx->m, x->px, x->us, x->vs, x->ws, ctx->f[EDDY_PLANEW], x->wout,
                                               phi, dvec, ralf, rdy2, lg, x->twr, x->twi, sp, rm);
  else
    k_fwd32<2><<<g, FT32, smem, ctx->stream>>>(d, ctx->m, x->px, x->us, x->vs, x->ws, ctx->f[EDDY_PLANEW], x->wout,
                                               phi, dvec, ralf, rdy2, lg, x->twr, x->twi, sp, rm);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

// the refined solve: mode 0 (divergence of the FP32 predictor velocities) or
// mode 1 (dvec given); solution into phi with DIRECT's ghosts
int refined_solve(eddy_ctx *ctx, int mode, double alfxdt, double *dvec, double *phi) {
  MixedState *x = ms(ctx);
  int sweeps = ctx->prm.refine_sweeps;
  int rc;
  EDDY_CUDA(cudaMemsetAsync(x->resid, 0, 4 * sizeof(double), ctx->stream));
  if ((rc = fwd32(ctx, mode, alfxdt, nullptr, dvec, 0))) return rc;
  if ((rc = solve32(ctx, phi, 0))) return rc;
  for (int s = 0; s < sweeps; s++) {
    if ((rc = fwd32(ctx, 2, alfxdt, phi, dvec, s))) return rc;
    if ((rc = solve32(ctx, phi, 1))) return rc;
  }
  return launch_dp_ghost(ctx, phi);
}

}  // namespace

// ---------------------------------------------------------------------------
int mixed_create(eddy_ctx *ctx) {
  const Dims &d = ctx->d;
  if (ctx->prm.refine_sweeps < 1 || ctx->prm.refine_sweeps > 3) {
    ctx->err = "refine_sweeps must be 1, 2 or 3 in the mixed form";
    return EDDY_EINVAL;
  }
  MixedState *x = new (std::nothrow) MixedState();
  if (!x) return EDDY_ENOMEM;
  ctx->mixed = x;
  x->px = (d.nx + 3) / 4 * 4;
  x->n32 = (size_t)x->px * d.ny * d.nz;
  float **fl[] = {&x->uo, &x->vo, &x->wo, &x->p, &x->tv, &x->kv, &x->us, &x->vs,
                  &x->ws, &x->ua, &x->va, &x->wa, &x->dens, &x->dens_alt, &x->rha};
  for (float **p : fl) {
    EDDY_CUDA(cudaMalloc(p, sizeof(float) * x->n32));
    EDDY_CUDA(cudaMemset(*p, 0, sizeof(float) * x->n32));
  }
  // metrics in FP32, one buffer
  float **dst[] = {nullptr, nullptr, &x->m.ap, &x->m.au, &x->m.av, &x->m.aw, nullptr, nullptr,
                   &x->m.bp, &x->m.bu, &x->m.bv, &x->m.bw, nullptr, nullptr, &x->m.cp, &x->m.cu,
                   &x->m.cv, &x->m.cw, &x->m.whx, &x->m.why, &x->m.whz, &x->m.dfxu, &x->m.dfxw,
                   &x->m.dfxul, &x->m.dfxwl, &x->m.dfxd, &x->m.dfxdl, &x->m.dens_bg};
  size_t tot = 0;
  for (int a = 0; a < 28; a++)
    if (dst[a]) tot += (ctx->h[a].size() + 31) / 32 * 32;
  std::vector<float> hb(tot, 0.f);
  EDDY_CUDA(cudaMalloc(&x->mbuf, sizeof(float) * tot));
  size_t off = 0;
  for (int a = 0; a < 28; a++) {
    if (!dst[a]) continue;
    for (size_t e = 0; e < ctx->h[a].size(); e++) hb[off + e] = (float)ctx->h[a][e];
    *dst[a] = x->mbuf + off;
    off += (ctx->h[a].size() + 31) / 32 * 32;
  }
  EDDY_CUDA(cudaMemcpy(x->mbuf, hb.data(), sizeof(float) * tot, cudaMemcpyHostToDevice));
  int L = ctx->pp.L;
  std::vector<float> twr(L), twi(L);
  for (int r = 0; r < L / 2; r++) {
    double angf = -2.0 * M_PI * (double)r / (double)L, angb = 2.0 * M_PI * (double)r / (double)L;
    twr[r] = (float)std::cos(angf);
    twi[r] = (float)std::sin(angf);
    twr[L / 2 + r] = (float)std::cos(angb);
    twi[L / 2 + r] = (float)std::sin(angb);
  }
  EDDY_CUDA(cudaMalloc(&x->twr, sizeof(float) * L));
  EDDY_CUDA(cudaMalloc(&x->twi, sizeof(float) * L));
  EDDY_CUDA(cudaMemcpy(x->twr, twr.data(), sizeof(float) * L, cudaMemcpyHostToDevice));
  EDDY_CUDA(cudaMemcpy(x->twi, twi.data(), sizeof(float) * L, cudaMemcpyHostToDevice));
  if (xform_supported(ctx->pp.M)) {
    int rc = xform_prepare(ctx, &x->xp);
    if (rc) return rc;
  }
  EDDY_CUDA(cudaMalloc(&x->wout, sizeof(double) * (size_t)d.nx * d.ny));
  EDDY_CUDA(cudaMemset(x->wout, 0, sizeof(double) * (size_t)d.nx * d.ny));
  EDDY_CUDA(cudaMalloc(&x->resid, 4 * sizeof(double)));
  EDDY_CUDA(cudaMemset(x->resid, 0, 4 * sizeof(double)));
  if (L < 8) {
    ctx->err = "the mixed form needs at least 8 cells along y";
    return EDDY_EINVAL;
  }
  // the correction solves keep the forward-eliminated right-hand side in FP32
  // in the (FP64-sized) c' buffer of the plan and read c' from cpz, computed
  // here once: it does not depend on the right-hand side
  {
    const PoissonPlan &pp = ctx->pp;
    const long long nl = (long long)pp.M * pp.L;
    EDDY_CUDA(cudaMalloc(&x->cpz, sizeof(float) * (size_t)nl * pp.N));
    const double *lam = x->xp.fmat ? x->xp.lam : pp.dlam;
    const int m0 = x->xp.fmat ? x->xp.m0 : pp.dm0;
    k_tridiag_cprime<float><<<(unsigned)((nl + 127) / 128), 128, 0, ctx->stream>>>(pp.M, pp.L, pp.N, m0, lam, pp.ak,
                                                                                  pp.an, pp.bn, pp.cn, x->cpz);
    EDDY_LAUNCHED(ctx);
  }
  size_t smem = fft32_smem(L);
  if (smem > 48 * 1024) {
    EDDY_CUDA(cudaFuncSetAttribute(k_fwd32<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    EDDY_CUDA(cudaFuncSetAttribute(k_fwd32<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    EDDY_CUDA(cudaFuncSetAttribute(k_fwd32<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    EDDY_CUDA(cudaFuncSetAttribute(k_bwd32<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    EDDY_CUDA(cudaFuncSetAttribute(k_bwd32<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  EDDY_CUDA(cudaFuncSetAttribute(k_rhs32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ring_smem_bytes<NFLD, TX, TY, float>()));
  EDDY_CUDA(cudaFuncSetAttribute(k_density32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ring_smem_bytes<DNF, DTX, DTY, float>()));
  return EDDY_OK;
}

void mixed_release(eddy_ctx *ctx) {
  MixedState *x = ms(ctx);
  if (!x) return;
  float *fl[] = {x->uo, x->vo, x->wo, x->p, x->tv, x->kv, x->us, x->vs,
                 x->ws, x->ua, x->va, x->wa, x->dens, x->dens_alt, x->rha, x->mbuf, x->twr, x->twi, x->cpz};
  for (float *p : fl) if (p) cudaFree(p);
  if (x->resid) cudaFree(x->resid);
  if (x->wout) cudaFree(x->wout);
  xform_release(&x->xp);
  delete x;
  ctx->mixed = nullptr;
}

// FP32 array that mirrors (or, for the FP32-master fields, holds) `field`
static float *mirror(MixedState *x, int field) {
  switch (field) {
    case EDDY_UO: return x->uo;
    case EDDY_VO: return x->vo;
    case EDDY_WO: return x->wo;
    case EDDY_P: return x->p;
    case EDDY_TV: return x->tv;
    case EDDY_DENS: return x->dens;
    case EDDY_US: return x->us;
    case EDDY_VS: return x->vs;
    case EDDY_WS: return x->ws;
    case EDDY_UA: return x->ua;
    case EDDY_VA: return x->va;
    case EDDY_WA: return x->wa;
    case EDDY_RHA: return x->rha;
    default: return nullptr;
  }
}

int mixed_from64(eddy_ctx *ctx, int field) {
  MixedState *x = ms(ctx);
  if (!x) return EDDY_OK;
  float *b = mirror(x, field);
  if (!b) return EDDY_OK;
  int rc = to32(ctx, ctx->f[field], b);
  if (rc) return rc;
  if (field == EDDY_DENS) return to32(ctx, ctx->f[field], x->dens_alt);
  if (field == EDDY_TV) return to32(ctx, ctx->f[field], x->kv);
  return EDDY_OK;
}

int mixed_to64(eddy_ctx *ctx, int field) {
  MixedState *x = ms(ctx);
  if (!x) return EDDY_OK;
  switch (field) {
    case EDDY_DENS: case EDDY_US: case EDDY_VS: case EDDY_WS:
    case EDDY_UA: case EDDY_VA: case EDDY_WA: case EDDY_RHA:
      return to64(ctx, mirror(x, field), ctx->f[field]);
    default:
      return EDDY_OK;
  }
}

// after the eddy viscosity (dynamic model or learned closure) is updated in
// FP64: FP32 copies for the stencils
int mixed_after_sgs(eddy_ctx *ctx) {
  MixedState *x = ms(ctx);
  ProfScope ps(ctx, PROF_CONVERT);
  if (ctx->prm.closure == 1) {
    int rc = to32(ctx, ctx->f[EDDY_TV], x->tv);
    if (rc) return rc;
    return to32(ctx, ctx->kappa, x->kv);
  }
  // the dynamic model's diffusivity is its viscosity: both copies in one pass
  k_to32x2<<<plane_grid(ctx->d), 256, 0, ctx->stream>>>(ctx->d, x->px, ctx->f[EDDY_TV], x->tv, x->kv);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

int mixed_turvis(eddy_ctx *ctx) {
  MixedState *x = ms(ctx);
  if (ctx->prm.isgs != 2) return launch_turvis(ctx);
  // FP32 scratch lives in the plain procedure's FP64 arrays (|S| holds px*ny*nz
  // floats in its nx*ny*nz doubles); the two procedures never run at once
  return launch_turvis32(ctx, x->px, x->uo, x->vo, x->wo, reinterpret_cast<float *>(ctx->gs),
                         reinterpret_cast<float *>(ctx->imm2), reinterpret_cast<float *>(ctx->ilm2));
}

int mixed_views(eddy_ctx *ctx, MixedViews *v) {
  MixedState *x = ms(ctx);
  if (!x) return EDDY_EINVAL;
  *v = MixedViews{x->uo, x->vo, x->wo, x->dens, x->tv, x->kv, x->px};
  return EDDY_OK;
}

// BOUNDINOUT predictor (src/boundary.f:694-944) on the FP32 u*: inlet plane,
// convective 730 outlet, then the outlet mass balance in FP64 on the outlet
// plane (inflow flux from the FP64 inlet plane)
static int boundinout_pred(eddy_ctx *ctx, double alfxdt) {
  MixedState *x = ms(ctx);
  const Dims &d = ctx->d;
  const int px = x->px;
  cudaStream_t st = ctx->stream;
  double *fin = ctx->scal + 8, *fout = ctx->scal + 10;
  int n2 = d.nx * d.ny, nin = (d.ix2 - d.ix1 + 1) * (d.jy2 - d.jy1 + 1);
  bct::k_inlet_plane<float><<<nblk(n2), 256, 0, st>>>(d, px, x->us, x->vs, x->ws, ctx->f[EDDY_PLANEU],
                                                      ctx->f[EDDY_PLANEV], ctx->f[EDDY_PLANEW]);
  EDDY_LAUNCHED(ctx);
  int rc;
  if ((rc = plane_flux<double>(ctx, d.nx, ctx->f[EDDY_PLANEW], 1, fin))) return rc;
  bct::k_outlet_convective<float, float><<<nblk(nin), 256, 0, st>>>(d, px, ctx->m, x->us, x->vs, x->ws, x->uo, x->vo,
                                                                    x->wo, fin, alfxdt);
  EDDY_LAUNCHED(ctx);
  bct::k_yper3<float><<<nblk((long long)d.nx * d.nz), 256, 0, st>>>(d, px, x->us, x->vs, x->ws);
  EDDY_LAUNCHED(ctx);
  k_plane_from32<<<nblk(n2), 256, 0, st>>>(d, px, x->ws, d.kz2, x->wout);
  EDDY_LAUNCHED(ctx);
  if ((rc = plane_flux<double>(ctx, d.nx, x->wout, 1, fout))) return rc;
  k_rescale_plane<<<nblk(nin), 256, 0, st>>>(d, px, x->wout, x->ws, fin, fout);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

int mixed_substep(eddy_ctx *ctx, double alfxdt, double gamxdt, double rhoxdt) {
  MixedState *x = ms(ctx);
  const Dims &d = ctx->d;
  const int px = x->px;
  double **f = ctx->f;
  int rc;
  {
    ProfScope ps(ctx, PROF_RHS_PRED);
    TmaMaps<NFLD> maps;
    const float *src[NFLD] = {x->uo, x->vo, x->wo, x->tv, x->p, x->dens, x->ua, x->va, x->wa};
    for (int q = 0; q < NFLD; q++) {
      const CUtensorMap *mp = tmap32(ctx, src[q], RingGeom<TX, TY, float>::PX, TY + 2);
      if (!mp) return EDDY_ECUDA;
      maps.m[q] = *mp;
    }
    dim3 g((d.ix2 - d.ix1 + TX) / TX, (d.jy2 - d.jy1 + TY) / TY, (d.kz2 - d.kz1 + KCHUNK) / KCHUNK);
    k_rhs32<<<g, dim3(TX, TY), ring_smem_bytes<NFLD, TX, TY, float>(), ctx->stream>>>(
        d, x->m, ctx->sc, px, maps, x->us, x->vs, x->ws, x->ua, x->va, x->wa, (float)alfxdt, (float)gamxdt,
        (float)rhoxdt, ctx->err_flag);
    EDDY_LAUNCHED(ctx);
    long long ng = 2LL * d.nx * d.ny + 2LL * d.nx * d.nz + 2LL * d.ny * d.nz;
    k_zero_faces32<<<nblk(ng), 256, 0, ctx->stream>>>(d, px, x->us, x->vs, x->ws);
    EDDY_LAUNCHED(ctx);
  }
  if ((rc = ib_overlap_regen(ctx))) return rc;
  // immersed body: momforc_mod2 + velinterior on the FP32 predictor velocities
  if (ctx->ib) {
    ProfScope ps(ctx, PROF_IB_FORCE);
    const double *vb = ib_velocity(ctx);
    if ((rc = ib_force32(ctx, 0, 0, x->us, px, vb[0], vb[0]))) return rc;
    if ((rc = ib_force32(ctx, 1, 1, x->vs, px, vb[1], vb[1]))) return rc;
    if ((rc = ib_force32(ctx, 2, 2, x->ws, px, vb[2], vb[2]))) return rc;
  }
  {
    ProfScope ps(ctx, PROF_BC);
    if ((rc = bc_boundary<float>(ctx, px, x->us, x->vs, x->ws))) return rc;
    if ((rc = boundinout_pred(ctx, alfxdt))) return rc;
    if ((rc = bc_boundary<float>(ctx, px, x->us, x->vs, x->ws))) return rc;
  }
  // FP64 divergence right-hand side kept in the (unused in this form) FP64 u* array
  if ((rc = refined_solve(ctx, 0, alfxdt, f[EDDY_US], f[EDDY_DP]))) return rc;
  {
    ProfScope ps(ctx, PROF_CORRECT);
    dim3 g((d.nx + BX - 1) / BX, (d.ny + BY - 1) / BY, (d.nz + BZ - 1) / BZ);
    k_correct_mixed<<<g, dim3(BX, BY, BZ), 0, ctx->stream>>>(d, ctx->m, px, x->us, x->vs, x->ws, f[EDDY_DP],
                                                             f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], x->uo, x->vo, x->wo,
                                                             alfxdt);
    EDDY_LAUNCHED(ctx);
  }
  {
    ProfScope ps(ctx, PROF_BC);
    if ((rc = bc_boundary<double>(ctx, d.nx, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO]))) return rc;
    if ((rc = bc_boundinout<double, float>(ctx, d.nx, px, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], x->us, x->vs, x->ws,
                                           alfxdt, 0)))
      return rc;
    k_plane_to64<<<nblk((long long)d.nx * d.ny), 256, 0, ctx->stream>>>(d, x->wout, f[EDDY_WO], d.kz2);
    EDDY_LAUNCHED(ctx);
    if ((rc = bc_boundary<double>(ctx, d.nx, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO]))) return rc;
    long long np = 3LL * d.ny * d.nz + 2LL * d.nx * d.nz + 3LL * d.nx * d.ny;
    k_sync_planes<<<nblk(np), 256, 0, ctx->stream>>>(d, px, f[EDDY_UO], f[EDDY_VO], f[EDDY_WO], x->uo, x->vo, x->wo);
    EDDY_LAUNCHED(ctx);
  }
  {
    ProfScope ps(ctx, PROF_PUPDATE);
    k_pref_m<<<1, 32, 0, ctx->stream>>>(d, f[EDDY_P], f[EDDY_DP], ctx->scal);
    EDDY_LAUNCHED(ctx);
    k_pupdate_m<<<plane_grid(d), 256, 0, ctx->stream>>>(d, px, f[EDDY_P], f[EDDY_DP], ctx->scal, x->p);
    EDDY_LAUNCHED(ctx);
    if (ctx->ib && (rc = ib_force(ctx, 3, 4, f[EDDY_P], 0.0, 0.0, x->p, px))) return rc;
    long long ng = 2LL * d.nx * d.ny + 2LL * d.nx * d.nz + 2LL * d.ny * d.nz;
    k_pghost_m<<<nblk(ng), 256, 0, ctx->stream>>>(d, px, f[EDDY_P], x->p);
    EDDY_LAUNCHED(ctx);
  }
  if (ctx->prm.idens == 1) {
    ProfScope ps(ctx, PROF_DENSITY);
    if ((rc = bc_boundinoutd_dens<float>(ctx, px, x->dens))) return rc;
    TmaMaps<DNF> maps;
    const float *src[DNF] = {x->dens, x->kv, x->uo, x->vo, x->wo, x->rha};
    for (int q = 0; q < DNF; q++) {
      const CUtensorMap *mp = tmap32(ctx, src[q], RingGeom<DTX, DTY, float>::PX, DTY + 2);
      if (!mp) return EDDY_ECUDA;
      maps.m[q] = *mp;
    }
    dim3 g((d.ix2 - d.ix1 + DTX) / DTX, (d.jy2 - d.jy1 + DTY) / DTY, (d.kz2 - d.kz1 + DKC) / DKC);
    k_density32<<<g, dim3(DTX, DTY), ring_smem_bytes<DNF, DTX, DTY, float>(), ctx->stream>>>(
        d, x->m, ctx->sc, px, maps, x->rha, x->dens_alt, (float)(ctx->sc.ru1 / ctx->sc.prn), (float)alfxdt,
        (float)gamxdt, (float)rhoxdt, ctx->err_flag);
    EDDY_LAUNCHED(ctx);
    long long ng = 2LL * d.nx * d.ny + 2LL * d.nx * d.nz + 2LL * d.ny * d.nz;
    k_dens_ghost32<<<nblk(ng), 256, 0, ctx->stream>>>(d, px, x->dens, x->dens_alt);
    EDDY_LAUNCHED(ctx);
    float *t = x->dens;
    x->dens = x->dens_alt;
    x->dens_alt = t;
    if ((rc = bc_boundinoutd_dens<float>(ctx, px, x->dens))) return rc;
    if (ctx->ib && (rc = ib_force32(ctx, 3, 4, x->dens, px, 0.0, 0.0))) return rc;
  }
  return EDDY_OK;
}

int mixed_poisson_rhs(eddy_ctx *ctx, const double *rhs, double *dp) {
  // mode 1 reads the right-hand side from dvec; refinement reads it again
  return refined_solve(ctx, 1, 1.0, const_cast<double *>(rhs), dp);
}

int mixed_residuals(eddy_ctx *ctx, double *out, int n) {
  MixedState *x = ms(ctx);
  if (!x || n < 1) return EDDY_EINVAL;
  double h[4];
  EDDY_CUDA(cudaMemcpyAsync(h, x->resid, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
  EDDY_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int s = 0; s < n && s < 4; s++) out[s] = h[s];
  return EDDY_OK;
}
