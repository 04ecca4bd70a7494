// bc_templates.cuh -- boundary-condition kernels shared by the FP64 (plain)
// and FP32 (mixed) storage forms.  Arrays have a row pitch (NX for FP64, NX
// rounded up to 4 for FP32 so TMA rows stay 16-byte aligned).
//
//   BOUNDARY     src/boundary.f:7-66 (BOUND050 :69, BOUND060 :125, BOUND082 :372,
//                BOUND500 :409)
//   BOUNDINOUT   src/boundary.f:505-994 (inlet 305 :694, outlets 710/730)
//   BOUNDINOUTD  src/boundary.f:2241-2281, BOUNDARY_DENS :2001-2197
#pragma once
#include "eddy_internal.h"

int launch_fill_plane(eddy_ctx *ctx, double *a, int axis, int dst, int src, double sgn, int zero);

namespace {
namespace bct {

template <class T>
__global__ void k_fill_plane(Dims d, int pitch, T *a, int axis, int dst, int src, T sgn, int zero) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int n1 = axis == 0 ? d.ny : d.nx;
  int n2 = axis == 2 ? d.ny : d.nz;
  if (t >= n1 * n2) return;
  int a1 = 1 + t % n1, a2 = 1 + t / n1;
  long long qd, qs;
  if (axis == 0) { qd = pidx(d, pitch, dst, a1, a2); qs = pidx(d, pitch, src, a1, a2); }
  else if (axis == 1) { qd = pidx(d, pitch, a1, dst, a2); qs = pidx(d, pitch, a1, src, a2); }
  else { qd = pidx(d, pitch, a1, a2, dst); qs = pidx(d, pitch, a1, a2, src); }
  a[qd] = zero ? T(0) : sgn * a[qs];
}

// up to FQ_MAX plane fills along one axis in one launch; the fills of a batch
// are independent (no fill reads or writes a plane another one writes in the
// same array), so one thread per in-plane position applies all of them
constexpr int FQ_MAX = 8;
template <class T>
struct FillBatch {
  T *a[FQ_MAX];
  int dst[FQ_MAX], src[FQ_MAX], zero[FQ_MAX];
  T sgn[FQ_MAX];
  int n;
};

template <class T>
__global__ void k_fill_planes(Dims d, int pitch, int axis, FillBatch<T> B) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int n1 = axis == 0 ? d.ny : d.nx;
  int n2 = axis == 2 ? d.ny : d.nz;
  if (t >= n1 * n2) return;
  int a1 = 1 + t % n1, a2 = 1 + t / n1;
  for (int o = 0; o < B.n; o++) {
    long long qd, qs;
    if (axis == 0) { qd = pidx(d, pitch, B.dst[o], a1, a2); qs = pidx(d, pitch, B.src[o], a1, a2); }
    else if (axis == 1) { qd = pidx(d, pitch, a1, B.dst[o], a2); qs = pidx(d, pitch, a1, B.src[o], a2); }
    else { qd = pidx(d, pitch, a1, a2, B.dst[o]); qs = pidx(d, pitch, a1, a2, B.src[o]); }
    B.a[o][qd] = B.zero[o] ? T(0) : B.sgn[o] * B.a[o][qs];
  }
}

// flux through the z plane k: sum over interior (i,j) of a/(ap bp) and of
// the areas, FP64; FLUXB blocks write partial sums, one warp adds them in a
// fixed order (deterministic)
constexpr int FLUXB = 148, FLUXT = 256;

template <class T>
__global__ void __launch_bounds__(FLUXT)
    k_plane_flux_part(Dims d, int pitch, DevMetrics m, const T *a, int k, double *part) {
  __shared__ double sf[FLUXT], sa[FLUXT];
  const int mi = d.ix2 - d.ix1 + 1, mj = d.jy2 - d.jy1 + 1;
  double f = 0., ar = 0.;
  for (int t = blockIdx.x * FLUXT + threadIdx.x; t < mi * mj; t += gridDim.x * FLUXT) {
    const int i = d.ix1 + t % mi, j = d.jy1 + t / mi;
    const double areaij = 1.0 / (m.ap[i] * m.bp[j]);
    f = f + (double)a[pidx(d, pitch, i, j, k)] * areaij;
    ar = ar + areaij;
  }
  sf[threadIdx.x] = f;
  sa[threadIdx.x] = ar;
  __syncthreads();
  for (int w = FLUXT / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      sf[threadIdx.x] += sf[threadIdx.x + w];
      sa[threadIdx.x] += sa[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sf[0];
    part[2 * blockIdx.x + 1] = sa[0];
  }
}

__global__ void k_plane_flux_final(const double *part, double *out) {
  double f = 0., ar = 0.;
  for (int b = threadIdx.x; b < FLUXB; b += 32) {
    f += part[2 * b];
    ar += part[2 * b + 1];
  }
  for (int o = 16; o > 0; o >>= 1) {
    f += __shfl_xor_sync(0xffffffffu, f, o);
    ar += __shfl_xor_sync(0xffffffffu, ar, o);
  }
  if (threadIdx.x == 0) {
    out[0] = f;
    out[1] = ar;
  }
}

template <class T>
__global__ void k_inlet_plane(Dims d, int pitch, T *ubc, T *vbc, T *wbc, const double *pu, const double *pv,
                              const double *pw) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.nx * d.ny) return;
  int i = 1 + t % d.nx, j = 1 + t / d.nx;
  long long q = pidx(d, pitch, i, j, 1);
  ubc[q] = (T)pu[t];
  vbc[q] = (T)pv[t];
  wbc[q] = (T)pw[t];
}

// 730 convective outflow, predictor (src/boundary.f:853-870)
template <class T, class TO>
__global__ void k_outlet_convective(Dims d, int pitch, DevMetrics m, T *ubc, T *vbc, T *wbc, const TO *uof,
                                    const TO *vof, const TO *wof, const double *flux_in, double alfxdt) {
  int mi = d.ix2 - d.ix1 + 1, mj = d.jy2 - d.jy1 + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= mi * mj) return;
  int i = d.ix1 + t % mi, j = d.jy1 + t / mi;
  double qin2 = flux_in[0] / flux_in[1];
  T coef = (T)(qin2 * alfxdt * m.cp[d.kz2]);
  long long qn = pidx(d, pitch, i, j, d.nz), qk = pidx(d, pitch, i, j, d.kz2), qkm = pidx(d, pitch, i, j, d.kz2 - 1);
  ubc[qn] = (T)uof[qn] - coef * ((T)uof[qn] - (T)uof[qk]);
  vbc[qn] = (T)vof[qn] - coef * ((T)vof[qn] - (T)vof[qk]);
  wbc[qk] = (T)wof[qk] - coef * ((T)wof[qk] - (T)wof[qkm]);
}

template <class T>
__global__ void k_yper3(Dims d, int pitch, T *a, T *b, T *c) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.nx * d.nz) return;
  int i = 1 + t % d.nx, k = 1 + t / d.nx;
  T *arr[3] = {a, b, c};
  for (int s = 0; s < 3; s++) {
    T *x = arr[s];
    x[pidx(d, pitch, i, 1, k)] = x[pidx(d, pitch, i, d.ny - 1, k)];
    x[pidx(d, pitch, i, d.ny, k)] = x[pidx(d, pitch, i, 2, k)];
  }
}

// outflow mass balance (src/boundary.f:920-944)
template <class T>
__global__ void k_outlet_rescale(Dims d, int pitch, T *wbc, const double *flux_in, const double *flux_out) {
  int mi = d.ix2 - d.ix1 + 1, mj = d.jy2 - d.jy1 + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= mi * mj) return;
  int i = d.ix1 + t % mi, j = d.jy1 + t / mi;
  long long q = pidx(d, pitch, i, j, d.kz2);
  double qin1 = flux_in[0], qout = flux_out[0];
  if (qout != 0.) {
    double c = qin1 / qout;
    wbc[q] = (T)((double)wbc[q] * c);
  } else {
    wbc[q] = (T)(qin1 / flux_out[1]);
  }
}

// corrector copies of the outlet planes (src/boundary.f:947-980)
template <class T, class TO>
__global__ void k_outlet_corrector(Dims d, int pitch, int opitch, T *ubc, T *vbc, T *wbc, const TO *uof,
                                   const TO *vof, const TO *wof, int t6) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.nx * d.ny) return;
  int i = 1 + t % d.nx, j = 1 + t / d.nx;
  long long qn = pidx(d, pitch, i, j, d.nz), qk = pidx(d, pitch, i, j, d.kz2);
  long long on = pidx(d, opitch, i, j, d.nz), ok = pidx(d, opitch, i, j, d.kz2);
  if (t6 == 730 || t6 == 731) {
    ubc[qn] = (T)uof[on];
    vbc[qn] = (T)vof[on];
    wbc[qk] = (T)wof[ok];
  } else if (t6 == 710) {
    ubc[qn] = (T)uof[ok];
    vbc[qn] = (T)vof[ok];
    wbc[qk] = (T)wof[ok];
  }
}

template <class T>
__global__ void k_dens_inlet(Dims d, int pitch, T *dens, const double *plane) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.nx * d.ny) return;
  int i = 1 + t % d.nx, j = 1 + t / d.nx;
  dens[pidx(d, pitch, i, j, 1)] = (T)plane[t];
}

}  // namespace bct

template <class T>
int bc_fill(eddy_ctx *ctx, int pitch, T *a, int axis, int dst, int src, double sgn, int zero) {
  const Dims &d = ctx->d;
  int n = axis == 0 ? d.ny * d.nz : (axis == 1 ? d.nx * d.nz : d.nx * d.ny);
  bct::k_fill_plane<T><<<(n + 255) / 256, 256, 0, ctx->stream>>>(d, pitch, a, axis, dst, src, (T)sgn, zero);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

// Plane fills in their given order, batched: consecutive fills along the same
// axis share one launch until a fill would touch a plane that a queued fill of
// the same array writes (or write one a queued fill reads), the axis changes
// or the batch is full.  Every batch is independent inside, so the result is
// that of the fills one after another.  flush() before anything else that
// reads or writes the arrays is launched.
template <class T>
struct FillQueue {
  eddy_ctx *ctx;
  int pitch;
  int axis = -1;
  bct::FillBatch<T> b{};
  FillQueue(eddy_ctx *c, int p) : ctx(c), pitch(p) { b.n = 0; }
  int flush() {
    if (b.n == 0) return EDDY_OK;
    const Dims &d = ctx->d;
    int n = axis == 0 ? d.ny * d.nz : (axis == 1 ? d.nx * d.nz : d.nx * d.ny);
    bct::k_fill_planes<T><<<(n + 255) / 256, 256, 0, ctx->stream>>>(d, pitch, axis, b);
    EDDY_LAUNCHED(ctx);
    b.n = 0;
    axis = -1;
    return EDDY_OK;
  }
  int add(T *a, int ax, int dst, int src, double sgn, int zero) {
    bool conflict = (axis >= 0 && ax != axis) || b.n == bct::FQ_MAX;
    for (int o = 0; o < b.n && !conflict; o++)
      if (b.a[o] == a && (b.dst[o] == dst || (!zero && b.dst[o] == src) || (!b.zero[o] && b.src[o] == dst)))
        conflict = true;
    if (conflict)
      if (int rc = flush()) return rc;
    axis = ax;
    b.a[b.n] = a;
    b.dst[b.n] = dst;
    b.src[b.n] = src;
    b.sgn[b.n] = (T)sgn;
    b.zero[b.n] = zero;
    b.n++;
    return EDDY_OK;
  }
};

// plane flux (out[0] flux, out[1] area) of the z plane k of `a`; partial
// sums in ctx->scal + 32
template <class T>
int plane_flux(eddy_ctx *ctx, int pitch, const T *a, int k, double *out) {
  double *part = ctx->scal + 32;
  bct::k_plane_flux_part<T><<<bct::FLUXB, bct::FLUXT, 0, ctx->stream>>>(ctx->d, pitch, ctx->m, a, k, part);
  EDDY_LAUNCHED(ctx);
  bct::k_plane_flux_final<<<1, 32, 0, ctx->stream>>>(part, out);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

// BOUNDARY (src/boundary.f:7-66): wall types first, then periodic x/y.
template <class T>
int bc_boundary(eddy_ctx *ctx, int pitch, T *u, T *v, T *w) {
  const Dims &d = ctx->d;
  int rc;
  FillQueue<T> q(ctx, pitch);
#define F(...) \
  if ((rc = q.add(__VA_ARGS__)) != EDDY_OK) return rc
  for (int ib = 1; ib <= 6; ib++) {
    int t = d.itype[ib];
    if (t == 50 || t == 60) {
      double sg = (t == 50) ? -1. : 1.;
      switch (ib) {
        case 1: F(u, 0, 1, 0, 0., 1); F(v, 0, 1, d.ix1, sg, 0); F(w, 0, 1, d.ix1, sg, 0); break;
        case 2: F(u, 0, d.ix2, 0, 0., 1); F(v, 0, d.nx, d.ix2, sg, 0); F(w, 0, d.nx, d.ix2, sg, 0); break;
        case 3: F(u, 1, 1, d.jy1, sg, 0); F(v, 1, 1, 0, 0., 1); F(w, 1, 1, d.jy1, sg, 0); break;
        case 4: F(u, 1, d.ny, d.jy2, sg, 0); F(v, 1, d.jy2, 0, 0., 1); F(w, 1, d.ny, d.jy2, sg, 0); break;
        case 5: F(u, 2, 1, d.kz1, sg, 0); F(v, 2, 1, d.kz1, sg, 0); F(w, 2, 1, 0, 0., 1); break;
        case 6: F(u, 2, d.nz, d.kz2, sg, 0); F(v, 2, d.nz, d.kz2, sg, 0); F(w, 2, d.kz2, 0, 0., 1); break;
      }
    } else if (t == 82) {
      if (ib == 1) { F(u, 0, 1, d.ix1, 1., 0); F(v, 0, 1, d.ix1, -1., 0); F(w, 0, 1, d.ix1, -1., 0); }
      if (ib == 2) { F(u, 0, d.nx, d.ix2, 1., 0); F(v, 0, d.nx, d.ix2, 1., 0); F(w, 0, d.nx, d.ix2, 1., 0); }
    }
  }
  if (d.itype[1] == 500) {
    F(u, 0, 1, d.ix2, 1., 0); F(v, 0, 1, d.ix2, 1., 0); F(w, 0, 1, d.ix2, 1., 0);
    F(u, 0, d.nx, d.ix1, 1., 0); F(v, 0, d.nx, d.ix1, 1., 0); F(w, 0, d.nx, d.ix1, 1., 0);
  }
  if (d.itype[3] == 500) {
    F(u, 1, 1, d.jy2, 1., 0); F(v, 1, 1, d.jy2, 1., 0); F(w, 1, 1, d.jy2, 1., 0);
    F(u, 1, d.ny, d.jy1, 1., 0); F(v, 1, d.ny, d.jy1, 1., 0); F(w, 1, d.ny, d.jy1, 1., 0);
  }
#undef F
  return q.flush();
}

// BOUNDINOUT (src/boundary.f:505-994) for inlet 305 and outlets 710/730;
// ubc (type T, pitch) from uof (type TO, pitch opitch).
template <class T, class TO>
int bc_boundinout(eddy_ctx *ctx, int pitch, int opitch, T *ubc, T *vbc, T *wbc, const TO *uof, const TO *vof,
                  const TO *wof, double alfxdt, int idiv) {
  const Dims &d = ctx->d;
  cudaStream_t st = ctx->stream;
  double *fin = ctx->scal + 8, *fout = ctx->scal + 10;
  int n2 = d.nx * d.ny, nin = (d.ix2 - d.ix1 + 1) * (d.jy2 - d.jy1 + 1);
  int iinq = idiv;
  if (d.itype[5] == 305) {
    bct::k_inlet_plane<T><<<(n2 + 255) / 256, 256, 0, st>>>(d, pitch, ubc, vbc, wbc, ctx->f[EDDY_PLANEU],
                                                            ctx->f[EDDY_PLANEV], ctx->f[EDDY_PLANEW]);
    EDDY_LAUNCHED(ctx);
  } else {
    iinq = 0;
  }
  int t6 = d.itype[6];
  if (idiv == 1) {
    if (t6 == 710 || t6 == 720) {
      ctx->err = "outlet types 710/720 are not on the restated hot path";
      return EDDY_EINVAL;
    }
    if (t6 != 730) return EDDY_OK;
    if (iinq != 1) {
      ctx->err = "convective outlet needs the 305 inlet flux";
      return EDDY_EINVAL;
    }
    if (pitch != opitch) {
      ctx->err = "predictor outlet: source and target pitches differ";
      return EDDY_EINVAL;
    }
    if (int rc = plane_flux<T>(ctx, pitch, wbc, 1, fin)) return rc;
    bct::k_outlet_convective<T, TO><<<(nin + 255) / 256, 256, 0, st>>>(d, pitch, ctx->m, ubc, vbc, wbc, uof, vof,
                                                                        wof, fin, alfxdt);
    EDDY_LAUNCHED(ctx);
    bct::k_yper3<T><<<(d.nx * d.nz + 255) / 256, 256, 0, st>>>(d, pitch, ubc, vbc, wbc);
    EDDY_LAUNCHED(ctx);
    if (int rc = plane_flux<T>(ctx, pitch, wbc, d.kz2, fout)) return rc;
    bct::k_outlet_rescale<T><<<(nin + 255) / 256, 256, 0, st>>>(d, pitch, wbc, fin, fout);
    EDDY_LAUNCHED(ctx);
  } else {
    if (t6 == 720) {
      ctx->err = "outlet type 720 is not on the restated hot path";
      return EDDY_EINVAL;
    }
    bct::k_outlet_corrector<T, TO><<<(n2 + 255) / 256, 256, 0, st>>>(d, pitch, opitch, ubc, vbc, wbc, uof, vof, wof,
                                                                      t6);
    EDDY_LAUNCHED(ctx);
  }
  return EDDY_OK;
}

// BOUNDINOUTD (src/boundary.f:2241-2281) then BOUNDARY_DENS (:2001-2044)
template <class T>
int bc_boundinoutd_dens(eddy_ctx *ctx, int pitch, T *dens) {
  const Dims &d = ctx->d;
  int rc;
  FillQueue<T> q(ctx, pitch);
#define F(...) \
  if ((rc = q.add(__VA_ARGS__)) != EDDY_OK) return rc
  if (d.itype[5] == 305) {
    bct::k_dens_inlet<T><<<(d.nx * d.ny + 255) / 256, 256, 0, ctx->stream>>>(d, pitch, dens, ctx->f[EDDY_PLANED]);
    EDDY_LAUNCHED(ctx);
    F(dens, 2, 2, 1, 1., 0);
  }
  if (d.itype[6] == 730) { F(dens, 2, d.kz2, d.kz2 - 1, 1., 0); F(dens, 2, d.nz, d.kz2, 1., 0); }
  if (d.itype[6] == 710) F(dens, 2, d.kz2, d.kz2 - 1, 1., 0);
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
  return q.flush();
}

}  // namespace
