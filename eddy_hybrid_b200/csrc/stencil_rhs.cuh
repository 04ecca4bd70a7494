// stencil_rhs.cuh -- explicit momentum right-hand side of src/rhs.f:4-438
// (Cartesian; with CN the terms the flags f select are returned as the
// Crank-Nicolson part in *cn, stencil_cn.cuh), templated on the
// arithmetic type T and on a neighbour accessor: S.u/v/w/t(di,dj,dk) return
// uo/vo/wo/tv at the offset from the current cell.  With T = double the
// operation order is exactly the reference's (the plain form is compiled with
// -fmad=false); with T = float the mixed form accumulates in FP32.
#pragma once
#include "stencil_cn.cuh"

// ---------------------------------------------------------------------------
// u-momentum explicit RHS at a u point (src/rhs.f:77-172)
template <class T, class M, class Acc, bool CN = false>
__device__ __forceinline__ T rhs_u(const Acc &S, const M &m, T ru1, int i, int j, int k, T *cn = nullptr,
                                    const CnFlags<T> *f = nullptr) {
  T qxp = (S.u(1, 0, 0) + S.u(0, 0, 0)) * T(0.5);
  T qxm = (S.u(0, 0, 0) + S.u(-1, 0, 0)) * T(0.5);
  T uxp = (S.u(1, 0, 0) + S.u(0, 0, 0)) * T(0.5);
  T uxm = (S.u(0, 0, 0) + S.u(-1, 0, 0)) * T(0.5);
  T uyp = (S.u(0, 1, 0) + S.u(0, 0, 0)) * T(0.5);
  T uym = (S.u(0, 0, 0) + S.u(0, -1, 0)) * T(0.5);
  T uzp = (S.u(0, 0, 1) + S.u(0, 0, 0)) * T(0.5);
  T uzm = (S.u(0, 0, 0) + S.u(0, 0, -1)) * T(0.5);
  T vxp = (S.v(1, 0, 0) + S.v(0, 0, 0)) * T(0.5);
  T vxm = (S.v(1, -1, 0) + S.v(0, -1, 0)) * T(0.5);
  T wxp = (S.w(1, 0, 0) + S.w(0, 0, 0)) * T(0.5);
  T wxm = (S.w(1, 0, -1) + S.w(0, 0, -1)) * T(0.5);
  T dqdxp = m.ap[i + 1] * (S.u(1, 0, 0) - S.u(0, 0, 0));
  T dqdxm = m.ap[i] * (S.u(0, 0, 0) - S.u(-1, 0, 0));
  T dudyp = m.bv[j] * (S.u(0, 1, 0) - S.u(0, 0, 0));
  T dudym = m.bv[j - 1] * (S.u(0, 0, 0) - S.u(0, -1, 0));
  T dudzp = m.cw[k] * (S.u(0, 0, 1) - S.u(0, 0, 0));
  T dudzm = m.cw[k - 1] * (S.u(0, 0, 0) - S.u(0, 0, -1));
  T dvdxp = m.au[i] * (S.v(1, 0, 0) - S.v(0, 0, 0));
  T dvdxm = m.au[i] * (S.v(1, -1, 0) - S.v(0, -1, 0));
  T dwdxp = m.au[i] * (S.w(1, 0, 0) - S.w(0, 0, 0));
  T dwdxm = m.au[i] * (S.w(1, 0, -1) - S.w(0, 0, -1));
  T tvjp = T(0.25) * (S.t(1, 0, 0) + S.t(0, 0, 0) + S.t(1, 1, 0) + S.t(0, 1, 0));
  T tvjm = T(0.25) * (S.t(1, 0, 0) + S.t(0, 0, 0) + S.t(1, -1, 0) + S.t(0, -1, 0));
  T tvkp = T(0.25) * (S.t(1, 0, 0) + S.t(0, 0, 0) + S.t(1, 0, 1) + S.t(0, 0, 1));
  T tvkm = T(0.25) * (S.t(1, 0, 0) + S.t(0, 0, 0) + S.t(1, 0, -1) + S.t(0, 0, -1));
  T txxp = (ru1 + T(2.) * S.t(1, 0, 0)) * dqdxp;
  T txxm = (ru1 + T(2.) * S.t(0, 0, 0)) * dqdxm;
  T tyyp = (ru1 + tvjp) * dudyp;
  T tyym = (ru1 + tvjm) * dudym;
  T tzzp = (ru1 + tvkp) * dudzp;
  T tzzm = (ru1 + tvkm) * dudzm;
  T txyp = tvjp * dvdxp;
  T txym = tvjm * dvdxm;
  T txzp = tvkp * dwdxp;
  T txzm = tvkm * dwdxm;
  T h11 = -m.au[i] * (qxp * uxp - qxm * uxm);
  T h22 = -m.bu[j] * (vxp * uyp - vxm * uym);
  T h33 = -m.cu[k] * (wxp * uzp - wxm * uzm);
  T t11 = m.au[i] * (txxp - txxm);
  T t22 = m.bu[j] * (tyyp - tyym);
  T t33 = m.cu[k] * (tzzp - tzzm);
  T s22 = m.bu[j] * (txyp - txym);
  T s33 = m.cu[k] * (txzp - txzm);
  if (CN) {
    // src/rhs.f:175-191 (ruimplx = ruimply = 1)
    *cn = cn_part(*f, t11, t22, h11, h22);
    return (T(1.) - f->fcx) * h11 + (T(1.) - f->fcy) * h22 + h33 + (T(1.) - f->fx) * t11 + (T(1.) - f->fy) * t22 +
           t33 + s22 + s33;
  }
  return h11 + h22 + h33 + t11 + t22 + t33 + s22 + s33;
}

// v-momentum (src/rhs.f:219-321)
template <class T, class M, class Acc, bool CN = false>
__device__ __forceinline__ T rhs_v(const Acc &S, const M &m, T ru1, int i, int j, int k, T *cn = nullptr,
                                    const CnFlags<T> *f = nullptr) {
  T vxp = (S.v(1, 0, 0) + S.v(0, 0, 0)) * T(0.5);
  T vxm = (S.v(0, 0, 0) + S.v(-1, 0, 0)) * T(0.5);
  T vyp = (S.v(0, 1, 0) + S.v(0, 0, 0)) * T(0.5);
  T vym = (S.v(0, 0, 0) + S.v(0, -1, 0)) * T(0.5);
  T vzp = (S.v(0, 0, 1) + S.v(0, 0, 0)) * T(0.5);
  T vzm = (S.v(0, 0, 0) + S.v(0, 0, -1)) * T(0.5);
  T qyp = (S.u(0, 1, 0) + S.u(0, 0, 0)) * T(0.5);
  T qym = (S.u(-1, 1, 0) + S.u(-1, 0, 0)) * T(0.5);
  T wyp = (S.w(0, 1, 0) + S.w(0, 0, 0)) * T(0.5);
  T wym = (S.w(0, 1, -1) + S.w(0, 0, -1)) * T(0.5);
  T dvdxp = m.au[i] * (S.v(1, 0, 0) - S.v(0, 0, 0));
  T dvdxm = m.au[i - 1] * (S.v(0, 0, 0) - S.v(-1, 0, 0));
  T dvdyp = m.bp[j + 1] * (S.v(0, 1, 0) - S.v(0, 0, 0));
  T dvdym = m.bp[j] * (S.v(0, 0, 0) - S.v(0, -1, 0));
  T dvdzp = m.cw[k] * (S.v(0, 0, 1) - S.v(0, 0, 0));
  T dvdzm = m.cw[k - 1] * (S.v(0, 0, 0) - S.v(0, 0, -1));
  T dudyp = m.bv[j] * (S.u(0, 1, 0) - S.u(0, 0, 0));
  T dudym = m.bv[j] * (S.u(-1, 1, 0) - S.u(-1, 0, 0));
  T dwdyp = m.bv[j] * (S.w(0, 1, 0) - S.w(0, 0, 0));
  T dwdym = m.bv[j] * (S.w(0, 1, -1) - S.w(0, 0, -1));
  T tvip = T(0.25) * (S.t(0, 1, 0) + S.t(0, 0, 0) + S.t(1, 1, 0) + S.t(1, 0, 0));
  T tvim = T(0.25) * (S.t(0, 1, 0) + S.t(0, 0, 0) + S.t(-1, 1, 0) + S.t(-1, 0, 0));
  T tvkp = T(0.25) * (S.t(0, 1, 0) + S.t(0, 0, 0) + S.t(0, 1, 1) + S.t(0, 0, 1));
  T tvkm = T(0.25) * (S.t(0, 1, 0) + S.t(0, 0, 0) + S.t(0, 1, -1) + S.t(0, 0, -1));
  T txxp = (ru1 + tvip) * dvdxp;
  T txxm = (ru1 + tvim) * dvdxm;
  T tyyp = (ru1 + T(2.) * S.t(0, 1, 0)) * dvdyp;
  T tyym = (ru1 + T(2.) * S.t(0, 0, 0)) * dvdym;
  T tzzp = (ru1 + tvkp) * dvdzp;
  T tzzm = (ru1 + tvkm) * dvdzm;
  T txyp = tvip * dudyp;
  T txym = tvim * dudym;
  T tyzp = tvkp * dwdyp;
  T tyzm = tvkm * dwdym;
  T h11 = -m.av[i] * (qyp * vxp - qym * vxm);
  T h22 = -m.bv[j] * (vyp * vyp - vym * vym);
  T h33 = -m.cv[k] * (wyp * vzp - wym * vzm);
  T t11 = m.av[i] * (txxp - txxm);
  T t22 = m.bv[j] * (tyyp - tyym);
  T t33 = m.cv[k] * (tzzp - tzzm);
  T s11 = m.av[i] * (txyp - txym);
  T s33 = m.cv[k] * (tyzp - tyzm);
  if (CN) {
    *cn = cn_part(*f, t11, t22, h11, h22);
    return (T(1.) - f->fcx) * h11 + (T(1.) - f->fcy) * h22 + h33 + (T(1.) - f->fx) * t11 + (T(1.) - f->fy) * t22 +
           t33 + s11 + s33;
  }
  return h11 + h22 + h33 + t11 + t22 + t33 + s11 + s33;
}

// w-momentum (src/rhs.f:347-422)
template <class T, class M, class Acc, bool CN = false>
__device__ __forceinline__ T rhs_w(const Acc &S, const M &m, T ru1, int i, int j, int k, T *cn = nullptr,
                                    const CnFlags<T> *f = nullptr) {
  T wxp = (S.w(1, 0, 0) + S.w(0, 0, 0)) * T(0.5);
  T wxm = (S.w(0, 0, 0) + S.w(-1, 0, 0)) * T(0.5);
  T wyp = (S.w(0, 1, 0) + S.w(0, 0, 0)) * T(0.5);
  T wym = (S.w(0, 0, 0) + S.w(0, -1, 0)) * T(0.5);
  T wzp = (S.w(0, 0, 1) + S.w(0, 0, 0)) * T(0.5);
  T wzm = (S.w(0, 0, 0) + S.w(0, 0, -1)) * T(0.5);
  T qzp = (S.u(0, 0, 1) + S.u(0, 0, 0)) * T(0.5);
  T qzm = (S.u(-1, 0, 1) + S.u(-1, 0, 0)) * T(0.5);
  T vzp = (S.v(0, 0, 1) + S.v(0, 0, 0)) * T(0.5);
  T vzm = (S.v(0, -1, 1) + S.v(0, -1, 0)) * T(0.5);
  T dwdxp = m.au[i] * (S.w(1, 0, 0) - S.w(0, 0, 0));
  T dwdxm = m.au[i - 1] * (S.w(0, 0, 0) - S.w(-1, 0, 0));
  T dwdyp = m.bv[j] * (S.w(0, 1, 0) - S.w(0, 0, 0));
  T dwdym = m.bv[j - 1] * (S.w(0, 0, 0) - S.w(0, -1, 0));
  T dwdzp = m.cp[k + 1] * (S.w(0, 0, 1) - S.w(0, 0, 0));
  T dwdzm = m.cp[k] * (S.w(0, 0, 0) - S.w(0, 0, -1));
  T dudzp = m.cw[k] * (S.u(0, 0, 1) - S.u(0, 0, 0));
  T dudzm = m.cw[k] * (S.u(-1, 0, 1) - S.u(-1, 0, 0));
  T dvdzp = m.cw[k] * (S.v(0, 0, 1) - S.v(0, 0, 0));
  T dvdzm = m.cw[k] * (S.v(0, -1, 1) - S.v(0, -1, 0));
  T tvip = T(0.25) * (S.t(0, 0, 1) + S.t(0, 0, 0) + S.t(1, 0, 1) + S.t(1, 0, 0));
  T tvim = T(0.25) * (S.t(0, 0, 1) + S.t(0, 0, 0) + S.t(-1, 0, 1) + S.t(-1, 0, 0));
  T tvjp = T(0.25) * (S.t(0, 0, 1) + S.t(0, 0, 0) + S.t(0, 1, 1) + S.t(0, 1, 0));
  T tvjm = T(0.25) * (S.t(0, 0, 1) + S.t(0, 0, 0) + S.t(0, -1, 1) + S.t(0, -1, 0));
  T txxp = (ru1 + tvip) * dwdxp;
  T txxm = (ru1 + tvim) * dwdxm;
  T tyyp = (ru1 + tvjp) * dwdyp;
  T tyym = (ru1 + tvjm) * dwdym;
  T tzzp = (ru1 + T(2.) * S.t(0, 0, 1)) * dwdzp;
  T tzzm = (ru1 + T(2.) * S.t(0, 0, 0)) * dwdzm;
  T txzp = tvip * dudzp;
  T txzm = tvim * dudzm;
  T tyzp = tvjp * dvdzp;
  T tyzm = tvjm * dvdzm;
  T h11 = -m.aw[i] * (qzp * wxp - qzm * wxm);
  T h22 = -m.bw[j] * (vzp * wyp - vzm * wym);
  T h33 = -m.cw[k] * (wzp * wzp - wzm * wzm);
  T t11 = m.aw[i] * (txxp - txxm);
  T t22 = m.bw[j] * (tyyp - tyym);
  T t33 = m.cw[k] * (tzzp - tzzm);
  T s11 = m.aw[i] * (txzp - txzm);
  T s22 = m.bw[j] * (tyzp - tyzm);
  if (CN) {
    *cn = cn_part(*f, t11, t22, h11, h22);
    return (T(1.) - f->fcx) * h11 + (T(1.) - f->fcy) * h22 + h33 + (T(1.) - f->fx) * t11 + (T(1.) - f->fy) * t22 +
           t33 + s11 + s22;
  }
  return h11 + h22 + h33 + t11 + t22 + t33 + s11 + s22;
}

