// stencil_density.cuh -- density right-hand side of src/rhs_density.f:55-165
// (Cartesian; with CN the terms the flags f select are returned as the
// Crank-Nicolson part in *cn, stencil_cn.cuh), templated on the arithmetic type T and on
// a neighbour accessor: S.at(f, di, dj, dk) with f = 0 density, 1 eddy
// diffusivity, 2 u, 3 v, 4 w.  With T = double the operation order is the
// reference's (the plain form is compiled with -fmad=false).
#pragma once
#include "stencil_cn.cuh"

template <class T, class M, class Acc, bool CN = false>
__device__ __forceinline__ T rhs_dens(const Acc &S, const M &m, T repr1, int i, int j, int k, T *cn = nullptr,
                                       const CnFlags<T> *f = nullptr) {
  auto dens = [&](int a, int b, int c) { return S.at(0, a, b, c); };
  auto kv = [&](int a, int b, int c) { return S.at(1, a, b, c); };
  T qxp = S.at(2, 0, 0, 0), qxm = S.at(2, -1, 0, 0);
  T rxp = (dens(1, 0, 0) + dens(0, 0, 0)) * T(0.5);
  T rxm = (dens(0, 0, 0) + dens(-1, 0, 0)) * T(0.5);
  T vyp = S.at(3, 0, 0, 0), vym = S.at(3, 0, -1, 0);
  T ryp = (dens(0, 1, 0) + dens(0, 0, 0)) * T(0.5);
  T rym = (dens(0, 0, 0) + dens(0, -1, 0)) * T(0.5);
  T wzp = S.at(4, 0, 0, 0), wzm = S.at(4, 0, 0, -1);
  T rzp = (dens(0, 0, 1) + dens(0, 0, 0)) * T(0.5);
  T rzm = (dens(0, 0, 0) + dens(0, 0, -1)) * T(0.5);
  T drdxp = m.au[i] * (dens(1, 0, 0) - dens(0, 0, 0));
  T drdxm = m.au[i - 1] * (dens(0, 0, 0) - dens(-1, 0, 0));
  T drdyp = m.bv[j] * (dens(0, 1, 0) - dens(0, 0, 0));
  T drdym = m.bv[j - 1] * (dens(0, 0, 0) - dens(0, -1, 0));
  T drdzp = m.cw[k] * (dens(0, 0, 1) - dens(0, 0, 0));
  T drdzm = m.cw[k - 1] * (dens(0, 0, 0) - dens(0, 0, -1));
  T kvip = T(0.5) * (kv(1, 0, 0) + kv(0, 0, 0));
  T kvim = T(0.5) * (kv(-1, 0, 0) + kv(0, 0, 0));
  T kvjp = T(0.5) * (kv(0, 1, 0) + kv(0, 0, 0));
  T kvjm = T(0.5) * (kv(0, -1, 0) + kv(0, 0, 0));
  T kvkp = T(0.5) * (kv(0, 0, 1) + kv(0, 0, 0));
  T kvkm = T(0.5) * (kv(0, 0, -1) + kv(0, 0, 0));
  T txxp = (repr1 + kvip) * drdxp;
  T txxm = (repr1 + kvim) * drdxm;
  T tyyp = (repr1 + kvjp) * drdyp;
  T tyym = (repr1 + kvjm) * drdym;
  T tzzp = (repr1 + kvkp) * drdzp;
  T tzzm = (repr1 + kvkm) * drdzm;
  T h11 = -m.ap[i] * (rxp * qxp - rxm * qxm);
  T h22 = -m.bp[j] * (ryp * vyp - rym * vym);
  T h33 = -m.cp[k] * (rzp * wzp - rzm * wzm);
  T t11 = m.ap[i] * (txxp - txxm);
  T t22 = m.bp[j] * (tyyp - tyym);
  T t33 = m.cp[k] * (tzzp - tzzm);
  if (CN) {
    // src/rhs_density.f:147-156
    *cn = cn_part(*f, t11, t22, h11, h22);
    return (T(1.) - f->fcx) * h11 + (T(1.) - f->fcy) * h22 + h33 + (T(1.) - f->fx) * t11 + (T(1.) - f->fy) * t22 +
           t33;
  }
  return h11 + h22 + h33 + t11 + t22 + t33;
}
