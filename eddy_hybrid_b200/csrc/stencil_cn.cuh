// stencil_cn.cuh -- the Crank-Nicolson split of the right-hand sides
// (src/rhs.f:175-191, src/rhs_density.f:147-156): the flags rflagx = IMPLX,
// rflagy = IMPLY, rflagcx = IMPLCX, rflagcy = IMPLCY (each 0 or 1) move the
// viscous / convective terms of their axes from the explicit right-hand side
// to the C.N. part, in the reference's expressions:
//   explicit = (1 - fcx) h11 + (1 - fcy) h22 + h33 + (1 - fx) t11 + (1 - fy) t22 + t33 (+ cross terms)
//   C.N.     = fx t11 + fy t22 + fcx h11 + fcy h22
#pragma once

template <class T>
struct CnFlags {
  T fx, fy, fcx, fcy;
};

template <class T>
__device__ __forceinline__ T cn_part(const CnFlags<T> &f, T t11, T t22, T h11, T h22) {
  return f.fx * t11 + f.fy * t22 + f.fcx * h11 + f.fcy * h22;
}
