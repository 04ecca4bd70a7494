// stencil_cn.cuh -- the Crank-Nicolson split of the viscous terms shared by
// the momentum and density right-hand sides (src/rhs.f:175-191,
// src/rhs_density.f:147-156): CN bit 0 = IMPLY, bit 1 = IMPLX; the convective
// flags IMPLCX, IMPLCY are 0.
#pragma once

// the implicit-axis flag (rflagx or rflagy) as a factor: 1 when set, else 0
template <class T, int F>
__device__ __forceinline__ constexpr T cn_flag() {
  return F ? T(1.) : T(0.);
}
// the C.N. part rflagx t11 + rflagy t22 (the convective flags are 0)
template <class T, int CN>
__device__ __forceinline__ T cn_part(T t11, T t22) {
  if ((CN & 3) == 3) return t11 + t22;
  return (CN & 2) ? t11 : t22;
}
