// k_sgs32.cu -- the mixed form's FP32 dynamic eddy viscosity: the fused
// y-marching TURVIS kernel of k_sgs_impl.cuh instantiated for float in its own
// translation unit, compiled with FMA contraction (the FP64 instantiation in
// k_sgs.cu keeps the reference's operation order under -fmad=false).
#include <cmath>
#include <vector>

#include "eddy_internal.h"

int launch_fill_plane(eddy_ctx *ctx, double *a, int axis, int dst, int src, double sgn, int zero);

namespace {
#include "k_sgs_impl.cuh"
}  // namespace

// FP32 dynamic procedure on the mixed form's FP32 velocities (row pitch px),
// the same fused march in single precision; TV (FP64) receives the result.
// gs32 (px-pitched field) and imm32/ilm32 ((NX,NZ)) are FP32 scratch.
int launch_turvis32(eddy_ctx *ctx, int px, const float *u, const float *v, const float *w, float *gs32,
                    float *imm32, float *ilm32) {
  int rc = turvis_dynamic<float>(ctx, px, u, v, w, gs32, imm32, ilm32);
  if (rc) return rc;
  return boundturb_tv(ctx);
}
