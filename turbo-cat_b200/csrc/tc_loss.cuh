// Per-row loss gradients of the reference, shared by the symmetric trainer
// (tc_train.cu) and the regular-tree trainer (tc_regular.cu).
#pragma once

#include <cuda_runtime.h>

#include "tcgpu.h"

namespace tc {

// fast_exp_avx2 lane arithmetic of the reference (src/boosting/loss.cpp:34-69).
__device__ __forceinline__ float ref_fast_exp(float x) {
  x = fmaxf(x, -88.0f);
  x = fminf(x, 88.0f);
  const float t = __fmul_rn(x, 1.4426950408889634f);
  const float ti = rintf(t);
  const float tf = __fsub_rn(t, ti);
  float poly = __fmaf_rn(0.0013333558146428443f, tf, 0.009618129107628477f);
  poly = __fmaf_rn(poly, tf, 0.05550410866482046f);
  poly = __fmaf_rn(poly, tf, 0.2402265069591007f);
  poly = __fmaf_rn(poly, tf, 0.6931471805599453f);
  poly = __fmaf_rn(poly, tf, 1.0f);
  const float pow2 = __int_as_float(((int)ti + 127) << 23);
  return __fmul_rn(poly, pow2);
}

__device__ __forceinline__ void loss_grad(int loss, float pred, float y, uint32_t i, uint32_t n_vec,
                                          float gamma, float alpha, float& g, float& h) {
  if (loss == TC_LOSS_MSE) {  // src/boosting/loss.cpp:348-362
    g = __fmul_rn(2.0f, __fsub_rn(pred, y));
    h = 2.0f;
  } else if (loss == TC_LOSS_LOGLOSS) {  // src/boosting/loss.cpp:123-211
    float p;
    if (i < n_vec) {
      float x = fminf(fmaxf(pred, -15.0f), 15.0f);
      p = __fdiv_rn(1.0f, __fadd_rn(1.0f, ref_fast_exp(__fsub_rn(0.0f, x))));
    } else {
      const float x = fmaxf(-15.0f, fminf(15.0f, pred));
      p = __fdiv_rn(1.0f, __fadd_rn(1.0f, expf(-x)));
    }
    g = __fsub_rn(p, y);
    h = fmaxf(__fmul_rn(p, __fsub_rn(1.0f, p)), 1e-6f);
  } else {  // TC_LOSS_FOCAL, src/boosting/loss.cpp:505-539 (class weights 1)
    const float p = __fdiv_rn(1.0f, __fadd_rn(1.0f, expf(-pred)));
    float pt = __fmaf_rn(y, p, __fmul_rn(__fsub_rn(1.0f, y), __fsub_rn(1.0f, p)));
    pt = fmaxf(pt, 1e-7f);
    const float at = __fmaf_rn(y, alpha, __fmul_rn(__fsub_rn(1.0f, y), __fsub_rn(1.0f, alpha)));
    const float fw = powf(__fsub_rn(1.0f, pt), gamma);
    const float coef = __fmul_rn(at, fw);
    g = __fmul_rn(coef, __fsub_rn(p, y));
    h = fmaxf(__fmul_rn(__fmul_rn(coef, p), __fsub_rn(1.0f, p)), 1e-6f);
  }
}

}  // namespace tc
