// FP32 tanh of the plain form, built only from correctly rounded operations.
//
// Every step is one IEEE single-precision operation (fused multiply-add, multiply, add, divide,
// round-to-integer, exponent construction), written with the _rn intrinsics so that the compiler
// contracts nothing. The result is therefore a function of the input alone, the same on any
// IEEE machine that performs the same operations in the same order -- which is what lets a CPU
// restatement of the plain network reproduce the device's outputs bit for bit (the ACA pivot
// search compares signed determinants of network outputs, so last-bit differences would choose
// other, equally valid pivots).
//
// Method, for a = |x| (sign restored at the end):
//   a < 0.8 : tanh(a) = a + a s P(s), s = a^2, P of degree 5: a weighted least-squares
//             (Lawson-iterated, i.e. minimax) fit of (tanh(a)/a - 1)/s on [0, 0.8],
//             |error| < 3.4e-9 relative to tanh(a)/a;
//   a < 9.5 : tanh(a) = 1 - 2 / (e + 1), e = exp(2a) = 2^k exp(r) with k = rint(2a / ln 2) and
//             r = 2a - k ln 2 by Cody-Waite reduction (ln 2 split into a 16-bit head and a tail),
//             exp(r) by its Taylor series to degree 7 (|r| <= ln 2 / 2: truncation < 6e-9);
//   a >= 9.5: 1 (tanh(9.5) rounds to 1 in FP32).
// The constants are written as the FP32 values they round to (hexadecimal literals).
// Maximum error over every FP32 input in [0, 10): 1.04 ulp (mean 0.03 ulp) against a
// double-precision tanh; CUDA's tanhf is documented at 2 ulp.
#pragma once

#include <cuda_runtime.h>

namespace hignn {

__device__ __forceinline__ float tanh_f32(float x) {
  const float a = fabsf(x);
  float t;
  if (a < 0.8f) {
    const float s = __fmul_rn(a, a);
    float p = 0x1.a19af4p-10f;
    p = __fmaf_rn(p, s, -0x1.e69e6cp-8f);
    p = __fmaf_rn(p, s, 0x1.5d356ep-6f);
    p = __fmaf_rn(p, s, -0x1.b92feap-5f);
    p = __fmaf_rn(p, s, 0x1.110b7ep-3f);
    p = __fmaf_rn(p, s, -0x1.55553ep-2f);
    t = __fmaf_rn(a, __fmul_rn(s, p), a);
  } else if (a < 9.5f) {
    const float y = __fadd_rn(a, a);
    const float kf = rintf(__fmul_rn(y, 0x1.715476p+0f));
    const float r = __fmaf_rn(kf, -0x1.7f7d1cp-20f, __fmaf_rn(kf, -0x1.62e4p-1f, y));
    float p = 0x1.a01a02p-13f;
    p = __fmaf_rn(p, r, 0x1.6c16c2p-10f);
    p = __fmaf_rn(p, r, 0x1.111112p-7f);
    p = __fmaf_rn(p, r, 0x1.555556p-5f);
    p = __fmaf_rn(p, r, 0x1.555556p-3f);
    p = __fmaf_rn(p, r, 0.5f);
    p = __fmaf_rn(p, r, 1.0f);
    p = __fmaf_rn(p, r, 1.0f);
    const float e = __fmul_rn(p, __int_as_float(((int)kf + 127) << 23));
    t = __fsub_rn(1.0f, __fdiv_rn(2.0f, __fadd_rn(e, 1.0f)));
  } else {
    t = (a == a) ? 1.0f : a;  // NaN stays NaN
  }
  return copysignf(t, x);
}

}  // namespace hignn
