// Seventh-order WENO reconstruction used by the hybrid scheme
// (OOP/spatial_operator.py:87-124), arranged for FP32 robustness.
//
// The reference evaluates each smoothness indicator IS_k as a quadratic form
// of the raw stencil values, whose terms are O(1e4 v^2) and cancel to the
// small true indicator; in FP32 that cancellation loses everything.  Here
// every standard Balsara-Shu indicator is written as an exact sum of three
// positive squares of linear combinations of first differences
// (an LDL^T factorisation of the same quadratic form over d1 = w1 - w0,
// d2 = w2 - w1, d3 = w3 - w2; coefficients are exact rationals).  The
// reference writes 544 where the published leading coefficient of IS_0 is
// 547, so its IS_0 equals the standard one minus 3 v1^2; that term is added
// back explicitly to reproduce the reference's weights.
#pragma once

namespace hitb200 {

// IS = D0 s1^2 + D1 s2^2 + D2 d3^2 with s1 = d1 + L10 d2 + L20 d3,
// s2 = d2 + L21 d3 (one line per stencil: D0, D1, D2, L10, L20, L21).
#define HITB200_WENO_IS(NAME, D0, D1, D2, L10, L20, L21)                         \
  template <typename T>                                                        \
  __device__ __forceinline__ T NAME(T w0, T w1, T w2, T w3) {                  \
    T d1 = w1 - w0, d2 = w2 - w1, d3 = w3 - w2;                                \
    T s1 = d1 + T(L10) * d2 + T(L20) * d3;                                     \
    T s2 = d2 + T(L21) * d3;                                                   \
    return T(D0) * s1 * s1 + T(D1) * s2 * s2 + T(D2) * d3 * d3;                \
  }
HITB200_WENO_IS(weno_is0, 547.0, 85040.0 / 547.0, 203060.0 / 1063.0, -1394.0 / 547.0,
                927.0 / 547.0, -3167.0 / 2126.0)
HITB200_WENO_IS(weno_is1, 267.0, 85040.0 / 267.0, 203060.0 / 1063.0, -554.0 / 267.0,
                247.0 / 267.0, -1345.0 / 2126.0)
HITB200_WENO_IS(weno_is2, 547.0, 293200.0 / 547.0, 40612.0 / 733.0, -714.0 / 547.0,
                247.0 / 547.0, -3167.0 / 7330.0)
HITB200_WENO_IS(weno_is3, 2107.0, 1083920.0 / 2107.0, 203060.0 / 13549.0, -2594.0 / 2107.0,
                927.0 / 2107.0, -13313.0 / 27098.0)
#undef HITB200_WENO_IS

// Value at the right face of v3 from v0..v6 (the reference's v1..v7).
// Nonlinear weights alpha_k = d_k / (eps + IS_k)^2 normalised by their sum.
// FP64: all four weights are scaled by prod_k (eps + IS_k)^2 so that the face
// value needs one division (the scaled weights stay within 1e-60 .. 1e40).
// FP32: that product would underflow, so each weight uses a fast reciprocal
// (2 ulp), which perturbs the convex combination far below FP32 flux error.
// The reference's IS_0 can be negative, so eps + IS_0 can cancel to (nearly)
// zero; its square is floored at 1e-30 so that the fast reciprocal stays
// finite.  The floored weight then exceeds every other by at least 1e10, so
// the face value is q_0 to FP32 precision, the exact limit of the weights.
template <typename T>
__device__ __forceinline__ T weno7(T v0, T v1, T v2, T v3, T v4, T v5, T v6) {
  const T eps = T(1e-10);
  const T q0 = T(-1.0 / 4.0) * v0 + T(13.0 / 12.0) * v1 - T(23.0 / 12.0) * v2 + T(25.0 / 12.0) * v3;
  const T q1 = T(1.0 / 12.0) * v1 - T(5.0 / 12.0) * v2 + T(13.0 / 12.0) * v3 + T(1.0 / 4.0) * v4;
  const T q2 = T(-1.0 / 12.0) * v2 + T(7.0 / 12.0) * v3 + T(7.0 / 12.0) * v4 - T(1.0 / 12.0) * v5;
  const T q3 = T(1.0 / 4.0) * v3 + T(13.0 / 12.0) * v4 - T(5.0 / 12.0) * v5 + T(1.0 / 12.0) * v6;
  const T e0 = eps + (weno_is0<T>(v0, v1, v2, v3) - T(3) * v0 * v0);
  const T e1 = eps + weno_is1<T>(v1, v2, v3, v4);
  const T e2 = eps + weno_is2<T>(v2, v3, v4, v5);
  const T e3 = eps + weno_is3<T>(v3, v4, v5, v6);
  const T s0 = e0 * e0, s1 = e1 * e1, s2 = e2 * e2, s3 = e3 * e3;
  if constexpr (sizeof(T) == 8) {
    const T p01 = s0 * s1, p23 = s2 * s3;
    const T w0 = T(1.0 / 35.0) * s1 * p23;
    const T w1 = T(12.0 / 35.0) * s0 * p23;
    const T w2 = T(18.0 / 35.0) * s3 * p01;
    const T w3 = T(4.0 / 35.0) * s2 * p01;
    return (w0 * q0 + w1 * q1 + w2 * q2 + w3 * q3) / (w0 + w1 + w2 + w3);
  } else {
    const float a0 = __fdividef(1.0f / 35.0f, fmaxf(s0, 1e-30f));
    const float a1 = __fdividef(12.0f / 35.0f, fmaxf(s1, 1e-30f));
    const float a2 = __fdividef(18.0f / 35.0f, fmaxf(s2, 1e-30f));
    const float a3 = __fdividef(4.0f / 35.0f, fmaxf(s3, 1e-30f));
    return __fdividef(a0 * q0 + a1 * q1 + a2 * q2 + a3 * q3, a0 + a1 + a2 + a3);
  }
}

}  // namespace hitb200
