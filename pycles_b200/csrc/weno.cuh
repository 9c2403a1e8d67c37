// WENO and central interpolants, Csrc/advection_interpolation.h.
//
// The templates keep the reference's operations and their order.  The FP64
// plain form instantiates them with double in a translation unit compiled
// without FMA contraction (advection_f64.cu), which reproduces the
// reference's roundings exactly: the WENO7 smoothness indicators are
// quadratic forms whose ~1e4 phi^2 terms cancel down to (dphi)^2, and the
// face values enter flux differences that cancel further, so any other
// rounding (a contracted FMA, a rearranged weight formula) moves tendencies
// of slow velocity components by ~1e-12 relative.  The FP32 forms are used
// by the precision path through weno_face<ORDER, true>:
// the stencil is shifted by its centre value in FP64, the WENO arithmetic
// (candidate polynomials, smoothness indicators, weights) runs in FP32 on
// the differences, and the centre is added back in FP64.  WENO is exactly
// invariant to that shift in real arithmetic, and working on differences
// keeps the FP32 smoothness indicators free of the rounding noise of the
// absolute values.
#pragma once

template <typename R>
__device__ __forceinline__ R interp_4(R phim1, R phi, R phip1, R phip2) {
  // advection_interpolation.h:12-14
  return R(7.0 / 12.0) * (phi + phip1) - R(1.0 / 12.0) * (phim1 + phip2);
}

template <typename R>
__device__ __forceinline__ R interp_6(R phim2, R phim1, R phi, R phip1, R phip2, R phip3) {
  // advection_interpolation.h:20-24
  return (R(37.0 / 60.0) * (phi + phip1) - R(2.0 / 15.0) * (phim1 + phip2) +
          R(1.0 / 60.0) * (phim2 + phip3));
}

template <typename R>
__device__ __forceinline__ R weno5(R phim2, R phim1, R phi, R phip1, R phip2) {
  // advection_interpolation.h:79-104
  const R p0 = R(1.0 / 3.0) * phim2 - R(7.0 / 6.0) * phim1 + R(11.0 / 6.0) * phi;
  const R p1 = R(-1.0 / 6.0) * phim1 + R(5.0 / 6.0) * phi + R(1.0 / 3.0) * phip1;
  const R p2 = R(1.0 / 3.0) * phi + R(5.0 / 6.0) * phip1 - R(1.0 / 6.0) * phip2;
  const R a2 = phi - R(2.0) * phip1 + phip2;
  const R b2 = R(3.0) * phi - R(4.0) * phip1 + phip2;
  const R beta2 = R(13.0 / 12.0) * a2 * a2 + R(0.25) * b2 * b2;
  const R a1 = phim1 - R(2.0) * phi + phip1;
  const R b1 = phim1 - phip1;
  const R beta1 = R(13.0 / 12.0) * a1 * a1 + R(0.25) * b1 * b1;
  const R a0 = phim2 - R(2.0) * phim1 + phi;
  const R b0 = phim2 - R(4.0) * phim1 + R(3.0) * phi;
  const R beta0 = R(13.0 / 12.0) * a0 * a0 + R(0.25) * b0 * b0;
  const R e0 = beta0 + R(1e-10);
  const R e1 = beta1 + R(1e-10);
  const R e2 = beta2 + R(1e-10);
  const R alpha0 = R(0.1) / (e0 * e0);
  const R alpha1 = R(0.6) / (e1 * e1);
  const R alpha2 = R(0.3) / (e2 * e2);
  const R alpha_sum_inv = R(1.0) / (alpha0 + alpha1 + alpha2);
  const R w0 = alpha0 * alpha_sum_inv;
  const R w1 = alpha1 * alpha_sum_inv;
  const R w2 = alpha2 * alpha_sum_inv;
  return w0 * p0 + w1 * p1 + w2 * p2;
}

template <typename R>
__device__ __forceinline__ R weno7(R phim3, R phim2, R phim1, R phi, R phip1, R phip2, R phip3) {
  // advection_interpolation.h:106-145
  const R p0 = R(-1.0 / 4.0) * phim3 + R(13.0 / 12.0) * phim2 + R(-23.0 / 12.0) * phim1 +
               R(25.0 / 12.0) * phi;
  const R p1 = R(1.0 / 12.0) * phim2 + R(-5.0 / 12.0) * phim1 + R(13.0 / 12.0) * phi +
               R(1.0 / 4.0) * phip1;
  const R p2 = R(-1.0 / 12.0) * phim1 + R(7.0 / 12.0) * phi + R(7.0 / 12.0) * phip1 +
               R(-1.0 / 12.0) * phip2;
  const R p3 = R(1.0 / 4.0) * phi + R(13.0 / 12.0) * phip1 + R(-5.0 / 12.0) * phip2 +
               R(1.0 / 12.0) * phip3;
  const R beta0 = (phim3 * (R(547.0) * phim3 - R(3882.0) * phim2 + R(4642.0) * phim1 - R(1854.0) * phi) +
                   phim2 * (R(7043.0) * phim2 - R(17246.0) * phim1 + R(7042.0) * phi) +
                   phim1 * (R(11003.0) * phim1 - R(9402.0) * phi) + R(2107.0) * phi * phi);
  const R beta1 = (phim2 * (R(267.0) * phim2 - R(1642.0) * phim1 + R(1602.0) * phi - R(494.0) * phip1) +
                   phim1 * (R(2843.0) * phim1 - R(5966.0) * phi + R(1922.0) * phip1) +
                   phi * (R(3443.0) * phi - R(2522.0) * phip1) + R(547.0) * phip1 * phip1);
  const R beta2 = (phim1 * (R(547.0) * phim1 - R(2522.0) * phi + R(1922.0) * phip1 - R(494.0) * phip2) +
                   phi * (R(3443.0) * phi - R(5966.0) * phip1 + R(1602.0) * phip2) +
                   phip1 * (R(2843.0) * phip1 - R(1642.0) * phip2) + R(267.0) * phip2 * phip2);
  const R beta3 = (phi * (R(2107.0) * phi - R(9402.0) * phip1 + R(7042.0) * phip2 - R(1854.0) * phip3) +
                   phip1 * (R(11003.0) * phip1 - R(17246.0) * phip2 + R(4642.0) * phip3) +
                   phip2 * (R(7043.0) * phip2 - R(3882.0) * phip3) + R(547.0) * phip3 * phip3);
  const R e0 = beta0 + R(1e-10);
  const R e1 = beta1 + R(1e-10);
  const R e2 = beta2 + R(1e-10);
  const R e3 = beta3 + R(1e-10);
  const R alpha0 = R(1.0 / 35.0) / (e0 * e0);
  const R alpha1 = R(12.0 / 35.0) / (e1 * e1);
  const R alpha2 = R(18.0 / 35.0) / (e2 * e2);
  const R alpha3 = R(4.0 / 35.0) / (e3 * e3);
  const R alpha_sum_inv = R(1.0) / (alpha0 + alpha1 + alpha2 + alpha3);
  const R w0 = alpha0 * alpha_sum_inv;
  const R w1 = alpha1 * alpha_sum_inv;
  const R w2 = alpha2 * alpha_sum_inv;
  const R w3 = alpha3 * alpha_sum_inv;
  return w0 * p0 + w1 * p1 + w2 * p2 + w3 * p3;
}

// FP32 value type whose division is the fast approximate one (__fdividef,
// ~2 ulp): the precision form's WENO weights are ratios of smoothness
// indicators and need no correctly rounded division.
struct FastF {
  float v;
  __device__ __forceinline__ FastF() : v(0.0f) {}
  __device__ __forceinline__ explicit FastF(float x) : v(x) {}
  __device__ __forceinline__ explicit FastF(double x) : v((float)x) {}
};
__device__ __forceinline__ FastF operator+(FastF a, FastF b) { return FastF(a.v + b.v); }
__device__ __forceinline__ FastF operator-(FastF a, FastF b) { return FastF(a.v - b.v); }
__device__ __forceinline__ FastF operator*(FastF a, FastF b) { return FastF(a.v * b.v); }
__device__ __forceinline__ FastF operator/(FastF a, FastF b) { return FastF(__fdividef(a.v, b.v)); }

// The FP32 interpolants on a stencil shifted by its centre value, with the
// zero centre folded out by hand: IEEE arithmetic does not let the compiler
// drop x * 0, and the folded terms are a quarter of the WENO7 work.  Real-
// arithmetic identical to weno5 / weno7 with phi = 0 (a* = phim*, b* = phip*).
//
// The arithmetic runs on packed FP32 pairs (FFMA2: two lanes per
// instruction).  The smoothness indicators pair up exactly: WENO7's beta0
// and beta3 are the same quadratic form of (a3, a2, a1) and (b3, b2, b1),
// beta1 and beta2 the same form of (a2, a1, b1) and (b2, b1, a1), WENO5's
// beta0 and beta2 the same form of (a2, a1) and (b2, b1); the candidate
// polynomials pair with per-lane coefficients.
__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }

__device__ __forceinline__ float weno5_c0(float a2, float a1, float b1, float b2) {
  const float2 X2 = f2(a2, b2), X1 = f2(a1, b1);
  // (p0, p2) = (1/3 a2 - 7/6 a1, -1/6 b2 + 5/6 b1); p1 = -1/6 a1 + 1/3 b1
  const float2 P02 = fma2(X2, f2(1.0f / 3.0f, -1.0f / 6.0f), mul2(X1, f2(-7.0f / 6.0f, 5.0f / 6.0f)));
  const float p1 = (-1.0f / 6.0f) * a1 + (1.0f / 3.0f) * b1;
  // (beta0, beta2) = 13/12 (X2 - 2 X1)^2 + 1/4 (X2 - 4 X1)^2
  const float2 Sa = fma2(X1, f2(-2.0f, -2.0f), X2);
  const float2 Sb = fma2(X1, f2(-4.0f, -4.0f), X2);
  // e_k = beta_k + 1e-10, all three scaled by kE (the weights d_k / e_k^2
  // over their sum do not change when every e_k is scaled alike)
  constexpr float kE = 1.0e4f;
  const float2 E02 = fma2(mul2(Sa, f2(kE * 13.0f / 12.0f, kE * 13.0f / 12.0f)), Sa,
                          fma2(mul2(Sb, f2(kE * 0.25f, kE * 0.25f)), Sb, f2(kE * 1e-10f, kE * 1e-10f)));
  const float s1a = a1 + b1, s1b = a1 - b1;
  const float e1 = (kE * 13.0f / 12.0f) * s1a * s1a + (kE * 0.25f) * s1b * s1b + kE * 1e-10f;
  // the weights with numerators and denominator multiplied by
  // e0^2 e1^2 e2^2: one reciprocal instead of four.  With the scaling the
  // products stay normal numbers: >= 1e-24 where every stencil is flat
  // (unscaled they reach 1e-40, which the packed multiplies flush to zero),
  // <= 3e38 for first differences up to ~600 (far beyond any velocity or
  // scalar jump between neighbouring cells; beyond it the face value is not
  // finite, which the thermodynamics' non-finite check reports).  Capping
  // the indicators instead cost 0.5 ms per step at 512x512x256.
  const float2 Q02 = mul2(E02, E02);
  const float q1 = e1 * e1;
  const float2 A02 = mul2(mul2(f2(0.1f, 0.3f), f2(Q02.y, Q02.x)), f2(q1, q1));  // (0.1 q1 q2, 0.3 q0 q1)
  const float a1w = 0.6f * Q02.x * Q02.y;
  const float2 acc = mul2(A02, P02);
  const float inv = __fdividef(1.0f, A02.x + A02.y + a1w);
  return (acc.x + acc.y + a1w * p1) * inv;
}

__device__ __forceinline__ float weno7_c0(float a3, float a2, float a1, float b1, float b2, float b3) {
  const float2 X3 = f2(a3, b3), X2 = f2(a2, b2), X1 = f2(a1, b1), X0 = f2(b1, a1);
  // (p0, p3) and (p1, p2)
  const float2 P03 = fma2(X3, f2(-0.25f, 1.0f / 12.0f),
                          fma2(X2, f2(13.0f / 12.0f, -5.0f / 12.0f), mul2(X1, f2(-23.0f / 12.0f, 13.0f / 12.0f))));
  const float2 P12 = fma2(X2, f2(1.0f / 12.0f, -1.0f / 12.0f),
                          fma2(X1, f2(-5.0f / 12.0f, 7.0f / 12.0f), mul2(X0, f2(0.25f, -1.0f / 12.0f))));
  // (beta0, beta3) = Q(X3, X2, X1), Q(x3, x2, x1) = x3 (547 x3 - 3882 x2 + 4642 x1)
  //                  + x2 (7043 x2 - 17246 x1) + 11003 x1^2
  const float2 t3 = fma2(X1, f2(4642.0f, 4642.0f), fma2(X2, f2(-3882.0f, -3882.0f), mul2(X3, f2(547.0f, 547.0f))));
  const float2 t2 = fma2(X1, f2(-17246.0f, -17246.0f), mul2(X2, f2(7043.0f, 7043.0f)));
  const float2 E03 = fma2(mul2(X1, f2(11003.0f, 11003.0f)), X1, fma2(X2, t2, fma2(X3, t3, f2(1e-10f, 1e-10f))));
  // (beta1, beta2) = Q'(X2, X1, X0), Q'(y2, y1, y0) = y2 (267 y2 - 1642 y1 - 494 y0)
  //                  + y1 (2843 y1 + 1922 y0) + 547 y0^2
  const float2 u2 = fma2(X0, f2(-494.0f, -494.0f), fma2(X1, f2(-1642.0f, -1642.0f), mul2(X2, f2(267.0f, 267.0f))));
  const float2 u1 = fma2(X0, f2(1922.0f, 1922.0f), mul2(X1, f2(2843.0f, 2843.0f)));
  const float2 E12 = fma2(mul2(X0, f2(547.0f, 547.0f)), X0, fma2(X1, u1, fma2(X2, u2, f2(1e-10f, 1e-10f))));
  const float2 Q03 = mul2(E03, E03), Q12 = mul2(E12, E12);
  const float al0 = __fdividef(1.0f / 35.0f, Q03.x);
  const float al3 = __fdividef(4.0f / 35.0f, Q03.y);
  const float al1 = __fdividef(12.0f / 35.0f, Q12.x);
  const float al2 = __fdividef(18.0f / 35.0f, Q12.y);
  const float2 A03 = f2(al0, al3), A12 = f2(al1, al2);
  const float2 S = add2(A03, A12);
  const float inv = __fdividef(1.0f, S.x + S.y);
  const float2 acc = fma2(A12, P12, mul2(A03, P03));
  return (acc.x + acc.y) * inv;
}

// Face value from a stencil held in an array: ORDER 5 reads v[0..4]
// (upwind-positive: centre v[2]), ORDER 7 reads v[0..6] (centre v[3]).
// F32 selects the shifted mixed-precision evaluation described above.
template <int ORDER, bool F32>
__device__ __forceinline__ double weno_face(double a0, double a1, double a2, double a3, double a4,
                                            double a5 = 0.0, double a6 = 0.0) {
  if constexpr (ORDER == 5) {
    if constexpr (!F32) {
      return weno5<double>(a0, a1, a2, a3, a4);
    } else {
      const float r = weno5_c0((float)(a0 - a2), (float)(a1 - a2), (float)(a3 - a2), (float)(a4 - a2));
      return a2 + (double)r;
    }
  } else {
    if constexpr (!F32) {
      return weno7<double>(a0, a1, a2, a3, a4, a5, a6);
    } else {
      const float r = weno7_c0((float)(a0 - a3), (float)(a1 - a3), (float)(a2 - a3), (float)(a4 - a3),
                               (float)(a5 - a3), (float)(a6 - a3));
      return a3 + (double)r;
    }
  }
}

// Upwind face flux 0.5*((u+|u|)phi+ + (u-|u|)phi-)*rho
// (Csrc/scalar_advection.h:363 and momentum_advection_weno.h:172).
__device__ __forceinline__ double upwind_flux(double vel, double phip, double phim, double rho) {
  return 0.5 * ((vel + fabs(vel)) * phip + (vel - fabs(vel)) * phim) * rho;
}

// Upwind-only evaluation.  Of the reference's two biased interpolants one is
// always multiplied by an exact zero ((u-|u|) for u >= 0, (u+|u|) for
// u <= 0), so only the upwind one is computed: from a window v[0..W-1]
// (W = ORDER+1; the face lies between v[W/2-1] and v[W/2]) the stencil is
// v[0..ORDER-1] for u >= 0 and v[W-1..1] for u < 0, picked element by
// element so lanes of one warp that see both signs do not diverge.  With
// phi the upwind value,
//   0.5*((u+|u|)*phi + (u-|u|)*phi)*rho
// equals the reference's flux for every finite input (the zero term adds
// +-0), rounding included, so the FP64 form stays bit-identical.
template <int ORDER, bool F32>
__device__ __forceinline__ double weno_upwind(bool pos, const double* v) {
  constexpr int W = ORDER + 1;
  double st[ORDER];
#pragma unroll
  for (int m = 0; m < ORDER; ++m) st[m] = pos ? v[m] : v[W - 1 - m];
  if constexpr (ORDER == 5)
    return weno_face<5, F32>(st[0], st[1], st[2], st[3], st[4]);
  else
    return weno_face<7, F32>(st[0], st[1], st[2], st[3], st[4], st[5], st[6]);
}

// The precision form's upwind face value from first differences: d[m] =
// (float)(phi[f-R+2+m] - phi[f-R+1+m]), m = 0 .. 2R-2 (R = (ORDER+1)/2, so
// d[R-1] = phi[f+1] - phi[f]), each formed once per cell in FP64 and
// rounded once.  The stencil's differences from its centre are partial sums
// of d: for u >= 0 (centre phi[f]) phi[f-o] - phi[f] = -(d_{f-1} + ... +
// d_{f-o}) and phi[f+o] - phi[f] = d_f + ... + d_{f+o-1}; for u < 0 (centre
// phi[f+1], stencil mirrored) the same with the roles of the sides swapped.
// Returns r with face value = centre + r.
template <int ORDER>
__device__ __forceinline__ float weno_delta(bool pos, const float* d) {
  if constexpr (ORDER == 5) {  // d_{f+o} = d[2 + o]
    const float a1 = pos ? -d[1] : d[3];
    const float a2 = a1 + (pos ? -d[0] : d[4]);
    const float b1 = pos ? d[2] : -d[2];
    const float b2 = b1 + (pos ? d[3] : -d[1]);
    return weno5_c0(a2, a1, b1, b2);
  } else {                     // d_{f+o} = d[3 + o]
    const float a1 = pos ? -d[2] : d[4];
    const float a2 = a1 + (pos ? -d[1] : d[5]);
    const float a3 = a2 + (pos ? -d[0] : d[6]);
    const float b1 = pos ? d[3] : -d[3];
    const float b2 = b1 + (pos ? d[4] : -d[2]);
    const float b3 = b2 + (pos ? d[5] : -d[1]);
    return weno7_c0(a3, a2, a1, b1, b2, b3);
  }
}

__device__ __forceinline__ double upwind_flux1(double vel, double phi, double rho) {
  return 0.5 * ((vel + fabs(vel)) * phi + (vel - fabs(vel)) * phi) * rho;
}
