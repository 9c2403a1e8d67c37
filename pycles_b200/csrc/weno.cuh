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
__device__ __forceinline__ float weno5_c0(float a2, float a1, float b1, float b2) {
  const float p0 = (1.0f / 3.0f) * a2 - (7.0f / 6.0f) * a1;
  const float p1 = (-1.0f / 6.0f) * a1 + (1.0f / 3.0f) * b1;
  const float p2 = (5.0f / 6.0f) * b1 - (1.0f / 6.0f) * b2;
  const float s2a = b2 - 2.0f * b1, s2b = b2 - 4.0f * b1;
  const float s1a = a1 + b1, s1b = a1 - b1;
  const float s0a = a2 - 2.0f * a1, s0b = a2 - 4.0f * a1;
  const float e0 = (13.0f / 12.0f) * s0a * s0a + 0.25f * s0b * s0b + 1e-10f;
  const float e1 = (13.0f / 12.0f) * s1a * s1a + 0.25f * s1b * s1b + 1e-10f;
  const float e2 = (13.0f / 12.0f) * s2a * s2a + 0.25f * s2b * s2b + 1e-10f;
  const float al0 = __fdividef(0.1f, e0 * e0);
  const float al1 = __fdividef(0.6f, e1 * e1);
  const float al2 = __fdividef(0.3f, e2 * e2);
  const float inv = __fdividef(1.0f, al0 + al1 + al2);
  return (al0 * inv) * p0 + (al1 * inv) * p1 + (al2 * inv) * p2;
}

__device__ __forceinline__ float weno7_c0(float a3, float a2, float a1, float b1, float b2, float b3) {
  const float p0 = -0.25f * a3 + (13.0f / 12.0f) * a2 + (-23.0f / 12.0f) * a1;
  const float p1 = (1.0f / 12.0f) * a2 + (-5.0f / 12.0f) * a1 + 0.25f * b1;
  const float p2 = (-1.0f / 12.0f) * a1 + (7.0f / 12.0f) * b1 + (-1.0f / 12.0f) * b2;
  const float p3 = (13.0f / 12.0f) * b1 + (-5.0f / 12.0f) * b2 + (1.0f / 12.0f) * b3;
  const float be0 = a3 * (547.0f * a3 - 3882.0f * a2 + 4642.0f * a1) + a2 * (7043.0f * a2 - 17246.0f * a1) +
                    11003.0f * a1 * a1;
  const float be1 = a2 * (267.0f * a2 - 1642.0f * a1 - 494.0f * b1) + a1 * (2843.0f * a1 + 1922.0f * b1) +
                    547.0f * b1 * b1;
  const float be2 = a1 * (547.0f * a1 + 1922.0f * b1 - 494.0f * b2) + b1 * (2843.0f * b1 - 1642.0f * b2) +
                    267.0f * b2 * b2;
  const float be3 = b1 * (11003.0f * b1 - 17246.0f * b2 + 4642.0f * b3) + b2 * (7043.0f * b2 - 3882.0f * b3) +
                    547.0f * b3 * b3;
  const float e0 = be0 + 1e-10f, e1 = be1 + 1e-10f, e2 = be2 + 1e-10f, e3 = be3 + 1e-10f;
  const float al0 = __fdividef(1.0f / 35.0f, e0 * e0);
  const float al1 = __fdividef(12.0f / 35.0f, e1 * e1);
  const float al2 = __fdividef(18.0f / 35.0f, e2 * e2);
  const float al3 = __fdividef(4.0f / 35.0f, e3 * e3);
  const float inv = __fdividef(1.0f, al0 + al1 + al2 + al3);
  return (al0 * inv) * p0 + (al1 * inv) * p1 + (al2 * inv) * p2 + (al3 * inv) * p3;
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

__device__ __forceinline__ double upwind_flux1(double vel, double phi, double rho) {
  return 0.5 * ((vel + fabs(vel)) * phi + (vel - fabs(vel)) * phi) * rho;
}
