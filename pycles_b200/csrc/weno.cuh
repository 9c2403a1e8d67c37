// WENO and central interpolants, Csrc/advection_interpolation.h.
//
// The FP64 forms keep the reference's term order (the compiler may contract
// a*b+c into FMAs, which moves results by at most a few ulp).  The FP32
// forms are used by the precision path through weno5_mixed / weno7_mixed:
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

// The same WENO5/WENO7 interpolants with a single division.  The normalised
// weights w_k = (d_k/q_k) / sum_j (d_j/q_j), q_k = (beta_k + eps)^2, equal
// n_k / sum_j n_j with n_k = d_k * prod_{j != k} q_j, so one reciprocal of
// the sum replaces the reference's 4 (WENO5) or 5 (WENO7) divisions.  In
// FP64 the products stay far from the range limits (q >= 1e-20, and q <= 1e10
// for any physical jump), and the result differs from the reference's
// formula by rounding only.  Used by the FP64 form: FP64 division is a
// multi-instruction sequence, and the advection is FP64-pipe bound.
__device__ __forceinline__ double weno5_1div(double phim2, double phim1, double phi, double phip1, double phip2) {
  const double p0 = (1.0 / 3.0) * phim2 - (7.0 / 6.0) * phim1 + (11.0 / 6.0) * phi;
  const double p1 = (-1.0 / 6.0) * phim1 + (5.0 / 6.0) * phi + (1.0 / 3.0) * phip1;
  const double p2 = (1.0 / 3.0) * phi + (5.0 / 6.0) * phip1 - (1.0 / 6.0) * phip2;
  const double a2 = phi - 2.0 * phip1 + phip2;
  const double b2 = 3.0 * phi - 4.0 * phip1 + phip2;
  const double a1 = phim1 - 2.0 * phi + phip1;
  const double b1 = phim1 - phip1;
  const double a0 = phim2 - 2.0 * phim1 + phi;
  const double b0 = phim2 - 4.0 * phim1 + 3.0 * phi;
  const double e0 = (13.0 / 12.0) * a0 * a0 + 0.25 * b0 * b0 + 1e-10;
  const double e1 = (13.0 / 12.0) * a1 * a1 + 0.25 * b1 * b1 + 1e-10;
  const double e2 = (13.0 / 12.0) * a2 * a2 + 0.25 * b2 * b2 + 1e-10;
  const double q0 = e0 * e0, q1 = e1 * e1, q2 = e2 * e2;
  const double n0 = 0.1 * (q1 * q2);
  const double n1 = 0.6 * (q0 * q2);
  const double n2 = 0.3 * (q0 * q1);
  return (n0 * p0 + n1 * p1 + n2 * p2) / (n0 + n1 + n2);
}

// a*(c0 a + c1 b + c2 c + c3 d) + b*(c4 b + c5 c + c6 d) + c*(c7 c + c8 d) + c9 d d,
// every product and sum rounded separately, left to right, as the C source
// of advection_interpolation.h:116-131 evaluates it.
__device__ __forceinline__ double w7_beta(double a, double b, double c, double d, double c0, double c1, double c2,
                                          double c3, double c4, double c5, double c6, double c7, double c8,
                                          double c9) {
  const double i1 = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(c0, a), __dmul_rn(c1, b)), __dmul_rn(c2, c)),
                              __dmul_rn(c3, d));
  const double i2 = __dadd_rn(__dadd_rn(__dmul_rn(c4, b), __dmul_rn(c5, c)), __dmul_rn(c6, d));
  const double i3 = __dadd_rn(__dmul_rn(c7, c), __dmul_rn(c8, d));
  const double g4 = __dmul_rn(__dmul_rn(c9, d), d);
  return __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(a, i1), __dmul_rn(b, i2)), __dmul_rn(c, i3)), g4);
}

__device__ __forceinline__ double weno7_1div(double phim3, double phim2, double phim1, double phi, double phip1,
                                             double phip2, double phip3) {
  const double p0 = (-1.0 / 4.0) * phim3 + (13.0 / 12.0) * phim2 + (-23.0 / 12.0) * phim1 + (25.0 / 12.0) * phi;
  const double p1 = (1.0 / 12.0) * phim2 + (-5.0 / 12.0) * phim1 + (13.0 / 12.0) * phi + (1.0 / 4.0) * phip1;
  const double p2 = (-1.0 / 12.0) * phim1 + (7.0 / 12.0) * phi + (7.0 / 12.0) * phip1 + (-1.0 / 12.0) * phip2;
  const double p3 = (1.0 / 4.0) * phi + (13.0 / 12.0) * phip1 + (-5.0 / 12.0) * phip2 + (1.0 / 12.0) * phip3;
  // The WENO7 smoothness indicators are quadratic forms in the stencil
  // values themselves, whose terms (~1e4 phi^2) cancel down to (dphi)^2: a
  // contracted FMA moves beta by ~1e-10 relative, which reaches the weights.
  // They are therefore evaluated with the reference's separately rounded
  // operations in its order.
  const double beta0 = w7_beta(phim3, phim2, phim1, phi, 547.0, -3882.0, 4642.0, -1854.0, 7043.0, -17246.0, 7042.0,
                               11003.0, -9402.0, 2107.0);
  const double beta1 = w7_beta(phim2, phim1, phi, phip1, 267.0, -1642.0, 1602.0, -494.0, 2843.0, -5966.0, 1922.0,
                               3443.0, -2522.0, 547.0);
  const double beta2 = w7_beta(phim1, phi, phip1, phip2, 547.0, -2522.0, 1922.0, -494.0, 3443.0, -5966.0, 1602.0,
                               2843.0, -1642.0, 267.0);
  const double beta3 = w7_beta(phi, phip1, phip2, phip3, 2107.0, -9402.0, 7042.0, -1854.0, 11003.0, -17246.0,
                               4642.0, 7043.0, -3882.0, 547.0);
  const double e0 = beta0 + 1e-10, e1 = beta1 + 1e-10, e2 = beta2 + 1e-10, e3 = beta3 + 1e-10;
  const double q0 = e0 * e0, q1 = e1 * e1, q2 = e2 * e2, q3 = e3 * e3;
  const double q01 = q0 * q1, q23 = q2 * q3;
  const double n0 = (1.0 / 35.0) * (q1 * q23);
  const double n1 = (12.0 / 35.0) * (q0 * q23);
  const double n2 = (18.0 / 35.0) * (q3 * q01);
  const double n3 = (4.0 / 35.0) * (q2 * q01);
  return (n0 * p0 + n1 * p1 + n2 * p2 + n3 * p3) / (n0 + n1 + n2 + n3);
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

// Face value from a stencil held in an array: ORDER 5 reads v[0..4]
// (upwind-positive: centre v[2]), ORDER 7 reads v[0..6] (centre v[3]).
// F32 selects the shifted mixed-precision evaluation described above.
template <int ORDER, bool F32>
__device__ __forceinline__ double weno_face(double a0, double a1, double a2, double a3, double a4,
                                            double a5 = 0.0, double a6 = 0.0) {
  if constexpr (ORDER == 5) {
    if constexpr (!F32) {
      return weno5_1div(a0, a1, a2, a3, a4);
    } else {
      const float r = weno5<FastF>(FastF((float)(a0 - a2)), FastF((float)(a1 - a2)), FastF(0.0f),
                                   FastF((float)(a3 - a2)), FastF((float)(a4 - a2))).v;
      return a2 + (double)r;
    }
  } else {
    if constexpr (!F32) {
      return weno7_1div(a0, a1, a2, a3, a4, a5, a6);
    } else {
      const float r = weno7<FastF>(FastF((float)(a0 - a3)), FastF((float)(a1 - a3)), FastF((float)(a2 - a3)),
                                   FastF(0.0f), FastF((float)(a4 - a3)), FastF((float)(a5 - a3)),
                                   FastF((float)(a6 - a3))).v;
      return a3 + (double)r;
    }
  }
}

// Upwind face flux 0.5*((u+|u|)phi+ + (u-|u|)phi-)*rho
// (Csrc/scalar_advection.h:363 and momentum_advection_weno.h:172).
__device__ __forceinline__ double upwind_flux(double vel, double phip, double phim, double rho) {
  return 0.5 * ((vel + fabs(vel)) * phip + (vel - fabs(vel)) * phim) * rho;
}
