// Correctly rounded exp and log for the FP64 plain form.
//
// Why: the reference evaluates exp/log with the C library, whose results are
// the correctly rounded ones in all but extremely rare cases.  In the
// saturation adjustment and the dry equation of state a one-ulp difference
// in the temperature reaches the buoyancy, g (alpha - alpha0)/alpha0, which
// cancels three to four digits, and from there w and the pressure-driven
// velocities: with 1-ulp-accurate device exp/log those fields differ from
// the reference by ~1e-12 relative after one step.  Evaluating exp and log
// to ~2^-100 in double-double arithmetic and rounding once reproduces the
// correctly rounded result except for inputs within ~2^-47 ulp of a
// rounding boundary.
//
// Methods (table-driven, after P. T. P. Tang, "Table-driven implementation
// of the exponential function in IEEE floating-point arithmetic", ACM TOMS
// 15 (1989), and "Table-driven implementation of the logarithm function",
// ACM TOMS 16 (1990)), with double-double arithmetic (Dekker's and Knuth's
// error-free transformations):
//   exp(x) = 2^m * 2^(j/128) * exp(r),  x = (128 m + j) ln2/128 + r,
//            |r| <= ln2/256, exp(r) by its Taylor series;
//   log(x) = e ln2 + ln(c_j) + log1p(v),  x = 2^e m, c_j = 1 + j/256 <= m,
//            v = (m - c_j)/c_j < 2^-8, log1p(v) by its Taylor series.
// Tables: crmath_tables.cuh (generated at 60 digits by gen_crmath_tables.py).
// Arguments outside the normal range go to the CUDA library function.
#pragma once

#include "crmath_tables.cuh"

namespace crm {

struct dd {
  double hi, lo;
};

__device__ __forceinline__ dd two_sum(double a, double b) {
  const double s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  const double e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
  return {s, e};
}

__device__ __forceinline__ dd fast_two_sum(double a, double b) {  // |a| >= |b|
  const double s = __dadd_rn(a, b);
  const double e = __dsub_rn(b, __dsub_rn(s, a));
  return {s, e};
}

__device__ __forceinline__ dd two_prod(double a, double b) {
  const double p = __dmul_rn(a, b);
  const double e = fma(a, b, -p);
  return {p, e};
}

__device__ __forceinline__ double exp(double x) {
  if (!(fabs(x) < 700.0)) return ::exp(x);
  const double kd = rint(x * CRM_INV_L);
  const int k = (int)kd;
  // r = x - k*ln2/128 in double-double (k*L1 exact, Sterbenz for the subtraction)
  const double t1 = fma(-kd, CRM_L1, x);
  const dd p2 = two_prod(kd, CRM_L2);
  dd r = two_sum(t1, -p2.hi);
  r.lo = __dsub_rn(__dsub_rn(r.lo, p2.lo), __dmul_rn(kd, CRM_L3));
  r = fast_two_sum(r.hi, r.lo);
  // exp(r) - 1 = r + r^2/2 + r^3 (1/6 + r/24 + r^2/120 + r^3/720)
  const double rh = r.hi;
  const double tail = rh * rh * rh * (1.0 / 6.0 + rh * (1.0 / 24.0 + rh * (1.0 / 120.0 + rh * (1.0 / 720.0))));
  const dd sq = two_prod(rh, rh);
  const double half_hi = 0.5 * sq.hi;  // exact
  dd p = two_sum(rh, half_hi);
  p.lo = __dadd_rn(p.lo, __dadd_rn(__dadd_rn(r.lo, 0.5 * sq.lo), __dadd_rn(__dmul_rn(rh, r.lo), tail)));
  p = fast_two_sum(p.hi, p.lo);
  // T * (1 + p), T = 2^(j/128) as double-double
  const int j = k & 127;
  const int m = (k - j) >> 7;
  const double Th = __ldg(CRM_EXP2_TAB + 2 * j);
  const double Tl = __ldg(CRM_EXP2_TAB + 2 * j + 1);
  const dd a = two_prod(Th, p.hi);
  const double lo = __dadd_rn(__dadd_rn(a.lo, __dmul_rn(Th, p.lo)), __dadd_rn(Tl, __dmul_rn(Tl, p.hi)));
  dd b = two_sum(Th, a.hi);
  const double res = __dadd_rn(b.hi, __dadd_rn(b.lo, lo));
  if (m < -1021 || m > 1022) return ::exp(x);
  return res * __longlong_as_double((long long)(m + 1023) << 52);
}

__device__ __forceinline__ double log(double x) {
  const long long bits = __double_as_longlong(x);
  const int be = (int)((bits >> 52) & 0x7ff);
  if (!(x > 0.0) || be == 0 || be == 0x7ff) return ::log(x);
  const int e = be - 1023;
  const long long mbits = bits & 0x000fffffffffffffLL;
  const double mm = __longlong_as_double(mbits | 0x3ff0000000000000LL);  // [1, 2)
  const int j = (int)(mbits >> 44);                                        // top 8 bits
  const double c = 1.0 + (double)j * (1.0 / 256.0);
  const double f = __dsub_rn(mm, c);  // exact
  // v = f/c to ~2^-105 without a division: vh = f*(1/c) is off by at most a
  // few ulp, the remainder f - vh*c is exact (FMA), and its quotient by c
  // needs only a relative accuracy of 2^-50
  const double rc = __ldg(CRM_INVC_TAB + j);
  const double vh0 = __dmul_rn(f, rc);
  const double vl0 = __dmul_rn(fma(-vh0, c, f), rc);
  const dd v = fast_two_sum(vh0, vl0);
  const double vh = v.hi;
  const double vl = v.lo;
  // log1p(v) = v - v^2/2 + v^3 (1/3 - v/4 + v^2/5 - v^3/6 + v^4/7 - v^5/8 + v^6/9)
  const double tail =
      vh * vh * vh *
      (1.0 / 3.0 + vh * (-0.25 + vh * (0.2 + vh * (-1.0 / 6.0 + vh * (1.0 / 7.0 + vh * (-0.125 + vh * (1.0 / 9.0)))))));
  const dd sq = two_prod(vh, vh);
  dd l = two_sum(vh, -0.5 * sq.hi);
  l.lo = __dadd_rn(l.lo, __dadd_rn(__dsub_rn(vl, 0.5 * sq.lo), __dsub_rn(tail, __dmul_rn(vh, vl))));
  // e ln2 + ln(c_j) + log1p(v)
  const double ed = (double)e;
  const double ch = __ldg(CRM_LOGC_TAB + 2 * j);
  const double cl = __ldg(CRM_LOGC_TAB + 2 * j + 1);
  const dd s1 = two_sum(ed * CRM_LN2_HI, ch);  // ed * LN2_HI exact
  const dd s2 = two_sum(s1.hi, l.hi);
  const double lo = __dadd_rn(__dadd_rn(s1.lo, s2.lo), __dadd_rn(__dadd_rn(ed * CRM_LN2_LO, cl), l.lo));
  return __dadd_rn(s2.hi, lo);
}

}  // namespace crm
