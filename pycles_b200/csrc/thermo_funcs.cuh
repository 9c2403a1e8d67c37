// Thermodynamic functions of the saturation adjustment, templated on the
// exp/log implementation M:
//   * ExactMath (crmath.cuh, correctly rounded) for the FP64 plain form,
//     instantiated only in thermo.cu, compiled with -fmad=false so the
//     temperature follows the reference's separately rounded C arithmetic;
//   * FastMath (CUDA's exp/log, FMA contraction on) for the precision form,
//     instantiated only in thermo_fast.cu and mlp.cu.
// Everything here has internal linkage: each translation unit gets its own
// copy compiled with its own flags.
#pragma once

#include "pb_common.cuh"

namespace {
namespace thermo_f {

using namespace pbc;

struct FastMath {
  static constexpr bool exact = false;  // free to reorder the reference's expressions
  static __device__ __forceinline__ double exp(double x) { return ::exp(x); }
  static __device__ __forceinline__ double log(double x) { return ::log(x); }
};

// ---- Csrc/thermodynamic_functions.h, Csrc/entropies.h
__device__ __forceinline__ double pd_c(double p0, double qt, double qv) {
  return p0 * (1.0 - qt) / (1.0 - qt + eps_vi * qv);
}
__device__ __forceinline__ double pv_c(double p0, double qt, double qv) {
  return p0 * eps_vi * qv / (1.0 - qt + eps_vi * qv);
}
__device__ __forceinline__ double qv_star_c(double p0, double qt, double pv) {
  return eps_v * (1.0 - qt) * pv / (p0 - pv);
}
// alpha and buoyancy: buoyancy cancels ~3 digits of alpha, so both keep the
// reference's separately rounded operations in either form.
__device__ __forceinline__ double alpha_c(double p0, double T, double qt, double qv) {
  return mul_rn((Rd * T) / p0, add_rn(sub_rn(1.0, qt), mul_rn(eps_vi, qv)));
}
__device__ __forceinline__ double buoyancy_c(double alpha0, double alpha) {
  return mul_rn(g, sub_rn(alpha, alpha0)) / alpha0;
}
__device__ __forceinline__ double cpm_c(double qt) { return (1.0 - qt) * cpd + qt * cpv; }
template <class M>
__device__ __forceinline__ double sd_c(double pd, double T) {
  return sd_tilde + cpd * M::log(T / T_tilde) - Rd * M::log(pd / p_tilde);
}
template <class M>
__device__ __forceinline__ double sv_c(double pv, double T) {
  return sv_tilde + cpv * M::log(T / T_tilde) - Rv * M::log(pv / p_tilde);
}
__device__ __forceinline__ double sc_c(double L, double T) { return -L / T; }
__device__ __forceinline__ double interp_2(double a, double b) { return 0.5 * (a + b); }

// latent_heat_variable with lambda_constant (Microphysics.pxd:65-75)
__device__ __forceinline__ double latent_heat(double T) {
  const double TC = T - 273.15;
  return (2500.8 - 2.36 * TC + 0.0016 * TC * TC - 0.00006 * TC * TC * TC) * 1000.0;
}

// lookup (Csrc/lookup.h:48-54) with a range check the reference lacks:
// out-of-table arguments flag PB_ERR_TABLE_RANGE and are clamped.
__device__ __forceinline__ double table_lookup(const pb_table& t, double x, unsigned int* err) {
  const double fi = floor((x - t.x_min) * t.dxi);
  long long indx;
  if (!(fi >= 0.0 && fi <= (double)(t.n - 2))) {
    pb_flag_at(err, PB_ERR_TABLE_RANGE);
    indx = (fi >= 0.0) ? t.n - 2 : 0;
  } else {
    indx = (long long)fi;
  }
  const double y1 = __ldg(t.y + indx);
  const double y2 = __ldg(t.y + indx + 1);
  const double x1 = t.x_min + t.dx * indx;
  return y1 + (x - x1) * (y2 - y1) * t.dxi;
}

// temperature_no_ql (Csrc/thermodynamics_sa.h:10-15).  The precision form
// multiplies by 1/p_tilde instead of dividing (FP64 division is a
// multi-instruction sequence).
template <class M>
__device__ __forceinline__ double temperature_no_ql(double pd, double pv, double s, double qt) {
  if constexpr (M::exact) {
    return T_tilde * M::exp((s - (1.0 - qt) * (sd_tilde - Rd * M::log(pd / p_tilde)) -
                             qt * (sv_tilde - Rv * M::log(pv / p_tilde))) /
                            ((1.0 - qt) * cpd + qt * cpv));
  } else {
    constexpr double ipt = 1.0 / p_tilde;
    return T_tilde * M::exp((s - (1.0 - qt) * (sd_tilde - Rd * M::log(pd * ipt)) -
                             qt * (sv_tilde - Rv * M::log(pv * ipt))) /
                            ((1.0 - qt) * cpd + qt * cpv));
  }
}

// Entropy of the saturated mixture at temperature T (the secant's s_1, s_2,
// Csrc/thermodynamics_sa.h:37,54): the reference's operations in the plain
// form; the precision form evaluates log(T/T_tilde) once for the dry and the
// vapour parts and multiplies by the constant reciprocals (three logarithms
// per secant iteration instead of four).
template <class M>
__device__ __forceinline__ double entropy_sat(double pd, double pv, double T, double qt, double L, double sigma) {
  if constexpr (M::exact) {
    return sd_c<M>(pd, T) * (1.0 - qt) + sv_c<M>(pv, T) * qt + sc_c(L, T) * sigma;
  } else {
    constexpr double ipt = 1.0 / p_tilde, iTt = 1.0 / T_tilde;
    const double lT = M::log(T * iTt);
    const double sd = sd_tilde + cpd * lT - Rd * M::log(pd * ipt);
    const double sv = sv_tilde + cpv * lT - Rv * M::log(pv * ipt);
    return sd * (1.0 - qt) + sv * qt + sc_c(L, T) * sigma;
  }
}

// The secant's first point (Csrc/thermodynamics_sa.h:22-24): the temperature
// with all water as vapour.  The learned seed is a correction to it.
template <class M>
__device__ __forceinline__ double first_point(double p0, double s, double qt) {
  const double pv_1 = pv_c(p0, qt, qt);
  const double pd_1 = p0 - pv_1;
  return temperature_no_ql<M>(pd_1, pv_1, s, qt);
}

struct EosOut {
  double T, qv, ql, qi;
  int iters;
  bool sat;
};

// eos_c (Csrc/thermodynamics_sa.h:17-66) in two parts, so that a caller can
// evaluate learned seeds for the saturated cells between them.
struct EosStart {
  double pd_1, pv_1, T_1, qv_star_1;
  bool sat;
};

template <class M>
__device__ __forceinline__ EosStart eos_start(const pb_table& LT, double p0, double s, double qt,
                                              unsigned int* err) {
  EosStart e;
  e.pv_1 = pv_c(p0, qt, qt);
  e.pd_1 = p0 - e.pv_1;
  e.T_1 = temperature_no_ql<M>(e.pd_1, e.pv_1, s, qt);
  const double pv_star_1 = table_lookup(LT, e.T_1, err);
  e.qv_star_1 = qv_star_c(p0, qt, pv_star_1);
  e.sat = !(qt <= e.qv_star_1);
  return e;
}

// The saturated branch (:33-64).  The secant loop is the reference's; it is
// capped at max_iter (the reference loops without a cap), reaching the cap
// sets PB_ERR_SECANT_CAP.  use_seed replaces the second secant point T_2
// (:39) by a learned guess; the loop and its stopping test stay the
// reference's.  The root lies between T_1 (no condensate) and the
// reference's T_2 (all of sigma_1 condensed at T_1's latent heat) -- over
// saturated states at 700-1020 hPa it sits at 0.20-0.87 of that interval --
// so the guess is clamped to [T_1 + (T_2 - T_1)/16, T_2]: a good guess is
// untouched, a wild one (or NaN) cannot take the secant off the saturation
// table, and T_2 != T_1 keeps the first secant step defined.
//
// The reference returns T from the loop's last update but qv and ql from the
// point before it (:44-63), whose distance from the root is up to the
// stopping tolerance (1e-3 K).  A seeded secant reaches the root by another
// path, so that point's error would differ from the plain secant's and act
// as a perturbation of the buoyancy in every seeded cloudy cell.  A seeded
// cell therefore takes qv and ql at the returned T: qv* is extrapolated from
// its last two evaluations (the secant step's own ratio, in FP32; the
// curvature term is ~1e-7 of qv*, far below the ~1e-3 K error it removes),
// so no table lookup or entropy evaluation is added.  T, qv and ql then
// agree with each other, and the difference left to the plain secant is the
// plain secant's own.  Measured over 1000 steps of the precision form
// against the FP64 plain form, u relative to its norm on a 32x32x32
// cloud-topped grid: 2.2e-6 with qv* looked up at the returned T, against
// 2.5e-5 with the reference's values (2.0e-4 at 512x512x256).  A point where
// the extrapolated saturation deficit falls outside [0, qt] keeps the
// reference's values.
template <class M>
__device__ __forceinline__ EosOut eos_finish(const pb_table& LT, const EosStart& e, double p0, double s, double qt,
                                             int max_iter, bool use_seed, double seed, unsigned int* err) {
  EosOut o;
  o.qv = qt;
  o.ql = 0.0;
  o.qi = 0.0;
  o.iters = 0;
  double T_1 = e.T_1;
  if (!e.sat) {
    o.T = T_1;
    o.sat = false;
    return o;
  }
  o.sat = true;
  const double sigma_1 = qt - e.qv_star_1;
  const double L_1 = latent_heat(T_1);
  const double s_1 = entropy_sat<M>(e.pd_1, e.pv_1, T_1, qt, L_1, sigma_1);
  double f_1 = s - s_1;
  double T_2 = T_1 + sigma_1 * L_1 / ((1.0 - qt) * cpd + e.qv_star_1 * cpv);
  if (use_seed) T_2 = fmin(fmax(seed, T_1 + 0.0625 * (T_2 - T_1)), T_2);
  double delta_T;
  double qv_star_2, sigma_2;
  double qv_1 = e.qv_star_1;            // qv* at T_1
  double T_p = T_1, qv_p = qv_1;        // the point before T_1
  int it = 0;
  do {
    const double pv_star_2 = table_lookup(LT, T_2, err);
    qv_star_2 = qv_star_c(p0, qt, pv_star_2);
    const double pv_2 = pv_c(p0, qt, qv_star_2);
    const double pd_2 = p0 - pv_2;
    sigma_2 = qt - qv_star_2;
    const double L_2 = latent_heat(T_2);
    const double s_2 = entropy_sat<M>(pd_2, pv_2, T_2, qt, L_2, sigma_2);
    const double f_2 = s - s_2;
    const double T_n = T_2 - f_2 * (T_2 - T_1) / (f_2 - f_1);
    T_p = T_1;
    qv_p = qv_1;
    T_1 = T_2;
    qv_1 = qv_star_2;
    T_2 = T_n;
    f_1 = f_2;
    delta_T = fabs(T_2 - T_1);
    ++it;
    if (it >= max_iter) {
      if (delta_T >= 1.0e-3 || sigma_2 < 0.0) pb_flag_at(err, PB_ERR_SECANT_CAP);
      break;
    }
  } while (delta_T >= 1.0e-3 || sigma_2 < 0.0);
  o.T = T_2;
  if (use_seed) {
    // T_1: where qv_star_2 was evaluated; T_p: the evaluation before it
    const float lam = __fdividef((float)(T_2 - T_1), (float)(T_1 - T_p));
    const double qv_star_f = qv_star_2 + (qv_star_2 - qv_p) * (double)lam;
    const double sigma_f = qt - qv_star_f;
    if (sigma_f >= 0.0 && sigma_f <= qt) {
      qv_star_2 = qv_star_f;
      sigma_2 = sigma_f;
    }
  }
  o.qv = qv_star_2;
  o.ql = 1.0 * sigma_2;  // lambda = 1
  o.qi = (1.0 - 1.0) * sigma_2;
  o.iters = it;
  return o;
}

template <class M>
__device__ __forceinline__ EosOut eos_sa(const pb_table& LT, double p0, double s, double qt, int max_iter,
                                         bool use_seed, double seed, unsigned int* err) {
  const EosStart e = eos_start<M>(LT, p0, s, qt, err);
  return eos_finish<M>(LT, e, p0, s, qt, max_iter, use_seed, seed, err);
}

}  // namespace thermo_f
}  // namespace
