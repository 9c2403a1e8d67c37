// Surface fluxes of the lowest model level (Surface.pyx): the schemes
// SullivanPatton (dry, Monin-Obukhov friction velocity), Bomex (fixed
// friction velocity and fluxes) and DYCOMS_RF01 (bulk formulae), and the
// flux-to-tendency step they share, SurfaceBase.update (Surface.pyx:116-178).
//
// FP64 in both arithmetic forms: the work is one horizontal plane (nlg0*nlg1
// columns, about 1/nlg2 of a 3-D pass).  This translation unit is compiled
// with -fmad=false and uses correctly rounded log (crmath.cuh), so the
// fluxes follow the reference's separately rounded C; pow and atan are
// CUDA's (within an ulp of the C library's).
//
// Two kernels per update:
//   surface_columns : per column, compute_windspeed, the scheme's friction
//                     velocity and scalar fluxes, and a per-block partial
//                     sum of the interior temperature at k = gw;
//   surface_apply   : per column, the scheme's momentum fluxes (they read
//                     the neighbours' wind speed and friction velocity
//                     written by the first kernel), the horizontal mean of
//                     the lowest-level temperature from the partial sums (a
//                     fixed-order reduction, so every block gets the same
//                     value), and SurfaceBase.update.
#include <string.h>

#include "pb_common.cuh"
#include "crmath.cuh"

namespace {
namespace sfc {

using namespace pbc;

// generate_parameters.py:44-49 (Byun's surface-layer constants)
constexpr double vkb = 0.35;
constexpr double beta_m = 4.7;
constexpr double gamma_m = 15.0;

constexpr int kThreads = 512;  // one column per thread at 512 x 512 (latency-bound plane work)
constexpr int kMaxBlocks = PB_SURFACE_SCRATCH;

__device__ __forceinline__ double interp_2(double a, double b) { return 0.5 * (a + b); }
__device__ __forceinline__ double exner_c(double p0) { return pow(p0 / p_tilde, kappa); }
__device__ __forceinline__ double pd_c(double p0, double qt, double qv) {
  return p0 * (1.0 - qt) / (1.0 - qt + eps_vi * qv);
}
__device__ __forceinline__ double pv_c(double p0, double qt, double qv) {
  return p0 * eps_vi * qv / (1.0 - qt + eps_vi * qv);
}
__device__ __forceinline__ double cpm_c(double qt) { return (1.0 - qt) * cpd + qt * cpv; }
// Csrc/entropies.h:5-11
__device__ __forceinline__ double sd_c(double pd, double T) {
  return sd_tilde + cpd * crm::log(T / T_tilde) - Rd * crm::log(pd / p_tilde);
}
__device__ __forceinline__ double sv_c(double pv, double T) {
  return sv_tilde + cpv * crm::log(T / T_tilde) - Rv * crm::log(pv / p_tilde);
}
// latent_heat_variable with lambda_constant (Microphysics.pxd:65-75)
__device__ __forceinline__ double latent_heat(double T) {
  const double TC = T - 273.15;
  return (2500.8 - 2.36 * TC + 0.0016 * TC * TC - 0.00006 * TC * TC * TC) * 1000.0;
}

// psi_m_unstable / psi_m_stable (Csrc/surface.h:6-25)
__device__ __forceinline__ double psi_m_unstable(double zeta, double zeta0) {
  const double x = pow((1.0 - gamma_m * zeta), 0.25);
  const double x0 = pow((1.0 - gamma_m * zeta0), 0.25);
  return 2.0 * crm::log((1.0 + x) / (1.0 + x0)) + crm::log((1.0 + x * x) / (1.0 + x0 * x0)) - 2.0 * atan(x) +
         2.0 * atan(x0);
}
__device__ __forceinline__ double psi_m_stable(double zeta, double zeta0) { return -beta_m * (zeta - zeta0); }

// compute_ustar (Csrc/surface.h:34-93).  The reference returns `ustar`, set
// to the first fixed-point iterate ustar1 before its secant loop (:52, :73)
// and never updated inside it, or the neutral guess when the buoyancy flux
// vanishes (:89); the loop's iterates do not reach the result, so only that
// first iterate is computed.
__device__ double compute_ustar(double windspeed, double buoyancy_flux, double z0, double zb) {
  const double logz = crm::log(zb / z0);
  const double ustar0 = windspeed * vkb / logz;
  if (!(fabs(buoyancy_flux) > 1.0e-20)) return ustar0;
  const double lmo = -ustar0 * ustar0 * ustar0 / (buoyancy_flux * vkb);
  const double zeta = zb / lmo;
  const double zeta0 = z0 / lmo;
  const double psi = zeta >= 0.0 ? psi_m_stable(zeta, zeta0) : psi_m_unstable(zeta, zeta0);
  return windspeed * vkb / (logz - psi);
}

// entropyflux_from_thetaflux_qtflux (Csrc/surface.h:95-106)
__device__ __forceinline__ double entropyflux(double thetaflux, double qtflux, double p0_b, double T_b,
                                              double qt_b, double qv_b) {
  const double exner_b = exner_c(p0_b);
  const double pd_b = pd_c(p0_b, qt_b, qv_b);
  const double pv_b = pv_c(p0_b, qt_b, qv_b);
  const double sd_b = sd_c(pd_b, T_b);
  const double sv_b = sv_c(pv_b, T_b);
  const double cp_b = cpm_c(qt_b);
  return cp_b * thetaflux * exner_b / T_b + qtflux * (sv_b - sd_b);
}

struct Args {
  pb_surface sc;
  pb_surface_fields f;
  const double* p0_half;
  const double* alpha0;
  const double* alpha0_half;
  const double* rho0_half;
  const double* u;
  const double* v;
  const double* T;
  const double* qt;
  const double* qv;
  const double* ql;
  double* ut;
  double* vt;
  double* st;
  double* qtt;
  long long n0, n1;       // nlg[0], nlg[1]
  long long is, js, gw;   // strides and ghost width of the 3-D fields
  double dz;
  double inv_nxy;         // 1 / (n[1] * n[0]), HorizontalMean's n_horizontal_i
};

// Fixed-order block sum; the result is valid on thread 0.
__device__ __forceinline__ double block_sum(double x, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = x;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kThreads / 32; ++w) t += sh[w];
  return t;
}

template <int SCHEME>
__global__ void __launch_bounds__(kThreads) surface_columns(Args a) {
  __shared__ double sh[kThreads / 32];
  const long long ncol = a.n0 * a.n1;
  const long long gw = a.gw;
  double tsum = 0.0;
  // SullivanPatton's buoyancy flux (Surface.pyx:253-255): a Python-level
  // expression of the reference state, the same in every column
  double bflux = 0.0, sflux_num = 0.0;
  if (SCHEME == PB_SURFACE_SULLIVAN_PATTON) {
    const double T0 = a.p0_half[gw] * a.alpha0_half[gw] / Rd;
    bflux = a.sc.theta_flux * exner_c(a.p0_half[gw]) * g / T0;
    sflux_num = cpd * a.sc.theta_flux * exner_c(a.p0_half[gw]);
  }
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncol;
       c += (long long)gridDim.x * blockDim.x) {
    const long long i = c / a.n1, j = c - i * a.n1;
    const long long ijk = i * a.is + j * a.js + gw;
    const double T = a.T[ijk];
    if (i >= gw && i < a.n0 - gw && j >= gw && j < a.n1 - gw) tsum += T;
    // compute_windspeed (Csrc/surface.h:157-185) over i, j >= 1; the row and
    // column 0 keep 0 (SullivanPatton and Bomex pass a fresh zeroed array,
    // DYCOMS_RF01's persistent one is never written there)
    double ws = 0.0;
    if (i >= 1 && j >= 1) {
      const double ui = interp_2(a.u[ijk - a.is], a.u[ijk]) + a.sc.u0;
      const double vi = interp_2(a.v[ijk - a.js], a.v[ijk]) + a.sc.v0;
      ws = fmax(sqrt(ui * ui + vi * vi), a.sc.gustiness);
    }
    a.f.windspeed[c] = ws;
    if (SCHEME == PB_SURFACE_SULLIVAN_PATTON) {  // Surface.pyx:258-278
      a.f.s_flux[c] = sflux_num / T;
      if (i >= 1 && j >= 1) a.f.friction_velocity[c] = compute_ustar(ws, bflux, a.sc.z0, a.dz / 2.0);
    } else if (SCHEME == PB_SURFACE_BOMEX) {     // Surface.pyx:344-350
      a.f.friction_velocity[c] = a.sc.ustar;
      a.f.s_flux[c] = entropyflux(a.sc.theta_flux, a.f.qt_flux[c], a.p0_half[gw], T, a.qt[ijk], a.qv[ijk]);
    } else {                                     // DYCOMS_RF01, Surface.pyx:536-547
      if (i >= gw - 1 && i < a.n0 - gw + 1 && j >= gw - 1 && j < a.n1 - gw + 1) {
        a.f.friction_velocity[c] = sqrt(a.sc.cm) * ws;
        const double lv = latent_heat(T);
        const double qt = a.qt[ijk];
        const double qv = qt - a.ql[ijk];
        const double pv = pv_c(a.p0_half[gw], qt, qv);
        const double pd = pd_c(a.p0_half[gw], qt, qv);
        const double sv = sv_c(pv, T);
        const double sd = sd_c(pd, T);
        a.f.qt_flux[c] = a.sc.fq / lv / 1.22;
        a.f.s_flux[c] = a.alpha0_half[gw] * (a.sc.ft / T + a.sc.fq * (sv - sd) / lv);
      }
    }
  }
  const double t = block_sum(tsum, sh);
  if (threadIdx.x == 0) a.f.scratch[blockIdx.x] = t;
}

template <int SCHEME>
__global__ void __launch_bounds__(kThreads) surface_apply(Args a, int nparts) {
  __shared__ double sh[kThreads / 32];
  __shared__ double t_mean_sh;
  // HorizontalMean of the temperature at k = gw (ParallelMPI.pyx:196-241):
  // the sum of the per-block partials in block order, times 1/(n0 n1)
  {
    double x = 0.0;
    for (int p = threadIdx.x; p < nparts; p += kThreads) x += a.f.scratch[p];
    const double t = block_sum(x, sh);
    if (threadIdx.x == 0) t_mean_sh = t * a.inv_nxy;
    __syncthreads();
  }
  const double t_mean = t_mean_sh;
  const long long gw = a.gw;
  const long long ncol = a.n0 * a.n1;
  const long long s2 = a.n1;  // istride_2d
  const double tendency_factor = a.alpha0_half[gw] / a.alpha0[gw - 1] * (1.0 / a.dz);
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncol;
       c += (long long)gridDim.x * blockDim.x) {
    const long long i = c / a.n1, j = c - i * a.n1;
    const long long ijk = i * a.is + j * a.js + gw;
    // the scheme's momentum fluxes
    if (SCHEME == PB_SURFACE_DYCOMS_RF01) {  // Surface.pyx:548-553, interior columns
      if (i >= gw && i < a.n0 - gw && j >= gw && j < a.n1 - gw) {
        const double* ws = a.f.windspeed;
        a.f.u_flux[c] = -a.sc.cm * interp_2(ws[c], ws[c + s2]) * (a.u[ijk] + a.sc.u0);
        a.f.v_flux[c] = -a.sc.cm * interp_2(ws[c], ws[c + 1]) * (a.v[ijk] + a.sc.v0);
      }
    } else if (i >= 1 && i < a.n0 - 1 && j >= 1 && j < a.n1 - 1) {  // Surface.pyx:279-287, 360-366
      const double* ws = a.f.windspeed;
      if (SCHEME == PB_SURFACE_SULLIVAN_PATTON) {
        const double* fv = a.f.friction_velocity;
        const double su = interp_2(fv[c], fv[c + s2]);
        const double sv = interp_2(fv[c], fv[c + 1]);
        a.f.u_flux[c] = -(su * su) / interp_2(ws[c], ws[c + s2]) * (a.u[ijk] + a.sc.u0);
        a.f.v_flux[c] = -(sv * sv) / interp_2(ws[c], ws[c + 1]) * (a.v[ijk] + a.sc.v0);
      } else {
        const double us2 = a.sc.ustar * a.sc.ustar;
        a.f.u_flux[c] = -us2 / interp_2(ws[c], ws[c + s2]) * (a.u[ijk] + a.sc.u0);
        a.f.v_flux[c] = -us2 / interp_2(ws[c], ws[c + 1]) * (a.v[ijk] + a.sc.v0);
      }
    }
    // SurfaceBase.update over the interior columns (Surface.pyx:116-178)
    if (!(i >= gw && i < a.n0 - gw && j >= gw && j < a.n1 - gw)) continue;
    const double T = a.T[ijk];
    const double fv = a.f.friction_velocity[c];
    const double uf = a.f.u_flux[c], vf = a.f.v_flux[c], sf = a.f.s_flux[c];
    double b;
    if (SCHEME == PB_SURFACE_SULLIVAN_PATTON) {  // dry_case
      const double shf = sf * a.rho0_half[gw] * T;
      b = shf * g * a.alpha0_half[gw] / cpd / t_mean;
      a.f.shf[c] = shf;
    } else {
      const double lv = latent_heat(T);
      const double qtf = a.f.qt_flux[c];
      const double lhf = qtf * a.rho0_half[gw] * lv;
      const double qt = a.qt[ijk];
      const double qv = qt - a.ql[ijk];
      const double pv = pv_c(a.p0_half[gw], qt, qv);
      const double pd = pd_c(a.p0_half[gw], qt, qv);
      const double sv = sv_c(pv, T);
      const double sd = sd_c(pd, T);
      const double shf = (sf * a.rho0_half[gw] - lhf / lv * (sv - sd)) * T;
      const double cp_ = cpm_c(qt);
      b = g * a.alpha0_half[gw] / cp_ / t_mean * (shf + (eps_vi - 1.0) * cp_ * t_mean * lhf / lv);
      a.f.lhf[c] = lhf;
      a.f.shf[c] = shf;
      a.qtt[ijk] += qtf * tendency_factor;
    }
    a.f.b_flux[c] = b;
    a.f.obukhov_length[c] = -fv * fv * fv / b / vkb;
    a.ut[ijk] += uf * tendency_factor;
    a.vt[ijk] += vf * tendency_factor;
    a.st[ijk] += sf * tendency_factor;
  }
}

template <int SCHEME>
int launch(const Args& a, cudaStream_t st) {
  const long long ncol = a.n0 * a.n1;
  long long nb = (ncol + kThreads - 1) / kThreads;
  if (nb > kMaxBlocks) nb = kMaxBlocks;
  surface_columns<SCHEME><<<(int)nb, kThreads, 0, st>>>(a);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  surface_apply<SCHEME><<<(int)nb, kThreads, 0, st>>>(a, (int)nb);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

}  // namespace sfc
}  // namespace

extern "C" int pb_surface_update(const pb_dims* dims, const pb_surface* surface, const double* p0_half,
                                 const double* alpha0, const double* alpha0_half, const double* rho0_half,
                                 const double* u, const double* v, const double* T, const double* qt,
                                 const double* qv, const double* ql, double* u_tend, double* v_tend,
                                 double* s_tend, double* qt_tend, const pb_surface_fields* fields,
                                 void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!surface) return PB_ERR_ARG;
  const int scheme = surface->scheme;
  if (scheme == PB_SURFACE_NONE) return PB_OK;
  if (scheme != PB_SURFACE_SULLIVAN_PATTON && scheme != PB_SURFACE_BOMEX && scheme != PB_SURFACE_DYCOMS_RF01)
    return PB_ERR_ARG;
  if (!fields || !p0_half || !alpha0 || !alpha0_half || !rho0_half || !u || !v || !T || !u_tend || !v_tend ||
      !s_tend)
    return PB_ERR_ARG;
  const pb_surface_fields& f = *fields;
  if (!f.u_flux || !f.v_flux || !f.qt_flux || !f.s_flux || !f.obukhov_length || !f.friction_velocity || !f.shf ||
      !f.lhf || !f.b_flux || !f.windspeed || !f.scratch)
    return PB_ERR_ARG;
  const bool moist = scheme != PB_SURFACE_SULLIVAN_PATTON;
  if (moist && (!qt || !ql || !qt_tend || (scheme == PB_SURFACE_BOMEX && !qv))) return PB_ERR_ARG;
  sfc::Args a;
  memset(&a, 0, sizeof(a));
  a.sc = *surface;
  a.f = f;
  a.p0_half = p0_half;
  a.alpha0 = alpha0;
  a.alpha0_half = alpha0_half;
  a.rho0_half = rho0_half;
  a.u = u;
  a.v = v;
  a.T = T;
  a.qt = qt;
  a.qv = qv;
  a.ql = ql;
  a.ut = u_tend;
  a.vt = v_tend;
  a.st = s_tend;
  a.qtt = qt_tend;
  a.n0 = dims->nlg[0];
  a.n1 = dims->nlg[1];
  a.is = (long long)dims->nlg[1] * dims->nlg[2];
  a.js = dims->nlg[2];
  a.gw = dims->gw;
  a.dz = dims->dx[2];
  a.inv_nxy = 1.0 / (double)(dims->n[1] * dims->n[0]);
  cudaStream_t st = as_stream(stream);
  if (scheme == PB_SURFACE_SULLIVAN_PATTON) return sfc::launch<PB_SURFACE_SULLIVAN_PATTON>(a, st);
  if (scheme == PB_SURFACE_BOMEX) return sfc::launch<PB_SURFACE_BOMEX>(a, st);
  return sfc::launch<PB_SURFACE_DYCOMS_RF01>(a, st);
}
