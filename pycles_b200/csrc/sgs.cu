// Subgrid scale: kinematics (strain-rate magnitude), the eddy viscosity and
// diffusivity (UniformViscosity, Smagorinsky), and the diffusion of the
// scalars and of momentum (Kinematics.pyx, SGS.pyx, ScalarDiffusion.pyx,
// MomentumDiffusion.pyx with Csrc/kinematics.h, sgs.h, scalar_diffusion.h,
// momentum_diffusion.h).
//
// The reference materialises nine velocity-gradient and nine strain-rate
// arrays and one flux array per (component, direction); here every gradient,
// strain-rate component and face flux is formed in registers from the
// velocity / scalar / viscosity stencil where it is consumed, so each kernel
// reads its fields once from HBM (neighbours come from L1/L2) and writes
// only its results:
//   kinematics_sgs      : strain-rate magnitude (kept: the momentum
//                         diffusion's entropy source reads it) and the
//                         viscosity and diffusivity, over all cells;
//   scalar_diffusion    : per interior cell and scalar, the three
//                         directions' face fluxes and their divergence
//                         (+ the qt-diffusion entropy source);
//   momentum_diffusion  : per interior cell, the nine stress fluxes, their
//                         divergence into u, v, w, and the entropy source.
// FP64 in both arithmetic forms (stencils of width 2: bound by memory, not
// arithmetic).  Compiled with -fmad=false and correctly rounded log so every
// value follows the reference's separately rounded C.
#include <math.h>
#include <string.h>

#include "pb_common.cuh"
#include "crmath.cuh"

namespace {
namespace sgsk {

using namespace pbc;

constexpr double vkb = 0.35;  // generate_parameters.py:44
constexpr int kThreads = 128;
constexpr int kMaxScalars = 8;

struct G {
  int n0, n1, n2;  // nlg
  long long is, js;
  int gw;
  double dxi[3];   // DimStruct.dxi (1/dx)
};

__device__ __forceinline__ long long stride_of(const G& g, int d) { return d == 0 ? g.is : (d == 1 ? g.js : 1); }

// velocity gradient dv_a/dx_b at flat index p (Csrc/kinematics.h:6-34)
__device__ __forceinline__ double vgrad(const G& g, const double* const* V, int a, int b, long long p) {
  return (__ldg(V[a] + p + stride_of(g, b)) - __ldg(V[a] + p)) * g.dxi[b];
}
// strain-rate component S_ab at p (Csrc/kinematics.h:37-69)
__device__ __forceinline__ double strain(const G& g, const double* const* V, int a, int b, long long p) {
  return 0.5 * (vgrad(g, V, a, b, p) + vgrad(g, V, b, a, p));
}

struct KArgs {
  G g;
  const double* V[3];
  const double* bvf;
  const double* zl_half;
  double* smag;
  double* visc;
  double* diff;
  int scheme;  // pb_sgs_scheme
  int length;  // pb_sgs_length
  double cs, prt, delta, const_visc, const_diff;
};

// Kinematics.update + SGS.update for one cell.  The strain-rate magnitude
// (Csrc/kinematics.h:72-131) is 0 outside [1, nlg-1)^3; inside, the
// diagonal components at ijk - s_d, then twice the square of the average
// of S over four cells for the pairs (0,0), (0,1), (0,2), (1,1), (1,2) --
// the pairs the reference's loops visit -- and sqrt(2 sum).  For a pair
// (a, a) the fourth cell is two cells back along a: from the plane a = 1
// the reference's flat index leaves the computed strain field (a wrap into
// the previous row for a = y, where the strain rate is never computed: 0;
// before the array for a = x), and 0 is used; with gw >= 3 no interior
// tendency reads the viscosity of those ghost planes.
template <int SCHEME, int LENGTH>
__global__ void __launch_bounds__(kThreads) kinematics_sgs(KArgs a) {
  const G& g = a.g;
  const int k = blockIdx.x * kThreads + threadIdx.x;
  const int j = blockIdx.y, i = blockIdx.z;
  if (k >= g.n2) return;
  const long long ijk = (long long)i * g.is + (long long)j * g.js + k;
  double m = 0.0;
  if (i >= 1 && i < g.n0 - 1 && j >= 1 && j < g.n1 - 1 && k >= 1 && k < g.n2 - 1) {
    const int c[3] = {i, j, k};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double t = strain(g, a.V, d, d, ijk - stride_of(g, d));
      m += t * t;
    }
#pragma unroll
    for (int v1 = 0; v1 < 2; ++v1) {
#pragma unroll
      for (int d = v1; d < 3; ++d) {
        const long long s1 = stride_of(g, v1), sd = stride_of(g, d);
        const double p1 = strain(g, a.V, v1, d, ijk);
        const double p2 = strain(g, a.V, v1, d, ijk - s1);
        const double p3 = strain(g, a.V, v1, d, ijk - sd);
        const double p4 = (v1 == d && c[v1] == 1) ? 0.0 : strain(g, a.V, v1, d, ijk - sd - s1);
        const double si = 0.25 * (p1 + p2 + p3 + p4);
        m += 2.0 * si * si;
      }
    }
  }
  const double S = sqrt(2.0 * m);
  a.smag[ijk] = S;
  if (SCHEME == 0) return;  // Kinematics.update alone
  if (SCHEME == PB_SGS_UNIFORM) {  // SGS.pyx:84-90
    a.visc[ijk] = a.const_visc;
    a.diff[ijk] = a.const_diff;
    return;
  }
  // Csrc/sgs.h:4-18 (grid length), :21-54 (wall), :56-89 (ILES)
  double nu;
  if (LENGTH == PB_SGS_LENGTH_GRID) {
    nu = a.cs * a.cs * a.delta * a.delta * S;
  } else {
    const double z = a.zl_half[k];
    const double ell = LENGTH == PB_SGS_LENGTH_WALL ? a.delta * vkb * (z) / (a.delta + vkb * (z))
                                                    : fmax(0.0, a.delta - vkb * z);
    nu = a.cs * a.cs * ell * ell * S;
  }
  const double n2 = a.bvf[ijk];
  if (n2 > 0.0) {
    const double fb = sqrt(fmax(1.0 - n2 / (a.prt * S * S), 0.0));
    nu = nu * fb;
  }
  a.visc[ijk] = nu;
  a.diff[ijk] = nu / a.prt;
}

struct SArgs {
  G g;
  const double* rho0;
  const double* rho0_half;
  const double* alpha0_half;
  const double* p0_half;
  const double* D;
  const double* qv;
  const double* T;
  int ns;
  const double* phi[kMaxScalars];
  double* tend[kMaxScalars];
  double factor[kMaxScalars];
  double dxi_div[3];  // 1/dx as second_order_diffusion forms it
  int qt_index;       // scalar whose diffusion feeds the entropy source, -1: none
  int s_index;
};

// second_order_diffusion (Csrc/scalar_diffusion.h:6-57) at face p along d:
// written over [gw-1, nlg-gw) in every dimension and 0 on the level
// k = gw-1; the flux array is 0 elsewhere (never written).
__device__ __forceinline__ double sflux(const SArgs& a, const double* phi, double factor, int d, long long p,
                                        int pi, int pj, int pk) {
  const G& g = a.g;
  const int lo = g.gw - 1;
  if (pi < lo || pj < lo || pk < lo || pi >= g.n0 - g.gw || pj >= g.n1 - g.gw || pk >= g.n2 - g.gw) return 0.0;
  if (pk == lo) return 0.0;
  const long long s = stride_of(g, d);
  const double rho = d == 2 ? a.rho0[pk] : a.rho0_half[pk];
  return -factor * (0.5 * (__ldg(a.D + p) + __ldg(a.D + p + s))) * (__ldg(phi + p + s) - __ldg(phi + p)) * rho *
         a.dxi_div[d];
}

// The same flux without the range tests, for a face inside [gw-1, nlg-gw)
// and off the level gw-1.
__device__ __forceinline__ double sflux_in(const SArgs& a, const double* phi, double factor, int d, long long p,
                                           int pk) {
  const long long s = stride_of(a.g, d);
  const double rho = d == 2 ? a.rho0[pk] : a.rho0_half[pk];
  return -factor * (0.5 * (__ldg(a.D + p) + __ldg(a.D + p + s))) * (__ldg(phi + p + s) - __ldg(phi + p)) * rho *
         a.dxi_div[d];
}

// ScalarDiffusion.update (ScalarDiffusion.pyx:112-150) for one interior
// cell: per scalar in order, per direction, the flux divergence
// (scalar_flux_divergence, Csrc/flux_divergence.h:4-32) and, for qt, the
// entropy source (compute_qt_diffusion_s_source,
// Csrc/scalar_diffusion.h:70-113).
__global__ void __launch_bounds__(kThreads, 8) scalar_diffusion(SArgs a) {
  const G& g = a.g;
  const int k = g.gw + blockIdx.x * kThreads + threadIdx.x;
  const int j = g.gw + blockIdx.y, i = g.gw + blockIdx.z;
  if (k >= g.n2 - g.gw) return;
  const long long ijk = (long long)i * g.is + (long long)j * g.js + k;
  for (int n = 0; n < a.ns; ++n) {
    const double* phi = a.phi[n];
    double t = a.tend[n][ijk];
    const bool src = n == a.qt_index;
    double sw_sd = 0.0;
    if (src) {
      const double qt = phi[ijk], qv = a.qv[ijk], T = a.T[ijk], p0 = a.p0_half[k];
      const double pd = p0 * (1.0 - qt) / (1.0 - qt + eps_vi * qv);
      const double sd = sd_tilde + cpd * crm::log(T / T_tilde) - Rd * crm::log(pd / p_tilde);
      const double pv = p0 * eps_vi * qv / (1.0 - qt + eps_vi * qv);
      const double sv = sv_tilde + cpv * crm::log(T / T_tilde) - Rv * crm::log(pv / p_tilde);
      const double TC = T - 273.15;
      const double L = (2500.8 - 2.36 * TC + 0.0016 * TC * TC - 0.00006 * TC * TC * TC) * 1000.0;
      const double sw = sv - (((qt - qv) / qt) * L / T);
      sw_sd = sw - sd;
    }
    for (int d = 0; d < 3; ++d) {
      const long long s = stride_of(g, d);
      // an interior cell's own face and the face below it lie inside the
      // flux range; only the face below the first level (k = gw) is 0
      const double fh = sflux_in(a, phi, a.factor[n], d, ijk, k);
      const double fl = (d == 2 && k == g.gw) ? 0.0 : sflux_in(a, phi, a.factor[n], d, ijk - s, d == 2 ? k - 1 : k);
      t -= a.alpha0_half[k] * (fh - fl) * g.dxi[d];
      if (src) {
        int hi[3] = {i, j, k};
        hi[d] += 1;
        const double fu = sflux(a, phi, a.factor[n], d, ijk + s, hi[0], hi[1], hi[2]);
        a.tend[a.s_index][ijk] -= sw_sd * a.alpha0_half[k] * (fu - fh) * a.dxi_div[d];
      }
    }
    a.tend[n][ijk] = t;
  }
}

struct MArgs {
  G g;
  const double* V[3];
  const double* rho0;
  const double* rho0_half;
  const double* alpha0;
  const double* alpha0_half;
  const double* nu;
  const double* smag;
  const double* T;
  double* tend[3];
  double* s_tend;
};

// compute_diffusive_flux_m (Csrc/momentum_diffusion.h:5-96) of S_{i1 i2}
// at p (inside the flux range [gw-1, nlg-gw) for every p the divergence
// reads); 0 on the level k = gw-1.
__device__ __forceinline__ double mflux(const MArgs& a, int i1, int i2, long long p, int pk) {
  const G& g = a.g;
  if (pk == g.gw - 1) return 0.0;
  const double S = strain(g, a.V, i1, i2, p);
  const long long s1 = stride_of(g, i1), s2 = stride_of(g, i2);
  if (i1 != 2 && i2 != 2) {
    if (i1 == i2) return -2.0 * S * __ldg(a.nu + p + s1) * a.rho0_half[pk];
    const double vi = 0.25 * (__ldg(a.nu + p) + __ldg(a.nu + p + s1) + __ldg(a.nu + p + s2) + __ldg(a.nu + p + s1 + s2));
    return -2.0 * S * vi * a.rho0_half[pk];
  }
  if (i1 == 2 && i2 == 2) return -2.0 * S * __ldg(a.nu + p + s1) * a.rho0_half[pk + 1];
  const double vi = 0.25 * (__ldg(a.nu + p) + __ldg(a.nu + p + s1) + __ldg(a.nu + p + s2) + __ldg(a.nu + p + s1 + s2));
  return -2.0 * S * vi * a.rho0[pk];
}

// MomentumDiffusion.update (MomentumDiffusion.pyx:52-78) for one interior
// cell: for u, v, w the divergence of the three stress fluxes
// (momentum_flux_divergence, Csrc/flux_divergence.h:34-60), then the
// entropy source S^2 nu / T (compute_entropy_source,
// Csrc/momentum_diffusion.h:98-118).
__global__ void __launch_bounds__(kThreads) momentum_diffusion(MArgs a) {
  const G& g = a.g;
  const int k = g.gw + blockIdx.x * kThreads + threadIdx.x;
  const int j = g.gw + blockIdx.y, i = g.gw + blockIdx.z;
  if (k >= g.n2 - g.gw) return;
  const long long ijk = (long long)i * g.is + (long long)j * g.js + k;
  // fully unrolled: the component indices fold into the stencil offsets
  // and the loads shared by the nine fluxes are issued once
#pragma unroll
  for (int i1 = 0; i1 < 3; ++i1) {
    double t = a.tend[i1][ijk];
    const double al = i1 != 2 ? a.alpha0_half[k] : a.alpha0[k];
#pragma unroll
    for (int i2 = 0; i2 < 3; ++i2) {
      const double fh = mflux(a, i1, i2, ijk, k);
      const double fl = mflux(a, i1, i2, ijk - stride_of(g, i2), i2 == 2 ? k - 1 : k);
      t -= al * (fh - fl) * g.dxi[i2];
    }
    a.tend[i1][ijk] = t;
  }
  const double S = a.smag[ijk];
  a.s_tend[ijk] += S * S * a.nu[ijk] / a.T[ijk];
}

G make_g(const pb_dims* d) {
  G g;
  g.n0 = (int)d->nlg[0];
  g.n1 = (int)d->nlg[1];
  g.n2 = (int)d->nlg[2];
  g.js = d->nlg[2];
  g.is = (long long)d->nlg[1] * d->nlg[2];
  g.gw = (int)d->gw;
  for (int q = 0; q < 3; ++q) g.dxi[q] = d->dxi[q];
  return g;
}

}  // namespace sgsk
}  // namespace

extern "C" int pb_kinematics_sgs(const pb_dims* dims, const pb_sgs* sgs, const double* u, const double* v,
                                 const double* w, const double* buoyancy_frequency, const double* zl_half,
                                 double* strain_rate_mag, double* viscosity, double* diffusivity, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!u || !v || !w || !strain_rate_mag) return PB_ERR_ARG;
  if (dims->nlg[1] > 65535 || dims->nlg[0] > 65535) return PB_ERR_UNSUPPORTED;
  const dim3 grid((unsigned)((dims->nlg[2] + sgsk::kThreads - 1) / sgsk::kThreads), (unsigned)dims->nlg[1],
                  (unsigned)dims->nlg[0]);
  cudaStream_t st = as_stream(stream);
  sgsk::KArgs a;
  memset(&a, 0, sizeof(a));
  a.g = sgsk::make_g(dims);
  a.V[0] = u;
  a.V[1] = v;
  a.V[2] = w;
  a.smag = strain_rate_mag;
  if (!sgs) {  // the strain-rate magnitude alone
    sgsk::kinematics_sgs<0, PB_SGS_LENGTH_GRID><<<grid, sgsk::kThreads, 0, st>>>(a);
    pb_note_launch();
    PB_LAUNCH_CHECK();
    return PB_OK;
  }
  if (!viscosity || !diffusivity) return PB_ERR_ARG;
  if (sgs->scheme != PB_SGS_UNIFORM && sgs->scheme != PB_SGS_SMAGORINSKY) return PB_ERR_ARG;
  if (sgs->length != PB_SGS_LENGTH_GRID && sgs->length != PB_SGS_LENGTH_WALL && sgs->length != PB_SGS_LENGTH_ILES)
    return PB_ERR_ARG;
  if (sgs->scheme == PB_SGS_SMAGORINSKY && !buoyancy_frequency) return PB_ERR_ARG;
  if (sgs->scheme == PB_SGS_SMAGORINSKY && sgs->length != PB_SGS_LENGTH_GRID && !zl_half) return PB_ERR_ARG;
  a.bvf = buoyancy_frequency;
  a.zl_half = zl_half;
  a.visc = viscosity;
  a.diff = diffusivity;
  a.scheme = sgs->scheme;
  a.length = sgs->length;
  a.cs = sgs->cs;
  a.prt = sgs->prt;
  // delta = cbrt(dx dy dz) (Csrc/sgs.h:7), formed by the host C library
  a.delta = cbrt(dims->dx[0] * dims->dx[1] * dims->dx[2]);
  a.const_visc = sgs->viscosity;
  a.const_diff = sgs->diffusivity;
  if (sgs->scheme == PB_SGS_UNIFORM)
    sgsk::kinematics_sgs<PB_SGS_UNIFORM, PB_SGS_LENGTH_GRID><<<grid, sgsk::kThreads, 0, st>>>(a);
  else if (sgs->length == PB_SGS_LENGTH_GRID)
    sgsk::kinematics_sgs<PB_SGS_SMAGORINSKY, PB_SGS_LENGTH_GRID><<<grid, sgsk::kThreads, 0, st>>>(a);
  else if (sgs->length == PB_SGS_LENGTH_WALL)
    sgsk::kinematics_sgs<PB_SGS_SMAGORINSKY, PB_SGS_LENGTH_WALL><<<grid, sgsk::kThreads, 0, st>>>(a);
  else
    sgsk::kinematics_sgs<PB_SGS_SMAGORINSKY, PB_SGS_LENGTH_ILES><<<grid, sgsk::kThreads, 0, st>>>(a);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

extern "C" int pb_scalar_diffusion(const pb_dims* dims, const double* rho0, const double* rho0_half,
                                   const double* alpha0_half, const double* diffusivity, int nscalars,
                                   const double* const* scalars, double* const* tendencies, const double* factors,
                                   int qt_index, int s_index, const double* p0_half, const double* qv,
                                   const double* T, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!rho0 || !rho0_half || !alpha0_half || !diffusivity || nscalars < 0 || (nscalars > 0 && (!scalars ||
      !tendencies)))
    return PB_ERR_ARG;
  if (nscalars > sgsk::kMaxScalars) return PB_ERR_UNSUPPORTED;
  if (qt_index >= nscalars || (qt_index >= 0 && (s_index < 0 || s_index >= nscalars || s_index == qt_index ||
                                                  !p0_half || !qv || !T)))
    return PB_ERR_ARG;
  if (dims->gw < 2) return PB_ERR_UNSUPPORTED;
  if (dims->n[1] > 65535 || dims->n[0] > 65535) return PB_ERR_UNSUPPORTED;
  if (nscalars == 0) return PB_OK;
  sgsk::SArgs a;
  memset(&a, 0, sizeof(a));
  a.g = sgsk::make_g(dims);
  a.rho0 = rho0;
  a.rho0_half = rho0_half;
  a.alpha0_half = alpha0_half;
  a.p0_half = p0_half;
  a.D = diffusivity;
  a.qv = qv;
  a.T = T;
  a.ns = nscalars;
  for (int n = 0; n < nscalars; ++n) {
    if (!scalars[n] || !tendencies[n]) return PB_ERR_ARG;
    a.phi[n] = scalars[n];
    a.tend[n] = tendencies[n];
    a.factor[n] = factors ? factors[n] : 1.0;
  }
  for (int q = 0; q < 3; ++q) a.dxi_div[q] = 1.0 / dims->dx[q];
  a.qt_index = qt_index;
  a.s_index = qt_index >= 0 ? s_index : -1;
  const dim3 grid((unsigned)((dims->n[2] + sgsk::kThreads - 1) / sgsk::kThreads), (unsigned)dims->n[1],
                  (unsigned)dims->n[0]);
  sgsk::scalar_diffusion<<<grid, sgsk::kThreads, 0, as_stream(stream)>>>(a);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}

extern "C" int pb_momentum_diffusion(const pb_dims* dims, const double* rho0, const double* rho0_half,
                                     const double* alpha0, const double* alpha0_half, const double* u,
                                     const double* v, const double* w, const double* viscosity,
                                     const double* strain_rate_mag, const double* T, double* ut, double* vt,
                                     double* wt, double* s_tend, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!rho0 || !rho0_half || !alpha0 || !alpha0_half || !u || !v || !w || !viscosity || !strain_rate_mag || !T ||
      !ut || !vt || !wt || !s_tend)
    return PB_ERR_ARG;
  if (dims->gw < 2) return PB_ERR_UNSUPPORTED;
  if (dims->n[1] > 65535 || dims->n[0] > 65535) return PB_ERR_UNSUPPORTED;
  sgsk::MArgs a;
  memset(&a, 0, sizeof(a));
  a.g = sgsk::make_g(dims);
  a.V[0] = u;
  a.V[1] = v;
  a.V[2] = w;
  a.rho0 = rho0;
  a.rho0_half = rho0_half;
  a.alpha0 = alpha0;
  a.alpha0_half = alpha0_half;
  a.nu = viscosity;
  a.smag = strain_rate_mag;
  a.T = T;
  a.tend[0] = ut;
  a.tend[1] = vt;
  a.tend[2] = wt;
  a.s_tend = s_tend;
  const dim3 grid((unsigned)((dims->n[2] + sgsk::kThreads - 1) / sgsk::kThreads), (unsigned)dims->n[1],
                  (unsigned)dims->n[0]);
  sgsk::momentum_diffusion<<<grid, sgsk::kThreads, 0, as_stream(stream)>>>(a);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}
