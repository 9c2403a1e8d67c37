// DYCOMS-RF01 radiation (Radiation.pyx:230-353): per interior column the
// inversion height zi (highest level with qt > 8 g/kg), the three flux terms
// of Stevens et al. 2005 eq. 3 (above-inversion cooling, the upward and the
// downward liquid-water-path terms), the heating rate as the flux
// divergence, and its entropy tendency and temperature tendency.
//
// One thread per column, three passes over its levels (zi; the downward
// path from the top, whose flux term is parked in the heating-rate array;
// the upward path with the flux and its divergence), each a sequential
// recurrence in the reference's order, so every flux value is the
// reference's.  FP64, compiled with -fmad=false, correctly rounded exp.
// The reference keeps zi and rhoi from the previous pencil when no level
// of a column has qt > 8e-3 (undefined for the first pencil); here such a
// column takes zi above the domain (the cubic term vanishes) -- see
// pb_dycoms_radiation.
#include <math.h>
#include <string.h>

#include "pb_common.cuh"
#include "crmath.cuh"

namespace {
namespace rdk {

using namespace pbc;

struct Args {
  long long n0, n1, n2, is, js;
  int gw, nz;
  double dz, dzi, f0, f1, kap, alpha_z, divergence;
  const double* rho0_half;
  const double* z;
  const double* ql;
  const double* qt;
  const double* T;
  double* s_tend;
  double* heating;
  double* dTdt;
};

__global__ void __launch_bounds__(128) dycoms_radiation(Args a) {
  const long long nl1 = a.n1 - 2 * a.gw;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= (a.n0 - 2 * a.gw) * nl1) return;
  const long long i = a.gw + c / nl1, j = a.gw + c % nl1;
  const long long col = i * a.is + j * a.js;
  const int g = a.gw, n = a.nz;
  const double* rh = a.rho0_half;
  // zi, rhoi: the highest level with qt > 8e-3
  double zi = INFINITY, rhoi = 0.0;
  for (int k = 0; k < n; ++k)
    if (a.qt[col + g + k] > 8e-3) {
      zi = a.z[g + k];
      rhoi = rh[g + k];
    }
  // downward path from the top: C_k = f0 exp(-q0(k)), q0 accumulated from
  // level n-1 down to k; C_n = f0 exp(-0).  C_k for k < n is parked in the
  // heating-rate array of level k.
  const double cn = a.f0 * crm::exp(-0.0);
  double q0 = 0.0;
  for (int k = n - 1; k >= 0; --k) {
    q0 += a.kap * rh[g + k] * a.ql[col + g + k] * a.dz;
    a.heating[col + g + k] = a.f0 * crm::exp(-q0);
  }
  // upward: F_k = (cubic term + f1 exp(-q1(k))) + C_k; heating[k-1] from
  // F_k - F_{k-1}
  double q1 = 0.0;
  double fprev = (0.0 + a.f1 * crm::exp(-q1)) + a.heating[col + g];  // F_0
  for (int k = 1; k <= n; ++k) {
    double f;
    const double zk = a.z[g + k - 1];
    if (zk >= zi) {
      const double cz = cbrt(zk - zi);
      f = rhoi * cpd * a.divergence * a.alpha_z * (pow(cz, 4.0) / 4.0 + zi * cz);
    } else {
      f = 0.0;
    }
    q1 += a.kap * rh[g + k - 1] * a.ql[col + g + k - 1] * a.dz;
    f += a.f1 * crm::exp(-q1);
    f += k < n ? a.heating[col + g + k] : cn;
    const long long o = col + g + k - 1;
    // Radiation.pyx:334-336 divides by rho0_half[k-1], without the ghost offset
    const double h = -(f - fprev) * a.dzi / rh[k - 1];
    a.heating[o] = h;
    a.s_tend[o] += h / a.T[o];
    const double qt = a.qt[o];
    a.dTdt[o] = h / ((1.0 - qt) * cpd + qt * cpv);
    fprev = f;
  }
}

}  // namespace rdk
}  // namespace

extern "C" int pb_dycoms_radiation(const pb_dims* dims, const pb_dycoms_radiation_params* prm,
                                   const double* rho0_half, const double* z, const double* ql, const double* qt,
                                   const double* T, double* s_tend, double* heating_rate, double* dTdt_rad,
                                   void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!prm || !rho0_half || !z || !ql || !qt || !T || !s_tend || !heating_rate || !dTdt_rad) return PB_ERR_ARG;
  rdk::Args a;
  memset(&a, 0, sizeof(a));
  a.n0 = dims->nlg[0];
  a.n1 = dims->nlg[1];
  a.n2 = dims->nlg[2];
  a.js = dims->nlg[2];
  a.is = (long long)dims->nlg[1] * dims->nlg[2];
  a.gw = (int)dims->gw;
  a.nz = (int)dims->n[2];
  a.dz = dims->dx[2];
  a.dzi = dims->dxi[2];
  a.f0 = prm->f0;
  a.f1 = prm->f1;
  a.kap = prm->kap;
  a.alpha_z = prm->alpha_z;
  a.divergence = prm->divergence;
  a.rho0_half = rho0_half;
  a.z = z;
  a.ql = ql;
  a.qt = qt;
  a.T = T;
  a.s_tend = s_tend;
  a.heating = heating_rate;
  a.dTdt = dTdt_rad;
  const long long ncol = (long long)dims->n[0] * dims->n[1];
  rdk::dycoms_radiation<<<(unsigned)((ncol + 127) / 128), 128, 0, as_stream(stream)>>>(a);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}
