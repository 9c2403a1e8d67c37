// DYCOMS-RF01 radiation (Radiation.pyx:230-353): per interior column the
// inversion height zi (highest level with qt > 8 g/kg), the three flux terms
// of Stevens et al. 2005 eq. 3 (above-inversion cooling, the upward and the
// downward liquid-water-path terms), the heating rate as the flux
// divergence, and its entropy tendency and temperature tendency.
//
// One warp per column: the running water-path sums in the reference's
// order on one lane, the exponentials, fluxes and divergence on all 32, so
// every flux value is the reference's.  FP64, compiled with -fmad=false,
// correctly rounded exp.
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

constexpr int kWarps = 4;  // columns per block

// One warp per column.  The warp stages the column's water-path increments
// kap rho0_half ql dz in shared memory (coalesced loads), lane 0 runs the
// two running sums in the reference's order (upward q1, downward q0: a
// chain of additions), then all lanes evaluate the exponentials, the cubic
// term and the flux on their levels and, after a warp barrier, the flux
// divergence.  Shared memory per warp: increments, q1, q0 and F on n+1
// levels.
__global__ void __launch_bounds__(kWarps * 32) dycoms_radiation(Args a) {
  extern __shared__ double sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long nl1 = a.n1 - 2 * a.gw;
  const long long c = (long long)blockIdx.x * kWarps + w;
  if (c >= (a.n0 - 2 * a.gw) * nl1) return;  // whole warps leave together
  const long long i = a.gw + c / nl1, j = a.gw + c % nl1;
  const long long col = i * a.is + j * a.js;
  const int g = a.gw, n = a.nz;
  const double* rh = a.rho0_half;
  double* inc = sm + (size_t)w * 4 * (n + 1);
  double* q1 = inc + (n + 1);
  double* q0 = q1 + (n + 1);
  double* F = q0 + (n + 1);
  // zi, rhoi: the highest level with qt > 8e-3 (warp maximum of the level)
  int kz = -1;
  for (int k = lane; k < n; k += 32) {
    if (a.qt[col + g + k] > 8e-3) kz = k;
    inc[k] = a.kap * rh[g + k] * a.ql[col + g + k] * a.dz;
  }
  kz = __reduce_max_sync(0xffffffffu, kz);
  const double zi = kz >= 0 ? a.z[g + kz] : INFINITY;
  const double rhoi = kz >= 0 ? rh[g + kz] : 0.0;
  __syncwarp();
  if (lane == 0) {  // the two independent chains interleaved (each in its own order)
    double s1 = 0.0, s0 = 0.0;
    q1[0] = s1;
    q0[n] = s0;
    for (int k = 1; k <= n; ++k) {
      s1 += inc[k - 1];
      q1[k] = s1;
      s0 += inc[n - k];
      q0[n - k] = s0;
    }
  }
  __syncwarp();
  for (int k = lane; k <= n; k += 32) {
    double f;
    if (k == 0) {
      f = 0.0;
    } else {
      const double zk = a.z[g + k - 1];
      if (zk >= zi) {
        const double cz = cbrt(zk - zi);
        f = rhoi * cpd * a.divergence * a.alpha_z * (pow(cz, 4.0) / 4.0 + zi * cz);
      } else {
        f = 0.0;
      }
    }
    f += a.f1 * crm::exp(-q1[k]);
    f += a.f0 * crm::exp(-q0[k]);
    F[k] = f;
  }
  __syncwarp();
  for (int k = lane; k < n; k += 32) {
    const long long o = col + g + k;
    // Radiation.pyx:334-336 divides by rho0_half[k], without the ghost offset
    const double h = -(F[k + 1] - F[k]) * a.dzi / rh[k];
    a.heating[o] = h;
    a.s_tend[o] += h / a.T[o];
    const double qt = a.qt[o];
    a.dTdt[o] = h / ((1.0 - qt) * cpd + qt * cpv);
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
  const size_t smem = (size_t)rdk::kWarps * 4 * (dims->n[2] + 1) * sizeof(double);
  if (smem > 227 * 1024) return PB_ERR_UNSUPPORTED;
  if (smem > 48 * 1024)
    PB_CUDA_TRY(cudaFuncSetAttribute(rdk::dycoms_radiation, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  rdk::dycoms_radiation<<<(unsigned)((ncol + rdk::kWarps - 1) / rdk::kWarps), rdk::kWarps * 32, smem,
                          as_stream(stream)>>>(a);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}
