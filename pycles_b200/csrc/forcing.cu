// Case forcing (Forcing.pyx): SullivanPatton (Coriolis :256-300), Bomex
// (large-scale pressure gradient, radiative cooling and drying, subsidence
// :102-254), DyCOMS_RF01 (subsidence and Coriolis :346-460), as one pass per
// RK stage over the interior columns: each thread owns one cell and applies
// the scheme's terms to its tendencies in the reference's order (per array
// the same sequence of subtractions and additions as the reference's
// successive loops).  The per-level profiles (ug, vg, the large-scale
// tendencies, the subsidence velocity) are set by the host as the schemes'
// initialize does; Bomex's horizontal means of u and v come from
// pb_horizontal_stat.  FP64, compiled with -fmad=false and correctly
// rounded log (the entropy source of the large-scale tendencies).
#include <string.h>

#include "pb_common.cuh"
#include "crmath.cuh"

namespace {
namespace fck {

using namespace pbc;

constexpr int kThreads = 128;

struct Args {
  long long n0, n1, n2, is, js;
  int gw, scheme;
  double dzi, f, u0, v0;
  const double* ug;
  const double* vg;
  const double* dtdt;
  const double* dqtdt;
  const double* sub;
  const double* umean;
  const double* vmean;
  const double* p0_half;
  const double* u;
  const double* v;
  const double* s;
  const double* qt;
  const double* ql;
  const double* T;
  double* ut;
  double* vt;
  double* st;
  double* qtt;
};

// apply_subsidence (Forcing.pyx:2013-2039) for one cell: below the top
// interior level the local difference; from it up (top level and ghosts)
// the difference of the level below it, subtracted again.
__device__ __forceinline__ double subs(const Args& a, const double* phi, long long ijk, long long k) {
  const long long kmax = a.n2 - a.gw - 1;
  const long long kk = k < kmax ? k : kmax - 1;
  const long long o = ijk - (k - kk);
  return (phi[o + 1] - phi[o]) * a.dzi * a.sub[kk];
}

// coriolis_force (Forcing.pyx:1954-1980) for one interior cell
__device__ __forceinline__ void coriolis(const Args& a, long long ijk, long long k, double& ut, double& vt) {
  const double u_at_v = 0.25 * (a.u[ijk] + a.u[ijk - a.is] + a.u[ijk - a.is + a.js] + a.u[ijk + a.js]) + a.u0;
  const double v_at_u = 0.25 * (a.v[ijk] + a.v[ijk + a.is] + a.v[ijk + a.is - a.js] + a.v[ijk - a.js]) + a.v0;
  ut = ut - a.f * (a.vg[k] - v_at_u);
  vt = vt + a.f * (a.ug[k] - u_at_v);
}

template <int SCHEME>
__global__ void __launch_bounds__(kThreads) forcing_kernel(Args a) {
  const long long k = a.gw + (long long)blockIdx.x * kThreads + threadIdx.x;
  const long long j = a.gw + blockIdx.y, i = a.gw + blockIdx.z;
  if (k >= a.n2) return;
  const bool interior = k < a.n2 - a.gw;
  const long long ijk = i * a.is + j * a.js + k;
  if (SCHEME == PB_FORCING_SULLIVAN_PATTON) {
    if (!interior) return;
    double ut = a.ut[ijk], vt = a.vt[ijk];
    coriolis(a, ijk, k, ut, vt);
    a.ut[ijk] = ut;
    a.vt[ijk] = vt;
    return;
  }
  double ut = a.ut[ijk], vt = a.vt[ijk], st = a.st[ijk], qtt = a.qtt[ijk];
  if (SCHEME == PB_FORCING_BOMEX && interior) {
    // large_scale_p_gradient (Forcing.pyx:1982-2011)
    const double u_at_v = a.umean[k] + a.u0;
    const double v_at_u = a.vmean[k] + a.v0;
    ut = ut - a.f * (a.vg[k] - v_at_u);
    vt = vt + a.f * (a.ug[k] - u_at_v);
    // large-scale sources (Forcing.pyx:186-197) with s_tendency_c
    // (Csrc/entropies.h:17-21)
    const double p0 = a.p0_half[k], qt = a.qt[ijk], qv = qt - a.ql[ijk], T = a.T[ijk];
    const double pv = p0 * eps_vi * qv / (1.0 - qt + eps_vi * qv);
    const double pd = p0 * (1.0 - qt) / (1.0 - qt + eps_vi * qv);
    const double sv = sv_tilde + cpv * crm::log(T / T_tilde) - Rv * crm::log(pv / p_tilde);
    const double sd = sd_tilde + cpd * crm::log(T / T_tilde) - Rd * crm::log(pd / p_tilde);
    const double cpm = (1.0 - qt) * cpd + qt * cpv;
    st += cpm * a.dtdt[k] / T + (sv - sd) * a.dqtdt[k];
    qtt += a.dqtdt[k];
  }
  // apply_subsidence of s, qt, u, v (Forcing.pyx:199-202, 400-403)
  st -= subs(a, a.s, ijk, k);
  qtt -= subs(a, a.qt, ijk, k);
  ut -= subs(a, a.u, ijk, k);
  vt -= subs(a, a.v, ijk, k);
  if (SCHEME == PB_FORCING_DYCOMS_RF01 && interior) coriolis(a, ijk, k, ut, vt);
  a.ut[ijk] = ut;
  a.vt[ijk] = vt;
  a.st[ijk] = st;
  a.qtt[ijk] = qtt;
}

}  // namespace fck
}  // namespace

extern "C" int pb_forcing_update(const pb_dims* dims, const pb_forcing* forcing, const double* p0_half,
                                 const double* umean, const double* vmean, const double* u, const double* v,
                                 const double* s, const double* qt, const double* ql, const double* T, double* ut,
                                 double* vt, double* s_tend, double* qt_tend, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!forcing) return PB_ERR_ARG;
  const int sc = forcing->scheme;
  if (sc == PB_FORCING_NONE) return PB_OK;
  if (sc != PB_FORCING_SULLIVAN_PATTON && sc != PB_FORCING_BOMEX && sc != PB_FORCING_DYCOMS_RF01)
    return PB_ERR_ARG;
  if (!u || !v || !ut || !vt || !forcing->ug || !forcing->vg) return PB_ERR_ARG;
  if (sc != PB_FORCING_SULLIVAN_PATTON && (!s || !qt || !s_tend || !qt_tend || !forcing->subsidence))
    return PB_ERR_ARG;
  if (sc == PB_FORCING_BOMEX && (!umean || !vmean || !p0_half || !ql || !T || !forcing->dtdt || !forcing->dqtdt))
    return PB_ERR_ARG;
  if (dims->gw < 2 || dims->n[2] < 2) return PB_ERR_UNSUPPORTED;
  if (dims->n[1] > 65535 || dims->n[0] > 65535) return PB_ERR_UNSUPPORTED;
  fck::Args a;
  memset(&a, 0, sizeof(a));
  a.n0 = dims->nlg[0];
  a.n1 = dims->nlg[1];
  a.n2 = dims->nlg[2];
  a.js = dims->nlg[2];
  a.is = (long long)dims->nlg[1] * dims->nlg[2];
  a.gw = (int)dims->gw;
  a.scheme = sc;
  a.dzi = dims->dxi[2];
  a.f = forcing->coriolis_param;
  a.u0 = forcing->u0;
  a.v0 = forcing->v0;
  a.ug = forcing->ug;
  a.vg = forcing->vg;
  a.dtdt = forcing->dtdt;
  a.dqtdt = forcing->dqtdt;
  a.sub = forcing->subsidence;
  a.umean = umean;
  a.vmean = vmean;
  a.p0_half = p0_half;
  a.u = u;
  a.v = v;
  a.s = s;
  a.qt = qt;
  a.ql = ql;
  a.T = T;
  a.ut = ut;
  a.vt = vt;
  a.st = s_tend;
  a.qtt = qt_tend;
  // interior columns, levels gw .. nlg2-1 (the subsidence reaches the top ghosts)
  const dim3 grid((unsigned)((dims->nlg[2] - dims->gw + fck::kThreads - 1) / fck::kThreads), (unsigned)dims->n[1],
                  (unsigned)dims->n[0]);
  cudaStream_t st = as_stream(stream);
  if (sc == PB_FORCING_SULLIVAN_PATTON)
    fck::forcing_kernel<PB_FORCING_SULLIVAN_PATTON><<<grid, fck::kThreads, 0, st>>>(a);
  else if (sc == PB_FORCING_BOMEX)
    fck::forcing_kernel<PB_FORCING_BOMEX><<<grid, fck::kThreads, 0, st>>>(a);
  else
    fck::forcing_kernel<PB_FORCING_DYCOMS_RF01><<<grid, fck::kThreads, 0, st>>>(a);
  pb_note_launch();
  PB_LAUNCH_CHECK();
  return PB_OK;
}
