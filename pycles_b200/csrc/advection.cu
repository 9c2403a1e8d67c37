// Advection entry points and the FP32 precision-form instantiations of the
// kernels in advection_kernels.cuh (the FP64 plain form is instantiated in
// advection_f64.cu, compiled without FMA contraction).
#include <cudaTypedefs.h>

#include "advection_kernels.cuh"
#include "momentum_tma.cuh"

int pb_make_plane_map(CUtensorMap* map, const double* field, const Geo& g, int box_k, int box_j) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return 1;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[3] = {(cuuint64_t)g.n2, (cuuint64_t)g.n1, (cuuint64_t)g.n0};
  const cuuint64_t strides[2] = {(cuuint64_t)g.n2 * 8, (cuuint64_t)(g.n1 * g.n2) * 8};
  const cuuint32_t box[3] = {(cuuint32_t)box_k, (cuuint32_t)box_j, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(field), dims, strides, box,
                            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : 1;
}

namespace pbadv {

// The precision form's momentum pass: the TMA plane ring where the fields
// allow it (even nlg2, 16-byte aligned arrays), else the register-prefetch
// plane kernel.
static bool use_tma(const Geo& g, const MomArgs& a) {
  return pb_tma_plane_ok(g, a.vel[0]) && pb_tma_plane_ok(g, a.vel[1]) && pb_tma_plane_ok(g, a.vel[2]);
}

cudaError_t scalar_fp32(int order, int ns, const Geo& g, ScalarArgs base, double* const* flux_dir[3],
                        const double* const vel[3], cudaStream_t st) {
  return order == 5 ? launch_scalar_ns<5, true>(ns, g, base, flux_dir, vel, st)
                    : launch_scalar_ns<7, true>(ns, g, base, flux_dir, vel, st);
}

cudaError_t momentum_fp32(int order, const Geo& g, const MomArgs& a, cudaStream_t st) {
  if (use_tma(g, a))
    return order == 5 ? launch_momentum_tma<5, false>(g, a, st) : launch_momentum_tma<7, false>(g, a, st);
  return order == 5 ? launch_momentum<5, true>(g, a, st) : launch_momentum<7, true>(g, a, st);
}

cudaError_t momentum_rk3_fp32(int order, const Geo& g, const MomArgs& a, cudaStream_t st) {
  if (use_tma(g, a))
    return order == 5 ? launch_momentum_tma<5, true>(g, a, st) : launch_momentum_tma<7, true>(g, a, st);
  return order == 5 ? launch_momentum_rk3<5>(g, a, st) : launch_momentum_rk3<7>(g, a, st);
}

}  // namespace pbadv

namespace {

using pbadv::kMaxScalars;
using pbadv::MomArgs;
using pbadv::ScalarArgs;

int check_order(const pb_dims* d, int order) {
  if (order != 5 && order != 7) return PB_ERR_UNSUPPORTED;
  const long R = (order + 1) / 2;
  if (d->gw < R) return PB_ERR_UNSUPPORTED;
  return PB_OK;
}
}  // namespace

extern "C" int pb_scalar_advection(const pb_dims* dims, const double* rho0, const double* rho0_half,
                                   const double* alpha0, const double* alpha0_half, const double* u,
                                   const double* v, const double* w, int nscalars,
                                   const double* const* scalars, double* const* tendencies, double* flux,
                                   int order, int precision, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!rho0 || !rho0_half || !alpha0 || !alpha0_half || !u || !v || !w) return PB_ERR_ARG;
  if (nscalars < 0 || (nscalars > 0 && (!scalars || !tendencies))) return PB_ERR_ARG;
  if (precision != PB_FP64 && precision != PB_FP32) return PB_ERR_ARG;
  if ((rc = check_order(dims, order))) return rc;
  if (nscalars == 0) return PB_OK;
  const Geo g = make_geo(dims);
  cudaStream_t st = as_stream(stream);
  const double* vel[3] = {u, v, w};
  for (int s0 = 0; s0 < nscalars; s0 += kMaxScalars) {
    const int ns = (nscalars - s0 < kMaxScalars) ? nscalars - s0 : kMaxScalars;
    ScalarArgs a{};
    a.rho0 = rho0;
    a.rho0_half = rho0_half;
    a.alpha0_half = alpha0_half;
    a.ns = ns;
    double* fx[kMaxScalars] = {};
    double* fy[kMaxScalars] = {};
    double* fz[kMaxScalars] = {};
    for (int q = 0; q < ns; ++q) {
      if (!scalars[s0 + q] || !tendencies[s0 + q]) return PB_ERR_ARG;
      a.s[q] = scalars[s0 + q];
      a.t[q] = tendencies[s0 + q];
      if (flux) {
        double* fs = flux + (long long)(s0 + q) * 3 * g.npg;
        fx[q] = fs;
        fy[q] = fs + g.npg;
        fz[q] = fs + 2 * g.npg;
      }
    }
    double* const* fdir[3] = {flux ? fx : nullptr, flux ? fy : nullptr, flux ? fz : nullptr};
    cudaError_t e;
    e = precision == PB_FP64 ? pbadv::scalar_fp64(order, ns, g, a, fdir, vel, st)
                             : pbadv::scalar_fp32(order, ns, g, a, fdir, vel, st);
    if (e != cudaSuccess) return PB_ERR_CUDA;
  }
  return PB_OK;
}

extern "C" int pb_scalar_advection_rk3(const pb_dims* dims, const double* rho0, const double* rho0_half,
                                       const double* alpha0, const double* alpha0_half, const double* u,
                                       const double* v, const double* w, int nscalars,
                                       const double* const* scalars, double* const* tendencies,
                                       double* const* new_values, double* const* copies, double dt, int rk_step,
                                       int order, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!rho0 || !rho0_half || !alpha0 || !alpha0_half || !u || !v || !w) return PB_ERR_ARG;
  if (nscalars < 0 || (nscalars > 0 && (!scalars || !tendencies || !new_values || !copies))) return PB_ERR_ARG;
  if (rk_step < 0 || rk_step > 2) return PB_ERR_ARG;
  if ((rc = check_order(dims, order))) return rc;
  if (nscalars == 0) return PB_OK;
  const Geo g = make_geo(dims);
  cudaStream_t st = as_stream(stream);
  const double* vel[3] = {u, v, w};
  for (int s0 = 0; s0 < nscalars; s0 += kMaxScalars) {
    const int ns = (nscalars - s0 < kMaxScalars) ? nscalars - s0 : kMaxScalars;
    ScalarArgs a{};
    a.rho0 = rho0;
    a.rho0_half = rho0_half;
    a.alpha0_half = alpha0_half;
    a.ns = ns;
    a.fused = 1;
    a.dt = dt;
    a.stage = rk_step;
    for (int q = 0; q < ns; ++q) {
      const int i = s0 + q;
      if (!scalars[i] || !tendencies[i] || !new_values[i] || !copies[i] || new_values[i] == scalars[i])
        return PB_ERR_ARG;
      a.s[q] = scalars[i];
      a.t[q] = tendencies[i];
      a.vnew[q] = new_values[i];
      a.copy[q] = copies[i];
    }
    double* const* fdir[3] = {nullptr, nullptr, nullptr};
    if (pbadv::scalar_fp32(order, ns, g, a, fdir, vel, st) != cudaSuccess) return PB_ERR_CUDA;
  }
  return PB_OK;
}

extern "C" int pb_momentum_advection(const pb_dims* dims, const double* rho0, const double* rho0_half,
                                     const double* alpha0, const double* alpha0_half, const double* u,
                                     const double* v, const double* w, double* ut, double* vt, double* wt,
                                     int order, int precision, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!rho0 || !rho0_half || !alpha0 || !alpha0_half || !u || !v || !w || !ut || !vt || !wt) return PB_ERR_ARG;
  if (precision != PB_FP64 && precision != PB_FP32) return PB_ERR_ARG;
  if ((rc = check_order(dims, order))) return rc;
  const Geo g = make_geo(dims);
  MomArgs a{};
  a.vel[0] = u;
  a.vel[1] = v;
  a.vel[2] = w;
  a.tend[0] = ut;
  a.tend[1] = vt;
  a.tend[2] = wt;
  a.rho0 = rho0;
  a.rho0_half = rho0_half;
  a.alpha0 = alpha0;
  a.alpha0_half = alpha0_half;
  a.err = pb_error_word_ptr();
  cudaStream_t st = as_stream(stream);
  cudaError_t e;
  e = precision == PB_FP64 ? pbadv::momentum_fp64(order, g, a, st) : pbadv::momentum_fp32(order, g, a, st);
  return e == cudaSuccess ? PB_OK : PB_ERR_CUDA;
}

extern "C" int pb_momentum_advection_rk3(const pb_dims* dims, const double* rho0, const double* rho0_half,
                                         const double* alpha0, const double* alpha0_half, const double* u,
                                         const double* v, const double* w, double* wt, double* u_new,
                                         double* v_new, double* w_new, double* u_copy, double* v_copy,
                                         double* w_copy, double dt, int rk_step, int order, void* stream) {
  int rc = pb_check_dims(dims);
  if (rc) return rc;
  if (!rho0 || !rho0_half || !alpha0 || !alpha0_half || !u || !v || !w || !wt || !u_new || !v_new || !w_new ||
      !u_copy || !v_copy || !w_copy)
    return PB_ERR_ARG;
  if (rk_step < 0 || rk_step > 2) return PB_ERR_ARG;
  if ((rc = check_order(dims, order))) return rc;
  // the new values go to other arrays than the ones the stencils read
  if (u_new == u || v_new == v || w_new == w) return PB_ERR_ARG;
  const Geo g = make_geo(dims);
  MomArgs a{};
  a.vel[0] = u;
  a.vel[1] = v;
  a.vel[2] = w;
  a.tend[2] = wt;
  a.rho0 = rho0;
  a.rho0_half = rho0_half;
  a.alpha0 = alpha0;
  a.alpha0_half = alpha0_half;
  a.vnew[0] = u_new;
  a.vnew[1] = v_new;
  a.vnew[2] = w_new;
  a.copy[0] = u_copy;
  a.copy[1] = v_copy;
  a.copy[2] = w_copy;
  a.err = pb_error_word_ptr();
  a.dt = dt;
  a.stage = rk_step;
  const cudaError_t e = pbadv::momentum_rk3_fp32(order, g, a, as_stream(stream));
  return e == cudaSuccess ? PB_OK : PB_ERR_CUDA;
}
