// Translation unit of the FP64 plain-form advection, compiled with
// -fmad=false: the WENO interpolants, upwind fluxes and flux divergences are
// evaluated with the operations and order of Csrc/advection_interpolation.h,
// Csrc/scalar_advection.h, Csrc/momentum_advection_weno.h and
// Csrc/flux_divergence.h, each rounded separately (the reference's C is
// built without FMA), divisions included, so the tendencies equal the
// reference's bit for bit.
#include "advection_kernels.cuh"

namespace pbadv {

cudaError_t scalar_fp64(int order, int ns, const Geo& g, ScalarArgs base, double* const* flux_dir[3],
                        const double* const vel[3], cudaStream_t st) {
  return order == 5 ? launch_scalar_ns<5, false>(ns, g, base, flux_dir, vel, st)
                    : launch_scalar_ns<7, false>(ns, g, base, flux_dir, vel, st);
}

cudaError_t momentum_fp64(int order, const Geo& g, const MomArgs& a, cudaStream_t st) {
  return order == 5 ? launch_momentum<5, false>(g, a, st) : launch_momentum<7, false>(g, a, st);
}

}  // namespace pbadv
