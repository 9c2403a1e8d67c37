// Saturation-adjustment and dry thermodynamics, precision form: the same
// kernels as the FP64 plain form (thermo_kernels.cuh) with CUDA's exp/log and
// FMA contraction, and optionally the learned secant seed evaluated inside
// the kernel.  Every quantity is still FP64 and the secant still runs to the
// reference's |dT| < 1e-3 K.
#include "thermo_kernels.cuh"

namespace thermo_k {

cudaError_t launch_sa_fast(const Geo& geo, const SaArgs& a, bool seeded, cudaStream_t st) {
  return seeded ? thermo_kk::launch_sa<thermo_f::FastMath, true>(geo, a, st)
                : thermo_kk::launch_sa<thermo_f::FastMath, false>(geo, a, st);
}

cudaError_t launch_dry_fast(const Geo& geo, const DryArgs& a, cudaStream_t st) {
  return thermo_kk::launch_dry<thermo_f::FastMath>(geo, a, st);
}

}  // namespace thermo_k
