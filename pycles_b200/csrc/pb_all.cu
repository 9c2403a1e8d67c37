// Translation unit 1 of libpycles_b200.so: time stepping, ghost fills,
// advection, pressure.  The thermodynamics are translation unit 2
// (thermo.cu), compiled without FMA contraction.
#include "timestep.cu"
#include "advection.cu"
#include "pressure.cu"
#include "pressure_shard.cu"
#include "pressure_noalloc.cu"
#include "mlp.cu"
