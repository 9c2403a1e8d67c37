// Single translation unit for libpycles_b200.so: the device error word and
// the shared helpers are visible to every kernel without relocatable
// device code.
#include "timestep.cu"
#include "advection.cu"
#include "thermo.cu"
#include "pressure.cu"
