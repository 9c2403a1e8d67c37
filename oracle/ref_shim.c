/*
 * Test infrastructure, not product code.
 *
 * Thin C shim that compiles the PyCLES reference kernels IN PLACE (the
 * headers under the reference's Csrc/ directory are included from where
 * they lie; nothing of them is copied here) into oracle/_ref/libpycles_ref.so.
 * Only the checker (tests/, __graft_entry__.smoke, bench.py's CPU legs)
 * loads the result.  It pins the numpy restatement in oracle/port.py and
 * generates the golden fixtures under tests/golden/.
 *
 * What this file adds on top of the reference headers:
 *  - the two latent-heat / phase-partition function pointers that the
 *    reference supplies from Cython (Microphysics.pxd:65-75: lambda_constant,
 *    latent_heat_variable), restated as C functions;
 *  - wrappers that pass those pointers, so ctypes can call eos_update,
 *    bvf_sa and thetali_update with plain pointers;
 *  - a LookupStruct constructor (init_table, Csrc/lookup.h:16-40) callable
 *    from ctypes;
 *  - wrappers of the surface-layer functions of Csrc/surface.h and of the
 *    qt-diffusion entropy source (Csrc/scalar_diffusion.h), which takes the
 *    latent-heat function pointers.
 * The dry-thermodynamics header defines eos_c/eos_update under the same
 * names as the saturation-adjustment header, so it is included with those
 * two names remapped.
 */
#include <stdlib.h>
#include <stdio.h>
#include <math.h>
#include <sys/types.h>

#include "parameters.h"
#include "grid.h"
#include "lookup.h"
#include "advection_interpolation.h"
#include "flux_divergence.h"
#include "scalar_advection.h"
#include "momentum_advection.h"
#include "thermodynamics_sa.h"
#include "prognostic_variables.h"
#include "surface.h"
#include "kinematics.h"
#include "sgs.h"
#include "scalar_diffusion.h"
#include "momentum_diffusion.h"

#define eos_c dry_eos_c
#define eos_update dry_eos_update
#include "thermodynamics_dry.h"
#undef eos_c
#undef eos_update

/* Microphysics.pxd:65-66 */
static double shim_lambda_constant(double T) { (void)T; return 1.0; }
/* Microphysics.pxd:71-75 */
static double shim_latent_heat_variable(double T, double Lambda) {
    (void)Lambda;
    double TC = T - 273.15;
    return (2500.8 - 2.36 * TC + 0.0016 * TC * TC - 0.00006 * TC * TC * TC) * 1000.0;
}

/* ---- lookup table ---------------------------------------------------- */
struct LookupStruct* ref_table_new(long n, double* x, double* y) {
    struct LookupStruct* LT = (struct LookupStruct*)calloc(1, sizeof(struct LookupStruct));
    init_table(LT, (size_t)n, x, y);
    return LT;
}
void ref_table_free(struct LookupStruct* LT) { free_table(LT); free(LT); }
double ref_table_lookup(struct LookupStruct* LT, double x) { return lookup(LT, x); }

double ref_latent_heat_variable(double T) { return shim_latent_heat_variable(T, shim_lambda_constant(T)); }

/* ---- saturation-adjustment thermodynamics ---------------------------- */
void ref_eos_c(struct LookupStruct* LT, double p0, double s, double qt,
               double* T, double* qv, double* ql, double* qi) {
    eos_c(LT, shim_lambda_constant, shim_latent_heat_variable, p0, s, qt, T, qv, ql, qi);
}

void ref_eos_update(struct DimStruct* dims, struct LookupStruct* LT, double* p0, double* s,
                    double* qt, double* T, double* qv, double* ql, double* qi, double* alpha) {
    eos_update(dims, LT, shim_lambda_constant, shim_latent_heat_variable, p0, s, qt, T, qv, ql, qi, alpha);
}

void ref_bvf_sa(struct DimStruct* dims, struct LookupStruct* LT, double* p0, double* T, double* qt,
                double* qv, double* theta_rho, double* bvf) {
    bvf_sa(dims, LT, shim_lambda_constant, shim_latent_heat_variable, p0, T, qt, qv, theta_rho, bvf);
}

void ref_thetali_update(struct DimStruct* dims, double* p0, double* T, double* qt, double* ql,
                        double* qi, double* thetali) {
    thetali_update(dims, shim_lambda_constant, shim_latent_heat_variable, p0, T, qt, ql, qi, thetali);
}

/* entropy as in ThermodynamicsSA.entropy (ThermodynamicsSA.pyx:140-159) */
double ref_entropy_sa(double p0, double T, double qt, double ql, double qi) {
    double qv = qt - ql - qi;
    double pd = pd_c(p0, qt, qv);
    double pv = pv_c(p0, qt, qv);
    double L = shim_latent_heat_variable(T, shim_lambda_constant(T));
    return sd_c(pd, T) * (1.0 - qt) + sv_c(pv, T) * qt + sc_c(L, T) * (ql + qi);
}

double ref_exner(double p0) { return exner_c(p0); }
double ref_dry_eos(double pd, double s) { return dry_eos_c(pd, s); }

/* ---- surface fluxes (Csrc/surface.h) --------------------------------- */
double ref_compute_ustar(double windspeed, double buoyancy_flux, double z0, double zb) {
    return compute_ustar(windspeed, buoyancy_flux, z0, zb);
}
void ref_compute_windspeed(struct DimStruct* dims, double* u, double* v, double* speed, double u0, double v0,
                           double gustiness) {
    compute_windspeed(dims, u, v, speed, u0, v0, gustiness);
}
double ref_entropyflux(double thetaflux, double qtflux, double p0_b, double T_b, double qt_b, double qv_b) {
    return entropyflux_from_thetaflux_qtflux(thetaflux, qtflux, p0_b, T_b, qt_b, qv_b);
}

/* ---- subgrid scale and diffusion (Csrc/kinematics.h, sgs.h, *_diffusion.h) */
void ref_compute_qt_diffusion_s_source(struct DimStruct* dims, double* p0_half, double* alpha0, double* alpha0_half,
                                       double* flux, double* qt, double* qv, double* T, double* tendency,
                                       double dx, ssize_t d) {
    compute_qt_diffusion_s_source(dims, p0_half, alpha0, alpha0_half, flux, qt, qv, T, tendency,
                                  shim_lambda_constant, shim_latent_heat_variable, dx, d);
}

/* Csrc/entropies.h:17-21 (the forcing's entropy source) */
double ref_s_tendency(double p0, double qt, double qv, double T, double qt_tendency, double T_tendency) {
    return s_tendency_c(p0, qt, qv, T, qt_tendency, T_tendency);
}
