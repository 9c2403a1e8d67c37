"""ctypes binding to the reference's own C kernels (test infrastructure).

The library ``oracle/_ref/libpycles_ref.so`` is built by ``build_ref.py``
from the reference headers in place.  Each wrapper calls exactly one
reference function with the arguments the reference's Cython glue passes.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

from .dims import Dims, DimStructC

_HERE = os.path.dirname(os.path.abspath(__file__))
_REF_DIR = os.path.join(_HERE, "_ref")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)


def available() -> bool:
    return os.path.exists(os.path.join(_REF_DIR, "libpycles_ref.so"))


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_REF_DIR, "libpycles_ref.so")
        if not os.path.exists(path):
            raise RuntimeError("reference checker library missing: run oracle/build_ref.py")
        L = ctypes.CDLL(path)
        L.ref_table_new.restype = ctypes.c_void_p
        L.ref_table_new.argtypes = [ctypes.c_long, _dp, _dp]
        L.ref_table_lookup.restype = ctypes.c_double
        L.ref_table_lookup.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.ref_table_free.argtypes = [ctypes.c_void_p]
        L.ref_latent_heat_variable.restype = ctypes.c_double
        L.ref_latent_heat_variable.argtypes = [ctypes.c_double]
        L.ref_eos_c.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                _dp, _dp, _dp, _dp]
        L.ref_entropy_sa.restype = ctypes.c_double
        L.ref_entropy_sa.argtypes = [ctypes.c_double] * 5
        L.ref_exner.restype = ctypes.c_double
        L.ref_exner.argtypes = [ctypes.c_double]
        L.ref_dry_eos.restype = ctypes.c_double
        L.ref_dry_eos.argtypes = [ctypes.c_double, ctypes.c_double]
        L.scalar_flux_divergence.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_ssize_t]
        L.compute_advective_fluxes_a.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int]
        L.compute_advective_tendencies_m.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                                     ctypes.c_ssize_t, ctypes.c_ssize_t, ctypes.c_int]
        _lib = L
    return _lib


def tdma_module():
    """The reference's cythonized TDMA wrapper, or None if it was not built."""
    if _REF_DIR not in sys.path:
        sys.path.insert(0, _REF_DIR)
    try:
        import tdma_ref  # type: ignore
        return tdma_ref
    except ImportError:
        return None


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


class Table:
    """LookupStruct built by the reference init_table (Csrc/lookup.h:16-40)."""

    def __init__(self, x, y):
        self.x = np.ascontiguousarray(x, dtype=np.float64)
        self.y = np.ascontiguousarray(y, dtype=np.float64)
        self.ptr = lib().ref_table_new(len(self.y), _p(self.x), _p(self.y))

    def __del__(self):
        try:
            lib().ref_table_free(self.ptr)
        except Exception:
            pass

    def lookup(self, x):
        return lib().ref_table_lookup(self.ptr, float(x))


# --------------------------------------------------------------------------
# kernels, called as the reference glue calls them
# --------------------------------------------------------------------------
def advective_fluxes_a(d: Dims, rho0, rho0_half, vel, scalar, flux, direction, order):
    """compute_advective_fluxes_a (Csrc/scalar_advection.h:689-730)."""
    dc = d.c()
    lib().compute_advective_fluxes_a(ctypes.byref(dc), _p(rho0), _p(rho0_half), _p(vel), _p(scalar),
                                     _p(flux), int(direction), int(order))


def scalar_flux_divergence(d: Dims, alpha0, alpha0_half, flux, tend, dx, direction):
    """scalar_flux_divergence (Csrc/flux_divergence.h:4-32)."""
    dc = d.c()
    lib().scalar_flux_divergence(ctypes.byref(dc), _p(alpha0), _p(alpha0_half), _p(flux), _p(tend),
                                 float(dx), int(direction))


def advective_tendencies_m(d: Dims, rho0, rho0_half, alpha0, alpha0_half, vel_advected, vel_advecting,
                           tend, d_advected, d_advecting, order):
    """compute_advective_tendencies_m (Csrc/momentum_advection.h:13-93)."""
    dc = d.c()
    lib().compute_advective_tendencies_m(ctypes.byref(dc), _p(rho0), _p(rho0_half), _p(alpha0),
                                         _p(alpha0_half), _p(vel_advected), _p(vel_advecting), _p(tend),
                                         int(d_advected), int(d_advecting), int(order))


def clip_qt(d: Dims, qt, clip_value):
    dc = d.c()
    lib().clip_qt(ctypes.byref(dc), _p(qt), ctypes.c_double(clip_value))


def eos_update_sa(d: Dims, table: Table, p0, s, qt, T, qv, ql, qi, alpha):
    dc = d.c()
    lib().ref_eos_update(ctypes.byref(dc), ctypes.c_void_p(table.ptr), _p(p0), _p(s), _p(qt), _p(T),
                         _p(qv), _p(ql), _p(qi), _p(alpha))


def buoyancy_update_sa(d: Dims, alpha0, alpha, buoyancy, wt):
    dc = d.c()
    lib().buoyancy_update_sa(ctypes.byref(dc), _p(alpha0), _p(alpha), _p(buoyancy), _p(wt))


def bvf_sa(d: Dims, table: Table, p0, T, qt, qv, theta_rho, bvf):
    dc = d.c()
    lib().ref_bvf_sa(ctypes.byref(dc), ctypes.c_void_p(table.ptr), _p(p0), _p(T), _p(qt), _p(qv),
                     _p(theta_rho), _p(bvf))


def thetali_update(d: Dims, p0, T, qt, ql, qi, thetali):
    dc = d.c()
    lib().ref_thetali_update(ctypes.byref(dc), _p(p0), _p(T), _p(qt), _p(ql), _p(qi), _p(thetali))


def eos_update_dry(d: Dims, pd, s, T, alpha):
    dc = d.c()
    lib().dry_eos_update(ctypes.byref(dc), _p(pd), _p(s), _p(T), _p(alpha))


def buoyancy_update_dry(d: Dims, alpha0, alpha, buoyancy, wt):
    dc = d.c()
    lib().buoyancy_update(ctypes.byref(dc), _p(alpha0), _p(alpha), _p(buoyancy), _p(wt))


def bvf_dry(d: Dims, p0, T, theta, bvf):
    dc = d.c()
    lib().bvf_dry(ctypes.byref(dc), _p(p0), _p(T), _p(theta), _p(bvf))


def build_buffer(nv_index, dim, s, d: Dims, values, buffer):
    dc = d.c()
    lib().build_buffer(ctypes.c_long(nv_index), ctypes.c_long(dim), ctypes.c_long(s), ctypes.byref(dc),
                       _p(values), _p(buffer))


def buffer_to_values(dim, s, d: Dims, values, buffer):
    dc = d.c()
    lib().buffer_to_values(ctypes.c_ssize_t(dim), ctypes.c_ssize_t(s), ctypes.byref(dc), _p(values), _p(buffer))


def set_bcs(dim, s, bc_factor, d: Dims, values):
    dc = d.c()
    lib().set_bcs(ctypes.c_ssize_t(dim), ctypes.c_ssize_t(s), ctypes.c_double(bc_factor), ctypes.byref(dc),
                  _p(values))


def eos_c(table: Table, p0, s, qt):
    T = ctypes.c_double()
    qv = ctypes.c_double()
    ql = ctypes.c_double()
    qi = ctypes.c_double()
    lib().ref_eos_c(ctypes.c_void_p(table.ptr), p0, s, qt, ctypes.byref(T), ctypes.byref(qv),
                    ctypes.byref(ql), ctypes.byref(qi))
    return T.value, qv.value, ql.value, qi.value


def entropy_sa(p0, T, qt, ql, qi):
    return lib().ref_entropy_sa(p0, T, qt, ql, qi)


# ---- surface layer (Csrc/surface.h) ---------------------------------------
def compute_ustar(windspeed, buoyancy_flux, z0, zb):
    f = lib().ref_compute_ustar
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_double] * 4
    return f(windspeed, buoyancy_flux, z0, zb)


def compute_windspeed(d: Dims, u, v, speed, u0, v0, gustiness):
    dc = d.c()
    f = lib().ref_compute_windspeed
    f.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    f(ctypes.byref(dc), _p(u), _p(v), _p(speed), u0, v0, gustiness)


def entropyflux_from_thetaflux_qtflux(thetaflux, qtflux, p0_b, T_b, qt_b, qv_b):
    f = lib().ref_entropyflux
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_double] * 6
    b = np.broadcast_arrays(*[np.asarray(x, dtype=np.float64) for x in (thetaflux, qtflux, p0_b, T_b, qt_b,
                                                                         qv_b)])
    out = np.empty(b[0].shape)
    for idx in np.ndindex(out.shape):
        out[idx] = f(*[float(x[idx]) for x in b])
    return out


# ---- subgrid scale and diffusion (Csrc/kinematics.h, sgs.h, *_diffusion.h) --
def _fn(name, argtypes, restype=None):
    f = getattr(lib(), name)
    f.argtypes = argtypes
    f.restype = restype
    return f


def compute_velocity_gradient(d: Dims, v, vgrad, direction):
    dc = d.c()
    _fn("compute_velocity_gradient", [ctypes.c_void_p, _dp, _dp, ctypes.c_ssize_t])(
        ctypes.byref(dc), _p(v), _p(vgrad), direction)


def compute_strain_rate(d: Dims, vgrad, strain_rate):
    dc = d.c()
    _fn("compute_strain_rate", [ctypes.c_void_p, _dp, _dp])(ctypes.byref(dc), _p(vgrad), _p(strain_rate))


def compute_strain_rate_mag(d: Dims, strain_rate, strain_rate_mag):
    dc = d.c()
    _fn("compute_strain_rate_mag", [ctypes.c_void_p, _dp, _dp])(ctypes.byref(dc), _p(strain_rate),
                                                               _p(strain_rate_mag))


def smagorinsky_update(d: Dims, visc, diff, buoy_freq, strain_rate_mag, cs, prt, variant="plain", zl_half=None):
    dc = d.c()
    if variant == "plain":
        _fn("smagorinsky_update", [ctypes.c_void_p, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double])(
            ctypes.byref(dc), _p(visc), _p(diff), _p(buoy_freq), _p(strain_rate_mag), cs, prt)
    else:
        name = "smagorinsky_update_wall" if variant == "wall" else "smagorinsky_update_iles"
        _fn(name, [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double])(
            ctypes.byref(dc), _p(zl_half), _p(visc), _p(diff), _p(buoy_freq), _p(strain_rate_mag), cs, prt)


def compute_diffusive_flux(d: Dims, rho0, rho0_half, diffusivity, scalar, flux, dx, direction, factor):
    dc = d.c()
    _fn("compute_diffusive_flux", [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_ssize_t,
                                   ctypes.c_ssize_t, ctypes.c_double])(
        ctypes.byref(dc), _p(rho0), _p(rho0_half), _p(diffusivity), _p(scalar), _p(flux), dx, direction, 2, factor)


def compute_qt_diffusion_s_source(d: Dims, p0_half, alpha0, alpha0_half, flux, qt, qv, T, tendency, dx, direction):
    dc = d.c()
    _fn("ref_compute_qt_diffusion_s_source", [ctypes.c_void_p] + [_dp] * 8 + [ctypes.c_double, ctypes.c_ssize_t])(
        ctypes.byref(dc), _p(p0_half), _p(alpha0), _p(alpha0_half), _p(flux), _p(qt), _p(qv), _p(T), _p(tendency),
        dx, direction)


def compute_diffusive_flux_m(d: Dims, strain_rate, viscosity, flux, rho0, rho0_half, i1, i2):
    dc = d.c()
    _fn("compute_diffusive_flux_m", [ctypes.c_void_p] + [_dp] * 5 + [ctypes.c_ssize_t, ctypes.c_ssize_t])(
        ctypes.byref(dc), _p(strain_rate), _p(viscosity), _p(flux), _p(rho0), _p(rho0_half), i1, i2)


def momentum_flux_divergence(d: Dims, alpha0, alpha0_half, flux, tendency, d_advected, d_advecting):
    dc = d.c()
    _fn("momentum_flux_divergence", [ctypes.c_void_p] + [_dp] * 4 + [ctypes.c_ssize_t, ctypes.c_ssize_t])(
        ctypes.byref(dc), _p(alpha0), _p(alpha0_half), _p(flux), _p(tendency), d_advected, d_advecting)


def compute_entropy_source(d: Dims, viscosity, strain_rate_mag, temperature, entropy_tendency):
    dc = d.c()
    _fn("compute_entropy_source", [ctypes.c_void_p] + [_dp] * 4)(
        ctypes.byref(dc), _p(viscosity), _p(strain_rate_mag), _p(temperature), _p(entropy_tendency))


def s_tendency_c(p0, qt, qv, T, qt_tendency, T_tendency):
    f = _fn("ref_s_tendency", [ctypes.c_double] * 6, ctypes.c_double)
    b = np.broadcast_arrays(*[np.asarray(x, dtype=np.float64) for x in (p0, qt, qv, T, qt_tendency, T_tendency)])
    out = np.empty(b[0].shape)
    for idx in np.ndindex(out.shape):
        out[idx] = f(*[float(x[idx]) for x in b])
    return out
