"""Surface fluxes (Surface.pyx) with the update on the GPU.

``SurfaceFactory`` picks the scheme by ``namelist['meta']['casename']`` as the
reference does (Surface.pyx:39-74); the schemes built are SullivanPatton
(dry, Monin-Obukhov friction velocity), Bomex (fixed friction velocity and
fluxes) and DYCOMS_RF01 (bulk formulae), each with SurfaceBase.update (the
fluxes' tendencies on the first interior level).  The reference's other
schemes raise NotImplementedError; any other case name, or none, gets
``SurfaceNone`` as in the reference.  The per-column arrays of SurfaceBase
(u_flux, v_flux, qt_flux, s_flux, obukhov_length, friction_velocity, shf,
lhf, b_flux) are device tensors of nlg0*nlg1 doubles, indexed i*nlg1 + j.
"""
from __future__ import annotations

import ctypes

import torch

from . import _capi


class SurfaceBase:
    scheme = _capi.PB_SURFACE_NONE
    dry_case = True

    def __init__(self):
        self.theta_flux = 0.0
        self.z0 = 0.0
        self.gustiness = 0.0
        self.ustar_ = 0.0
        self.cm = self.ft = self.fq = 0.0
        self.fields = {}

    def initialize(self, Gr, Ref, NS=None, Pa=None):
        """SurfaceBase.initialize (Surface.pyx:82-113): the per-column arrays,
        zeroed, plus the scratch of the lowest-level temperature mean."""
        n2 = int(Gr.dims.nlg[0] * Gr.dims.nlg[1])
        dev = getattr(Gr, "device", "cuda")
        for n in _capi.SURFACE_FIELDS:
            size = _capi.PB_SURFACE_SCRATCH if n == "scratch" else n2
            self.fields[n] = torch.zeros(size, dtype=torch.float64, device=dev)
        for n in _capi.SURFACE_FIELDS[:9]:
            setattr(self, n, self.fields[n])
        self.T_surface = getattr(Ref, "Tg", None)

    def _struct(self, Ref):
        return _capi.PbSurface(self.scheme, self.theta_flux, self.z0, self.gustiness, self.ustar_, self.cm,
                               self.ft, self.fq, float(getattr(Ref, "u0", 0.0)), float(getattr(Ref, "v0", 0.0)))

    def update(self, Gr, Ref, PV, DV, Pa=None, TS=None, stream=None):
        """Surface<scheme>.update + SurfaceBase.update in one library call."""
        if self.scheme == _capi.PB_SURFACE_NONE:
            return
        L = _capi.load()

        def pv(name):
            return _capi.ptr(PV.values[PV.get_varshift(Gr, name):]) if name in PV.index_name else None

        def pt(name):
            return _capi.ptr(PV.tendencies[PV.get_varshift(Gr, name):]) if name in PV.index_name else None

        def dv(name):
            return _capi.ptr(DV.values[DV.get_varshift(Gr, name):]) if name in DV.index_name else None

        f = _capi.PbSurfaceFields(*[_capi.ptr(self.fields[n]) for n in _capi.SURFACE_FIELDS])
        sc = self._struct(Ref)
        rc = L.pb_surface_update(ctypes.byref(Gr.dims), ctypes.byref(sc), _capi.ptr(Ref.d_p0_half),
                                 _capi.ptr(Ref.d_alpha0), _capi.ptr(Ref.d_alpha0_half), _capi.ptr(Ref.d_rho0_half),
                                 pv("u"), pv("v"), dv("temperature"), pv("qt"), dv("qv"), dv("ql"), pt("u"),
                                 pt("v"), pt("s"), pt("qt"), ctypes.byref(f), _capi.stream_handle(stream))
        _capi.check(rc, "pb_surface_update")

    def stats_io(self, Gr, NS=None, Pa=None):
        """Statistics output is not part of this library."""
        return


class SurfaceNone(SurfaceBase):
    """Surface.pyx:203-213."""

    def initialize(self, Gr, Ref, NS=None, Pa=None):
        return


class SurfaceSullivanPatton(SurfaceBase):
    """Surface.pyx:216-294: dry; theta flux 0.24 K m/s, roughness length
    0.1 m, gustiness 0.001 m/s."""
    scheme = _capi.PB_SURFACE_SULLIVAN_PATTON
    dry_case = True

    def __init__(self, LH=None):
        super().__init__()
        self.theta_flux = 0.24
        self.z0 = 0.1
        self.gustiness = 0.001


class SurfaceBomex(SurfaceBase):
    """Surface.pyx:297-377: theta flux 8e-3 K m/s, qt flux 5.2e-5 m/s,
    friction velocity 0.28 m/s (gustiness is never set: 0)."""
    scheme = _capi.PB_SURFACE_BOMEX
    dry_case = False

    def __init__(self, LH=None):
        super().__init__()

    def initialize(self, Gr, Ref, NS=None, Pa=None):
        super().initialize(Gr, Ref, NS, Pa)
        self.qt_flux.add_(5.2e-5)  # Surface.pyx:306
        self.theta_flux = 8.0e-3
        self.ustar_ = 0.28
        self.theta_surface = 299.1
        self.qt_surface = 22.45e-3


class SurfaceDYCOMS_RF01(SurfaceBase):
    """Surface.pyx:474-561: bulk drag coefficient 0.0011, sensible and latent
    heat fluxes 15 and 115 W/m^2, no gustiness."""
    scheme = _capi.PB_SURFACE_DYCOMS_RF01
    dry_case = False

    def __init__(self, namelist=None, LH=None):
        super().__init__()
        self.ft = 15.0
        self.fq = 115.0
        self.gustiness = 0.0
        self.cm = 0.0011

    def initialize(self, Gr, Ref, NS=None, Pa=None):
        super().initialize(Gr, Ref, NS, Pa)
        self.T_surface = 292.5


def SurfaceFactory(namelist, LH=None, Par=None):
    """Surface.pyx:39-74 restricted to the schemes built here (the
    reference's other schemes raise NotImplementedError); an unknown case
    name gets SurfaceNone, and so does a namelist without one."""
    casename = (namelist or {}).get("meta", {}).get("casename")
    if casename == "SullivanPatton":
        return SurfaceSullivanPatton(LH)
    if casename == "Bomex":
        return SurfaceBomex(LH)
    if casename == "DYCOMS_RF01":
        return SurfaceDYCOMS_RF01(namelist, LH)
    if casename in ("Gabls", "DYCOMS_RF02", "Rico", "Isdac", "IsdacCC", "Mpace", "Sheba", "CGILS", "ZGILS"):
        raise NotImplementedError(f"surface scheme of case {casename!r} is not built in this library")
    return SurfaceNone()
