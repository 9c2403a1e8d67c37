"""Radiation (Radiation.pyx) with the update on the GPU: RadiationFactory
(Radiation.pyx:30-57) gives the DYCOMS_RF01 and DYCOMS_RF02 cases the
DYCOMS radiation (Radiation.pyx:230-353), built here; RRTM and the SMOKE and
Isdac schemes raise NotImplementedError; every other case has none."""
from __future__ import annotations

import ctypes

import torch

from . import _capi


class RadiationNone:
    active = False

    def initialize(self, Gr, NS=None, Pa=None):
        return

    def initialize_profiles(self, *args, **kwargs):
        return

    def update(self, Gr, Ref, PV, DV, Sur=None, TS=None, Pa=None, stream=None):
        return

    def stats_io(self, *args, **kwargs):
        return


class RadiationDyCOMS_RF01(RadiationNone):
    active = True

    def __init__(self, namelist=None):
        self.params = _capi.PbDycomsRadiation(
            float((namelist or {}).get("radiation", {}).get("dycoms_f0", 70.0)), 22.0, 85.0, 1.0, 3.75e-6)

    def initialize(self, Gr, NS=None, Pa=None):
        """RadiationBase.initialize (Radiation.pyx:65-70): heating rate and
        temperature tendency, npg each."""
        dev = getattr(Gr, "device", "cuda")
        self.heating_rate = torch.zeros(Gr.dims.npg, dtype=torch.float64, device=dev)
        self.dTdt_rad = torch.zeros(Gr.dims.npg, dtype=torch.float64, device=dev)
        self._z = torch.as_tensor(Gr.z, dtype=torch.float64, device=dev).contiguous()

    def update(self, Gr, Ref, PV, DV, Sur=None, TS=None, Pa=None, stream=None):
        dv = lambda n: _capi.ptr(DV.values[DV.get_varshift(Gr, n):])
        rc = _capi.load().pb_dycoms_radiation(
            ctypes.byref(Gr.dims), ctypes.byref(self.params), _capi.ptr(Ref.d_rho0_half), _capi.ptr(self._z),
            dv("ql"), _capi.ptr(PV.values[PV.get_varshift(Gr, "qt"):]), dv("temperature"),
            _capi.ptr(PV.tendencies[PV.get_varshift(Gr, "s"):]), _capi.ptr(self.heating_rate),
            _capi.ptr(self.dTdt_rad), _capi.stream_handle(stream))
        _capi.check(rc, "pb_dycoms_radiation")


def RadiationFactory(namelist, LH=None, Pa=None):
    rad = (namelist or {}).get("radiation", {})
    if rad.get("use_RRTM", False):
        raise NotImplementedError("RRTM radiation is not built in this library")
    casename = (namelist or {}).get("meta", {}).get("casename")
    if casename in ("DYCOMS_RF01", "DYCOMS_RF02"):
        return RadiationDyCOMS_RF01(namelist)
    if casename in ("SMOKE", "Isdac", "IsdacCC", "CGILS", "ZGILS"):
        raise NotImplementedError(f"radiation of case {casename!r} is not built in this library")
    return RadiationNone()
