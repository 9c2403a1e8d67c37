"""Case forcing (Forcing.pyx) with the update on the GPU.

``ForcingFactory`` picks the scheme by ``namelist['meta']['casename']`` as
Forcing.__init__ does (Forcing.pyx:29-67): SullivanPatton (Coriolis), Bomex
(large-scale pressure gradient, cooling and drying, subsidence) and
DYCOMS_RF01 (subsidence, Coriolis) are built; the reference's other schemes
raise NotImplementedError; no case name: no forcing.  The per-level profiles
are computed on the host in ``initialize`` with the reference's formulas and
kept on the device.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _capi

_OMEGA = 7.2921151467064e-5  # Earth's rotation rate, generate_parameters.py:38
_P_TILDE, _KAPPA = 100000.0, 0.2859561752988048


def _exner(p0):
    return math.pow(p0 / _P_TILDE, _KAPPA)


class ForcingNone:
    scheme = _capi.PB_FORCING_NONE

    def initialize(self, Gr, RS, Th=None, NS=None, Pa=None):
        return

    def update(self, Gr, RS, PV, DV, Pa=None, stream=None):
        return

    def stats_io(self, *args, **kwargs):
        return


class _ForcingBase(ForcingNone):
    def initialize(self, Gr, RS, Th=None, NS=None, Pa=None):
        z = np.asarray(Gr.zl_half, dtype=np.float64)
        n = len(z)
        prof = {k: np.zeros(n) for k in ("ug", "vg", "dtdt", "dqtdt", "subsidence")}
        self._profiles(z, np.asarray(RS.p0_half, dtype=np.float64), prof)
        dev = getattr(Gr, "device", "cuda")
        self.prof = {k: torch.as_tensor(v, dtype=torch.float64, device=dev) for k, v in prof.items()}
        self.host_profiles = prof
        self._stats = None

    def update(self, Gr, RS, PV, DV, Pa=None, stream=None):
        f = _capi.PbForcing(self.scheme, self.coriolis_param, float(RS.u0), float(RS.v0),
                            *[_capi.ptr(self.prof[k]) for k in ("ug", "vg", "dtdt", "dqtdt", "subsidence")])

        def pv(name, arr):
            return _capi.ptr(arr[PV.get_varshift(Gr, name):]) if name in PV.index_name else None

        def dv(name):
            return _capi.ptr(DV.values[DV.get_varshift(Gr, name):]) if name in DV.index_name else None

        umean = vmean = None
        if self.scheme == _capi.PB_FORCING_BOMEX:  # Forcing.pyx:176-177
            from .statistics import HorizontalStatistics
            if self._stats is None:
                self._stats = HorizontalStatistics(Gr)
            umean = self._stats.HorizontalMean(Gr, PV.field("u", Gr), stream=stream)
            vmean = self._stats.HorizontalMean(Gr, PV.field("v", Gr), stream=stream)
        rc = _capi.load().pb_forcing_update(
            ctypes.byref(Gr.dims), ctypes.byref(f), _capi.ptr(RS.d_p0_half), _capi.ptr(umean), _capi.ptr(vmean),
            pv("u", PV.values), pv("v", PV.values), pv("s", PV.values), pv("qt", PV.values), dv("ql"),
            dv("temperature"), pv("u", PV.tendencies), pv("v", PV.tendencies), pv("s", PV.tendencies),
            pv("qt", PV.tendencies), _capi.stream_handle(stream))
        _capi.check(rc, "pb_forcing_update")


class ForcingSullivanPatton(_ForcingBase):
    """Forcing.pyx:256-300: geostrophic wind (1, 0) m/s, f = 1e-4 1/s."""
    scheme = _capi.PB_FORCING_SULLIVAN_PATTON
    coriolis_param = 1.0e-4

    def _profiles(self, z, p0, P):
        P["ug"][:] = 1.0


class ForcingBomex(_ForcingBase):
    """Forcing.pyx:102-254."""
    scheme = _capi.PB_FORCING_BOMEX
    coriolis_param = 0.376e-4

    def _profiles(self, z, p0, P):  # Forcing.pyx:117-142
        for k in range(len(z)):
            P["ug"][k] = -10.0 + (1.8e-3) * z[k]
            ex = _exner(p0[k])
            if z[k] <= 1500.0:
                P["dtdt"][k] = (-2.0 / (3600 * 24.0)) * ex
            if z[k] > 1500.0:
                P["dtdt"][k] = (-2.0 / (3600 * 24.0) + (z[k] - 1500.0) * (0.0 - -2.0 / (3600 * 24.0))
                                / (3000.0 - 1500.0)) * ex
            if z[k] <= 300.0:
                P["dqtdt"][k] = -1.2e-8
            if 300.0 < z[k] <= 500.0:
                P["dqtdt"][k] = -1.2e-8 + (z[k] - 300.0) * (0.0 - -1.2e-8) / (500.0 - 300.0)
            if z[k] <= 1500.0:
                P["subsidence"][k] = 0.0 + z[k] * (-0.65 / 100.0 - 0.0) / (1500.0 - 0.0)
            if 1500.0 < z[k] <= 2100.0:
                P["subsidence"][k] = -0.65 / 100 + (z[k] - 1500.0) * (0.0 - -0.65 / 100.0) / (2100.0 - 1500.0)


class ForcingDyCOMS_RF01(_ForcingBase):
    """Forcing.pyx:346-460 (the RF01 profiles; RF02 is not built)."""
    scheme = _capi.PB_FORCING_DYCOMS_RF01
    coriolis_param = 2.0 * _OMEGA * math.sin(31.5 * math.pi / 180.0)

    def _profiles(self, z, p0, P):  # Forcing.pyx:373-378
        P["subsidence"][:] = -z * 3.75e-6
        P["ug"][:] = 7.0
        P["vg"][:] = -5.5


def ForcingFactory(namelist, LH=None, Pa=None):
    casename = (namelist or {}).get("meta", {}).get("casename")
    if casename == "SullivanPatton":
        return ForcingSullivanPatton()
    if casename == "Bomex":
        return ForcingBomex()
    if casename == "DYCOMS_RF01":
        return ForcingDyCOMS_RF01()
    if casename in ("Gabls", "DYCOMS_RF02", "Rico", "Isdac", "IsdacCC", "Mpace", "Sheba", "CGILS", "ZGILS"):
        raise NotImplementedError(f"forcing of case {casename!r} is not built in this library")
    return ForcingNone()
