"""ScalarAdvection and MomentumAdvection with the update on the GPU.

``update`` keeps the reference signatures (ScalarAdvection.pxd:20,
MomentumAdvection.pxd:12) so Simulation3d's call sites need no change.
"""
from __future__ import annotations

import ctypes

import torch

from . import _capi


def _precision(namelist):
    return _capi.precision_of(namelist)


class ScalarAdvection:
    """ScalarAdvection (ScalarAdvection.pyx:31-123), sedimentation excluded."""

    def __init__(self, namelist, LH=None, Pa=None):
        try:
            self.order = int(namelist["scalar_transport"]["order"])
        except KeyError as e:
            raise ValueError("scalar_transport order not given in namelist") from e
        self.precision = _precision(namelist)
        self.keep_fluxes = bool(namelist.get("gpu", {}).get("keep_scalar_fluxes", False))
        self.flux = None

    def initialize(self, Gr, PV, NS=None, Pa=None):
        if self.keep_fluxes:
            self.flux = torch.zeros(PV.nv_scalars * Gr.dims.npg * Gr.dims.dims, dtype=torch.float64,
                                    device=PV.values.device)

    def update(self, Gr, Rs, PV, DV=None, Pa=None, stream=None):
        """ScalarAdvection.update (ScalarAdvection.pyx:69-123).  Precision
        form with fused stages: recorded on PV and run by TimeStepping.update
        together with the SSP-RK3 stage (or when PV.tendencies is read)."""
        if self.precision == _capi.PB_FP32 and self.flux is None and PV.fused_stepping_ok():
            PV.defer_advection("scalar", self, Gr, Rs, DV, stream)
            return
        self.update_now(Gr, Rs, PV, DV, stream=stream)

    def update_now(self, Gr, Rs, PV, DV=None, stream=None):
        scal = [PV.index_name[i] for i in range(PV.nv) if PV.var_type[i] == 1]
        if not scal:
            return
        n = len(scal)
        sp = (ctypes.c_void_p * n)(*[_capi.ptr(PV.field(nm, Gr)) for nm in scal])
        tp = (ctypes.c_void_p * n)(*[_capi.ptr(PV.tendency(nm, Gr)) for nm in scal])
        vel = [PV.values[int(PV.velocity_directions[d]) * Gr.dims.npg:] for d in range(3)]
        rc = _capi.load().pb_scalar_advection(
            ctypes.byref(Gr.dims), _capi.ptr(Rs.d_rho0), _capi.ptr(Rs.d_rho0_half), _capi.ptr(Rs.d_alpha0),
            _capi.ptr(Rs.d_alpha0_half), _capi.ptr(vel[0]), _capi.ptr(vel[1]), _capi.ptr(vel[2]), n, sp, tp,
            _capi.ptr(self.flux) if self.flux is not None else None, self.order, self.precision,
            _capi.stream_handle(stream))
        _capi.check(rc, "pb_scalar_advection")


class MomentumAdvection:
    """MomentumAdvection (MomentumAdvection.pyx:20-69)."""

    def __init__(self, namelist, Pa=None):
        try:
            self.order = int(namelist["momentum_transport"]["order"])
        except KeyError as e:
            raise ValueError("momentum_transport order not given in namelist") from e
        self.precision = _precision(namelist)

    def initialize(self, Gr, PV, NS=None, Pa=None):
        return

    def update(self, Gr, Rs, PV, Pa=None, stream=None):
        """MomentumAdvection.update (MomentumAdvection.pyx:41-69).  Precision
        form with fused stages: recorded on PV and run by TimeStepping.update
        together with the SSP-RK3 stage (or when PV.tendencies is read)."""
        if self.precision == _capi.PB_FP32 and PV.fused_stepping_ok():
            PV.defer_advection("momentum", self, Gr, Rs, None, stream)
            return
        self.update_now(Gr, Rs, PV, stream=stream)

    def update_now(self, Gr, Rs, PV, DV=None, stream=None):
        npg = Gr.dims.npg
        vs = [int(PV.velocity_directions[d]) * npg for d in range(3)]
        rc = _capi.load().pb_momentum_advection(
            ctypes.byref(Gr.dims), _capi.ptr(Rs.d_rho0), _capi.ptr(Rs.d_rho0_half), _capi.ptr(Rs.d_alpha0),
            _capi.ptr(Rs.d_alpha0_half), _capi.ptr(PV.values[vs[0]:]), _capi.ptr(PV.values[vs[1]:]),
            _capi.ptr(PV.values[vs[2]:]), _capi.ptr(PV.tendencies[vs[0]:]), _capi.ptr(PV.tendencies[vs[1]:]),
            _capi.ptr(PV.tendencies[vs[2]:]), self.order, self.precision, _capi.stream_handle(stream))
        _capi.check(rc, "pb_momentum_advection")
