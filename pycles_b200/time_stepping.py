"""TimeStepping (TimeStepping.pyx) -- SSP-RK3 with a fixed time step.

Adaptive time stepping (adjust_timestep, compute_cfl_max) is not part of the
hot path built here; the configurations run at fixed dt.
"""
from __future__ import annotations

import ctypes

import torch

from . import _capi


class TimeStepping:
    def __init__(self):
        self.rk_step = 0
        self.n_rk_steps = 3
        self.t = 0.0
        self.dt = 1.0
        self.value_copies = None
        self.fused_stages = 0  # stages run through the fused advection + RK3 kernels
        self.fused_values = None  # during a fused stage: the buffer its passes write the new values to

    def initialize(self, namelist, PV, Pa=None):
        ts = namelist["time_stepping"]
        self.ts_type = int(ts.get("ts_type", 3))
        if self.ts_type != 3:
            raise ValueError("only ts_type = 3 (SSP-RK3) is built")
        self.dt = float(ts.get("dt_initial", 1.0))
        self.dt_max = float(ts.get("dt_max", self.dt))
        self.t = float(ts.get("t", 0.0))
        self.t_max = float(ts.get("t_max", 0.0))
        self.n_rk_steps = 3
        self.value_copies = torch.zeros_like(PV.values).view(1, -1)

    def update(self, Gr, PV, Pa=None, stream=None, mark=None):
        """TimeStepping.update_third (TimeStepping.pyx:131-151).

        When the precision form's advection was deferred on PV (see
        PrognosticVariables), the stage runs as the advection passes that
        apply it: the scalars' passes, then the u, v, w pass, each writing the
        new values to PV's second value buffer; the w tendency (the
        thermodynamics' buoyancy) is consumed and cleared, and every other
        tendency was never stored, so all tendencies are left at zero as the
        reference leaves them.  The two value buffers then swap (or, with
        PV.stable_values, the new values are copied back so that PV.values
        keeps its device address).  mark(2) / mark(3), if given, are called
        after the scalar and the momentum passes; during the fused stage
        `fused_values` names the buffer that receives the new values."""
        pend = PV.take_pending_advection() if PV._pending else {}
        nscal = sum(1 for i in range(PV.nv) if PV.var_type[i] == 1)
        if "momentum" in pend and ("scalar" in pend or nscal == 0):
            self._fused_stage(Gr, PV, pend, stream, mark)
        else:
            if pend:  # not fusable: run what was recorded as plain advection
                PV._pending = pend
                PV.flush_advection()
            n = PV.nv * Gr.dims.npg
            rc = _capi.load().pb_rk3_update(_capi.ptr(PV.values), _capi.ptr(PV.tendencies),
                                            _capi.ptr(self.value_copies), n, self.dt, self.rk_step,
                                            _capi.stream_handle(stream))
            _capi.check(rc, "pb_rk3_update")
        if self.rk_step == 2:
            self.t += self.dt

    def _fused_stage(self, Gr, PV, pend, stream, mark):
        m = mark if mark is not None else (lambda i: None)
        npg = Gr.dims.npg
        L = _capi.load()
        sh = _capi.stream_handle(stream)
        nxt = PV.values_next
        if nxt is None or nxt.shape != PV.values.shape or nxt.device != PV.values.device:
            nxt = PV.values_next = torch.zeros_like(PV.values)
        cp = self.value_copies.view(-1)
        tend = PV._tendencies
        self.fused_values = nxt
        scal = [i for i in range(PV.nv) if PV.var_type[i] == 1]
        if scal:
            SA, _, Rs, _, _ = pend["scalar"]
            n = len(scal)
            arr = lambda t: (ctypes.c_void_p * n)(*[_capi.ptr(t[i * npg:]) for i in scal])
            rc = L.pb_scalar_advection_rk3(
                ctypes.byref(Gr.dims), _capi.ptr(Rs.d_rho0), _capi.ptr(Rs.d_rho0_half), _capi.ptr(Rs.d_alpha0),
                _capi.ptr(Rs.d_alpha0_half), _capi.ptr(PV.values[0:]), _capi.ptr(PV.values[npg:]),
                _capi.ptr(PV.values[2 * npg:]), n, arr(PV.values), arr(tend), arr(nxt), arr(cp), self.dt,
                self.rk_step, SA.order, sh)
            _capi.check(rc, "pb_scalar_advection_rk3")
            # the scalar passes leave the stage's advection tendency in the
            # tendency array; it is cleared before any plain update reads it
            PV._scalar_tendencies_stale = True
        m(2)
        MA, _, Rs, _, _ = pend["momentum"]
        rc = L.pb_momentum_advection_rk3(
            ctypes.byref(Gr.dims), _capi.ptr(Rs.d_rho0), _capi.ptr(Rs.d_rho0_half), _capi.ptr(Rs.d_alpha0),
            _capi.ptr(Rs.d_alpha0_half), _capi.ptr(PV.values[0:]), _capi.ptr(PV.values[npg:]),
            _capi.ptr(PV.values[2 * npg:]), _capi.ptr(tend[2 * npg:]), _capi.ptr(nxt[0:]), _capi.ptr(nxt[npg:]),
            _capi.ptr(nxt[2 * npg:]), _capi.ptr(cp[0:]), _capi.ptr(cp[npg:]), _capi.ptr(cp[2 * npg:]), self.dt,
            self.rk_step, MA.order, sh)
        _capi.check(rc, "pb_momentum_advection_rk3")
        st = stream if stream is not None else torch.cuda.current_stream(PV.values.device)
        with torch.cuda.stream(st):
            tend[2 * npg:3 * npg].zero_()  # the w tendency, consumed by the pass
        m(3)
        if PV.stable_values:
            with torch.cuda.stream(st):
                PV.values.copy_(nxt)
        else:
            PV.values, PV.values_next = nxt, PV.values
        self.fused_values = None
        self.fused_stages += 1
