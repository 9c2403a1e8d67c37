"""TimeStepping (TimeStepping.pyx) -- SSP-RK3 with a fixed time step.

Adaptive time stepping (adjust_timestep, compute_cfl_max) is not part of the
hot path built here; the configurations run at fixed dt.
"""
from __future__ import annotations

import torch

from . import _capi


class TimeStepping:
    def __init__(self):
        self.rk_step = 0
        self.n_rk_steps = 3
        self.t = 0.0
        self.dt = 1.0
        self.value_copies = None

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

    def update(self, Gr, PV, Pa=None, stream=None):
        """TimeStepping.update_third (TimeStepping.pyx:131-151)."""
        n = PV.nv * Gr.dims.npg
        rc = _capi.load().pb_rk3_update(_capi.ptr(PV.values), _capi.ptr(PV.tendencies),
                                        _capi.ptr(self.value_copies), n, self.dt, self.rk_step,
                                        _capi.stream_handle(stream))
        _capi.check(rc, "pb_rk3_update")
        if self.rk_step == 2:
            self.t += self.dt
