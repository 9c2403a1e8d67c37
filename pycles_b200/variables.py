"""PrognosticVariables / DiagnosticVariables held in GPU memory.

Same bookkeeping as PrognosticVariables.pyx:18-79 and
DiagnosticVariables.pyx:20-57 (name_index, bc_type, var_type,
velocity_directions, flat [var][npg] arrays); ``values`` and ``tendencies``
are CUDA float64 tensors instead of numpy arrays.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi


class PrognosticVariables:
    def __init__(self, Gr):
        self.name_index = {}
        self.index_name = []
        self.units = {}
        self.nice_name = {}
        self.desc = {}
        self.nv = 0
        self.nv_scalars = 0
        self.nv_velocities = 0
        self.bc_type = np.array([], dtype=np.double)
        self.var_type = np.array([], dtype=np.int64)
        self.velocity_directions = np.zeros((Gr.dims.dims,), dtype=np.int64)
        self.velocity_names_directional = ["" for _ in range(Gr.dims.dims)]
        self.values = None
        self._tendencies = None
        # Deferred advection of the precision form.  ScalarAdvection.update
        # and MomentumAdvection.update record their work here instead of
        # launching when fused stepping is possible (fuse_stages, velocities
        # first); TimeStepping.update then runs the advection kernels that
        # apply the SSP-RK3 stage in the same pass.  Reading `tendencies`
        # (as the surface, subgrid-scale, forcing and radiation updates do
        # between the advection and the time step) first launches the
        # recorded work as plain advection, so every caller sees the
        # reference's tendencies.
        self.fuse_stages = True
        self.stable_values = False  # fused stages copy the new values back instead of swapping buffers
        self.values_next = None     # second value buffer of fused stages
        self._pending = {}
        self._scalar_tendencies_stale = False

    @property
    def tendencies(self):
        if self._pending:
            self.flush_advection()
        if self._scalar_tendencies_stale:
            self._clear_stale_scalar_tendencies()
        return self._tendencies

    def _clear_stale_scalar_tendencies(self):
        """A fused stage leaves its scalar advection tendency behind (the
        scalar passes hand it from one direction to the next); the
        reference's time step leaves zeros.  Cleared before the first read."""
        self._scalar_tendencies_stale = False
        npg = self._tendencies.numel() // max(self.nv, 1)
        for i in range(self.nv):
            if self.var_type[i] == 1:
                self._tendencies[i * npg:(i + 1) * npg].zero_()

    @tendencies.setter
    def tendencies(self, t):
        self._tendencies = t

    def fused_stepping_ok(self):
        """Whether advection may be deferred into the time step: fused stages
        on and u, v, w the first three variables."""
        return self.fuse_stages and [int(i) for i in self.velocity_directions] == [0, 1, 2]

    def defer_advection(self, kind, component, Gr, Rs, DV=None, stream=None):
        self._pending[kind] = (component, Gr, Rs, DV, stream)

    def take_pending_advection(self):
        pend, self._pending = self._pending, {}
        return pend

    def flush_advection(self):
        """Launch deferred advection as plain (unfused) updates, scalars first
        as the reference calls them."""
        pend = self.take_pending_advection()
        for kind in ("scalar", "momentum"):
            if kind in pend:
                comp, Gr, Rs, DV, stream = pend[kind]
                comp.update_now(Gr, Rs, self, DV, stream=stream)

    def add_variable(self, name, units, nice_name, desc, bc_type, var_type, Pa=None):
        """PrognosticVariables.add_variable (PrognosticVariables.pyx:34-64)."""
        self.name_index[name] = self.nv
        self.index_name.append(name)
        self.units[name] = units
        self.nice_name[name] = nice_name
        self.desc[name] = desc
        self.nv = len(self.name_index)
        if bc_type == "sym":
            self.bc_type = np.append(self.bc_type, [1.0])
        elif bc_type == "asym":
            self.bc_type = np.append(self.bc_type, [-1.0])
        else:
            raise ValueError("Not a valid bc_type")
        if var_type == "velocity":
            self.var_type = np.append(self.var_type, 0)
            self.nv_velocities += 1
        elif var_type == "scalar":
            self.var_type = np.append(self.var_type, 1)
            self.nv_scalars += 1
        else:
            raise ValueError("Not a valid var_type")

    def set_velocity_direction(self, name, direction, Pa=None):
        self.velocity_directions[direction] = self.name_index[name]
        self.velocity_names_directional[direction] = name

    def initialize(self, Gr, NS=None, Pa=None, device="cuda"):
        npg = Gr.dims.npg
        self.values = torch.zeros(self.nv * npg, dtype=torch.float64, device=device)
        self.tendencies = torch.zeros(self.nv * npg, dtype=torch.float64, device=device)

    def get_nv(self, name):
        return self.name_index[name]

    def get_varshift(self, Gr, name):
        return self.name_index[name] * Gr.dims.npg

    def get_variable_array(self, name, Gr):
        i = self.name_index[name]
        npg = Gr.dims.npg
        return self.values[i * npg:(i + 1) * npg].view(*Gr.shape)

    def get_tendency_array(self, name, Gr):
        return self.tendency(name, Gr).view(*Gr.shape)

    def field(self, name, Gr):
        i = self.name_index[name]
        return self.values[i * Gr.dims.npg:(i + 1) * Gr.dims.npg]

    def tendency(self, name, Gr):
        i = self.name_index[name]
        if self._pending:
            self.flush_advection()
        if self.var_type[i] == 1 and self._scalar_tendencies_stale:
            self._clear_stale_scalar_tendencies()
        return self._tendencies[i * Gr.dims.npg:(i + 1) * Gr.dims.npg]

    def Update_all_bcs(self, Gr, Pa=None, stream=None):
        """PrognosticVariables.update_all_bcs (PrognosticVariables.pyx:183-233)."""
        bc = (ctypes.c_double * self.nv)(*[float(b) for b in self.bc_type])
        _capi.check(_capi.load().pb_update_all_bcs(ctypes.byref(Gr.dims), _capi.ptr(self.values), bc, self.nv,
                                                   _capi.stream_handle(stream)), "pb_update_all_bcs")

    update_all_bcs = Update_all_bcs

    def update_bcs_range(self, Gr, first, count, stream=None, values=None):
        """Ghost fill of the variables first .. first+count-1 only, of
        PV.values or of another buffer of the same layout."""
        bc = (ctypes.c_double * count)(*[float(b) for b in self.bc_type[first:first + count]])
        base = (self.values if values is None else values)[first * Gr.dims.npg:]
        _capi.check(_capi.load().pb_update_all_bcs(ctypes.byref(Gr.dims), _capi.ptr(base), bc, count,
                                                   _capi.stream_handle(stream)), "pb_update_all_bcs")


class DiagnosticVariables:
    def __init__(self):
        self.name_index = {}
        self.index_name = []
        self.units = {}
        self.nv = 0
        self.bc_type = np.array([], dtype=np.double)
        self.values = None
        self._npg = None

    def add_variables(self, name, units, nice_name, desc, bc_type, Pa=None):
        """DiagnosticVariables.add_variables (DiagnosticVariables.pyx:39-57)."""
        if name in self.name_index:
            return
        self.name_index[name] = self.nv
        self.index_name.append(name)
        self.units[name] = units
        if bc_type == "sym":
            self.bc_type = np.append(self.bc_type, [1.0])
        elif bc_type == "asym":
            self.bc_type = np.append(self.bc_type, [-1.0])
        else:
            raise ValueError("Not a valid bc_type")
        self.nv = len(self.name_index)
        if self.values is not None:  # grow an already allocated array
            extra = torch.zeros(self._npg, dtype=self.values.dtype, device=self.values.device)
            self.values = torch.cat([self.values, extra])

    def initialize(self, Gr, NS=None, Pa=None, device="cuda"):
        self._npg = Gr.dims.npg
        self.values = torch.zeros(self.nv * Gr.dims.npg, dtype=torch.float64, device=device)

    def get_varshift(self, Gr, name):
        return self.name_index[name] * Gr.dims.npg

    def field(self, name, Gr):
        i = self.name_index[name]
        return self.values[i * Gr.dims.npg:(i + 1) * Gr.dims.npg]

    def get_variable_array(self, name, Gr):
        return self.field(name, Gr).view(*Gr.shape)

    def communicate_variable(self, Gr, PM, nv, stream=None):
        """DiagnosticVariables.communicate_variable (DiagnosticVariables.pyx:65-112)."""
        bc = (ctypes.c_double * 1)(float(self.bc_type[nv]))
        f = self.values[nv * Gr.dims.npg:(nv + 1) * Gr.dims.npg]
        _capi.check(_capi.load().pb_update_all_bcs(ctypes.byref(Gr.dims), _capi.ptr(f), bc, 1,
                                                   _capi.stream_handle(stream)), "pb_update_all_bcs")
