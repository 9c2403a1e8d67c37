"""PressureSolver (PressureSolver.pyx:22-80) with the solve on the GPU.

The reference's PressureFFTParallel pencils become the single-GPU layout
inside ``pb_pressure_solve``; this class owns the device workspace (the
spectral array, the Thomas scratch and the grid constants that
PressureFFTParallel.initialize computes).
"""
from __future__ import annotations

import ctypes

import torch

from . import _capi


class PressureSolver:
    def __init__(self, namelist=None):
        self.workspace = None
        gpu = (namelist or {}).get("gpu", {})
        p = str(gpu.get("precision", "fp64")).lower()
        self.precision = _capi.PB_FP32 if p in ("fp32", "mixed", "precision") else _capi.PB_FP64
        self.refine_sweeps = int(gpu.get("pressure_refine_sweeps", 1))

    def initialize(self, namelist, Gr, RS, DV, PM=None):
        DV.add_variables("dynamic_pressure", "Pa", "p", "dynamic pressure", "sym", PM)
        DV.add_variables("divergence", "1/s", "d", "3d divergence", "sym", PM)

    def _ensure_workspace(self, Gr, device):
        L = _capi.load()
        nbytes = int(L.pb_pressure_workspace_bytes(ctypes.byref(Gr.dims)))
        if nbytes < 0:
            raise _capi.PbError("invalid grid for the pressure solver")
        if self.workspace is None or self.workspace.numel() < nbytes or self.workspace.device != device:
            # torch's caching allocator returns 512-byte aligned blocks
            self.workspace = torch.empty(nbytes, dtype=torch.uint8, device=device)
            _capi.check(L.pb_pressure_init(ctypes.byref(Gr.dims), _capi.ptr(self.workspace), nbytes),
                        "pb_pressure_init")
        return nbytes

    def update(self, Gr, RS, DV, PV, PM=None, stream=None):
        """PressureSolver.update (PressureSolver.pyx:38-80)."""
        self.solve(Gr, RS, DV, PV, stream=stream)
        PV.update_all_bcs(Gr, PM, stream=stream)

    def solve(self, Gr, RS, DV, PV, stream=None):
        """PressureSolver.update up to its final ghost fill of PV."""
        nbytes = self._ensure_workspace(Gr, PV.values.device)
        u, v, w = (PV.field(n, Gr) for n in PV.velocity_names_directional)
        rc = _capi.load().pb_pressure_solve(
            ctypes.byref(Gr.dims), _capi.ptr(RS.d_rho0), _capi.ptr(RS.d_rho0_half), _capi.ptr(RS.d_alpha0),
            _capi.ptr(RS.d_alpha0_half), _capi.ptr(u), _capi.ptr(v), _capi.ptr(w),
            _capi.ptr(DV.field("divergence", Gr)), _capi.ptr(DV.field("dynamic_pressure", Gr)),
            _capi.ptr(self.workspace), nbytes, self.precision, self.refine_sweeps, _capi.stream_handle(stream))
        _capi.check(rc, "pb_pressure_solve")
