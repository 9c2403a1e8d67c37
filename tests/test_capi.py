"""The C-ABI library: it loads, exports every entry point include/*.h
declares, and rejects invalid arguments before touching a device (no GPU
needed for any of these)."""
import ctypes
import glob
import os
import re

import pytest

from helpers import ROOT

from pycles_b200 import _capi
from pycles_b200.grid import Grid
from pycles_b200.simulation import namelist_for


def _declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*[\s\*]+(pb_[A-Za-z0-9_]+)\s*\(", txt, re.M):
            names.add(m.group(1))
    return names


def test_library_builds_and_loads():
    L = _capi.load()
    assert os.path.exists(_capi.lib_path())
    assert L.pb_status_string(0) == b"ok"


def test_every_declared_symbol_is_exported():
    L = _capi.load()
    declared = _declared_functions()
    assert len(declared) >= 12
    for name in declared:
        assert hasattr(L, name), name
        assert name in _capi.SIGNATURES, f"{name} has no ctypes signature"


def test_dims_struct_matches_reference_layout():
    # DimStruct (Csrc/grid.h): 1 + 4*3 + 4 + 4*3 longs, then 6 doubles
    assert ctypes.sizeof(_capi.PbDims) == (1 + 12 + 4 + 12) * 8 + 6 * 8
    # pb_surface: int (padded to 8) + 9 doubles; pb_surface_fields: 11 pointers
    assert ctypes.sizeof(_capi.PbSurface) == 8 + 9 * 8
    assert ctypes.sizeof(_capi.PbSurfaceFields) == 11 * 8


def test_workspace_size_and_dims_validation():
    L = _capi.load()
    Gr = Grid(namelist_for("bomex", 64, 64, 75, 100.0, 100.0, 40.0))
    n = L.pb_pressure_workspace_bytes(ctypes.byref(Gr.dims))
    assert n >= (64 // 2 + 1) * 64 * 75 * 24  # complex x-half-spectrum + FP64 Thomas scratch
    bad = Grid(namelist_for("bomex", 64, 64, 75, 100.0, 100.0, 40.0))
    bad.dims.nlg[0] = 3
    assert L.pb_pressure_workspace_bytes(ctypes.byref(bad.dims)) == -1


def test_invalid_arguments_rejected_without_device():
    L = _capi.load()
    Gr = Grid(namelist_for("bomex", 16, 16, 16, 100.0, 100.0, 40.0))
    d = ctypes.byref(Gr.dims)
    assert L.pb_momentum_advection(d, None, None, None, None, None, None, None, None, None, None, 5, 0,
                                   None) == _capi.PB_ERR_ARG
    p = ctypes.c_void_p(16)  # never dereferenced: rejected before any launch
    assert L.pb_momentum_advection(d, p, p, p, p, p, p, p, p, p, p, 9, 0, None) == _capi.PB_ERR_UNSUPPORTED
    assert L.pb_momentum_advection(d, p, p, p, p, p, p, p, p, p, p, 5, 7, None) == _capi.PB_ERR_ARG
    Gr3 = Grid(namelist_for("bomex", 16, 16, 16, 100.0, 100.0, 40.0, gw=3))
    assert L.pb_scalar_advection(ctypes.byref(Gr3.dims), p, p, p, p, p, p, p, 0, None, None, None, 7, 0,
                                 None) == _capi.PB_ERR_UNSUPPORTED  # WENO7 needs gw >= 4
    assert L.pb_rk3_update(p, p, p, 10, 1.0, 3, None) == _capi.PB_ERR_ARG
    assert L.pb_pressure_solve(d, p, p, p, p, p, p, p, p, p, None, 0, 0, 0, None) == _capi.PB_ERR_WORKSPACE
    assert L.pb_status_string(3) == b"unsupported configuration"
    sc = _capi.PbSurface(_capi.PB_SURFACE_NONE)
    assert L.pb_surface_update(d, ctypes.byref(sc), *([None] * 14), None, None) == _capi.PB_OK
    sc.scheme = 9
    assert L.pb_surface_update(d, ctypes.byref(sc), *([p] * 14), None, None) == _capi.PB_ERR_ARG
    fields = _capi.PbSurfaceFields(*([16] * len(_capi.SURFACE_FIELDS)))
    sc.scheme = _capi.PB_SURFACE_BOMEX  # moist: needs qt, qv, ql and the qt tendency
    args = [p] * 14
    args[7] = None  # qt
    assert L.pb_surface_update(d, ctypes.byref(sc), *args, ctypes.byref(fields), None) == _capi.PB_ERR_ARG
    assert L.pb_horizontal_stat(d, _capi.PB_STAT_MEAN, p, None, None, None, p, None, 0, None) == \
        _capi.PB_ERR_WORKSPACE
    assert L.pb_horizontal_stat(d, _capi.PB_STAT_MEAN_CUBES, p, p, None, None, p, p, 1 << 30, None) == \
        _capi.PB_ERR_ARG
    assert L.pb_horizontal_stat(d, 99, p, p, p, p, p, p, 1 << 30, None) == _capi.PB_ERR_ARG
    assert L.pb_stat_workspace_bytes(d) == 2 * 296 * Gr.dims.nlg[2] * 8
    fields.scratch = None
    sc.scheme = _capi.PB_SURFACE_SULLIVAN_PATTON
    assert L.pb_surface_update(d, ctypes.byref(sc), *([p] * 14), ctypes.byref(fields), None) == _capi.PB_ERR_ARG


def test_no_cpu_fallback():
    """The product path refuses CPU tensors instead of computing on the host."""
    import torch
    with pytest.raises(_capi.PbError):
        _capi.ptr(torch.zeros(4))
