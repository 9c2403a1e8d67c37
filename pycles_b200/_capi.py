"""ctypes binding of libpycles_b200.so (the C ABI of include/pycles_b200.h).

There is no fallback: if the library is missing or a call fails, this
module raises.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

_L3 = ctypes.c_long * 3
_D3 = ctypes.c_double * 3
_vp = ctypes.c_void_p


class PbDims(ctypes.Structure):
    """struct pb_dims == struct DimStruct (Csrc/grid.h:2-24), field for field."""
    _fields_ = [
        ("dims", ctypes.c_long),
        ("n", _L3), ("ng", _L3), ("nl", _L3), ("nlg", _L3),
        ("npd", ctypes.c_long), ("npl", ctypes.c_long), ("npg", ctypes.c_long),
        ("gw", ctypes.c_long),
        ("indx_lo", _L3), ("indx_lo_g", _L3),
        ("nbuffer", _L3), ("ghosted_stride", _L3),
        ("dx", _D3), ("dxi", _D3),
    ]


class PbTable(ctypes.Structure):
    _fields_ = [("y", _vp), ("n", ctypes.c_long), ("x_min", ctypes.c_double),
                ("dx", ctypes.c_double), ("dxi", ctypes.c_double)]


class PbMlp(ctypes.Structure):
    _fields_ = [("w1", _vp), ("b1", _vp), ("w2", _vp), ("b2", _vp), ("w3", _vp), ("b3", _vp),
                ("in_lo", ctypes.c_float * 3), ("in_hi", ctypes.c_float * 3),
                ("out_mean", ctypes.c_float), ("out_scale", ctypes.c_float), ("seed_y", _vp),
                ("seed_refresh", ctypes.c_int)]


class PbSurface(ctypes.Structure):
    _fields_ = [("scheme", ctypes.c_int), ("theta_flux", ctypes.c_double), ("z0", ctypes.c_double),
                ("gustiness", ctypes.c_double), ("ustar", ctypes.c_double), ("cm", ctypes.c_double),
                ("ft", ctypes.c_double), ("fq", ctypes.c_double), ("u0", ctypes.c_double),
                ("v0", ctypes.c_double)]


SURFACE_FIELDS = ("u_flux", "v_flux", "qt_flux", "s_flux", "obukhov_length", "friction_velocity", "shf",
                  "lhf", "b_flux", "windspeed", "scratch")


class PbSurfaceFields(ctypes.Structure):
    _fields_ = [(n, _vp) for n in SURFACE_FIELDS]


PB_OK, PB_ERR_ARG, PB_ERR_CUDA, PB_ERR_UNSUPPORTED, PB_ERR_WORKSPACE = 0, 1, 2, 3, 4
PB_FP64, PB_FP32 = 0, 1
PB_SURFACE_NONE, PB_SURFACE_SULLIVAN_PATTON, PB_SURFACE_BOMEX, PB_SURFACE_DYCOMS_RF01 = 0, 1, 2, 3
PB_SURFACE_SCRATCH = 512
PB_SGS_UNIFORM, PB_SGS_SMAGORINSKY = 1, 2
PB_FORCING_NONE, PB_FORCING_SULLIVAN_PATTON, PB_FORCING_BOMEX, PB_FORCING_DYCOMS_RF01 = 0, 1, 2, 3


class PbDycomsRadiation(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("f0", "f1", "kap", "alpha_z", "divergence")]


class PbForcing(ctypes.Structure):
    _fields_ = [("scheme", ctypes.c_int), ("coriolis_param", ctypes.c_double), ("u0", ctypes.c_double),
                ("v0", ctypes.c_double), ("ug", _vp), ("vg", _vp), ("dtdt", _vp), ("dqtdt", _vp),
                ("subsidence", _vp)]
(PB_STAT_MEAN, PB_STAT_MEAN_SQUARES, PB_STAT_MEAN_CUBES, PB_STAT_MAX, PB_STAT_MIN, PB_STAT_MEAN_SURFACE,
 PB_STAT_MEAN_CONDITIONAL, PB_STAT_MEAN_SQUARES_CONDITIONAL) = range(8)
PB_SGS_LENGTH_GRID, PB_SGS_LENGTH_WALL, PB_SGS_LENGTH_ILES = 0, 1, 2


class PbSgs(ctypes.Structure):
    _fields_ = [("scheme", ctypes.c_int), ("length", ctypes.c_int), ("cs", ctypes.c_double),
                ("prt", ctypes.c_double), ("viscosity", ctypes.c_double), ("diffusivity", ctypes.c_double)]


def precision_of(namelist) -> int:
    """The namelist's gpu.precision: "fp64" (plain form, default) or "fp32"
    (precision form)."""
    p = str((namelist or {}).get("gpu", {}).get("precision", "fp64")).lower()
    return PB_FP32 if p in ("fp32", "mixed", "precision") else PB_FP64
ERR_TABLE_RANGE, ERR_SECANT_CAP, ERR_NONFINITE = 0x1, 0x2, 0x4
MLP_NPARAM = 4481

# name -> (restype, argtypes); every symbol include/pycles_b200.h declares
_I, _LL, _D, _P = ctypes.c_int, ctypes.c_longlong, ctypes.c_double, ctypes.c_void_p
_DIMS = ctypes.POINTER(PbDims)
SIGNATURES = {
    "pb_scalar_advection": (_I, [_DIMS, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P, _I, _I, _P]),
    "pb_momentum_advection": (_I, [_DIMS, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _P]),
    "pb_scalar_advection_rk3": (_I, [_DIMS, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _D, _I, _I, _P]),
    "pb_momentum_advection_rk3": (_I, [_DIMS, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D, _I, _I,
                                       _P]),
    "pb_thermo_sa": (_I, [_DIMS, _P, _P, ctypes.POINTER(PbTable), _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                          _P, _I, ctypes.POINTER(PbMlp), _P, _I, _I, _P]),
    "pb_eos_sa": (_I, [ctypes.POINTER(PbTable), _P, _P, _P, _P, _P, _P, _P, _P, _P, _LL, _I, _P]),
    "pb_mlp_forward": (_I, [ctypes.POINTER(PbMlp), _P, _P, _P, _P, _LL, _P]),
    "pb_mlp_refresh_seed": (_I, [ctypes.POINTER(PbMlp), _DIMS, _P, _P, _P, _P, _P]),
    "pb_mlp_grad_workspace_bytes": (_LL, [_LL]),
    "pb_mlp_grad": (_I, [ctypes.POINTER(PbMlp), _P, _P, _LL, _P, _P, _P, _LL, _P]),
    "pb_mlp_adam": (_I, [_P, _P, _P, _P, _I, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                         ctypes.c_float, _P, _P, _P, _P, _P, _P, _P]),
    "pb_thermo_dry": (_I, [_DIMS, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P]),
    "pb_rk3_update": (_I, [_P, _P, _P, _LL, _D, _I, _P]),
    "pb_rk3_update_to": (_I, [_P, _P, _P, _P, _LL, _D, _I, _P]),
    "pb_update_all_bcs": (_I, [_DIMS, _P, _P, _I, _P]),
    "pb_pressure_workspace_bytes": (_LL, [_DIMS]),
    "pb_pressure_init": (_I, [_DIMS, _P, _LL]),
    "pb_pressure_solve": (_I, [_DIMS, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _LL, _I, _I, _P]),
    "pb_pressure_solve_noalloc": (_I, [_DIMS, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "pb_pressure_spectral_offset": (_LL, [_DIMS]),
    "pb_horizontal_sums": (_I, [_DIMS, _P, _P, _P]),
    "pb_pressure_divergence": (_I, [_DIMS, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P]),
    "pb_pressure_residual": (_I, [_DIMS, _P, _P, _P, _P, _P, _P]),
    "pb_pressure_fft_forward": (_I, [_DIMS, _P, _LL, _P, _I, _P]),
    "pb_pressure_fft_columns": (_I, [_DIMS, _P, _P, _DIMS, _P, _P, _P, _I, _I, _P]),
    "pb_pressure_fft_inverse": (_I, [_DIMS, _P, _LL, _P, _I, _P]),
    "pb_pressure_correct": (_I, [_DIMS, _P, _P, _P, _P, _P, _P]),
    "pb_surface_update": (_I, [_DIMS, ctypes.POINTER(PbSurface), _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                               _P, _P, ctypes.POINTER(PbSurfaceFields), _P]),
    "pb_kinematics_sgs": (_I, [_DIMS, ctypes.POINTER(PbSgs), _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "pb_scalar_diffusion": (_I, [_DIMS, _P, _P, _P, _P, _I, _P, _P, _P, _I, _I, _P, _P, _P, _P]),
    "pb_momentum_diffusion": (_I, [_DIMS] + [_P] * 15),
    "pb_stat_workspace_bytes": (_LL, [_DIMS]),
    "pb_horizontal_stat": (_I, [_DIMS, _I, _P, _P, _P, _P, _P, _P, _LL, _P]),
    "pb_forcing_update": (_I, [_DIMS, ctypes.POINTER(PbForcing)] + [_P] * 14),
    "pb_dycoms_radiation": (_I, [_DIMS, ctypes.POINTER(PbDycomsRadiation)] + [_P] * 9),
    "pb_get_error": (_I, [ctypes.POINTER(ctypes.c_uint)]),
    "pb_clear_error": (_I, [_P]),
    "pb_status_string": (ctypes.c_char_p, [_I]),
    "pb_launch_count": (_LL, []),
}

_lib = None


class PbError(RuntimeError):
    pass


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load the library (building it in-tree first if it is missing or stale
    and nvcc is available).  Raises if it cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if build_if_missing and _build.needs_build():
        try:
            _build.build()
        except Exception as e:  # pragma: no cover - build environment specific
            if not os.path.exists(path):
                raise PbError(f"libpycles_b200.so is missing and could not be built: {e}") from e
    if not os.path.exists(path):
        raise PbError(f"libpycles_b200.so not found at {path}; run python -m pycles_b200.build")
    L = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc: int, what: str) -> None:
    if rc != PB_OK:
        msg = load().pb_status_string(rc).decode()
        raise PbError(f"{what} failed: {msg} (status {rc})")


def ptr(t) -> int:
    """Device address of a CUDA tensor (or None)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise PbError("pycles_b200 kernels take CUDA tensors; got a CPU tensor")
    return t.data_ptr()


def stream_handle(stream=None) -> int:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def get_error() -> int:
    w = ctypes.c_uint(0)
    check(load().pb_get_error(ctypes.byref(w)), "pb_get_error")
    return w.value


def clear_error(stream=None) -> None:
    check(load().pb_clear_error(stream_handle(stream)), "pb_clear_error")
