"""Subgrid scale on the GPU: Kinematics (Kinematics.pyx), SGS with the
UniformViscosity and Smagorinsky schemes (SGS.pyx), ScalarDiffusion
(ScalarDiffusion.pyx) and MomentumDiffusion (MomentumDiffusion.pyx), with
the reference's update signatures.

Kinematics keeps only the strain-rate magnitude (the velocity gradients and
the nine strain-rate components the reference stores are formed in
registers where they are used), and the diffusion classes keep no flux
arrays.  ``SGS.update`` forms the strain-rate magnitude and the viscosity
and diffusivity in one kernel (the velocities do not change between the
stage's ``Ke.update`` and ``SGS.update``), so a step driver may skip
``Ke.update``.
"""
from __future__ import annotations

import ctypes

import torch

from . import _capi


class Kinematics:
    def __init__(self):
        self.strain_rate_mag = None

    def initialize(self, Gr, NS=None, Pa=None):
        dev = getattr(Gr, "device", "cuda")
        self.strain_rate_mag = torch.zeros(Gr.dims.npg, dtype=torch.float64, device=dev)

    def update(self, Gr, PV, stream=None):
        """Kinematics.update (Kinematics.pyx:42-58): the strain-rate magnitude."""
        npg = Gr.dims.npg
        vel = [PV.values[int(PV.velocity_directions[d]) * npg:] for d in range(3)]
        rc = _capi.load().pb_kinematics_sgs(ctypes.byref(Gr.dims), None, _capi.ptr(vel[0]), _capi.ptr(vel[1]),
                                            _capi.ptr(vel[2]), None, None, _capi.ptr(self.strain_rate_mag), None,
                                            None, _capi.stream_handle(stream))
        _capi.check(rc, "pb_kinematics_sgs")


class SGS:
    """SGS (SGS.pyx:33-55): ``namelist['sgs']['scheme']`` picks
    UniformViscosity or Smagorinsky; TKE is not built."""

    def __init__(self, namelist):
        sgs = namelist["sgs"]
        scheme = sgs["scheme"]
        self.struct = _capi.PbSgs()
        if scheme == "UniformViscosity":  # SGS.pyx:57-70
            u = sgs.get("UniformViscosity", {})
            self.struct.scheme = _capi.PB_SGS_UNIFORM
            self.struct.diffusivity = float(u.get("diffusivity", 0.0))
            self.struct.viscosity = float(u.get("viscosity", 0.0))
        elif scheme == "Smagorinsky":  # SGS.pyx:101-125
            s = sgs.get("Smagorinsky", {})
            self.struct.scheme = _capi.PB_SGS_SMAGORINSKY
            self.struct.cs = float(s.get("cs", 0.17))
            self.struct.prt = float(s.get("prt", 1.0 / 3.0))
            wall, iles = bool(s.get("wall", False)), bool(s.get("iles", False))
            # iles, read last, switches the wall adjustment off (SGS.pyx:109-122)
            self.struct.length = (_capi.PB_SGS_LENGTH_ILES if iles else
                                  _capi.PB_SGS_LENGTH_WALL if wall else _capi.PB_SGS_LENGTH_GRID)
        else:
            raise NotImplementedError(f"SGS scheme {scheme!r} is not built in this library")
        self.scheme = scheme
        self._zl_half = None

    def initialize(self, Gr, PV=None, NS=None, Pa=None):
        dev = getattr(Gr, "device", "cuda")
        self._zl_half = torch.as_tensor(Gr.zl_half, dtype=torch.float64, device=dev).contiguous()

    def update(self, Gr, DV, PV, Ke, Sur=None, Pa=None, stream=None):
        """Kinematics' strain-rate magnitude and SGS.update's viscosity and
        diffusivity in one launch."""
        npg = Gr.dims.npg
        vel = [PV.values[int(PV.velocity_directions[d]) * npg:] for d in range(3)]
        bvf = DV.values[DV.get_varshift(Gr, "buoyancy_frequency"):] if "buoyancy_frequency" in DV.index_name \
            else None
        rc = _capi.load().pb_kinematics_sgs(
            ctypes.byref(Gr.dims), ctypes.byref(self.struct), _capi.ptr(vel[0]), _capi.ptr(vel[1]),
            _capi.ptr(vel[2]), _capi.ptr(bvf), _capi.ptr(self._zl_half), _capi.ptr(Ke.strain_rate_mag),
            _capi.ptr(DV.values[DV.get_varshift(Gr, "viscosity"):]),
            _capi.ptr(DV.values[DV.get_varshift(Gr, "diffusivity"):]), _capi.stream_handle(stream))
        _capi.check(rc, "pb_kinematics_sgs")

    def stats_io(self, *args, **kwargs):
        """Statistics output is not part of this library."""
        return


class ScalarDiffusion:
    """ScalarDiffusion (ScalarDiffusion.pyx:27-150)."""

    def __init__(self, namelist, LH=None, DV=None, Pa=None):
        DV.add_variables("diffusivity", r"m^2s^{-1}", "D_t", "eddy diffusivity", "sym", Pa)
        self.qt_entropy_source = bool((namelist or {}).get("diffusion", {}).get("qt_entropy_source", False))

    def initialize(self, Gr, PV=None, DV=None, NS=None, Pa=None):
        return

    def update(self, Gr, RS, PV, DV, stream=None):
        npg = Gr.dims.npg
        scal = [i for i in range(PV.nv) if PV.var_type[i] == 1]
        if not scal:
            return
        n = len(scal)
        vals = (ctypes.c_void_p * n)(*[_capi.ptr(PV.values[i * npg:]) for i in scal])
        tends = (ctypes.c_void_p * n)(*[_capi.ptr(PV.tendencies[i * npg:]) for i in scal])
        # flux factor 2 for a TKE variable 'e' (ScalarDiffusion.pyx:122-127)
        factors = (ctypes.c_double * n)(*[2.0 if PV.index_name[i] == "e" else 1.0 for i in scal])
        names = [PV.index_name[i] for i in scal]
        qt_index = names.index("qt") if (self.qt_entropy_source and "qt" in names) else -1
        s_index = names.index("s") if qt_index >= 0 else -1

        def dv(name):
            return _capi.ptr(DV.values[DV.get_varshift(Gr, name):]) if name in DV.index_name else None

        rc = _capi.load().pb_scalar_diffusion(
            ctypes.byref(Gr.dims), _capi.ptr(RS.d_rho0), _capi.ptr(RS.d_rho0_half), _capi.ptr(RS.d_alpha0_half),
            dv("diffusivity"), n, vals, tends, factors, qt_index, s_index,
            _capi.ptr(RS.d_p0_half) if qt_index >= 0 else None, dv("qv") if qt_index >= 0 else None,
            dv("temperature") if qt_index >= 0 else None, _capi.stream_handle(stream))
        _capi.check(rc, "pb_scalar_diffusion")

    def stats_io(self, *args, **kwargs):
        return


class MomentumDiffusion:
    """MomentumDiffusion (MomentumDiffusion.pyx:27-78)."""

    def __init__(self, DV, Pa=None):
        DV.add_variables("viscosity", r"m^2s^{-1}", r"\nu_t", "eddy viscosity", "sym", Pa)

    def initialize(self, Gr, PV=None, DV=None, NS=None, Pa=None):
        return

    def update(self, Gr, RS, PV, DV, Ke, stream=None):
        npg = Gr.dims.npg
        vel = [int(PV.velocity_directions[d]) * npg for d in range(3)]
        s = PV.get_varshift(Gr, "s")
        rc = _capi.load().pb_momentum_diffusion(
            ctypes.byref(Gr.dims), _capi.ptr(RS.d_rho0), _capi.ptr(RS.d_rho0_half), _capi.ptr(RS.d_alpha0),
            _capi.ptr(RS.d_alpha0_half), *[_capi.ptr(PV.values[o:]) for o in vel],
            _capi.ptr(DV.values[DV.get_varshift(Gr, "viscosity"):]), _capi.ptr(Ke.strain_rate_mag),
            _capi.ptr(DV.values[DV.get_varshift(Gr, "temperature"):]),
            *[_capi.ptr(PV.tendencies[o:]) for o in vel], _capi.ptr(PV.tendencies[s:]), _capi.stream_handle(stream))
        _capi.check(rc, "pb_momentum_diffusion")

    def stats_io(self, *args, **kwargs):
        return
