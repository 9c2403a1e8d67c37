"""Restatement of the subgrid-scale glue (Kinematics.pyx, SGS.pyx,
ScalarDiffusion.pyx, MomentumDiffusion.pyx) on the state of an
``OracleSim`` -- TEST INFRASTRUCTURE ONLY.

``OracleSGS`` holds Kinematics' arrays (velocity gradients, strain rate and
its magnitude, Kinematics.pyx:27-35) and the DV fields 'viscosity' and
'diffusivity', and performs, in the reference's order and arithmetic:

* ``Kinematics.update`` (Kinematics.pyx:42-58) at the start of an RK stage;
* ``SGS.update`` (SGS.pyx:48-53) with UniformViscosity (:57-97) or
  Smagorinsky (:101-149: plain, wall-adjusted or ILES length scale);
* ``ScalarDiffusion.update`` (ScalarDiffusion.pyx:79-150);
* ``MomentumDiffusion.update`` (MomentumDiffusion.pyx:52-78).

The kernels come from the simulation's backend (oracle/ref.py or
oracle/port.py).
"""
from __future__ import annotations

import numpy as np


def scheme_from_namelist(namelist: dict) -> dict:
    """SGS.__init__ (SGS.pyx:35-44) with the schemes' own namelist reads
    (UniformViscosity :57-70, Smagorinsky :101-125) and
    ScalarDiffusion.__init__'s qt_entropy_source (ScalarDiffusion.pyx:30-34)."""
    sgs = namelist["sgs"]
    c = {"scheme": sgs["scheme"]}
    if c["scheme"] == "UniformViscosity":
        u = sgs.get("UniformViscosity", {})
        c["diffusivity"] = float(u.get("diffusivity", 0.0))
        c["viscosity"] = float(u.get("viscosity", 0.0))
    elif c["scheme"] == "Smagorinsky":
        s = sgs.get("Smagorinsky", {})
        c["cs"] = float(s.get("cs", 0.17))
        c["prt"] = float(s.get("prt", 1.0 / 3.0))
        wall = bool(s.get("wall", False))
        iles = bool(s.get("iles", False))
        # the try blocks of SGS.pyx:109-122: iles, read last, switches wall off
        c["variant"] = "iles" if iles else ("wall" if wall else "plain")
    else:
        raise ValueError(f"SGS scheme {c['scheme']!r} is not restated")
    c["qt_entropy_source"] = bool(namelist.get("diffusion", {}).get("qt_entropy_source", False))
    return c


class OracleSGS:
    def __init__(self, config: dict, d, zl_half):
        self.c = config
        self.d = d
        npg = d.npg
        self.vgrad = np.zeros(9 * npg)
        self.strain_rate = np.zeros(9 * npg)
        self.strain_rate_mag = np.zeros(npg)
        self.viscosity = np.zeros(npg)
        self.diffusivity = np.zeros(npg)
        self.zl_half = np.ascontiguousarray(zl_half, dtype=np.float64)
        self.is_init = False
        self.sd_flux = None
        self.md_flux = np.zeros(9 * npg)

    def ke_update(self, sim):
        """Kinematics.update (Kinematics.pyx:42-58)."""
        K, d = sim.K, self.d
        npg = d.npg
        count = 0
        for vi1, name in enumerate(("u", "v", "w")):
            for dd in range(3):
                K.compute_velocity_gradient(d, sim.var(name), self.vgrad[count * npg:(count + 1) * npg], dd)
                count += 1
        K.compute_strain_rate(d, self.vgrad, self.strain_rate)
        K.compute_strain_rate_mag(d, self.strain_rate, self.strain_rate_mag)

    def sgs_update(self, sim):
        """SGS.update: UniformViscosity sets the constants once (SGS.pyx:
        84-90), Smagorinsky every call (:127-145)."""
        K, d, c = sim.K, self.d, self.c
        if c["scheme"] == "UniformViscosity":
            if not self.is_init:
                self.diffusivity[:] = c["diffusivity"]
                self.viscosity[:] = c["viscosity"]
                self.is_init = True
            return
        K.smagorinsky_update(d, self.viscosity, self.diffusivity, sim.dv["buoyancy_frequency"],
                             self.strain_rate_mag, c["cs"], c["prt"], c["variant"], self.zl_half)

    def sd_update(self, sim):
        """ScalarDiffusion.update (ScalarDiffusion.pyx:79-150) for the
        scalars s[, qt] (no TKE variable: flux factor 1)."""
        K, d, rs = sim.K, self.d, sim.rs
        npg = d.npg
        scalars = sim.names[3:]
        if self.sd_flux is None:
            self.sd_flux = np.zeros(len(scalars) * 3 * npg)
        for si, name in enumerate(scalars):
            for dd in range(3):
                F = self.sd_flux[(si * 3 + dd) * npg:(si * 3 + dd + 1) * npg]
                K.compute_diffusive_flux(d, rs["rho0"], rs["rho0_half"], self.diffusivity, sim.var(name), F,
                                         d.dx[dd], dd, 1.0)
                K.scalar_flux_divergence(d, rs["alpha0"], rs["alpha0_half"], F, sim.tend(name), d.dx[dd], dd)
                if name == "qt" and self.c["qt_entropy_source"]:
                    K.compute_qt_diffusion_s_source(d, rs["p0_half"], rs["alpha0"], rs["alpha0_half"], F,
                                                    sim.var("qt"), sim.dv["qv"], sim.dv["temperature"],
                                                    sim.tend("s"), d.dx[dd], dd)

    def md_update(self, sim):
        """MomentumDiffusion.update (MomentumDiffusion.pyx:52-78)."""
        K, d, rs = sim.K, self.d, sim.rs
        npg = d.npg
        count = 0
        for i1, name in enumerate(("u", "v", "w")):
            for i2 in range(3):
                sl = slice(count * npg, (count + 1) * npg)
                K.compute_diffusive_flux_m(d, self.strain_rate[sl], self.viscosity, self.md_flux[sl], rs["rho0"],
                                           rs["rho0_half"], i1, i2)
                K.momentum_flux_divergence(d, rs["alpha0"], rs["alpha0_half"], self.md_flux[sl], sim.tend(name),
                                           i1, i2)
                count += 1
        K.compute_entropy_source(d, self.viscosity, self.strain_rate_mag, sim.dv["temperature"], sim.tend("s"))
