"""Restatement of the surface schemes' update methods (Surface.pyx) on the
state of an ``OracleSim`` -- TEST INFRASTRUCTURE ONLY.

``OracleSurface`` holds SurfaceBase's per-column arrays (Surface.pyx:82-96,
nlg0*nlg1 doubles, indexed i*nlg1 + j) and performs, in the reference's loop
order and arithmetic:

* ``SurfaceSullivanPatton.update`` (Surface.pyx:236-291),
* ``SurfaceBomex.update`` (Surface.pyx:319-371),
* ``SurfaceDYCOMS_RF01.update`` (Surface.pyx:502-556),

each followed by ``SurfaceBase.update`` (Surface.pyx:116-178).  The
surface-layer functions (compute_ustar, compute_windspeed,
entropyflux_from_thetaflux_qtflux) come from the simulation's backend: the
reference's own C (oracle/ref.py) or the restatement (oracle/port.py).
"""
from __future__ import annotations

import math

import numpy as np

from . import port

SULLIVAN_PATTON, BOMEX, DYCOMS_RF01 = "SullivanPatton", "Bomex", "DYCOMS_RF01"


def scheme_constants(scheme: str) -> dict:
    """The attributes each scheme's __init__/initialize sets."""
    if scheme == SULLIVAN_PATTON:  # Surface.pyx:217-226
        return dict(theta_flux=0.24, z0=0.1, gustiness=0.001, dry=True)
    if scheme == BOMEX:  # Surface.pyx:298-316; gustiness is never set (a cdef double: 0)
        return dict(theta_flux=8.0e-3, ustar=0.28, gustiness=0.0, qt_flux=5.2e-5, dry=False)
    if scheme == DYCOMS_RF01:  # Surface.pyx:475-491
        return dict(ft=15.0, fq=115.0, gustiness=0.0, cm=0.0011, dry=False)
    raise ValueError(f"surface scheme {scheme!r} is not restated")


class OracleSurface:
    NAMES = ("u_flux", "v_flux", "qt_flux", "s_flux", "obukhov_length", "friction_velocity", "shf", "lhf",
             "b_flux", "windspeed")

    def __init__(self, scheme: str, d, u0: float = 0.0, v0: float = 0.0):
        self.scheme = scheme
        self.c = scheme_constants(scheme)
        self.d = d
        self.u0, self.v0 = float(u0), float(v0)
        n2 = d.nlg[0] * d.nlg[1]
        for n in self.NAMES:
            setattr(self, n, np.zeros(n2))
        if scheme == BOMEX:  # Surface.pyx:306
            self.qt_flux = np.add(self.qt_flux, self.c["qt_flux"])

    # SurfaceSullivanPatton / SurfaceBomex / SurfaceDYCOMS_RF01 ----------------
    def update(self, sim):
        d, rs, K = self.d, sim.rs, sim.K
        gw = d.gw
        n0, n1 = d.nlg[0], d.nlg[1]
        sh = d.shape
        T = sim.dv["temperature"].reshape(sh)[:, :, gw]
        u, v = sim.var("u"), sim.var("v")
        c = self.c
        if self.scheme == SULLIVAN_PATTON:
            T0 = rs["p0_half"][gw] * rs["alpha0_half"][gw] / port.Rd
            buoyancy_flux = c["theta_flux"] * float(port.exner_c(rs["p0_half"][gw])) * port.g / T0
            s2 = self.s_flux.reshape(n0, n1)
            s2[:, :] = port.cpd * c["theta_flux"] * float(port.exner_c(rs["p0_half"][gw])) / T
            windspeed = np.zeros(n0 * n1)
            K.compute_windspeed(d, u, v, windspeed, self.u0, self.v0, c["gustiness"])
            ws2 = windspeed.reshape(n0, n1)
            fv2 = self.friction_velocity.reshape(n0, n1)
            for i in range(1, n0):
                for j in range(1, n1):
                    fv2[i, j] = K.compute_ustar(float(ws2[i, j]), buoyancy_flux, c["z0"], d.dx[2] / 2.0)
            U = u.reshape(sh)[:, :, gw]
            V = v.reshape(sh)[:, :, gw]
            uf = self.u_flux.reshape(n0, n1)
            vf = self.v_flux.reshape(n0, n1)
            a = port.interp_2(fv2[1:n0 - 1, 1:n1 - 1], fv2[2:n0, 1:n1 - 1])
            b = port.interp_2(fv2[1:n0 - 1, 1:n1 - 1], fv2[1:n0 - 1, 2:n1])
            uf[1:n0 - 1, 1:n1 - 1] = -(a * a) / port.interp_2(ws2[1:n0 - 1, 1:n1 - 1], ws2[2:n0, 1:n1 - 1]) * (
                U[1:n0 - 1, 1:n1 - 1] + self.u0)
            vf[1:n0 - 1, 1:n1 - 1] = -(b * b) / port.interp_2(ws2[1:n0 - 1, 1:n1 - 1], ws2[1:n0 - 1, 2:n1]) * (
                V[1:n0 - 1, 1:n1 - 1] + self.v0)
            self.windspeed = windspeed
        elif self.scheme == BOMEX:
            qt = sim.var("qt").reshape(sh)[:, :, gw]
            qv = sim.dv["qv"].reshape(sh)[:, :, gw]
            self.friction_velocity[:] = c["ustar"]
            s2 = self.s_flux.reshape(n0, n1)
            s2[:, :] = K.entropyflux_from_thetaflux_qtflux(c["theta_flux"], self.qt_flux.reshape(n0, n1),
                                                           rs["p0_half"][gw], T, qt, qv)
            windspeed = np.zeros(n0 * n1)
            K.compute_windspeed(d, u, v, windspeed, self.u0, self.v0, c["gustiness"])
            ws2 = windspeed.reshape(n0, n1)
            U = u.reshape(sh)[:, :, gw]
            V = v.reshape(sh)[:, :, gw]
            uf = self.u_flux.reshape(n0, n1)
            vf = self.v_flux.reshape(n0, n1)
            us2 = c["ustar"] ** 2
            uf[1:n0 - 1, 1:n1 - 1] = -us2 / port.interp_2(ws2[1:n0 - 1, 1:n1 - 1], ws2[2:n0, 1:n1 - 1]) * (
                U[1:n0 - 1, 1:n1 - 1] + self.u0)
            vf[1:n0 - 1, 1:n1 - 1] = -us2 / port.interp_2(ws2[1:n0 - 1, 1:n1 - 1], ws2[1:n0 - 1, 2:n1]) * (
                V[1:n0 - 1, 1:n1 - 1] + self.v0)
            self.windspeed = windspeed
        else:  # DYCOMS_RF01
            K.compute_windspeed(d, u, v, self.windspeed, self.u0, self.v0, c["gustiness"])
            ws2 = self.windspeed.reshape(n0, n1)
            qt3 = sim.var("qt").reshape(sh)[:, :, gw]
            ql3 = sim.dv["ql"].reshape(sh)[:, :, gw]
            r = (slice(gw - 1, n0 - gw + 1), slice(gw - 1, n1 - gw + 1))
            self.friction_velocity.reshape(n0, n1)[r] = math.sqrt(c["cm"]) * ws2[r]
            Tr = T[r]
            lv = port.latent_heat_variable(Tr)
            p0 = rs["p0_half"][gw]
            qv = qt3[r] - ql3[r]
            pv = port.pv_c(p0, qt3[r], qv)
            pd = port.pd_c(p0, qt3[r], qv)
            sv = port.sv_c(pv, Tr)
            sd = port.sd_c(pd, Tr)
            self.qt_flux.reshape(n0, n1)[r] = c["fq"] / lv / 1.22
            self.s_flux.reshape(n0, n1)[r] = rs["alpha0_half"][gw] * (c["ft"] / Tr + c["fq"] * (sv - sd) / lv)
            U = u.reshape(sh)[:, :, gw]
            V = v.reshape(sh)[:, :, gw]
            ii = slice(gw, n0 - gw)
            jj = slice(gw, n1 - gw)
            self.u_flux.reshape(n0, n1)[ii, jj] = -c["cm"] * port.interp_2(
                ws2[ii, jj], ws2[gw + 1:n0 - gw + 1, jj]) * (U[ii, jj] + self.u0)
            self.v_flux.reshape(n0, n1)[ii, jj] = -c["cm"] * port.interp_2(
                ws2[ii, jj], ws2[ii, gw + 1:n1 - gw + 1]) * (V[ii, jj] + self.v0)
        self.base_update(sim)

    # SurfaceBase.update (Surface.pyx:116-178) ----------------------------------
    def base_update(self, sim):
        d, rs = self.d, sim.rs
        gw = d.gw
        n0, n1 = d.nlg[0], d.nlg[1]
        sh = d.shape
        t_mean = port.horizontal_mean(d, sim.dv["temperature"])
        dzi = 1.0 / d.dx[2]
        tendency_factor = rs["alpha0_half"][gw] / rs["alpha0"][gw - 1] * dzi
        ii, jj = slice(gw, n0 - gw), slice(gw, n1 - gw)
        T = sim.dv["temperature"].reshape(sh)[ii, jj, gw]
        f2 = {n: getattr(self, n).reshape(n0, n1) for n in self.NAMES}
        fv = f2["friction_velocity"][ii, jj]
        if self.c["dry"]:
            f2["shf"][ii, jj] = f2["s_flux"][ii, jj] * rs["rho0_half"][gw] * T
            f2["b_flux"][ii, jj] = f2["shf"][ii, jj] * port.g * rs["alpha0_half"][gw] / port.cpd / t_mean[gw]
        else:
            qt = sim.var("qt").reshape(sh)[ii, jj, gw]
            ql = sim.dv["ql"].reshape(sh)[ii, jj, gw]
            lv = port.latent_heat_variable(T)
            f2["lhf"][ii, jj] = f2["qt_flux"][ii, jj] * rs["rho0_half"][gw] * lv
            p0 = rs["p0_half"][gw]
            pv = port.pv_c(p0, qt, qt - ql)
            pd = port.pd_c(p0, qt, qt - ql)
            sv = port.sv_c(pv, T)
            sd = port.sd_c(pd, T)
            f2["shf"][ii, jj] = (f2["s_flux"][ii, jj] * rs["rho0_half"][gw] - f2["lhf"][ii, jj] / lv * (sv - sd)) * T
            cp_ = port.cpm_c(qt)
            f2["b_flux"][ii, jj] = port.g * rs["alpha0_half"][gw] / cp_ / t_mean[gw] * (
                f2["shf"][ii, jj] + (port.eps_vi - 1.0) * cp_ * t_mean[gw] * f2["lhf"][ii, jj] / lv)
        f2["obukhov_length"][ii, jj] = -fv * fv * fv / f2["b_flux"][ii, jj] / port.vkb
        names = ("u", "v", "s") + (() if self.c["dry"] else ("qt",))
        flux = {"u": "u_flux", "v": "v_flux", "s": "s_flux", "qt": "qt_flux"}
        for n in names:
            sim.tend(n).reshape(sh)[ii, jj, gw] += f2[flux[n]][ii, jj] * tendency_factor
