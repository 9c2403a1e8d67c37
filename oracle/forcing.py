"""Restatement of the case forcing (Forcing.pyx: ForcingSullivanPatton
:256-300, ForcingBomex :102-254, ForcingDyCOMS_RF01 :346-460) on the state
of an ``OracleSim`` -- TEST INFRASTRUCTURE ONLY.  The update order of each
scheme is the reference's; s_tendency_c comes from the simulation's backend
(the reference C or oracle/port.py), the rest of the forcing is Cython in the
reference and restated in oracle/port.py.
"""
from __future__ import annotations

from . import port


class OracleForcing:
    def __init__(self, scheme: str, d, p0_half, zl_half, u0=0.0, v0=0.0):
        self.scheme = scheme
        self.d = d
        self.P = port.forcing_profiles(scheme, zl_half, p0_half)
        self.u0, self.v0 = float(u0), float(v0)

    def update(self, sim):
        d, rs, P = self.d, sim.rs, self.P
        f = P["coriolis_param"]
        u, v = sim.var("u"), sim.var("v")
        ut, vt = sim.tend("u"), sim.tend("v")
        if self.scheme == "SullivanPatton":  # Forcing.pyx:269-277
            port.coriolis_force(d, u, v, ut, vt, P["ug"], P["vg"], f, self.u0, self.v0)
            return
        if self.scheme == "Bomex":  # Forcing.pyx:154-203
            umean = port.horizontal_stat(d, "mean", u)
            vmean = port.horizontal_stat(d, "mean", v)
            port.large_scale_p_gradient(d, umean, vmean, ut, vt, P["ug"], P["vg"], f, self.u0, self.v0)
            sh = d.shape
            g_ = d.gw
            r = (slice(g_, sh[0] - g_), slice(g_, sh[1] - g_), slice(g_, sh[2] - g_))
            qt = sim.var("qt").reshape(sh)[r]
            qv = qt - sim.dv["ql"].reshape(sh)[r]
            T = sim.dv["temperature"].reshape(sh)[r]
            p0 = rs["p0_half"][None, None, g_:sh[2] - g_]
            dq = P["dqtdt"][None, None, g_:sh[2] - g_]
            dt = P["dtdt"][None, None, g_:sh[2] - g_]
            sim.tend("s").reshape(sh)[r] += sim.K.s_tendency_c(p0, qt, qv, T, dq, dt)
            sim.tend("qt").reshape(sh)[r] += dq
            for n in ("s", "qt", "u", "v"):
                port.apply_subsidence(d, rs["rho0"], rs["rho0_half"], P["subsidence"], sim.var(n), sim.tend(n))
            return
        if self.scheme == "DYCOMS_RF01":  # Forcing.pyx:391-407
            for n in ("s", "qt", "u", "v"):
                port.apply_subsidence(d, rs["rho0"], rs["rho0_half"], P["subsidence"], sim.var(n), sim.tend(n))
            port.coriolis_force(d, u, v, ut, vt, P["ug"], P["vg"], f, self.u0, self.v0)
            return
        raise ValueError(self.scheme)
