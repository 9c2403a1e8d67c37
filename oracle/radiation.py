"""Restatement of RadiationDyCOMS_RF01 (Radiation.pyx:230-353) on the state
of an ``OracleSim`` -- TEST INFRASTRUCTURE ONLY (the reference's radiation is
Cython; the loops are restated in oracle/port.py).  RadiationFactory
(Radiation.pyx:30-57) gives it to the DYCOMS_RF01 and DYCOMS_RF02 cases."""
from __future__ import annotations

import numpy as np

from . import port


class OracleRadiation:
    def __init__(self, d, z, f0=70.0):
        self.d = d
        self.z = np.asarray(z, dtype=np.float64)
        self.f0 = f0
        self.heating_rate = np.zeros(d.npg)
        self.dTdt_rad = np.zeros(d.npg)

    def update(self, sim):
        port.dycoms_radiation(self.d, sim.rs["rho0_half"], self.z, sim.dv["ql"], sim.var("qt"),
                              sim.dv["temperature"], sim.tend("s"), self.heating_rate, self.dTdt_rad, f0=self.f0)
