"""ReferenceState (ReferenceState.pyx:39-135).

The hydrostatic reference profiles are integrated once, on the host, in
FP64 with scipy's odeint as in the reference, then copied to the GPU
(``d_*`` attributes).  Nothing here runs per time step.
"""
from __future__ import annotations

import numpy as np
import torch

from .thermodynamics import Rd, eps_vi, g


class ReferenceState:
    def __init__(self, Gr):
        n = Gr.dims.nlg[2]
        for name in ("p0", "p0_half", "alpha0", "alpha0_half", "rho0", "rho0_half"):
            setattr(self, name, np.zeros(n))
        self.Pg = self.Tg = self.qtg = None
        self.u0 = 0.0
        self.v0 = 0.0

    def initialize(self, Gr, Thermodynamics, NS=None, Pa=None, device="cuda"):
        from scipy.integrate import odeint
        gw = Gr.dims.gw
        self.sg = Thermodynamics.entropy(self.Pg, self.Tg, self.qtg, 0.0, 0.0)
        sg, qtg = self.sg, self.qtg

        def rhs(p, z):
            T, ql, qi = Thermodynamics.eos(np.exp(p[0] if np.ndim(p) else p), sg, qtg)
            return -g / (Rd * T * (1.0 - qtg + eps_vi * (qtg - ql - qi)))

        z = np.array(Gr.z[gw - 1:-gw + 1])
        z_half = np.append([0.0], np.array(Gr.z_half[gw:-gw]))
        p0 = np.log(self.Pg)
        ng2 = Gr.dims.ng[2]
        p = np.zeros(ng2)
        p_half = np.zeros(ng2)
        p[gw - 1:-gw + 1] = odeint(rhs, p0, z, hmax=1.0)[:, 0]
        p_half[gw:-gw] = odeint(rhs, p0, z_half, hmax=1.0)[1:, 0]
        p[:gw - 1] = p[2 * gw - 2:gw - 1:-1]
        p[-gw + 1:] = p[-gw - 1:-2 * gw:-1]
        p_half[:gw] = p_half[2 * gw - 1:gw - 1:-1]
        p_half[-gw:] = p_half[-gw - 1:-2 * gw - 1:-1]
        p = np.exp(p)
        p_half = np.exp(p_half)
        alpha = np.zeros(ng2)
        alpha_half = np.zeros(ng2)
        for k in range(ng2):
            T, ql, qi = Thermodynamics.eos(p[k], sg, qtg)
            alpha[k] = Thermodynamics.alpha(p[k], T, qtg, qtg - (ql + qi))
            T, ql, qi = Thermodynamics.eos(p_half[k], sg, qtg)
            alpha_half[k] = Thermodynamics.alpha(p_half[k], T, qtg, qtg - (ql + qi))
            # entropy constancy check (ReferenceState.pyx:115-121)
            s = Thermodynamics.entropy(p_half[k], T, qtg, ql, qi)
            if abs(s - sg) / sg > 0.01:
                raise RuntimeError("Error in reference profiles entropy not constant")
        self.p0, self.p0_half = p, p_half
        self.alpha0, self.alpha0_half = alpha, alpha_half
        self.rho0 = 1.0 / alpha
        self.rho0_half = 1.0 / alpha_half
        self.to_device(device)

    def set_profiles(self, profiles: dict, device="cuda"):
        """Install precomputed profiles (e.g. from a restart dict), and the
        Galilean shift u0, v0 when the dict carries it."""
        for k in ("p0", "p0_half", "alpha0", "alpha0_half", "rho0", "rho0_half"):
            setattr(self, k, np.ascontiguousarray(profiles[k], dtype=np.float64))
        for k in ("u0", "v0"):
            if k in profiles:
                setattr(self, k, float(profiles[k]))
        self.to_device(device)

    def to_device(self, device="cuda"):
        for k in ("p0", "p0_half", "alpha0", "alpha0_half", "rho0", "rho0_half"):
            setattr(self, "d_" + k, torch.as_tensor(getattr(self, k), dtype=torch.float64, device=device).contiguous())

    def profiles(self) -> dict:
        """The six profiles (arrays of nlg2) and the Galilean shift u0, v0."""
        out = {k: np.array(getattr(self, k)) for k in ("p0", "p0_half", "alpha0", "alpha0_half", "rho0",
                                                       "rho0_half")}
        out["u0"], out["v0"] = float(self.u0), float(self.v0)
        return out
