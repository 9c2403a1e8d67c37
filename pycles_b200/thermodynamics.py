"""Thermodynamics components: ClausiusClapeyron table, ThermodynamicsSA,
ThermodynamicsDry.

``update`` runs on the GPU through the C ABI.  The scalar methods
``entropy``/``eos``/``alpha`` are the host-side helpers the reference also
evaluates on the host (ThermodynamicsSA.pyx:140-174): they serve the
reference-state integration and the initial conditions only, never the
time step.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _capi

# generate_parameters.py:19-41
g = 9.80665
Rd = 287.1
Rv = 461.5
eps_v = 0.6221018418201517
eps_vi = 1.6074538488331591
cpd = 1004.0
cpv = 1859.0
kappa = 0.2859561752988048
Tt = 273.16
T_tilde = 298.15
p_tilde = 100000.0
pv_star_t = 611.7
sd_tilde = 6864.8
sv_tilde = 10513.6


# --- host helpers (initialisation only), Csrc/thermodynamic_functions.h -------
def exner(p0):
    return np.power(np.asarray(p0, dtype=np.float64) / p_tilde, kappa)


def latent_heat_variable(T, lam=1.0):
    """Microphysics.pxd:71-75."""
    TC = T - 273.15
    return (2500.8 - 2.36 * TC + 0.0016 * TC * TC - 0.00006 * TC * TC * TC) * 1000.0


def _pd(p0, qt, qv):
    return p0 * (1.0 - qt) / (1.0 - qt + eps_vi * qv)


def _pv(p0, qt, qv):
    return p0 * eps_vi * qv / (1.0 - qt + eps_vi * qv)


def _sd(pd, T):
    return sd_tilde + cpd * np.log(T / T_tilde) - Rd * np.log(pd / p_tilde)


def _sv(pv, T):
    return sv_tilde + cpv * np.log(T / T_tilde) - Rv * np.log(pv / p_tilde)


def _qv_star(p0, qt, pv):
    return eps_v * (1.0 - qt) * pv / (p0 - pv)


def entropy_sa(p0, T, qt, ql, qi):
    """ThermodynamicsSA.entropy (ThermodynamicsSA.pyx:140-159), vectorised."""
    qv = qt - ql - qi
    pd = _pd(p0, qt, qv)
    pv = _pv(p0, qt, qv)
    L = latent_heat_variable(T)
    return _sd(pd, T) * (1.0 - qt) + _sv(pv, T) * qt + (-L / T) * (ql + qi)


def entropy_dry(p0, T):
    """ThermodynamicsDry.entropy (ThermodynamicsDry.pyx:87-92): sd_c(p0, T)."""
    return _sd(p0, T)


class ClausiusClapeyron:
    """pv*(T) table (Thermodynamics.pyx:45-116), integrated once on the host
    with scipy's odeint exactly as the reference does, then uploaded."""

    def __init__(self, namelist=None):
        cc = (namelist or {}).get("ClausiusClapeyron", {})
        self.Tmin = float(cc.get("temperature_min", 100.15))
        self.Tmax = float(cc.get("temperature_max", 380.0))
        self.n_lookup = int(cc.get("n_lookup", 512))
        self.T, self.pv = self._integrate()
        self.x_min = float(np.min(self.T))
        self.dx = float(self.T[1] - self.T[0])
        self.dxi = 1.0 / self.dx
        self._dev = None

    def _integrate(self):
        from scipy.integrate import odeint
        T = np.linspace(self.Tmin, self.Tmax, self.n_lookup)
        tp_close_index = np.max(np.where(T <= Tt))
        if T[tp_close_index] == Tt:
            raise ValueError("ClausiusClapeyron lookup table contains Tt; pick another Tmin/Tmax")
        T_above_Tt = np.append([Tt], T[tp_close_index + 1:])
        T_below_Tt = np.append(T[:tp_close_index + 1], [Tt])[::-1]

        def rhs(z, T_):
            return latent_heat_variable(T_, 1.0) / (Rv * T_ * T_)

        pv0 = np.log(pv_star_t)
        pv_above = np.exp(odeint(rhs, pv0, T_above_Tt, hmax=0.1)[1:])
        pv_below = np.exp(odeint(rhs, pv0, T_below_Tt, hmax=0.1)[1:])[::-1]
        pv = np.append(pv_below, pv_above)
        pv[pv < 1e-11] = 1e-11
        return T, pv

    def lookup(self, x):
        """Host lookup (Csrc/lookup.h:48-54), initialisation only."""
        indx = np.floor((x - self.x_min) * self.dxi).astype(np.int64)
        y1 = self.pv[indx]
        y2 = self.pv[indx + 1]
        x1 = self.x_min + self.dx * indx
        return y1 + (x - x1) * (y2 - y1) * self.dxi

    def device_table(self, device="cuda"):
        if self._dev is None:
            y = torch.as_tensor(self.pv, dtype=torch.float64, device=device).contiguous()
            t = _capi.PbTable()
            t.y = y.data_ptr()
            t.n = len(self.pv)
            t.x_min = self.x_min
            t.dx = self.dx
            t.dxi = self.dxi
            self._dev = (y, t)
        return self._dev[1]


def eos_sa_host(CC, p0, s, qt, T2_seed=None, max_iter=100):
    """Vectorised eos_c (Csrc/thermodynamics_sa.h:17-66) for initialisation
    and for generating training pairs of the learned seed.  Returns T, ql,
    qi, iterations."""
    p0, s, qt = (np.asarray(a, dtype=np.float64) for a in (p0, s, qt))
    p0, s, qt = np.broadcast_arrays(p0, s, qt)
    shape = s.shape
    p0, s, qt = p0.ravel(), s.ravel(), qt.ravel()
    pv_1 = _pv(p0, qt, qt)
    pd_1 = p0 - pv_1
    T_1 = T_tilde * np.exp((s - (1.0 - qt) * (sd_tilde - Rd * np.log(pd_1 / p_tilde))
                            - qt * (sv_tilde - Rv * np.log(pv_1 / p_tilde)))
                           / ((1.0 - qt) * cpd + qt * cpv))
    qvs1 = _qv_star(p0, qt, CC.lookup(T_1))
    T = T_1.copy()
    ql = np.zeros_like(T)
    qi = np.zeros_like(T)
    its = np.zeros(T.shape, dtype=np.int64)
    sat = np.nonzero(qt > qvs1)[0]
    if sat.size:
        P, S, Q = p0[sat], s[sat], qt[sat]
        t1 = T_1[sat]
        q1 = qvs1[sat]
        sig1 = Q - q1
        L1 = latent_heat_variable(t1)
        s1 = _sd(pd_1[sat], t1) * (1.0 - Q) + _sv(pv_1[sat], t1) * Q + (-L1 / t1) * sig1
        f1 = S - s1
        t2 = t1 + sig1 * L1 / ((1.0 - Q) * cpd + q1 * cpv)
        if T2_seed is not None:  # clamped to the bracket of the root, as on the device
            guess = np.asarray(T2_seed, dtype=np.float64).ravel()[sat]
            t2 = np.fmin(np.fmax(guess, t1 + 0.0625 * (t2 - t1)), t2)
        outT = t2.copy()
        outs = np.zeros_like(t2)
        outit = np.zeros(t2.shape, dtype=np.int64)
        act = np.arange(sat.size)
        it = 0
        while act.size and it < max_iter:
            it += 1
            qvs2 = _qv_star(P[act], Q[act], CC.lookup(t2[act]))
            pv2 = _pv(P[act], Q[act], qvs2)
            pd2 = P[act] - pv2
            sig2 = Q[act] - qvs2
            L2 = latent_heat_variable(t2[act])
            s2 = _sd(pd2, t2[act]) * (1.0 - Q[act]) + _sv(pv2, t2[act]) * Q[act] + (-L2 / t2[act]) * sig2
            f2 = S[act] - s2
            tn = t2[act] - f2 * (t2[act] - t1[act]) / (f2 - f1[act])
            t1[act] = t2[act]
            t2[act] = tn
            f1[act] = f2
            outT[act] = tn
            outs[act] = sig2
            outit[act] = it
            keep = (np.abs(tn - t1[act]) >= 1.0e-3) | (sig2 < 0.0)
            act = act[keep]
        T[sat] = outT
        ql[sat] = outs
        its[sat] = outit
    return T.reshape(shape), ql.reshape(shape), qi.reshape(shape), its.reshape(shape)


class ThermodynamicsSA:
    """ThermodynamicsSA (ThermodynamicsSA.pyx) with the update on the GPU."""

    thermodynamics_type = "SA"

    def __init__(self, namelist=None, LH=None, Par=None):
        namelist = namelist or {}
        self.CC = ClausiusClapeyron(namelist)
        th = namelist.get("thermodynamics", {})
        self.do_qt_clipping = bool(th.get("do_qt_clipping", True))
        self.max_secant_iter = int(namelist.get("gpu", {}).get("secant_max_iter", 100))
        self.precision = _capi.precision_of(namelist)
        self.mlp = None          # learned seed (pycles_b200.learned.SeedMLP, precision form) or None
        self.iter_stats = None   # device int64[2]: secant iterations, saturated cells
        self._seed_y = None      # device float32[npg]: the network's output per cell
        self._seed_for = None    # the network seed_y belongs to
        self._seed_calls = 0
        # updates between re-evaluations of the network (12: every fourth
        # SSP-RK3 time step; 1: every update).  The network's output for a
        # cell moves ~1e-4 K over a few steps against its own ~1e-2 K error,
        # and the secant decides every result.  Measured at 512x512x256
        # (thermodynamics ms per time step, seeded against unseeded 10.76):
        # interval 6: 10.89 (1.94 secant iterations per saturated cell),
        # 12: 10.67 (2.02), 24: 10.86 (2.23: more cells saturate between
        # refreshes and start from the reference's point).
        self.seed_refresh_interval = max(1, int(namelist.get("gpu", {}).get("seed_refresh_interval", 12)))

    def initialize(self, Gr, PV, DV, NS=None, Pa=None):
        PV.add_variable("s", "J kg^-1 K^-1", "s", "specific entropy", "sym", "scalar", Pa)
        PV.add_variable("qt", "kg/kg", "q_t", "total water mass fraction", "sym", "scalar", Pa)
        for name in ("buoyancy", "alpha", "temperature", "buoyancy_frequency", "qv", "ql", "qi",
                     "theta_rho", "thetali"):
            DV.add_variables(name, "", name, name, "sym", Pa)

    # host scalar helpers (reference-state integration, initial conditions)
    def entropy(self, p0, T, qt, ql, qi):
        return float(entropy_sa(p0, T, qt, ql, qi))

    def alpha(self, p0, T, qt, qv):
        return (Rd * T) / p0 * (1.0 - qt + eps_vi * qv)

    def eos(self, p0, s, qt):
        T, ql, qi, _ = eos_sa_host(self.CC, p0, s, qt)
        return float(T), float(ql), float(qi)

    def get_pv_star(self, T):
        return self.CC.lookup(T)

    def update(self, Gr, RS, PV, DV, stream=None):
        """ThermodynamicsSA.update (ThermodynamicsSA.pyx:176-213) on the GPU."""
        L = _capi.load()
        f = DV.field
        if self.iter_stats is None or self.iter_stats.device != PV.values.device:
            self.iter_stats = torch.zeros(2, dtype=torch.int64, device=PV.values.device)
        mlp_struct = None
        if self.mlp is not None:
            # learned seed for the secant's second point (no counterpart in the
            # reference; precision form only): the library refreshes the
            # network's output per cell for the cells saturated at the
            # previous update, then starts their secant from it
            if self.precision != _capi.PB_FP32:
                raise ValueError("the learned seed belongs to the precision form (gpu.precision = 'fp32')")
            npg = int(Gr.dims.npg)
            dev = PV.values.device
            if (self._seed_y is None or self._seed_for is not self.mlp or self._seed_y.numel() != npg
                    or self._seed_y.device != dev):
                self._seed_y = torch.zeros(npg, dtype=torch.float32, device=dev)
                self._seed_for = self.mlp
                self._seed_calls = 0
            self._mlp_struct = self.mlp.struct()
            self._mlp_struct.seed_y = self._seed_y.data_ptr()
            self._mlp_struct.seed_refresh = 1 if self._seed_calls % self.seed_refresh_interval == 0 else 0
            self._seed_calls += 1
            mlp_struct = ctypes.byref(self._mlp_struct)
        table = self.CC.device_table(PV.values.device)
        rc = L.pb_thermo_sa(ctypes.byref(Gr.dims), _capi.ptr(RS.d_p0_half), _capi.ptr(RS.d_alpha0_half),
                            ctypes.byref(table), _capi.ptr(PV.field("s", Gr)), _capi.ptr(PV.field("qt", Gr)),
                            _capi.ptr(f("temperature", Gr)), _capi.ptr(f("qv", Gr)), _capi.ptr(f("ql", Gr)),
                            _capi.ptr(f("qi", Gr)), _capi.ptr(f("alpha", Gr)), _capi.ptr(f("buoyancy", Gr)),
                            _capi.ptr(f("theta_rho", Gr)), _capi.ptr(f("buoyancy_frequency", Gr)),
                            _capi.ptr(f("thetali", Gr)), _capi.ptr(PV.tendency("w", Gr)),
                            1 if self.do_qt_clipping else 0, mlp_struct, _capi.ptr(self.iter_stats),
                            self.max_secant_iter, self.precision, _capi.stream_handle(stream))
        _capi.check(rc, "pb_thermo_sa")


class ThermodynamicsDry:
    """ThermodynamicsDry (ThermodynamicsDry.pyx) with the update on the GPU."""

    thermodynamics_type = "dry"

    def __init__(self, namelist=None, LH=None, Par=None):
        self.CC = ClausiusClapeyron(namelist)
        self.precision = _capi.precision_of(namelist)

    def initialize(self, Gr, PV, DV, NS=None, Pa=None):
        PV.add_variable("s", "J kg^-1 K^-1", "s", "specific entropy", "sym", "scalar", Pa)
        for name in ("buoyancy", "alpha", "temperature", "buoyancy_frequency", "theta"):
            DV.add_variables(name, "", name, name, "sym", Pa)

    def entropy(self, p0, T, qt, ql, qi):
        return float(entropy_dry(p0, T))

    def eos(self, p0, s, qt):
        return float(T_tilde * (math.exp((s - sd_tilde + Rd * math.log(p0 / p_tilde)) / cpd))), 0.0, 0.0

    def alpha(self, p0, T, qt, qv):
        return (Rd * T) / p0 * (1.0 - 0.0 + eps_vi * 0.0)

    def update(self, Gr, RS, PV, DV, stream=None):
        """ThermodynamicsDry.update (ThermodynamicsDry.pyx:105-120) on the GPU."""
        L = _capi.load()
        f = DV.field
        rc = L.pb_thermo_dry(ctypes.byref(Gr.dims), _capi.ptr(RS.d_p0_half), _capi.ptr(RS.d_alpha0_half),
                             _capi.ptr(PV.field("s", Gr)), _capi.ptr(f("temperature", Gr)),
                             _capi.ptr(f("alpha", Gr)), _capi.ptr(f("buoyancy", Gr)), _capi.ptr(f("theta", Gr)),
                             _capi.ptr(f("buoyancy_frequency", Gr)), _capi.ptr(PV.tendency("w", Gr)),
                             self.precision, _capi.stream_handle(stream))
        _capi.check(rc, "pb_thermo_dry")
