"""Restatement of the reference's Cython glue around the hot-path kernels --
TEST INFRASTRUCTURE ONLY.

``OracleSim`` reproduces one rank of ``Simulation3d.run`` (Simulation3d.pyx:
140-189) restricted to the hot-path components, in the reference's order per
RK stage: [Ke.update,] Th.update, SA.update, MA.update, [Sur.update,]
[SGS.update, SD.update, MD.update,] [Fo.update,] [Ra.update,] TS.update,
PV.Update_all_bcs, Pr.update.  The kernels come from one of two backends:

* ``"ref"``  -- the reference's own C (oracle/ref.py), TDMA from the
               reference's cythonized SparseSolvers when it was built;
* ``"port"`` -- the numpy restatement (oracle/port.py).

The glue itself (PressureSolver/PressureFFTParallel, TimeStepping,
HorizontalMean, ClausiusClapeyron, ReferenceState) is restated here, citing
file:line.
"""
from __future__ import annotations

import numpy as np

from . import port
from .dims import Dims


# ---------------------------------------------------------------------------
# ClausiusClapeyron.initialize (Thermodynamics.pyx:45-116)
# ---------------------------------------------------------------------------
def cc_table(Tmin=100.15, Tmax=380.0, n_lookup=512):
    from scipy.integrate import odeint
    T = np.linspace(Tmin, Tmax, n_lookup)
    tp_close_index = np.max(np.where(T <= port.Tt))
    if T[tp_close_index] == port.Tt:
        raise ValueError("ClausiusClapeyron table contains Tt")
    T_above_Tt = np.append([port.Tt], T[tp_close_index + 1:])
    T_below_Tt = np.append(T[:tp_close_index + 1], [port.Tt])[::-1]

    def rhs(z, T_):
        lam = 1.0
        L = port.latent_heat_variable(T_, lam)
        return L / (port.Rv * T_ * T_)

    pv0 = np.log(port.pv_star_t)
    pv_above_Tt = np.exp(odeint(rhs, pv0, T_above_Tt, hmax=0.1)[1:])
    pv_below_Tt = np.exp(odeint(rhs, pv0, T_below_Tt, hmax=0.1)[1:])[::-1]
    pv = np.append(pv_below_Tt, pv_above_Tt)
    pv_a = np.array(pv)
    pv_a[pv_a < 1e-11] = 1e-11
    return T, pv_a


# ---------------------------------------------------------------------------
# ReferenceState.initialize (ReferenceState.pyx:39-135)
# ---------------------------------------------------------------------------
def reference_state(d: Dims, Pg, Tg, qtg, moist=True, backend="ref", table_xy=None):
    """Returns dict p0, p0_half, alpha0, alpha0_half, rho0, rho0_half (length nlg[2])."""
    from scipy.integrate import odeint
    g_ = d.gw
    if moist:
        x, y = table_xy if table_xy is not None else cc_table()
        if backend == "ref":
            from . import ref
            LT = ref.Table(x, y)

            def eos(p, s, qt):
                T, qv, ql, qi = ref.eos_c(LT, p, s, qt)
                return T, ql, qi

            def entropy(p0, T, qt, ql, qi):
                return ref.entropy_sa(p0, T, qt, ql, qi)
        else:
            LT = port.Table(x, y)

            def eos(p, s, qt):
                T, qv, ql, qi, _ = port.eos_c(LT, p, s, qt)
                return float(T), float(ql), float(qi)

            def entropy(p0, T, qt, ql, qi):
                return float(port.entropy_sa(p0, T, qt, ql, qi))

        def alpha(p0, T, qt, qv):
            return port.alpha_c(p0, T, qt, qv)
    else:
        # ThermodynamicsDry.entropy/eos/alpha (ThermodynamicsDry.pyx:87-103)
        def eos(p, s, qt):
            return float(port.dry_eos_c(p, s)), 0.0, 0.0

        def entropy(p0, T, qt, ql, qi):
            return float(port.sd_c(p0, T))

        def alpha(p0, T, qt, qv):
            return port.alpha_c(p0, T, 0.0, 0.0)

    sg = entropy(Pg, Tg, qtg, 0.0, 0.0)

    def rhs(p, z):
        T, ql, qi = eos(float(np.exp(p[0])), sg, qtg)
        return -port.g / (port.Rd * T * (1.0 - qtg + port.eps_vi * (qtg - ql - qi)))

    z = np.array(d.z[g_ - 1:-g_ + 1])
    z_half = np.append([0.0], np.array(d.z_half[g_:-g_]))
    p0 = np.log(Pg)
    ng2 = d.nlg[2]
    p = np.zeros(ng2)
    p_half = np.zeros(ng2)
    p[g_ - 1:-g_ + 1] = odeint(rhs, p0, z, hmax=1.0)[:, 0]
    p_half[g_:-g_] = odeint(rhs, p0, z_half, hmax=1.0)[1:, 0]
    p[:g_ - 1] = p[2 * g_ - 2:g_ - 1:-1]
    p[-g_ + 1:] = p[-g_ - 1:-2 * g_:-1]
    p_half[:g_] = p_half[2 * g_ - 1:g_ - 1:-1]
    p_half[-g_:] = p_half[-g_ - 1:-2 * g_ - 1:-1]
    p = np.exp(p)
    p_half = np.exp(p_half)
    alpha_ = np.zeros(ng2)
    alpha_half = np.zeros(ng2)
    for k in range(ng2):
        T, ql, qi = eos(p[k], sg, qtg)
        qv = qtg - (ql + qi)
        alpha_[k] = alpha(p[k], T, qtg, qv)
        T, ql, qi = eos(p_half[k], sg, qtg)
        qv = qtg - (ql + qi)
        alpha_half[k] = alpha(p_half[k], T, qtg, qv)
    return dict(p0=p, p0_half=p_half, alpha0=alpha_, alpha0_half=alpha_half,
                rho0=1.0 / alpha_, rho0_half=1.0 / alpha_half)


# ---------------------------------------------------------------------------
# single-rank hot-path simulation
# ---------------------------------------------------------------------------
class OracleSim:
    """PV/DV state plus the hot-path component updates of one rank.

    Variable order u, v, w, s[, qt] as Simulation3d.initialize (:70-75) and
    Th.initialize (ThermodynamicsSA.pyx:85-86) add them; bc types sym/asym.
    """

    def __init__(self, d: Dims, rs: dict, moist: bool, scalar_order=5, momentum_order=5,
                 dt=1.0, backend="port", table_xy=None, clip_qt=True):
        self.d = d
        self.rs = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in rs.items()}
        self.moist = moist
        self.backend = backend
        self.sorder = scalar_order
        self.morder = momentum_order
        self.dt = dt
        self.do_clip = clip_qt
        self.names = ["u", "v", "w", "s"] + (["qt"] if moist else [])
        self.bc_type = np.array([1.0, 1.0, -1.0, 1.0] + ([1.0] if moist else []))
        self.nv = len(self.names)
        npg = d.npg
        self.values = np.zeros(self.nv * npg)
        self.tendencies = np.zeros(self.nv * npg)
        self.value_copy = np.zeros(self.nv * npg)
        dv = ["buoyancy", "alpha", "temperature", "buoyancy_frequency"]
        dv += ["qv", "ql", "qi", "theta_rho", "thetali"] if moist else ["theta"]
        dv += ["dynamic_pressure", "divergence"]
        self.dv = {n: np.zeros(npg) for n in dv}
        self.nscalars = self.nv - 3
        self.flux = np.zeros(self.nscalars * 3 * npg)
        self.secant_iters = None
        self.surface = None  # an oracle.surface.OracleSurface, updated after MA as Simulation3d.pyx:167
        self.sgs = None  # an oracle.sgs.OracleSGS: Ke at the stage start, SGS/SD/MD after Sur (:159-172)
        self.forcing = None  # an oracle.forcing.OracleForcing, after SD/MD (:173)
        self.radiation = None  # an oracle.radiation.OracleRadiation, after Fo (:174)
        if moist:
            x, y = table_xy if table_xy is not None else cc_table()
            self.table_xy = (x, y)
            if backend == "ref":
                from . import ref
                self.LT = ref.Table(x, y)
            else:
                self.LT = port.Table(x, y)

    # views ----------------------------------------------------------------
    def var(self, name):
        i = self.names.index(name)
        return self.values[i * self.d.npg:(i + 1) * self.d.npg]

    def tend(self, name):
        i = self.names.index(name)
        return self.tendencies[i * self.d.npg:(i + 1) * self.d.npg]

    @property
    def K(self):
        if self.backend == "ref":
            from . import ref
            return ref
        return port

    # components ------------------------------------------------------------
    def th_update(self):
        """ThermodynamicsSA.update (ThermodynamicsSA.pyx:176-213) or
        ThermodynamicsDry.update (ThermodynamicsDry.pyx:105-120)."""
        K, d, rs, dv = self.K, self.d, self.rs, self.dv
        if self.moist:
            qt = self.var("qt")
            if self.do_clip:
                K.clip_qt(d, qt, 1e-11)
            it = K.eos_update_sa(d, self.LT, rs["p0_half"], self.var("s"), qt, dv["temperature"], dv["qv"],
                                 dv["ql"], dv["qi"], dv["alpha"])
            self.secant_iters = it
            K.buoyancy_update_sa(d, rs["alpha0_half"], dv["alpha"], dv["buoyancy"], self.tend("w"))
            K.bvf_sa(d, self.LT, rs["p0_half"], dv["temperature"], qt, dv["qv"], dv["theta_rho"],
                     dv["buoyancy_frequency"])
            K.thetali_update(d, rs["p0_half"], dv["temperature"], qt, dv["ql"], dv["qi"], dv["thetali"])
        else:
            K.eos_update_dry(d, rs["p0_half"], self.var("s"), dv["temperature"], dv["alpha"])
            K.buoyancy_update_dry(d, rs["alpha0_half"], dv["alpha"], dv["buoyancy"], self.tend("w"))
            K.bvf_dry(d, rs["p0_half"], dv["temperature"], dv["theta"], dv["buoyancy_frequency"])

    def sa_update(self):
        """ScalarAdvection.update (ScalarAdvection.pyx:69-123) without sedimentation."""
        K, d, rs = self.K, self.d, self.rs
        npg = d.npg
        vel = [self.var(n) for n in ("u", "v", "w")]
        for si, name in enumerate(self.names[3:]):
            for direction in range(3):
                fs = si * 3 * npg + direction * npg
                F = self.flux[fs:fs + npg]
                K.advective_fluxes_a(d, rs["rho0"], rs["rho0_half"], vel[direction], self.var(name), F,
                                     direction, self.sorder)
                K.scalar_flux_divergence(d, rs["alpha0"], rs["alpha0_half"], F, self.tend(name),
                                         d.dx[direction], direction)

    def ma_update(self):
        """MomentumAdvection.update (MomentumAdvection.pyx:41-69)."""
        K, d, rs = self.K, self.d, self.rs
        vel = [self.var(n) for n in ("u", "v", "w")]
        tnd = [self.tend(n) for n in ("u", "v", "w")]
        for ia in range(3):
            for ig in range(3):
                K.advective_tendencies_m(d, rs["rho0"], rs["rho0_half"], rs["alpha0"], rs["alpha0_half"],
                                         vel[ia], vel[ig], tnd[ia], ia, ig, self.morder)

    def ts_update(self, rk_step):
        port.update_third(self.values, self.tendencies, self.value_copy, rk_step, self.dt)

    def update_all_bcs(self):
        if self.backend == "ref":
            self._update_all_bcs_ref()
        else:
            port.update_all_bcs(self.d, self.values, self.bc_type)

    def _update_all_bcs_ref(self, values=None, bc_type=None):
        """PrognosticVariables.update_all_bcs (PrognosticVariables.pyx:183-233), one rank:
        MPI_Sendrecv to self in x and y, set_bcs in z."""
        from . import ref
        d = self.d
        values = self.values if values is None else values
        bc_type = self.bc_type if bc_type is None else bc_type
        nv = len(bc_type)
        dc = d.c()
        for dim in range(3):
            nbuf = dc.nbuffer[dim]
            send = np.zeros(nv * nbuf)
            for s in (-1, 1):
                if dim < 2:
                    for i in range(nv):
                        ref.build_buffer(i, dim, s, d, values, send)
                    recv = send.copy()
                    for i in range(nv):
                        ref.buffer_to_values(dim, s, d, values[i * d.npg:(i + 1) * d.npg],
                                             np.ascontiguousarray(recv[nbuf * i:]))
                else:
                    for i in range(nv):
                        ref.set_bcs(dim, s, bc_type[i], d, values[i * d.npg:(i + 1) * d.npg])

    def pr_update(self):
        """PressureSolver.update (PressureSolver.pyx:38-80)."""
        d, rs, dv = self.d, self.rs, self.dv
        u, v, w = self.var("u"), self.var("v"), self.var("w")
        u3_mean = port.horizontal_mean(d, w)
        w.reshape(d.shape)[...] -= u3_mean[None, None, :]
        div = dv["divergence"]
        div[:] = 0.0
        for direction, vel in enumerate((u, v, w)):
            port.second_order_divergence(d, rs["alpha0"], rs["alpha0_half"], vel, div, direction)
        p = dv["dynamic_pressure"]
        if self.backend == "ref":
            self._poisson_ref(div, p)
        else:
            port.poisson_solve(d, rs["rho0"], rs["rho0_half"], div, p)
        if self.backend == "ref":
            self._update_all_bcs_ref(p, np.array([1.0]))
        else:
            port.fill_ghosts(d, p, 1.0)
        port.pressure_correction(d, p, u, v, w)
        self.update_all_bcs()

    def _poisson_ref(self, div, pres):
        """As port.poisson_solve, but each column solved by the reference TDMA."""
        from . import ref
        mod = ref.tdma_module()
        if mod is None:
            return port.poisson_solve(self.d, self.rs["rho0"], self.rs["rho0_half"], div, pres)
        from scipy.fftpack import fft, ifft
        d = self.d
        D = div.reshape(d.shape)[d.interior()]
        H = fft(fft(D, axis=0), axis=1)
        kx2, ky2 = port.modified_wave_numbers(d)
        a, c = port.off_diagonals(d, self.rs["rho0"])
        Z = np.zeros_like(H)
        for i in range(d.n[0]):
            for j in range(d.n[1]):
                b = port.diagonal(d, self.rs["rho0"], self.rs["rho0_half"], np.array(kx2[i] + ky2[j]))
                dkr = np.ascontiguousarray(H[i, j].real)
                dki = np.ascontiguousarray(H[i, j].imag)
                mod.tdma_solve(dkr, a, np.ascontiguousarray(b), c)
                mod.tdma_solve(dki, a, np.ascontiguousarray(b), c)
                if i != 0 or j != 0:
                    Z[i, j] = dkr + dki * 1j
        Z = ifft(ifft(Z, axis=1), axis=0)
        P = pres.reshape(d.shape)
        P[...] = 0.0
        P[d.interior()] = Z.real

    # driver ------------------------------------------------------------------
    def stage(self, rk_step):
        """One RK stage of Simulation3d.run (:158-180) over the hot path."""
        if self.sgs is not None:
            self.sgs.ke_update(self)
        self.th_update()
        self.sa_update()
        self.ma_update()
        if self.surface is not None:
            self.surface.update(self)
        if self.sgs is not None:
            self.sgs.sgs_update(self)
            self.sgs.sd_update(self)
            self.sgs.md_update(self)
        if self.forcing is not None:
            self.forcing.update(self)
        if self.radiation is not None:
            self.radiation.update(self)
        self.ts_update(rk_step)
        self.update_all_bcs()
        self.pr_update()

    def step(self):
        for rk in range(3):
            self.stage(rk)
