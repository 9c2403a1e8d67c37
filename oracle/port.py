"""numpy restatement of the PyCLES hot-path kernels -- TEST INFRASTRUCTURE ONLY.

Every function follows one reference function (file:line cited) and keeps
its loop ranges and its floating-point evaluation order, so that on the same
inputs it agrees with the reference's C to rounding of the transcendental
functions (bit-exact for the polynomial parts).  Arrays are 3-D views
``[i, j, k]`` of the flat ghosted fields (k contiguous), shape ``dims.nlg``.

Pinned against the compiled reference (``oracle.ref``) by
``tests/test_oracle_pin.py``.
"""
from __future__ import annotations

import math

import numpy as np

from .dims import Dims

# The reference evaluates exp/log/pow with the C library; numpy's vectorised
# versions differ from it in the last bit now and then, which the buoyancy's
# cancellation amplifies.  These call the C library (Python's math module)
# elementwise so the restatement matches the reference's transcendentals
# bit for bit.
_vlog = np.frompyfunc(math.log, 1, 1)
_vexp = np.frompyfunc(math.exp, 1, 1)
_vpow = np.frompyfunc(math.pow, 2, 1)


def _log(x):
    r = _vlog(np.asarray(x, dtype=np.float64))
    return np.asarray(r, dtype=np.float64)


def _exp(x):
    r = _vexp(np.asarray(x, dtype=np.float64))
    return np.asarray(r, dtype=np.float64)


def _pow(x, y):
    r = _vpow(np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64))
    return np.asarray(r, dtype=np.float64)

# generate_parameters.py:19-41 (values as written to parameters.h)
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
pi = 3.141592653589793


# ---------------------------------------------------------------------------
# interpolants, Csrc/advection_interpolation.h
# ---------------------------------------------------------------------------
def interp_2(phi, phip1):  # :4-6
    return 0.5 * (phi + phip1)


def interp_4(phim1, phi, phip1, phip2):  # :12-14
    return (7.0 / 12.0) * (phi + phip1) - (1.0 / 12.0) * (phim1 + phip2)


def interp_6(phim2, phim1, phi, phip1, phip2, phip3):  # :20-24
    return ((37.0 / 60.0) * (phi + phip1) - (2.0 / 15.0) * (phim1 + phip2)
            + (1.0 / 60.0) * (phim2 + phip3))


def interp_weno5(phim2, phim1, phi, phip1, phip2):  # :79-104
    p0 = (1.0 / 3.0) * phim2 - (7.0 / 6.0) * phim1 + (11.0 / 6.0) * phi
    p1 = (-1.0 / 6.0) * phim1 + (5.0 / 6.0) * phi + (1.0 / 3.0) * phip1
    p2 = (1.0 / 3.0) * phi + (5.0 / 6.0) * phip1 - (1.0 / 6.0) * phip2
    t2a = phi - 2.0 * phip1 + phip2
    t2b = 3.0 * phi - 4.0 * phip1 + phip2
    beta2 = 13.0 / 12.0 * t2a * t2a + 0.25 * t2b * t2b
    t1a = phim1 - 2.0 * phi + phip1
    t1b = phim1 - phip1
    beta1 = 13.0 / 12.0 * t1a * t1a + 0.25 * t1b * t1b
    t0a = phim2 - 2.0 * phim1 + phi
    t0b = phim2 - 4.0 * phim1 + 3.0 * phi
    beta0 = 13.0 / 12.0 * t0a * t0a + 0.25 * t0b * t0b
    alpha0 = 0.1 / ((beta0 + 1e-10) * (beta0 + 1e-10))
    alpha1 = 0.6 / ((beta1 + 1e-10) * (beta1 + 1e-10))
    alpha2 = 0.3 / ((beta2 + 1e-10) * (beta2 + 1e-10))
    alpha_sum_inv = 1.0 / (alpha0 + alpha1 + alpha2)
    w0 = alpha0 * alpha_sum_inv
    w1 = alpha1 * alpha_sum_inv
    w2 = alpha2 * alpha_sum_inv
    return w0 * p0 + w1 * p1 + w2 * p2


def interp_weno7(phim3, phim2, phim1, phi, phip1, phip2, phip3):  # :106-145
    p0 = (-1.0 / 4.0) * phim3 + (13.0 / 12.0) * phim2 + (-23.0 / 12.0) * phim1 + (25.0 / 12.0) * phi
    p1 = (1.0 / 12.0) * phim2 + (-5.0 / 12.0) * phim1 + (13.0 / 12.0) * phi + (1.0 / 4.0) * phip1
    p2 = (-1.0 / 12.0) * phim1 + (7.0 / 12.0) * phi + (7.0 / 12.0) * phip1 + (-1.0 / 12.0) * phip2
    p3 = (1.0 / 4.0) * phi + (13.0 / 12.0) * phip1 + (-5.0 / 12.0) * phip2 + (1.0 / 12.0) * phip3
    beta0 = (phim3 * (547.0 * phim3 - 3882.0 * phim2 + 4642.0 * phim1 - 1854.0 * phi)
             + phim2 * (7043.0 * phim2 - 17246.0 * phim1 + 7042.0 * phi)
             + phim1 * (11003.0 * phim1 - 9402.0 * phi)
             + 2107.0 * phi * phi)
    beta1 = (phim2 * (267.0 * phim2 - 1642.0 * phim1 + 1602.0 * phi - 494.0 * phip1)
             + phim1 * (2843.0 * phim1 - 5966.0 * phi + 1922.0 * phip1)
             + phi * (3443.0 * phi - 2522.0 * phip1)
             + 547.0 * phip1 * phip1)
    beta2 = (phim1 * (547.0 * phim1 - 2522.0 * phi + 1922.0 * phip1 - 494.0 * phip2)
             + phi * (3443.0 * phi - 5966.0 * phip1 + 1602.0 * phip2)
             + phip1 * (2843.0 * phip1 - 1642.0 * phip2)
             + 267.0 * phip2 * phip2)
    beta3 = (phi * (2107.0 * phi - 9402.0 * phip1 + 7042.0 * phip2 - 1854.0 * phip3)
             + phip1 * (11003.0 * phip1 - 17246.0 * phip2 + 4642.0 * phip3)
             + phip2 * (7043.0 * phip2 - 3882.0 * phip3)
             + 547.0 * phip3 * phip3)
    alpha0 = (1.0 / 35.0) / ((beta0 + 1e-10) * (beta0 + 1e-10))
    alpha1 = (12.0 / 35.0) / ((beta1 + 1e-10) * (beta1 + 1e-10))
    alpha2 = (18.0 / 35.0) / ((beta2 + 1e-10) * (beta2 + 1e-10))
    alpha3 = (4.0 / 35.0) / ((beta3 + 1e-10) * (beta3 + 1e-10))
    alpha_sum_inv = 1.0 / (alpha0 + alpha1 + alpha2 + alpha3)
    w0 = alpha0 * alpha_sum_inv
    w1 = alpha1 * alpha_sum_inv
    w2 = alpha2 * alpha_sum_inv
    w3 = alpha3 * alpha_sum_inv
    return w0 * p0 + w1 * p1 + w2 * p2 + w3 * p3


# ---------------------------------------------------------------------------
# index helpers
# ---------------------------------------------------------------------------
def _region(shape, lo, hi_off):
    return tuple(slice(lo, n - hi_off) for n in shape)


def _sh(A, reg, d, o):
    """View of A over region ``reg`` shifted by ``o`` cells along axis d."""
    s = list(reg)
    s[d] = slice(reg[d].start + o, reg[d].stop + o)
    return A[tuple(s)]


def _kvec(v, reg, ko=0):
    """1-D profile over the k-range of ``reg`` (shifted by ko), broadcastable."""
    return v[reg[2].start + ko: reg[2].stop + ko][None, None, :]


# ---------------------------------------------------------------------------
# scalar advection, Csrc/scalar_advection.h
# ---------------------------------------------------------------------------
def advective_fluxes_a(d: Dims, rho0, rho0_half, vel, scalar, flux, direction, order):
    """weno_fifth_order_a (:319-394) / weno_seventh_order_a (:396-480)."""
    sh = d.shape
    V = vel.reshape(sh)
    S = scalar.reshape(sh)
    F = flux.reshape(sh)
    if order == 7:
        reg = _region(sh, 3, 4)
        phip = interp_weno7(*[_sh(S, reg, direction, o) for o in (-3, -2, -1, 0, 1, 2, 3)])
        phim = interp_weno7(*[_sh(S, reg, direction, o) for o in (4, 3, 2, 1, 0, -1, -2)])
    elif order == 5:
        reg = _region(sh, 2, 3)
        phip = interp_weno5(*[_sh(S, reg, direction, o) for o in (-2, -1, 0, 1, 2)])
        phim = interp_weno5(*[_sh(S, reg, direction, o) for o in (3, 2, 1, 0, -1)])
    else:
        raise ValueError("oracle restates WENO5/WENO7 only")
    u = V[reg]
    rho = _kvec(rho0 if direction == 2 else rho0_half, reg)
    F[reg] = 0.5 * ((u + np.abs(u)) * phip + (u - np.abs(u)) * phim) * rho


def scalar_flux_divergence(d: Dims, alpha0, alpha0_half, flux, tend, dx, direction):
    """Csrc/flux_divergence.h:4-32 (uses dims->dxi[d])."""
    sh = d.shape
    F = flux.reshape(sh)
    T = tend.reshape(sh)
    reg = _region(sh, d.gw, d.gw)
    a = _kvec(alpha0_half, reg)
    T[reg] -= a * (F[reg] - _sh(F, reg, direction, -1)) * d.dxi[direction]


def momentum_flux_divergence(d: Dims, alpha0, alpha0_half, flux, tend, d_advected, d_advecting):
    """Csrc/flux_divergence.h:34-60."""
    sh = d.shape
    F = flux.reshape(sh)
    T = tend.reshape(sh)
    reg = _region(sh, d.gw, d.gw)
    a = _kvec(alpha0_half if d_advected != 2 else alpha0, reg)
    T[reg] -= a * (F[reg] - _sh(F, reg, d_advecting, -1)) * d.dxi[d_advecting]


def advective_tendencies_m(d: Dims, rho0, rho0_half, alpha0, alpha0_half, vel_advected, vel_advecting,
                           tend, d_advected, d_advecting, order):
    """weno_fifth_order_m (Csrc/momentum_advection_weno.h:113-245) and
    weno_seventh_order_m (:247-400), followed by momentum_flux_divergence."""
    sh = d.shape
    A = vel_advected.reshape(sh)
    G = vel_advecting.reshape(sh)
    flux = np.zeros(sh)
    ed, ing = d_advecting, d_advected
    if order == 7:
        reg = _region(sh, 3, 4)
        phip = interp_weno7(*[_sh(A, reg, ed, o) for o in (-3, -2, -1, 0, 1, 2, 3)])
        phim = interp_weno7(*[_sh(A, reg, ed, o) for o in (4, 3, 2, 1, 0, -1, -2)])
        vel_adv = interp_6(*[_sh(G, reg, ing, o) for o in (-2, -1, 0, 1, 2, 3)])
    elif order == 5:
        reg = _region(sh, 2, 3)
        phip = interp_weno5(*[_sh(A, reg, ed, o) for o in (-2, -1, 0, 1, 2)])
        phim = interp_weno5(*[_sh(A, reg, ed, o) for o in (3, 2, 1, 0, -1)])
        vel_adv = interp_4(*[_sh(G, reg, ing, o) for o in (-1, 0, 1, 2)])
    else:
        raise ValueError("oracle restates WENO5/WENO7 only")
    if d_advected != 2 and d_advecting != 2:
        rho = _kvec(rho0_half, reg)
    elif d_advected == 2 and d_advecting == 2:
        rho = _kvec(rho0_half, reg, 1)
    else:
        rho = _kvec(rho0, reg)
    flux[reg] = 0.5 * ((vel_adv + np.abs(vel_adv)) * phip + (vel_adv - np.abs(vel_adv)) * phim) * rho
    momentum_flux_divergence(d, alpha0, alpha0_half, flux.reshape(-1), tend, d_advected, d_advecting)


# ---------------------------------------------------------------------------
# thermodynamic functions, Csrc/thermodynamic_functions.h, Csrc/entropies.h
# ---------------------------------------------------------------------------
def exner_c(p0):
    return _pow(p0 / p_tilde, kappa)


def pd_c(p0, qt, qv):
    return p0 * (1.0 - qt) / (1.0 - qt + eps_vi * qv)


def pv_c(p0, qt, qv):
    return p0 * eps_vi * qv / (1.0 - qt + eps_vi * qv)


def qv_star_c(p0, qt, pv):
    return eps_v * (1.0 - qt) * pv / (p0 - pv)


def alpha_c(p0, T, qt, qv):
    return (Rd * T) / p0 * (1.0 - qt + eps_vi * qv)


def buoyancy_c(alpha0, alpha):
    return g * (alpha - alpha0) / alpha0


def cpm_c(qt):
    return (1.0 - qt) * cpd + qt * cpv


def sd_c(pd, T):
    return sd_tilde + cpd * _log(T / T_tilde) - Rd * _log(pd / p_tilde)


def sv_c(pv, T):
    return sv_tilde + cpv * _log(T / T_tilde) - Rv * _log(pv / p_tilde)


def sc_c(L, T):
    return -L / T


def latent_heat_variable(T, lam=1.0):
    """Microphysics.pxd:71-75."""
    TC = T - 273.15
    return (2500.8 - 2.36 * TC + 0.0016 * TC * TC - 0.00006 * TC * TC * TC) * 1000.0


class Table:
    """init_table / lookup (Csrc/lookup.h:16-54)."""

    def __init__(self, x, y):
        x = np.asarray(x, dtype=np.float64)
        self.y = np.ascontiguousarray(y, dtype=np.float64)
        self.x_min = float(np.min(x))
        self.x_max = float(np.max(x))
        self.dx = float(x[1] - x[0])
        self.dxi = 1.0 / self.dx

    def lookup(self, x):
        indx = np.floor((x - self.x_min) * self.dxi).astype(np.int64)
        y1 = self.y[indx]
        y2 = self.y[indx + 1]
        x1 = self.x_min + self.dx * indx
        return y1 + (x - x1) * (y2 - y1) * self.dxi


def temperature_no_ql(pd, pv, s, qt):
    """Csrc/thermodynamics_sa.h:10-15."""
    return T_tilde * _exp((s - (1.0 - qt) * (sd_tilde - Rd * _log(pd / p_tilde))
                           - qt * (sv_tilde - Rv * _log(pv / p_tilde)))
                          / ((1.0 - qt) * cpd + qt * cpv))


def eos_c(LT: Table, p0, s, qt, max_iter=10_000, T2_seed=None):
    """Vectorised eos_c (Csrc/thermodynamics_sa.h:17-66).

    Returns T, qv, ql, qi, iterations.  ``T2_seed`` (optional) replaces the
    first secant point T_2 of :39 -- the learned-guess variant -- clamped to
    [T_1 + (T_2 - T_1)/16, T_2], the interval that holds the root; the loop
    itself is unchanged.
    """
    p0 = np.asarray(p0, dtype=np.float64)
    s = np.asarray(s, dtype=np.float64)
    qt = np.asarray(qt, dtype=np.float64)
    p0, s, qt = np.broadcast_arrays(p0, s, qt)
    shape = s.shape
    p0 = p0.reshape(-1).copy()
    s = s.reshape(-1).copy()
    qt = qt.reshape(-1).copy()
    T = np.empty_like(s)
    qv = qt.copy()
    ql = np.zeros_like(s)
    qi = np.zeros_like(s)
    iters = np.zeros(s.shape, dtype=np.int64)
    pv_1 = pv_c(p0, qt, qt)
    pd_1 = p0 - pv_1
    T_1 = temperature_no_ql(pd_1, pv_1, s, qt)
    pv_star_1 = LT.lookup(T_1)
    qv_star_1 = qv_star_c(p0, qt, pv_star_1)
    unsat = qt <= qv_star_1
    T[unsat] = T_1[unsat]
    sat = np.nonzero(~unsat)[0]
    if sat.size:
        P, S, Q = p0[sat], s[sat], qt[sat]
        t1 = T_1[sat]
        pd1, pv1 = pd_1[sat], pv_1[sat]
        qvs1 = qv_star_1[sat]
        sigma_1 = Q - qvs1
        L_1 = latent_heat_variable(t1)
        s_1 = sd_c(pd1, t1) * (1.0 - Q) + sv_c(pv1, t1) * Q + sc_c(L_1, t1) * sigma_1
        f_1 = S - s_1
        t2 = t1 + sigma_1 * L_1 / ((1.0 - Q) * cpd + qvs1 * cpv)
        if T2_seed is not None:
            guess = np.asarray(T2_seed, dtype=np.float64).reshape(-1)[sat]
            t2 = np.fmin(np.fmax(guess, t1 + 0.0625 * (t2 - t1)), t2)
        out_T = np.empty_like(t1)
        out_qv = np.empty_like(t1)
        out_sig = np.empty_like(t1)
        out_lam = np.ones_like(t1)
        out_it = np.zeros(t1.shape, dtype=np.int64)
        act = np.arange(sat.size)
        it = 0
        while act.size and it < max_iter:
            it += 1
            P_, Q_, S_ = P[act], Q[act], S[act]
            T1_, T2_, F1_ = t1[act], t2[act], f_1[act]
            pv_star_2 = LT.lookup(T2_)
            qv_star_2 = qv_star_c(P_, Q_, pv_star_2)
            pv_2 = pv_c(P_, Q_, qv_star_2)
            pd_2 = P_ - pv_2
            sigma_2 = Q_ - qv_star_2
            L_2 = latent_heat_variable(T2_)
            s_2 = sd_c(pd_2, T2_) * (1.0 - Q_) + sv_c(pv_2, T2_) * Q_ + sc_c(L_2, T2_) * sigma_2
            f_2 = S_ - s_2
            T_n = T2_ - f_2 * (T2_ - T1_) / (f_2 - F1_)
            t1[act] = T2_
            t2[act] = T_n
            f_1[act] = f_2
            delta_T = np.abs(T_n - T2_)
            out_T[act] = T_n
            out_qv[act] = qv_star_2
            out_sig[act] = sigma_2
            out_it[act] = it
            keep = (delta_T >= 1.0e-3) | (sigma_2 < 0.0)
            act = act[keep]
        T[sat] = out_T
        qv[sat] = out_qv
        ql[sat] = out_lam * out_sig
        qi[sat] = (1.0 - out_lam) * out_sig
        iters[sat] = out_it
    return (T.reshape(shape), qv.reshape(shape), ql.reshape(shape), qi.reshape(shape),
            iters.reshape(shape))


def clip_qt(d: Dims, qt, clip_value):
    """Csrc/thermodynamics_sa.h:213-219."""
    np.maximum(qt, clip_value, out=qt)


def eos_update_sa(d: Dims, LT: Table, p0, s, qt, T, qv, ql, qi, alpha):
    """Csrc/thermodynamics_sa.h:68-96 (all ghosted cells)."""
    sh = d.shape
    P = np.broadcast_to(p0[None, None, :], sh)
    T_, qv_, ql_, qi_, it = eos_c(LT, P, s.reshape(sh), qt.reshape(sh))
    T[:] = T_.reshape(-1)
    qv[:] = qv_.reshape(-1)
    ql[:] = ql_.reshape(-1)
    qi[:] = qi_.reshape(-1)
    alpha[:] = alpha_c(P, T.reshape(sh), qt.reshape(sh), qv.reshape(sh)).reshape(-1)
    return it


def buoyancy_update_sa(d: Dims, alpha0, alpha, buoyancy, wt):
    """Csrc/thermodynamics_sa.h:98-132."""
    sh = d.shape
    A = alpha.reshape(sh)
    B = buoyancy.reshape(sh)
    W = wt.reshape(sh)
    n2 = sh[2]
    B[:, :, 0:n2 - 1] = buoyancy_c(alpha0[None, None, 0:n2 - 1], A[:, :, 0:n2 - 1])
    W[:, :, 1:n2 - 3] = W[:, :, 1:n2 - 3] + interp_2(B[:, :, 1:n2 - 3], B[:, :, 2:n2 - 2])


def bvf_sa(d: Dims, LT: Table, p0, T, qt, qv, theta_rho, bvf):
    """Csrc/thermodynamics_sa.h:134-182."""
    sh = d.shape
    n2 = sh[2]
    Tt_ = T.reshape(sh)
    QT = qt.reshape(sh)
    QV = qv.reshape(sh)
    TR = theta_rho.reshape(sh)
    BV = bvf.reshape(sh)
    dzi = 1.0 / d.dx[2]
    k = slice(1, n2 - 1)
    TR[:, :, k] = Tt_[:, :, k] * (1.0 - QT[:, :, k] + eps_vi * QV[:, :, k]) / exner_c(p0[None, None, k])
    k = slice(2, n2 - 2)
    km = slice(1, n2 - 3)
    kp = slice(3, n2 - 1)
    Tk, Tm, Tp = Tt_[:, :, k], Tt_[:, :, km], Tt_[:, :, kp]
    Qk, Qm, Qp = QT[:, :, k], QT[:, :, km], QT[:, :, kp]
    sat = QV[:, :, k] < Qk
    P = np.broadcast_to(p0[None, None, k], Tk.shape)
    Lv = latent_heat_variable(Tk)
    pv_star = LT.lookup(Tk)
    rsl = eps_v * pv_star / (P - pv_star)
    gamma_w = (g / cpd * (1.0 / (1.0 - Qk)) * (1.0 + Lv * rsl / (Rd * Tk))
               / (cpm_c(Qk) / cpd + Lv * Lv * (eps_v + rsl) * rsl / (cpd * Rd * Tk * Tk)))
    dTdz = (interp_2(Tk, Tp) - interp_2(Tm, Tk)) * dzi
    dqtdz = (interp_2(Qk, Qp) - interp_2(Qm, Qk)) * dzi
    moist = g / Tk * (dTdz + gamma_w) * (1.0 + Lv * rsl / (Rd * Tk)) - dqtdz / (1.0 - Qk)
    Rk, Rm, Rp = TR[:, :, k], TR[:, :, km], TR[:, :, kp]
    dry = g / Rk * (interp_2(Rk, Rp) - interp_2(Rm, Rk)) * dzi
    BV[:, :, k] = np.where(sat, moist, dry)


def thetali_update(d: Dims, p0, T, qt, ql, qi, thetali):
    """Csrc/thermodynamics_sa.h:185-211 with thetali_c (thermodynamic_functions.h:15-18)."""
    sh = d.shape
    P = p0[None, None, :]
    Tt_ = T.reshape(sh)
    Lv = latent_heat_variable(Tt_)
    Q = qt.reshape(sh)
    theta = Tt_ / exner_c(P)
    thetali[:] = (theta * _exp(-Lv * (ql.reshape(sh) / (1.0 - Q) + qi.reshape(sh) / (1.0 - Q))
                               / (Tt_ * cpd))).reshape(-1)


# dry thermodynamics, Csrc/thermodynamics_dry.h ------------------------------
def dry_eos_c(pd, s):  # :8-10
    return T_tilde * (_exp((s - sd_tilde + Rd * _log(pd / p_tilde)) / cpd))


def eos_update_dry(d: Dims, pd, s, T, alpha):  # :12-37
    sh = d.shape
    P = pd[None, None, :]
    T[:] = dry_eos_c(P, s.reshape(sh)).reshape(-1)
    alpha[:] = alpha_c(P, T.reshape(sh), 0.0, 0.0).reshape(-1)


def buoyancy_update_dry(d: Dims, alpha0, alpha, buoyancy, wt):  # :39-73
    sh = d.shape
    A = alpha.reshape(sh)
    B = buoyancy.reshape(sh)
    W = wt.reshape(sh)
    i = slice(0, sh[0] - 1)
    j = slice(0, sh[1] - 1)
    k = slice(0, sh[2] - 1)
    B[i, j, k] = buoyancy_c(alpha0[None, None, k], A[i, j, k])
    W[i, j, k] += interp_2(B[i, j, k], B[i, j, 1:sh[2]])


def bvf_dry(d: Dims, p0, T, theta, bvf):  # :75-110
    sh = d.shape
    n2 = sh[2]
    TH = theta.reshape(sh)
    BV = bvf.reshape(sh)
    dzi = 1.0 / d.dx[2]
    k = slice(1, n2)
    TH[:, :, k] = T.reshape(sh)[:, :, k] / exner_c(p0[None, None, k])
    k = slice(2, n2 - 1)
    BV[:, :, k] = g / TH[:, :, k] * (interp_2(TH[:, :, k], TH[:, :, 3:n2])
                                     - interp_2(TH[:, :, 1:n2 - 2], TH[:, :, k])) * dzi


def entropy_sa(p0, T, qt, ql, qi):
    """ThermodynamicsSA.entropy (ThermodynamicsSA.pyx:140-159)."""
    qv = qt - ql - qi
    pd = pd_c(p0, qt, qv)
    pv = pv_c(p0, qt, qv)
    L = latent_heat_variable(T)
    return sd_c(pd, T) * (1.0 - qt) + sv_c(pv, T) * qt + sc_c(L, T) * (ql + qi)


# ---------------------------------------------------------------------------
# halos, Csrc/prognostic_variables.h + PrognosticVariables.pyx:183-233
# ---------------------------------------------------------------------------
def set_bcs(d: Dims, V, dim, s, bc_factor):
    """set_bcs (Csrc/prognostic_variables.h:205-270) on a 3-D view."""
    assert dim == 2
    gw = d.gw
    n2 = d.shape[2]
    if s == -1:
        b = n2 - gw
        if bc_factor == 1.0:
            for k in range(gw):
                V[:, :, b + k] = V[:, :, b - k - 1]
        elif bc_factor == 2.0:
            for k in range(gw):
                V[:, :, b + k] = V[:, :, b - 1]
        else:
            V[:, :, b] = 0.0
            for k in range(1, gw):
                V[:, :, b + k] = bc_factor * V[:, :, b - k]
    else:
        b = gw - 1
        if bc_factor == 1.0:
            for k in range(gw):
                V[:, :, b - k] = V[:, :, b + k + 1]
        elif bc_factor == 2.0:
            for k in range(gw):
                V[:, :, b - k] = V[:, :, b + 1]
        else:
            V[:, :, b] = 0.0
            for k in range(1, gw):
                V[:, :, b - k] = bc_factor * V[:, :, b + k]


def fill_ghosts(d: Dims, field, bc_factor):
    """One variable of update_all_bcs on a single periodic-x,y rank:
    x then y self-exchange (build_buffer/buffer_to_values, :11-203),
    then the z boundary conditions (set_bcs)."""
    V = field.reshape(d.shape)
    gw = d.gw
    for dim in (0, 1):
        n = d.shape[dim]
        idx = [slice(None)] * 3
        src = [slice(None)] * 3
        # s = -1: upper ghosts receive the lower interior planes
        idx[dim] = slice(n - gw, n)
        src[dim] = slice(gw, 2 * gw)
        V[tuple(idx)] = V[tuple(src)]
        # s = +1: lower ghosts receive the upper interior planes
        idx[dim] = slice(0, gw)
        src[dim] = slice(n - 2 * gw, n - gw)
        V[tuple(idx)] = V[tuple(src)]
    set_bcs(d, V, 2, -1, bc_factor)
    set_bcs(d, V, 2, 1, bc_factor)


def update_all_bcs(d: Dims, values, bc_type):
    for v, bc in enumerate(bc_type):
        fill_ghosts(d, values[v * d.npg:(v + 1) * d.npg], bc)


# ---------------------------------------------------------------------------
# time stepping, TimeStepping.pyx:131-151
# ---------------------------------------------------------------------------
def update_third(values, tendencies, value_copy, rk_step, dt):
    if rk_step == 0:
        value_copy[:] = values
        values += tendencies * dt
    elif rk_step == 1:
        values[:] = 0.75 * value_copy + 0.25 * (values + tendencies * dt)
    else:
        values[:] = (1.0 / 3.0) * value_copy + (2.0 / 3.0) * (values + tendencies * dt)
    tendencies[:] = 0.0


# ---------------------------------------------------------------------------
# pressure, PressureSolver.pyx + PressureFFTParallel.pyx (one rank)
# ---------------------------------------------------------------------------
def horizontal_mean(d: Dims, values):
    """ParallelMPI.HorizontalMean (ParallelMPI.pyx:196-241), one rank: every
    level's sum is accumulated in the reference's order, i outer, j inner,
    one rounded addition per column (:219-226), then scaled by
    1/(n0 n1) (:232-236).  The order matters: w's horizontal mean is a
    cancelling sum, and the pressure solve subtracts it from every cell."""
    V = values.reshape(d.shape)
    g_ = d.gw
    s = np.zeros(d.shape[2])
    for i in range(g_, d.shape[0] - g_):
        Vi = V[i]
        for j in range(g_, d.shape[1] - g_):
            s += Vi[j]
    return s * (1.0 / float(d.n[1] * d.n[0]))


def modified_wave_numbers(d: Dims):
    """PressureFFTParallel.compute_modified_wave_numbers (:64-98)."""
    import math
    out = []
    for dim in (0, 1):
        n = d.n[dim]
        k2 = np.empty(n)
        for i in range(n):
            xi = float(i) if i <= n / 2 else float(i - n)
            # libm cos, as the reference's `from libc.math cimport cos`
            k2[i] = (2.0 * math.cos((2.0 * pi / n) * xi) - 2.0) / d.dx[dim] / d.dx[dim]
        k2[0] = 0.0
        out.append(k2)
    return out


def off_diagonals(d: Dims, rho0):
    """PressureFFTParallel.compute_off_diagonals (:100-127)."""
    n = d.n[2]
    gw = d.gw
    dzi = d.dxi[2]
    a = np.zeros(n)
    c = np.zeros(n)
    a[0] = 0.0
    c[0] = dzi * dzi * rho0[gw]
    for k in range(1, n - 1):
        a[k] = dzi * dzi * rho0[k + gw - 1]
        c[k] = dzi * dzi * rho0[k + gw]
    k = n - 1
    a[k] = dzi * dzi * rho0[k + gw - 1]
    c[k] = 0.0
    return a, c


def diagonal(d: Dims, rho0, rho0_half, kx2ky2):
    """PressureFFTParallel.compute_diagonal (:129-148), vectorised over columns.
    ``kx2ky2`` holds kx2[i] + ky2[j] per column; returns b[..., k]."""
    n = d.n[2]
    gw = d.gw
    dzi = d.dxi[2]
    K = np.asarray(kx2ky2)[..., None]
    b = np.empty(K.shape[:-1] + (n,))
    b[..., 0] = rho0_half[gw] * K[..., 0] - (rho0[gw]) * dzi * dzi
    kk = np.arange(1, n - 1)
    b[..., 1:n - 1] = rho0_half[kk + gw] * K - (rho0[kk + gw] + rho0[kk + gw - 1]) * dzi * dzi
    k = n - 1
    b[..., k] = rho0_half[k + gw] * K[..., 0] - (rho0[k + gw - 1]) * dzi * dzi
    return b


def tdma(x, a, b, c):
    """TDMA.solve (SparseSolvers.pyx:24-44) over the last axis, batched."""
    n = x.shape[-1]
    scratch = np.empty_like(b)
    scratch[..., 0] = c[0] / b[..., 0]
    x[..., 0] = x[..., 0] / b[..., 0]
    for i in range(1, n):
        m = 1.0 / (b[..., i] - a[i] * scratch[..., i - 1])
        scratch[..., i] = c[i] * m
        x[..., i] = (x[..., i] - a[i] * x[..., i - 1]) * m
    for i in range(n - 2, -1, -1):
        x[..., i] = x[..., i] - scratch[..., i] * x[..., i + 1]
    return x


def poisson_solve(d: Dims, rho0, rho0_half, div, pres):
    """PressureFFTParallel.solve (:150-219), one rank: the pencil transposes
    are identity re-layouts, so x-FFT, y-FFT, per-column TDMA on the real and
    imaginary parts, mode (0,0) zeroed, inverse y then x, real part; ghost
    cells of the result are zero."""
    from scipy.fftpack import fft, ifft
    import warnings
    D = div.reshape(d.shape)[d.interior()]
    H = fft(D, axis=0)
    H = fft(H, axis=1)
    kx2, ky2 = modified_wave_numbers(d)
    a, c = off_diagonals(d, rho0)
    b = diagonal(d, rho0, rho0_half, kx2[:, None] + ky2[None, :])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        xr = tdma(np.ascontiguousarray(H.real), a, b, c)
        xi = tdma(np.ascontiguousarray(H.imag), a, b, c)
    Z = xr + 1j * xi
    Z[0, 0, :] = 0.0
    Z = ifft(Z, axis=1)
    Z = ifft(Z, axis=0)
    P = pres.reshape(d.shape)
    P[...] = 0.0
    P[d.interior()] = Z.real


def second_order_divergence(d: Dims, alpha0, alpha0_half, vel, div, direction):
    """PressureSolver.pyx:138-175."""
    sh = d.shape
    V = vel.reshape(sh)
    D = div.reshape(sh)
    reg = _region(sh, d.gw, d.gw)
    dxi = 1.0 / d.dx[direction]
    if direction != 2:
        ah = _kvec(alpha0_half, reg)
        D[reg] += (V[reg] / ah - _sh(V, reg, direction, -1) / ah) * dxi
    else:
        D[reg] += ((V[reg]) / _kvec(alpha0, reg) - (_sh(V, reg, 2, -1)) / _kvec(alpha0, reg, -1)) * dxi


def pressure_correction(d: Dims, p, u, v, w):
    """PressureSolver.pyx:83-110: range [0, nlg-1) in every dimension."""
    sh = d.shape
    P = p.reshape(sh)
    reg = (slice(0, sh[0] - 1), slice(0, sh[1] - 1), slice(0, sh[2] - 1))
    Pc = P[reg]
    u.reshape(sh)[reg] -= (_sh(P, reg, 0, 1) - Pc) * d.dxi[0]
    v.reshape(sh)[reg] -= (_sh(P, reg, 1, 1) - Pc) * d.dxi[1]
    w.reshape(sh)[reg] -= (_sh(P, reg, 2, 1) - Pc) * d.dxi[2]


# ---------------------------------------------------------------------------
# surface layer, Csrc/surface.h (constants generate_parameters.py:44-49)
# ---------------------------------------------------------------------------
vkb = 0.35
Pr0 = 0.74
beta_m = 4.7
beta_h = beta_m / Pr0
gamma_m = 15.0
gamma_h = 9.0


def psi_m_unstable(zeta, zeta0):
    """Csrc/surface.h:6-12 (scalars)."""
    x = math.pow((1.0 - gamma_m * zeta), 0.25)
    x0 = math.pow((1.0 - gamma_m * zeta0), 0.25)
    return (2.0 * math.log((1.0 + x) / (1.0 + x0)) + math.log((1.0 + x * x) / (1.0 + x0 * x0))
            - 2.0 * math.atan(x) + 2.0 * math.atan(x0))


def psi_m_stable(zeta, zeta0):
    """Csrc/surface.h:22-25."""
    return -beta_m * (zeta - zeta0)


def compute_ustar(windspeed, buoyancy_flux, z0, zb):
    """Csrc/surface.h:34-93 (scalars).  The reference returns ``ustar``, which
    it sets to the first iterate ustar1 = windspeed vkb / (log(zb/z0) - psi_m)
    from the neutral guess before its secant loop (:52, :73) and does not
    update inside it; the loop's iterates never reach the result, so this
    restatement stops at that iterate."""
    logz = math.log(zb / z0)
    ustar0 = windspeed * vkb / logz
    if not (math.fabs(buoyancy_flux) > 1.0e-20):
        return ustar0
    lmo = -ustar0 * ustar0 * ustar0 / (buoyancy_flux * vkb)
    zeta = zb / lmo
    zeta0 = z0 / lmo
    psi = psi_m_stable(zeta, zeta0) if zeta >= 0.0 else psi_m_unstable(zeta, zeta0)
    return windspeed * vkb / (logz - psi)


def compute_windspeed(d: Dims, u, v, speed, u0, v0, gustiness):
    """Csrc/surface.h:157-185: speed[i*nlg1+j] over i, j >= 1 from the
    lowest interior level k = gw."""
    U = u.reshape(d.shape)[:, :, d.gw]
    V = v.reshape(d.shape)[:, :, d.gw]
    S = speed.reshape(d.nlg[0], d.nlg[1])
    ui = interp_2(U[:-1, 1:], U[1:, 1:]) + u0
    vi = interp_2(V[1:, :-1], V[1:, 1:]) + v0
    S[1:, 1:] = np.fmax(np.sqrt(ui * ui + vi * vi), gustiness)


def entropyflux_from_thetaflux_qtflux(thetaflux, qtflux, p0_b, T_b, qt_b, qv_b):
    """Csrc/surface.h:95-106 (arrays)."""
    exner_b = exner_c(p0_b)
    pd_b = pd_c(p0_b, qt_b, qv_b)
    pv_b = pv_c(p0_b, qt_b, qv_b)
    sd_b = sd_c(pd_b, T_b)
    sv_b = sv_c(pv_b, T_b)
    cp_b = cpm_c(qt_b)
    return cp_b * thetaflux * exner_b / T_b + qtflux * (sv_b - sd_b)


# ---------------------------------------------------------------------------
# kinematics, Csrc/kinematics.h
# ---------------------------------------------------------------------------
def compute_velocity_gradient(d: Dims, v, vgrad, direction):
    """Csrc/kinematics.h:6-34: vgrad = (v[ijk + s_d] - v[ijk]) dxi_d over
    [0, nlg-1) in every dimension."""
    sh = d.shape
    V = v.reshape(sh)
    G = vgrad.reshape(sh)
    reg = _region(sh, 0, 1)
    G[reg] = (_sh(V, reg, direction, 1) - V[reg]) * d.dxi[direction]


def compute_strain_rate(d: Dims, vgrad, strain_rate):
    """Csrc/kinematics.h:37-69: S[3 vi1 + d] = (vgrad[vi1][d] + vgrad[d][vi1]) / 2."""
    sh = d.shape
    npg = d.npg
    reg = _region(sh, 0, 1)
    for vi1 in range(3):
        for dd in range(3):
            a = vgrad[(3 * vi1 + dd) * npg:(3 * vi1 + dd + 1) * npg].reshape(sh)
            b = vgrad[(3 * dd + vi1) * npg:(3 * dd + vi1 + 1) * npg].reshape(sh)
            S = strain_rate[(3 * vi1 + dd) * npg:(3 * vi1 + dd + 1) * npg].reshape(sh)
            S[reg] = 0.5 * (a[reg] + b[reg])


def compute_strain_rate_mag(d: Dims, strain_rate, strain_rate_mag):
    """Csrc/kinematics.h:72-131: zero everywhere; over [1, nlg-1) add the
    diagonal components S_dd at ijk - s_d, then for the pairs (vi1, d) with
    vi1 in {0, 1} and d >= vi1 -- (0,0), (0,1), (0,2), (1,1), (1,2), as the
    reference loops run -- twice the square of S averaged over ijk, ijk -
    s_vi1, ijk - s_d, ijk - s_d - s_vi1; finally sqrt(2 sum) over all
    cells."""
    sh = d.shape
    npg = d.npg
    M = strain_rate_mag.reshape(sh)
    M[...] = 0.0
    reg = _region(sh, 1, 1)

    def comp(c):
        return strain_rate[c * npg:(c + 1) * npg].reshape(sh)

    for dd in range(3):
        S = comp(4 * dd)
        t = _sh(S, reg, dd, -1)
        M[reg] += t * t
    strides = (d.nlg[1] * d.nlg[2], d.nlg[2], 1)
    ii, jj, kk = np.meshgrid(*[np.arange(r.start, r.stop) for r in reg], indexing="ij")
    flat = ii * strides[0] + jj * strides[1] + kk
    for vi1 in range(2):
        for dd in range(vi1, 3):
            c = 3 * vi1 + dd
            S = comp(c)
            p2 = _sh(S, reg, vi1, -1)
            p3 = _sh(S, reg, dd, -1)
            # the fourth point by its flat offset, as the reference indexes it:
            # for vi1 = d it is two cells back along vi1, which from j = 1
            # wraps to the previous x row (a cell the strain rate is never
            # computed on: 0) and from i = 1 falls before the array (read
            # as 0 here; no interior tendency depends on it when gw >= 3)
            q = flat - strides[vi1] - strides[dd]
            Sf = strain_rate[c * npg:(c + 1) * npg]
            p4 = np.where(q >= 0, Sf[np.clip(q, 0, None)], 0.0)
            s_interp = 0.25 * (S[reg] + p2 + p3 + p4)
            M[reg] += 2.0 * s_interp * s_interp
    M[...] = np.sqrt(2.0 * M)


# ---------------------------------------------------------------------------
# Smagorinsky, Csrc/sgs.h
# ---------------------------------------------------------------------------
def smagorinsky_update(d: Dims, visc, diff, buoy_freq, strain_rate_mag, cs, prt, variant="plain", zl_half=None):
    """Csrc/sgs.h:4-18 (plain), :21-54 (wall), :56-89 (iles), over all npg
    cells; delta = cbrt(dx dy dz)."""
    sh = d.shape
    delta = _cbrt(d.dx[0] * d.dx[1] * d.dx[2])
    S = strain_rate_mag.reshape(sh)
    N2 = buoy_freq.reshape(sh)
    if variant == "plain":
        nu = cs * cs * delta * delta * S
    else:
        z = np.asarray(zl_half, dtype=np.float64)[None, None, :]
        if variant == "wall":
            ell = delta * vkb * z / (delta + vkb * z)
        else:
            ell = np.fmax(0.0, delta - vkb * z)
        nu = cs * cs * ell * ell * S
    pos = N2 > 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        fb = np.sqrt(np.fmax(1.0 - N2 / (prt * S * S), 0.0))
        nu = np.where(pos, nu * fb, nu)
    visc.reshape(sh)[...] = nu
    diff.reshape(sh)[...] = nu / prt


def _cbrt(x):
    """C's cbrt (the reference's delta); Python's math.cbrt is the C library's."""
    return math.cbrt(x)


# ---------------------------------------------------------------------------
# scalar diffusion, Csrc/scalar_diffusion.h
# ---------------------------------------------------------------------------
def compute_diffusive_flux(d: Dims, rho0, rho0_half, diffusivity, scalar, flux, dx, direction, factor):
    """Csrc/scalar_diffusion.h:6-57 (second_order_diffusion): over [gw-1,
    nlg-gw) in every dimension F = -factor interp_2(D, D[+s]) (phi[+s] -
    phi) rho dxi, rho = rho0[k] for d = 2 else rho0_half[k]; then F = 0 on
    the level k = gw-1."""
    sh = d.shape
    D = diffusivity.reshape(sh)
    P = scalar.reshape(sh)
    F = flux.reshape(sh)
    reg = tuple(slice(d.gw - 1, n - d.gw) for n in sh)
    rho = _kvec(rho0 if direction == 2 else rho0_half, reg)
    dxi = 1.0 / dx
    F[reg] = (-factor * interp_2(D[reg], _sh(D, reg, direction, 1)) * (_sh(P, reg, direction, 1) - P[reg])
              * rho * dxi)
    F[reg[0], reg[1], d.gw - 1] = 0.0


def compute_qt_diffusion_s_source(d: Dims, p0_half, alpha0, alpha0_half, flux, qt, qv, T, tendency, dx, direction):
    """Csrc/scalar_diffusion.h:70-113: the entropy tendency of the qt
    diffusion, -(sw - sd) alpha0_half (F[+s] - F) dxi over the interior."""
    sh = d.shape
    reg = _region(sh, d.gw, d.gw)
    F = flux.reshape(sh)
    Q = qt.reshape(sh)[reg]
    V = qv.reshape(sh)[reg]
    Tm = T.reshape(sh)[reg]
    p0 = _kvec(p0_half, reg)
    pd = pd_c(p0, Q, V)
    sd = sd_c(pd, Tm)
    pv = pv_c(p0, Q, V)
    sv = sv_c(pv, Tm)
    L = latent_heat_variable(Tm)
    sw = sv - (((Q - V) / Q) * L / Tm)
    dxi = 1.0 / dx
    tendency.reshape(sh)[reg] -= (sw - sd) * _kvec(alpha0_half, reg) * (_sh(F, reg, direction, 1) - F[reg]) * dxi


# ---------------------------------------------------------------------------
# momentum diffusion, Csrc/momentum_diffusion.h
# ---------------------------------------------------------------------------
def compute_diffusive_flux_m(d: Dims, strain_rate, viscosity, flux, rho0, rho0_half, i1, i2):
    """Csrc/momentum_diffusion.h:5-96: F = -2 S_{i1 i2} nu rho over [gw-1,
    nlg-gw); nu at ijk + s_i1 for the diagonal components, else averaged
    over the four cells around the edge; rho = rho0_half[k] (i1, i2 != 2),
    rho0_half[k+1] (i1 = i2 = 2), rho0[k] (one of them 2); F = 0 on the
    level k = gw-1."""
    sh = d.shape
    S = strain_rate.reshape(sh)
    N = viscosity.reshape(sh)
    F = flux.reshape(sh)
    reg = tuple(slice(d.gw - 1, n - d.gw) for n in sh)
    if i1 == i2:
        nu = _sh(N, reg, i1, 1)
    else:
        s4 = list(reg)
        s4[i1] = slice(reg[i1].start + 1, reg[i1].stop + 1)
        s4[i2] = slice(reg[i2].start + 1, reg[i2].stop + 1)
        nu = 0.25 * (N[reg] + _sh(N, reg, i1, 1) + _sh(N, reg, i2, 1) + N[tuple(s4)])
    if i1 != 2 and i2 != 2:
        rho = _kvec(rho0_half, reg)
    elif i1 == 2 and i2 == 2:
        rho = _kvec(rho0_half, reg, 1)
    else:
        rho = _kvec(rho0, reg)
    F[reg] = -2.0 * S[reg] * nu * rho
    F[reg[0], reg[1], d.gw - 1] = 0.0


def compute_entropy_source(d: Dims, viscosity, strain_rate_mag, temperature, entropy_tendency):
    """Csrc/momentum_diffusion.h:98-118: s tendency += S^2 nu / T over the interior."""
    sh = d.shape
    reg = _region(sh, d.gw, d.gw)
    S = strain_rate_mag.reshape(sh)[reg]
    entropy_tendency.reshape(sh)[reg] += S * S * viscosity.reshape(sh)[reg] / temperature.reshape(sh)[reg]


# ---------------------------------------------------------------------------
# horizontal statistics, ParallelMPI.pyx:196-540 (one rank; the loops'
# sequential order: per level, i then j over the interior columns)
# ---------------------------------------------------------------------------
def _hsum(d: Dims, col, combine=None, init=0.0):
    sh = d.shape
    g_ = d.gw
    acc = np.full(sh[2], init, dtype=np.float64)
    for i in range(g_, sh[0] - g_):
        for j in range(g_, sh[1] - g_):
            v = col(i, j)
            acc = acc + v if combine is None else combine(acc, v)
    return acc


def horizontal_stat(d: Dims, kind, v1, v2=None, v3=None, mask=None):
    """HorizontalMean (:196-241), ...ofSquares (:243-289), ...ofCubes
    (:291-325), HorizontalMaximum (:327-357), HorizontalMinimum (:359-389),
    HorizontalMeanSurface (:391-428), HorizontalMeanConditional (:430-483),
    HorizontalMeanofSquaresConditional (:485-540)."""
    sh = d.shape
    n_horizontal_i = 1.0 / float(d.n[1] * d.n[0])
    A = v1.reshape(sh) if kind != "surface" else v1.reshape(sh[0], sh[1])
    B = v2.reshape(sh) if v2 is not None else None
    C = v3.reshape(sh) if v3 is not None else None
    M = mask.reshape(sh) if mask is not None else None
    if kind == "mean":
        return _hsum(d, lambda i, j: A[i, j]) * n_horizontal_i
    if kind == "squares":
        return _hsum(d, lambda i, j: A[i, j] * B[i, j]) * n_horizontal_i
    if kind == "cubes":
        return _hsum(d, lambda i, j: A[i, j] * B[i, j] * C[i, j]) * n_horizontal_i
    if kind == "max":
        return _hsum(d, lambda i, j: A[i, j], np.fmax, -9e12)
    if kind == "min":
        return _hsum(d, lambda i, j: A[i, j], np.fmin, 9e12)
    if kind == "surface":
        g_ = d.gw
        s = 0.0
        for i in range(g_, sh[0] - g_):
            for j in range(g_, sh[1] - g_):
                s += A[i, j]
        return s * n_horizontal_i
    if kind in ("conditional", "squares_conditional"):
        prod = (lambda i, j: A[i, j] * M[i, j]) if kind == "conditional" else (lambda i, j: A[i, j] * B[i, j] * M[i, j])
        return _hsum(d, prod) / np.maximum(_hsum(d, lambda i, j: M[i, j]), 1.0)
    raise ValueError(kind)


# ---------------------------------------------------------------------------
# case forcing, Forcing.pyx (Cython, restated) + s_tendency_c (Csrc/entropies.h:17-21)
# ---------------------------------------------------------------------------
omega = 7.2921151467064e-5  # generate_parameters.py:38


def s_tendency_c(p0, qt, qv, T, qt_tendency, T_tendency):
    """Csrc/entropies.h:17-21."""
    pv = pv_c(p0, qt, qv)
    pd = pd_c(p0, qt, qv)
    return cpm_c(qt) * T_tendency / T + (sv_c(pv, T) - sd_c(pd, T)) * qt_tendency


def forcing_profiles(scheme, zl_half, p0_half):
    """The profiles each forcing's initialize sets (Forcing.pyx: SullivanPatton
    :260-268, Bomex :106-152, DyCOMS_RF01 :347-389), from Grid.zl_half."""
    n = len(zl_half)
    z = np.asarray(zl_half, dtype=np.float64)
    P = {k: np.zeros(n) for k in ("ug", "vg", "dtdt", "dqtdt", "subsidence")}
    if scheme == "SullivanPatton":
        P["ug"][:] = 1.0
        P["coriolis_param"] = 1.0e-4
    elif scheme == "Bomex":
        P["coriolis_param"] = 0.376e-4
        for k in range(n):
            P["ug"][k] = -10.0 + (1.8e-3) * z[k]
            ex = float(exner_c(p0_half[k]))
            if z[k] <= 1500.0:
                P["dtdt"][k] = (-2.0 / (3600 * 24.0)) * ex
            if z[k] > 1500.0:
                P["dtdt"][k] = (-2.0 / (3600 * 24.0) + (z[k] - 1500.0) * (0.0 - -2.0 / (3600 * 24.0))
                                / (3000.0 - 1500.0)) * ex
            if z[k] <= 300.0:
                P["dqtdt"][k] = -1.2e-8
            if z[k] > 300.0 and z[k] <= 500.0:
                P["dqtdt"][k] = -1.2e-8 + (z[k] - 300.0) * (0.0 - -1.2e-8) / (500.0 - 300.0)
            if z[k] <= 1500.0:
                P["subsidence"][k] = 0.0 + z[k] * (-0.65 / 100.0 - 0.0) / (1500.0 - 0.0)
            if z[k] > 1500.0 and z[k] <= 2100.0:
                P["subsidence"][k] = -0.65 / 100 + (z[k] - 1500.0) * (0.0 - -0.65 / 100.0) / (2100.0 - 1500.0)
    elif scheme == "DYCOMS_RF01":
        divergence = 3.75e-6
        P["coriolis_param"] = 2.0 * omega * math.sin(31.5 * pi / 180.0)
        for k in range(n):
            P["subsidence"][k] = -z[k] * divergence
        P["ug"][:] = 7.0
        P["vg"][:] = -5.5
    else:
        raise ValueError(scheme)
    return P


def apply_subsidence(d: Dims, rho0, rho0_half, subsidence, values, tendencies):
    """Forcing.pyx:2013-2039: over the interior columns, for k in [gw,
    nlg2-gw-1) tend = (phi[k+1] - phi[k]) dzi sub[k] is subtracted; the
    levels from nlg2-gw-1 up (the top interior level and the ghosts) get the
    last tend subtracted again."""
    sh = d.shape
    g_ = d.gw
    V = values.reshape(sh)[g_:sh[0] - g_, g_:sh[1] - g_, :]
    T = tendencies.reshape(sh)[g_:sh[0] - g_, g_:sh[1] - g_, :]
    kmax = sh[2] - g_ - 1
    tend = (V[:, :, g_ + 1:kmax + 1] - V[:, :, g_:kmax]) * d.dxi[2] * subsidence[None, None, g_:kmax]
    T[:, :, g_:kmax] -= tend
    T[:, :, kmax:] -= tend[:, :, -1:]


def coriolis_force(d: Dims, u, v, ut, vt, ug, vg, coriolis_param, u0, v0):
    """Forcing.pyx:1954-1980."""
    sh = d.shape
    r = _region(sh, d.gw, d.gw)
    U, V = u.reshape(sh), v.reshape(sh)
    def at(A, di, dj):
        return A[r[0].start + di:r[0].stop + di, r[1].start + dj:r[1].stop + dj, r[2]]
    u_at_v = 0.25 * (U[r] + at(U, -1, 0) + at(U, -1, 1) + at(U, 0, 1)) + u0
    v_at_u = 0.25 * (V[r] + at(V, 1, 0) + at(V, 1, -1) + at(V, 0, -1)) + v0
    k = _kvec(np.asarray(vg), r)
    ut.reshape(sh)[r] = ut.reshape(sh)[r] - coriolis_param * (k - v_at_u)
    vt.reshape(sh)[r] = vt.reshape(sh)[r] + coriolis_param * (_kvec(np.asarray(ug), r) - u_at_v)


def large_scale_p_gradient(d: Dims, umean, vmean, ut, vt, ug, vg, coriolis_param, u0, v0):
    """Forcing.pyx:1982-2011."""
    sh = d.shape
    r = _region(sh, d.gw, d.gw)
    u_at_v = _kvec(np.asarray(umean), r) + u0
    v_at_u = _kvec(np.asarray(vmean), r) + v0
    ut.reshape(sh)[r] = ut.reshape(sh)[r] - coriolis_param * (_kvec(np.asarray(vg), r) - v_at_u)
    vt.reshape(sh)[r] = vt.reshape(sh)[r] + coriolis_param * (_kvec(np.asarray(ug), r) - u_at_v)


# ---------------------------------------------------------------------------
# DYCOMS radiation, Radiation.pyx:230-353 (Cython, restated)
# ---------------------------------------------------------------------------
def dycoms_radiation(d: Dims, rho0_half, z, ql, qt, T, s_tend, heating_rate, dTdt_rad, f0=70.0, f1=22.0,
                     kap=85.0, alpha_z=1.0, divergence=3.75e-6):
    """RadiationDyCOMS_RF01.update on one rank: per interior column (z
    pencils in i, j order) zi/rhoi at the highest level with qt > 8e-3 (kept
    from the previous column when none qualifies, as the reference's
    variables are), the three flux terms of Stevens et al. 2005 eq. 3, the
    heating rate -(F[k+1] - F[k]) dzi / rho0_half[k] (the reference indexes
    rho0_half without the ghost offset here), then s_tend += heating / T and
    dTdt_rad = heating / cpm(qt)."""
    sh = d.shape
    g_ = d.gw
    n2 = d.n[2]
    dz, dzi = d.dx[2], d.dxi[2]
    QL, QT = ql.reshape(sh), qt.reshape(sh)
    H = heating_rate.reshape(sh)
    zi = rhoi = float("nan")
    for i in range(g_, sh[0] - g_):
        for j in range(g_, sh[1] - g_):
            for k in range(n2):
                if QT[i, j, g_ + k] > 8e-3:
                    zi = z[g_ + k]
                    rhoi = rho0_half[g_ + k]
            f = [0.0] * (n2 + 1)
            for k in range(n2):
                if z[g_ + k] >= zi:
                    c = math.cbrt(z[g_ + k] - zi)
                    f[k + 1] = rhoi * cpd * divergence * alpha_z * (math.pow(c, 4) / 4.0 + zi * c)
                else:
                    f[k + 1] = 0.0
            q1 = 0.0
            f[0] += f1 * math.exp(-q1)
            for k in range(1, n2 + 1):
                q1 += kap * rho0_half[g_ + k - 1] * QL[i, j, g_ + k - 1] * dz
                f[k] += f1 * math.exp(-q1)
            q0 = 0.0
            f[n2] += f0 * math.exp(-q0)
            for k in range(n2 - 1, -1, -1):
                q0 += kap * rho0_half[g_ + k] * QL[i, j, g_ + k] * dz
                f[k] += f0 * math.exp(-q0)
            for k in range(n2):
                H[i, j, g_ + k] = -(f[k + 1] - f[k]) * dzi / rho0_half[k]
    r = _region(sh, g_, g_)
    s_tend.reshape(sh)[r] += H[r] / T.reshape(sh)[r]
    dTdt_rad.reshape(sh)[r] = H[r] / cpm_c(QT[r])
