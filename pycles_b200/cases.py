"""Seeded synthetic initial states for the hot-path configurations.

Each case follows the structure of a reference initialiser (profiles in z,
perturbations from ``np.random.seed(rank)`` + ``random_sample(npg)`` drawn in
[i][j][k] order, Galilean shift) with the amplitudes of the benchmark
configurations.  The functions fill host numpy arrays; the
caller uploads them.  Vectorised: levels without perturbation are computed
once per level and broadcast.

* ``dry_cbl``   -- InitSullivanPatton (Initialization.pyx:191-258) structure:
                   theta 300 K up to 800 m, +6 K/km above, +-0.1 K below 200 m,
                   u0 = 1 Galilean shift, dry thermodynamics.
* ``bomex``     -- InitBomex (Initialization.pyx:260-368): thetal/qt/u
                   profiles, +-0.1 K and +-2.5e-5 kg/kg below 1600 m.
* ``dycoms``    -- InitDYCOMS_RF01 (Initialization.pyx:447-580): qt 9/1.5 g/kg,
                   thetal 289 K / 297.5+(z-840)^(1/3) K, +-0.1 K below 200 m,
                   thetal inverted to T with the same secant.
"""
from __future__ import annotations

import numpy as np

from . import thermodynamics as th


def _perturbation(npg, seed, amplitude):
    """(U[0,1) - 0.5) * 2 * amplitude, legacy MT19937 as the reference draws it."""
    np.random.seed(seed)
    return (np.random.random_sample(npg) - 0.5) * (2.0 * amplitude)


def dry_cbl(Gr, RS, Th, seed=0, amplitude=0.1):
    """Returns dict of host arrays u, v, w, s (each npg) and sets RS.u0/v0."""
    RS.Pg, RS.Tg, RS.qtg = 1.0e5, 300.0, 0.0
    RS.u0, RS.v0 = 1.0, 0.0
    RS.initialize(Gr, Th, device=getattr(Gr, "device", "cuda"))
    sh = Gr.shape
    z = Gr.z_half
    theta = np.where(z <= 800.0, 300.0, 300.0 + (z - 800.0) * 0.006)
    pert = _perturbation(Gr.npg, seed, amplitude).reshape(sh)
    p0 = RS.p0_half
    ex = th.exner(p0)
    s = np.empty(sh)
    s[...] = th.entropy_dry(p0, theta * ex)[None, None, :]
    low = np.nonzero(z < 200.0)[0]
    if low.size:
        t = (theta[low][None, None, :] + pert[:, :, low]) * ex[low][None, None, :]
        s[:, :, low] = th.entropy_dry(p0[low][None, None, :], t)
    u = np.full(sh, 1.0 - RS.u0)
    v = np.full(sh, 0.0 - RS.v0)
    w = np.zeros(sh)
    return {"u": u.ravel(), "v": v.ravel(), "w": w.ravel(), "s": s.ravel()}


def bomex(Gr, RS, Th, seed=0, theta_amp=0.1, qt_amp=2.5e-5):
    RS.Pg, RS.Tg, RS.qtg = 1.015e5, 300.4, 0.02245
    RS.initialize(Gr, Th, device=getattr(Gr, "device", "cuda"))
    sh = Gr.shape
    z = Gr.z_half
    thetal = np.empty_like(z)
    qt = np.empty_like(z)
    u = np.empty_like(z)
    for k, zk in enumerate(z):
        if zk <= 520.0:
            thetal[k] = 298.7
        elif zk <= 1480.0:
            thetal[k] = 298.7 + (zk - 520) * (302.4 - 298.7) / (1480.0 - 520.0)
        elif zk <= 2000:
            thetal[k] = 302.4 + (zk - 1480.0) * (308.2 - 302.4) / (2000.0 - 1480.0)
        else:
            thetal[k] = 308.2 + (zk - 2000.0) * (311.85 - 308.2) / (3000.0 - 2000.0)
        if zk <= 520:
            qt[k] = 17.0 + zk * (16.3 - 17.0) / 520.0
        elif zk <= 1480.0:
            qt[k] = 16.3 + (zk - 520.0) * (10.7 - 16.3) / (1480.0 - 520.0)
        elif zk <= 2000.0:
            qt[k] = 10.7 + (zk - 1480.0) * (4.2 - 10.7) / (2000.0 - 1480.0)
        else:
            qt[k] = 4.2 + (zk - 2000.0) * (3.0 - 4.2) / (3000.0 - 2000.0)
        qt[k] /= 1000.0
        u[k] = -8.75 if zk <= 700.0 else -8.75 + (zk - 700.0) * (-4.61 - -8.75) / (3000.0 - 700.0)
    RS.v0 = 0.0
    RS.u0 = 0.5 * (np.amax(u) + np.amin(u))
    np.random.seed(seed)
    theta_pert = (np.random.random_sample(Gr.npg) - 0.5) * (2.0 * theta_amp)
    qt_pert = (np.random.random_sample(Gr.npg) - 0.5) * (2.0 * qt_amp)
    p0 = RS.p0_half
    ex = th.exner(p0)
    S = np.empty(sh)
    QT = np.empty(sh)
    S[...] = th.entropy_sa(p0, thetal * ex, qt, 0.0, 0.0)[None, None, :]
    QT[...] = qt[None, None, :]
    low = np.nonzero(z <= 1600.0)[0]
    if low.size:
        tp = theta_pert.reshape(sh)[:, :, low]
        qp = qt_pert.reshape(sh)[:, :, low]
        temp = (thetal[low][None, None, :] + tp) * ex[low][None, None, :]
        q_ = qt[low][None, None, :] + qp
        S[:, :, low] = th.entropy_sa(p0[low][None, None, :], temp, q_, 0.0, 0.0)
        QT[:, :, low] = q_
    U = np.empty(sh)
    U[...] = (u - RS.u0)[None, None, :]
    V = np.full(sh, 0.0 - RS.v0)
    W = np.zeros(sh)
    return {"u": U.ravel(), "v": V.ravel(), "w": W.ravel(), "s": S.ravel(), "qt": QT.ravel()}


def _sat_adjst_thetal(Th, p, thetal, qt):
    """Vectorised sat_adjst of InitDYCOMS_RF01 (Initialization.pyx:504-540):
    thetal, qt -> T, ql with the reference's secant (tolerance 1e-9 K)."""
    p, thetal, qt = np.broadcast_arrays(np.asarray(p, float), np.asarray(thetal, float), np.asarray(qt, float))
    shape = p.shape
    p, thetal, qt = p.ravel(), thetal.ravel(), qt.ravel()

    def compute_thetal(p_, T_, ql_):
        theta_ = T_ / (p_ / th.p_tilde) ** (287.0 / 1015.0)
        return theta_ * np.exp(-2.47e6 * ql_ / (1015.0 * T_))

    t_1 = thetal * (p / th.p_tilde) ** (287.0 / 1015.0)
    qs_1 = th._qv_star(p, qt, Th.CC.lookup(t_1))
    T = t_1.copy()
    ql = np.zeros_like(T)
    sat = np.nonzero(qt > qs_1)[0]
    if sat.size:
        P, TL, Q = p[sat], thetal[sat], qt[sat]
        t1 = t_1[sat]
        ql_1 = Q - qs_1[sat]
        f_1 = TL - compute_thetal(P, t1, ql_1)
        t2 = t1 + 2.47e6 * ql_1 / 1015.0
        ql2 = Q - th._qv_star(P, Q, Th.CC.lookup(t2))
        act = np.arange(sat.size)
        for _ in range(200):
            act = act[np.abs(t2[act] - t1[act]) >= 1e-9]
            if not act.size:
                break
            qs_2 = th._qv_star(P[act], Q[act], Th.CC.lookup(t2[act]))
            ql_2 = Q[act] - qs_2
            f_2 = TL[act] - compute_thetal(P[act], t2[act], ql_2)
            t_n = t2[act] - f_2 * (t2[act] - t1[act]) / (f_2 - f_1[act])
            t1[act] = t2[act]
            t2[act] = t_n
            f_1[act] = f_2
            ql2[act] = ql_2
        T[sat] = t2
        ql[sat] = ql2
    return T.reshape(shape), ql.reshape(shape)


def dycoms(Gr, RS, Th, seed=0, amplitude=0.1):
    RS.Pg = 1017.8 * 100.0
    RS.qtg = 9.0 / 1000.0
    RS.u0 = 7.0
    RS.v0 = -5.5
    RS.Tg = 289.0 * (RS.Pg / th.p_tilde) ** (287.0 / 1015.0)
    RS.initialize(Gr, Th, device=getattr(Gr, "device", "cuda"))
    sh = Gr.shape
    z = Gr.z_half
    thetal = np.where(z <= 840.0, 289.0, 297.5 + np.cbrt(np.maximum(z - 840.0, 0.0)))
    qt = np.where(z <= 840.0, 9.0 / 1000.0, 1.5 / 1000.0)
    p0 = RS.p0_half
    T0, ql0 = _sat_adjst_thetal(Th, p0, thetal, qt)
    S = np.empty(sh)
    S[...] = th.entropy_sa(p0, T0, qt, ql0, 0.0)[None, None, :]
    pert = _perturbation(Gr.npg, seed, amplitude).reshape(sh)
    low = np.nonzero(z < 200.0)[0]
    if low.size:
        P = np.broadcast_to(p0[low][None, None, :], pert[:, :, low].shape)
        Q = np.broadcast_to(qt[low][None, None, :], P.shape)
        T, ql = _sat_adjst_thetal(Th, P, thetal[low][None, None, :] + pert[:, :, low], Q)
        S[:, :, low] = th.entropy_sa(P, T, Q, ql, 0.0)
    QT = np.empty(sh)
    QT[...] = qt[None, None, :]
    zero = np.zeros(sh)
    return {"u": zero.ravel(), "v": zero.ravel().copy(), "w": zero.ravel().copy(), "s": S.ravel(),
            "qt": QT.ravel()}


CASES = {"dry_cbl": dry_cbl, "bomex": bomex, "dycoms": dycoms}
