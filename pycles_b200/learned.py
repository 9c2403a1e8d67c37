"""Learned initial guess for the saturation-adjustment secant.

A 3 -> 64 -> 64 -> 1 SiLU MLP maps (p0, s, qt), each normalised to [-1, 1]
over p0 in [5e4, 1.02e5] Pa, s in [6800, 7100] J/kg/K, qt in [0, 0.025],
to the correction T - T_1 between the converged temperature and the
secant's first point T_1 (the all-vapour temperature of
Csrc/thermodynamics_sa.h:22-24).  The seed T_1 + correction replaces the
secant's linearised second point (:39).  The secant loop itself is
unchanged and still runs to the reference tolerance, so the network can only
change how many iterations a cell takes.  Learning the correction rather
than T itself keeps the target's scale at ~1 K, so the BF16 network's
relative error costs millikelvins.

Training pairs come from the plain FP64 secant (pb_eos_sa) on saturated
(p0, s, qt) samples; training runs on the GPU with this library's own BF16
tensor-core forward/backward kernels (pb_mlp_grad) and Adam (pb_mlp_adam).
No counterpart in the reference.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _capi

IN_LO = (5.0e4, 6800.0, 0.0)
IN_HI = (1.02e5, 7100.0, 0.025)
H = 64
OFF = {"w1": (0, H * 3), "b1": (H * 3, H), "w2": (H * 3 + H, H * H), "b2": (H * 3 + H + H * H, H),
       "w3": (H * 3 + 2 * H + H * H, H), "b3": (H * 3 + 3 * H + H * H, 1)}


class SeedMLP:
    def __init__(self, device="cuda", seed=0, out_mean=0.5, out_scale=1.0):
        self.device = torch.device(device)
        g = torch.Generator().manual_seed(seed)
        p = torch.zeros(_capi.MLP_NPARAM, dtype=torch.float32)
        # He-style initialisation of the weights, zero biases
        for name, fan_in in (("w1", 3), ("w2", H), ("w3", H)):
            o, n = OFF[name]
            p[o:o + n] = torch.randn(n, generator=g) * math.sqrt(2.0 / fan_in)
        self.params = p.to(self.device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        self._grad_ws = None  # pb_mlp_grad's per-block partial sums
        self.step_count = 0
        self.out_mean = float(out_mean)
        self.out_scale = float(out_scale)
        self.w1 = torch.empty(H * 3, dtype=torch.bfloat16, device=self.device)
        self.w2 = torch.empty(H * H, dtype=torch.bfloat16, device=self.device)
        self.w3 = torch.empty(H, dtype=torch.bfloat16, device=self.device)
        self.b1 = torch.empty(H, dtype=torch.float32, device=self.device)
        self.b2 = torch.empty(H, dtype=torch.float32, device=self.device)
        self.b3 = torch.empty(1, dtype=torch.float32, device=self.device)
        self._sync_copies()

    def _sync_copies(self):
        for name in ("w1", "w2", "w3", "b1", "b2", "b3"):
            o, n = OFF[name]
            getattr(self, name).copy_(self.params[o:o + n].to(getattr(self, name).dtype))

    def struct(self) -> _capi.PbMlp:
        s = _capi.PbMlp()
        s.w1, s.b1, s.w2, s.b2, s.w3, s.b3 = (getattr(self, n).data_ptr() for n in ("w1", "b1", "w2", "b2", "w3", "b3"))
        for i in range(3):
            s.in_lo[i] = IN_LO[i]
            s.in_hi[i] = IN_HI[i]
        s.out_mean = self.out_mean
        s.out_scale = self.out_scale
        s.seed_y = None  # the per-cell seed state belongs to the thermodynamics that uses the network
        s.seed_refresh = 0
        return s

    # ------------------------------------------------------------------
    @staticmethod
    def normalise(p0, s, qt):
        x = torch.stack([2.0 * (a - lo) / (hi - lo) - 1.0 for a, lo, hi in zip((p0, s, qt), IN_LO, IN_HI)], dim=1)
        return x.to(torch.float32).contiguous()

    def forward(self, p0, s, qt, stream=None):
        """Seeds for point lists (CUDA float64 tensors) through pb_mlp_forward."""
        out = torch.empty_like(p0)
        st = self.struct()
        _capi.check(_capi.load().pb_mlp_forward(ctypes.byref(st), p0.data_ptr(), s.data_ptr(), qt.data_ptr(),
                                                out.data_ptr(), p0.numel(), _capi.stream_handle(stream)),
                    "pb_mlp_forward")
        return out

    def grad_batch(self, x, target, stream=None):
        """Zeroes and fills self.grad / self.loss for one batch (pb_mlp_grad,
        deterministic: the same batch gives the same gradient bit for bit)."""
        L = _capi.load()
        need = int(L.pb_mlp_grad_workspace_bytes(x.shape[0]))
        if self._grad_ws is None or self._grad_ws.numel() < need:
            self._grad_ws = torch.empty(max(need, 16), dtype=torch.uint8, device=self.device)
        self.grad.zero_()
        self.loss.zero_()
        st = self.struct()
        _capi.check(L.pb_mlp_grad(ctypes.byref(st), x.data_ptr(), target.data_ptr(), x.shape[0],
                                  self.grad.data_ptr(), self.loss.data_ptr(), self._grad_ws.data_ptr(),
                                  self._grad_ws.numel(), _capi.stream_handle(stream)), "pb_mlp_grad")

    def adam(self, lr, n, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        self.step_count += 1
        _capi.check(_capi.load().pb_mlp_adam(
            self.params.data_ptr(), self.m.data_ptr(), self.v.data_ptr(), self.grad.data_ptr(), self.step_count,
            lr, beta1, beta2, eps, 1.0 / float(n), self.w1.data_ptr(), self.b1.data_ptr(), self.w2.data_ptr(),
            self.b2.data_ptr(), self.w3.data_ptr(), self.b3.data_ptr(), _capi.stream_handle(stream)), "pb_mlp_adam")

    def train(self, p0, s, qt, T, T1, epochs=3, batch=16384, lr=3e-3, lr_final=1e-4, seed=0, log=None):
        """Mini-batch Adam on (p0, s, qt) -> T - T1 pairs (CUDA float64
        tensors; T1 the secant's first point); cosine learning-rate decay."""
        x = self.normalise(p0, s, qt)
        y = ((T - T1 - self.out_mean) / self.out_scale).to(torch.float32).contiguous()
        n = x.shape[0]
        g = torch.Generator(device=x.device).manual_seed(seed)
        nb = max(1, n // batch)
        total = epochs * nb
        it = 0
        hist = []
        for ep in range(epochs):
            perm = torch.randperm(n, device=x.device, generator=g)
            for b in range(nb):
                sel = perm[b * batch:(b + 1) * batch]
                xb = x[sel].contiguous()
                yb = y[sel].contiguous()
                self.grad_batch(xb, yb)
                lr_t = lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * it / max(1, total)))
                self.adam(lr_t, xb.shape[0])
                it += 1
            hist.append(float(self.loss.item()) / float(batch))
            if log:
                log(f"epoch {ep}: batch loss {hist[-1]:.3e}")
        return hist


def training_pairs(thermo, p0, s, qt, max_iter=100):
    """(p0, s, qt) -> (T, T_1, secant iterations) from the plain FP64 secant
    (pb_eos_sa); keeps the saturated points (iterations > 0)."""
    table = thermo.CC.device_table(p0.device)
    T = torch.empty_like(p0)
    T1 = torch.empty_like(p0)
    its = torch.empty(p0.numel(), dtype=torch.int32, device=p0.device)
    _capi.check(_capi.load().pb_eos_sa(ctypes.byref(table), p0.data_ptr(), s.data_ptr(), qt.data_ptr(), None,
                                       T.data_ptr(), None, None, T1.data_ptr(), its.data_ptr(), p0.numel(),
                                       max_iter, _capi.stream_handle(None)), "pb_eos_sa")
    # saturated points whose secant converged to a finite temperature within
    # the cap (a draw can leave the saturation table's range)
    keep = (its > 0) & (its < max_iter) & torch.isfinite(T) & torch.isfinite(T1)
    return p0[keep], s[keep], qt[keep], T[keep], T1[keep], its[keep]


def secant_iterations(thermo, p0, s, qt, seed=None, max_iter=100):
    """Per-point secant iterations (and T) with or without a seed."""
    table = thermo.CC.device_table(p0.device)
    T = torch.empty_like(p0)
    its = torch.empty(p0.numel(), dtype=torch.int32, device=p0.device)
    _capi.check(_capi.load().pb_eos_sa(ctypes.byref(table), p0.data_ptr(), s.data_ptr(), qt.data_ptr(),
                                       seed.data_ptr() if seed is not None else None, T.data_ptr(), None, None,
                                       None, its.data_ptr(), p0.numel(), max_iter, _capi.stream_handle(None)),
                "pb_eos_sa")
    return T, its


def sample_inputs(states, n, rng_seed=0, jitter=(200.0, 3.0, 5e-4), device="cuda"):
    """n (p0, s, qt) samples drawn from simulation states (list of (p0 per cell,
    s, qt) flat tensors) with a small seeded jitter, clipped to the input box."""
    g = torch.Generator(device=device).manual_seed(rng_seed)
    P = torch.cat([st[0] for st in states])
    S = torch.cat([st[1] for st in states])
    Q = torch.cat([st[2] for st in states])
    idx = torch.randint(0, P.numel(), (n,), device=device, generator=g)
    out = []
    for a, j, lo, hi in zip((P, S, Q), jitter, IN_LO, IN_HI):
        v = a[idx] + j * (2.0 * torch.rand(n, device=device, generator=g, dtype=torch.float64) - 1.0)
        out.append(v.clamp(lo, hi))
    return out


def cell_inputs(sim):
    """(p0 per cell, s, qt) of a simulation's current state: the network's
    inputs for every ghosted cell (CUDA float64 tensors, views where they can
    be)."""
    Gr = sim.Gr
    n2 = int(Gr.dims.nlg[2])
    p0 = sim.RS.d_p0_half.repeat(int(Gr.npg) // n2)
    return p0, sim.PV.field("s", Gr), sim.PV.field("qt", Gr)


def train_seed(thermo, states, n_pairs=10_000_000, jitter=(200.0, 3.0, 5e-4), held_out_states=None,
               n_held_out=1_000_000, epochs=12, batch=16384, seed=0, draw=10_000_000, max_draws=8, device="cuda"):
    """Trains a SeedMLP on (p0, s, qt) -> T pairs from the plain FP64 secant
    (pb_eos_sa).  Inputs are drawn from simulation states (a list of (p0, s,
    qt) flat tensors, e.g. ``cell_inputs`` of runs saved along the way) with
    a seeded uniform jitter of the given half-widths, in batches of ``draw``,
    until ``n_pairs`` saturated samples are collected (only saturated points
    are pairs: elsewhere the secant does not run).  Evaluated on pairs drawn
    the same way from ``held_out_states`` (default: the training states,
    another seed).  Returns (mlp, info); mlp is None when the draws hold too
    few saturated points."""
    import time
    # the jittered draws reach outside the saturation table (those pairs are
    # dropped), which flags the device error word; leave it as it was found
    word0 = _capi.get_error()
    parts = [[] for _ in range(5)]
    got, draws = 0, 0
    while got < n_pairs and draws < max_draws:
        P, S, Q = sample_inputs(states, draw, rng_seed=1 + seed + 7919 * draws, jitter=jitter, device=device)
        P, S, Q, T, T1, _ = training_pairs(thermo, P, S, Q)
        for lst, t in zip(parts, (P, S, Q, T, T1)):
            lst.append(t)
        got += P.numel()
        draws += 1
    P, S, Q, T, T1 = (torch.cat(lst)[:n_pairs] for lst in parts)
    if word0 == 0:
        _capi.clear_error()
    info = {"training_pairs": int(P.numel()), "samples_drawn": draws * draw, "epochs": epochs,
            "jitter_half_widths": list(jitter)}
    if P.numel() < 1000:
        return None, info
    r = T - T1
    mlp = SeedMLP(device=device, seed=seed, out_mean=float(r.mean()), out_scale=2.0 * float(r.std()))
    torch.cuda.synchronize()
    t0 = time.time()
    hist = mlp.train(P, S, Q, T, T1, epochs=epochs, batch=batch, seed=seed)
    torch.cuda.synchronize()
    info["train_seconds"] = round(time.time() - t0, 2)
    info["final_batch_loss"] = hist[-1]
    del P, S, Q, T, T1, r
    held = held_out_states or states
    hj = jitter if held_out_states is None else (0.0, 0.0, 0.0)
    Ph, Sh, Qh = sample_inputs(held, n_held_out, rng_seed=1000 + seed, jitter=hj, device=device)
    Ph, Sh, Qh, Th, _, its_h = training_pairs(thermo, Ph, Sh, Qh)
    if Ph.numel():
        guess = mlp.forward(Ph, Sh, Qh)
        _, it_seed = secant_iterations(thermo, Ph, Sh, Qh, seed=guess)
    if word0 == 0:
        _capi.clear_error()
    if Ph.numel():
        info.update({"held_out_pairs": int(Ph.numel()),
                     "seed_mean_abs_error_K": float((guess - Th).abs().mean()),
                     "pointwise_mean_iterations_plain": float(its_h.double().mean()),
                     "pointwise_mean_iterations_seeded": float(it_seed.double().mean())})
    return mlp, info
