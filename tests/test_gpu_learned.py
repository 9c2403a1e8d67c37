"""The learned secant seed: BF16 tensor-core forward/backward kernels against
an FP64 CPU MLP (gradient check), training on pairs from the plain secant,
and what the trained network gains over the method without it.

Tolerances: forward and gradient within 3e-2 relative (BF16 operands of the
64x64 layer; the CPU reference evaluates the same BF16-rounded weights in
FP64).  The secant still runs to |dT| < 1e-3 K, so seeded and plain
temperatures agree to that tolerance.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _cpu_mlp(params, x, out_mean, out_scale, bf16):
    """FP64 forward/backward of the same network (CPU oracle of the MLP)."""
    from pycles_b200.learned import H, OFF
    P = params.astype(np.float64)

    def get(n):
        o, k = OFF[n]
        return P[o:o + k]

    def q(a):  # round to BF16 like the kernels' stored weights/operands
        if not bf16:
            return a
        t = torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).to(torch.float64)
        return t.numpy()

    W1 = q(get("w1")).reshape(H, 3)
    b1 = get("b1")
    W2 = q(get("w2")).reshape(H, H)
    b2 = get("b2")
    w3 = q(get("w3"))
    b3 = get("b3")[0]
    z1 = x @ W1.T + b1
    h1 = z1 / (1.0 + np.exp(-z1))
    h1q = q(h1)
    z2 = h1q @ W2.T + b2
    h2 = z2 / (1.0 + np.exp(-z2))
    y = h2 @ w3 + b3
    return y, (W1, W2, w3, z1, h1q, z2, h2)


def _cpu_grad(params, x, t):
    from pycles_b200.learned import H
    y, (W1, W2, w3, z1, h1q, z2, h2) = _cpu_mlp(params, x, 0, 1, True)
    sg = lambda z: (1 / (1 + np.exp(-z))) * (1 + z * (1 - 1 / (1 + np.exp(-z))))
    dy = y - t
    gw3 = h2.T @ dy
    gb3 = dy.sum()
    dz2 = dy[:, None] * w3[None, :] * sg(z2)
    gW2 = dz2.T @ h1q
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * sg(z1)
    gW1 = dz1.T @ x
    gb1 = dz1.sum(0)
    return np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])


def test_mlp_forward_and_gradient_vs_cpu():
    from pycles_b200.learned import SeedMLP
    mlp = SeedMLP(seed=3)
    rng = np.random.default_rng(0)
    n = 1000
    x = rng.uniform(-1, 1, size=(n, 3))
    t = rng.standard_normal(n) * 0.5
    xt = torch.tensor(x, dtype=torch.float32, device="cuda")
    tt = torch.tensor(t, dtype=torch.float32, device="cuda")
    mlp.grad_batch(xt, tt)
    g_gpu = mlp.grad.cpu().numpy().astype(np.float64)
    params = mlp.params.cpu().numpy()
    g_cpu = _cpu_grad(params, xt.cpu().numpy().astype(np.float64), tt.cpu().numpy().astype(np.float64))
    rel = np.linalg.norm(g_gpu - g_cpu) / np.linalg.norm(g_cpu)
    print("gradient rel L2 vs FP64 CPU MLP:", rel)
    assert rel < 3e-2
    # forward through pb_mlp_forward on physical inputs
    from pycles_b200.learned import IN_HI, IN_LO
    phys = [lo + (x[:, i] + 1) * 0.5 * (hi - lo) for i, (lo, hi) in enumerate(zip(IN_LO, IN_HI))]
    p0, s, qt = (torch.tensor(a, dtype=torch.float64, device="cuda") for a in phys)
    y_gpu = mlp.forward(p0, s, qt).cpu().numpy()
    y_cpu, _ = _cpu_mlp(params, mlp.normalise(p0, s, qt).cpu().numpy().astype(np.float64), 0, 1, True)
    # the seed is the secant's first point plus the network's correction
    from oracle import port
    P, S, Q = phys
    pv1 = port.pv_c(P, Q, Q)
    T1 = port.temperature_no_ql(P - pv1, pv1, S, Q)
    y_cpu = T1 + mlp.out_mean + mlp.out_scale * y_cpu
    assert np.max(np.abs(y_gpu - y_cpu)) / mlp.out_scale < 3e-2


def test_gradient_and_training_are_deterministic():
    """pb_mlp_grad adds per-block partial sums in a fixed order (no
    floating-point atomics): the same batch gives the same gradient bit for
    bit, and the same pairs give the same trained network."""
    from pycles_b200.learned import SeedMLP
    rng = np.random.default_rng(2)
    n = 50_000  # several hundred blocks of partial sums
    xt = torch.tensor(rng.uniform(-1, 1, size=(n, 3)), dtype=torch.float32, device="cuda")
    tt = torch.tensor(rng.standard_normal(n) * 0.5, dtype=torch.float32, device="cuda")
    mlp = SeedMLP(seed=4)
    grads = []
    for _ in range(3):
        mlp.grad_batch(xt, tt)
        grads.append((mlp.grad.clone(), mlp.loss.clone()))
    for g, l in grads[1:]:
        assert torch.equal(g, grads[0][0]) and torch.equal(l, grads[0][1])
    P = 8.0e4 + 2.0e4 * torch.tensor(rng.uniform(size=n), device="cuda")
    S = 6900.0 + 100.0 * torch.tensor(rng.uniform(size=n), device="cuda")
    Q = 0.01 + 0.01 * torch.tensor(rng.uniform(size=n), device="cuda")
    T1 = 280.0 + torch.tensor(rng.uniform(size=n), device="cuda")
    T = T1 + 2.0 + torch.tensor(rng.uniform(size=n), device="cuda")
    nets = []
    for _ in range(2):
        m = SeedMLP(seed=0, out_mean=2.5, out_scale=1.0)
        m.train(P, S, Q, T, T1, epochs=2, batch=8192)
        nets.append(m.params.clone())
    assert torch.equal(nets[0], nets[1])


def test_trained_seed_cuts_secant_iterations():
    from pycles_b200 import learned
    from pycles_b200.thermodynamics import ThermodynamicsSA
    th = ThermodynamicsSA({})
    g = torch.Generator(device="cuda").manual_seed(1)
    n = 400_000
    # saturated-range inputs: boundary-layer to cloud-layer pressures, entropies, moisture
    p0 = 7.0e4 + 3.2e4 * torch.rand(n, device="cuda", dtype=torch.float64, generator=g)
    s = 6850.0 + 200.0 * torch.rand(n, device="cuda", dtype=torch.float64, generator=g)
    qt = 0.004 + 0.02 * torch.rand(n, device="cuda", dtype=torch.float64, generator=g)
    P, S, Q, T, T1, its = learned.training_pairs(th, p0, s, qt)
    assert P.numel() > 10_000
    ntr = P.numel() * 9 // 10
    r = T - T1
    mlp = learned.SeedMLP(seed=0, out_mean=float(r.mean()), out_scale=float(r.std()) * 2)
    hist = mlp.train(P[:ntr], S[:ntr], Q[:ntr], T[:ntr], T1[:ntr], epochs=6, batch=8192)
    assert hist[-1] < hist[0]
    # held-out points: iterations with and without the seed, same answer
    Pt, St, Qt, Tt = P[ntr:], S[ntr:], Q[ntr:], T[ntr:]
    seed = mlp.forward(Pt, St, Qt)
    T_plain, it_plain = learned.secant_iterations(th, Pt, St, Qt)
    T_seed, it_seed = learned.secant_iterations(th, Pt, St, Qt, seed=seed)
    err = float((seed - Tt).abs().mean())
    mp, ms = float(it_plain.double().mean()), float(it_seed.double().mean())
    print(f"seed mean |error| {err:.3e} K; mean secant iterations plain {mp:.3f}, seeded {ms:.3f}")
    assert ms < mp
    assert float((T_seed - T_plain).abs().max()) < 2e-3


def test_fused_seed_in_thermodynamics():
    """The learned seed inside the precision-form thermodynamics update (the
    network refreshed for the cells saturated at the previous update, then
    the secant started from it): same temperatures as the plain form to the
    secant's tolerance, fewer secant iterations than the precision form
    without the seed."""
    from helpers import gpu_dv, gpu_sim, host_case
    from pycles_b200 import learned
    nl, rs, f = host_case(case="dycoms", nx=16, ny=16, nz=256, dx=35.0, dy=35.0, dz=5.0, gw=4, dt=0.25,
                          scalar_order=7, momentum_order=5)
    plain = gpu_sim(nl, rs, f)
    fast = gpu_sim(nl, rs, f, precision="fp32")
    seeded = gpu_sim(nl, rs, f, precision="fp32")
    n2 = plain.Gr.dims.nlg[2]
    s = torch.as_tensor(f["s"], device="cuda")
    qt = torch.as_tensor(f["qt"], device="cuda")
    p0 = seeded.RS.d_p0_half.repeat(s.numel() // n2)
    P, S, Q = learned.sample_inputs([(p0, s, qt)], 600_000, rng_seed=1)
    P, S, Q, T, T1, _ = learned.training_pairs(seeded.Th, P, S, Q)
    r = T - T1
    mlp = learned.SeedMLP(seed=0, out_mean=float(r.mean()), out_scale=2.0 * float(r.std()))
    mlp.train(P, S, Q, T, T1, epochs=8, batch=8192)
    seeded.Th.mlp = mlp
    seeded.Th.seed_refresh_interval = 1  # re-evaluate the network at every update
    stats = {}
    for name, g in (("plain", plain), ("fast", fast), ("seeded", seeded)):
        g.PV.Update_all_bcs(g.Gr)
        g.Th.update(g.Gr, g.RS, g.PV, g.DV)  # the condensate the seed refresh keys on
        g.Th.iter_stats = None
        g.Th.update(g.Gr, g.RS, g.PV, g.DV)
        it, nsat = g.Th.iter_stats.cpu().tolist()
        stats[name] = (it / max(nsat, 1), nsat, gpu_dv(g))
    print({k: v[:2] for k, v in stats.items()})
    assert stats["plain"][1] == stats["fast"][1] == stats["seeded"][1] > 1000
    Tp, Tf, Ts = (stats[k][2]["temperature"] for k in ("plain", "fast", "seeded"))
    assert np.max(np.abs(Tf - Tp)) < 1e-6
    assert np.max(np.abs(Ts - Tp)) < 2e-3
    assert stats["seeded"][0] < stats["fast"][0]


def test_seed_with_refresh_is_faster_on_a_cloudy_grid():
    """What the trained network gains in time, not only in iterations: on a
    grid whose boundary layer is mostly saturated, 12 precision-form
    thermodynamics updates with the learned seed (the refresh of the
    network's outputs that the default interval of 12 updates runs included)
    take less device time than 12 updates started from the reference's
    point.  CUDA events on the launching stream, best of 5 repeats."""
    from helpers import gpu_sim, host_case
    from pycles_b200 import learned
    nl, rs, f = host_case(case="dycoms", nx=192, ny=192, nz=64, dx=35.0, dy=35.0, dz=15.0, gw=4, dt=0.25,
                          scalar_order=7, momentum_order=5)
    f = dict(f, qt=f["qt"] + 3.0e-3)  # moister: most of the boundary layer saturated
    sims = {name: gpu_sim(nl, rs, f, precision="fp32") for name in ("plain", "seeded")}
    g = sims["seeded"]
    mlp, info = learned.train_seed(g.Th, [learned.cell_inputs(g)], n_pairs=1_000_000, draw=3_000_000,
                                   n_held_out=200_000)
    assert mlp is not None, info
    g.Th.mlp = mlp
    assert g.Th.seed_refresh_interval == 12
    stream = torch.cuda.current_stream()
    times, iters = {}, {}
    for name, sim in sims.items():
        sim.PV.Update_all_bcs(sim.Gr)
        for _ in range(12):  # warm-up; leaves the condensate the refresh keys on
            sim.Th.update(sim.Gr, sim.RS, sim.PV, sim.DV)
        sim.Th.iter_stats.zero_()
        best = float("inf")
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(12):
                sim.Th.update(sim.Gr, sim.RS, sim.PV, sim.DV, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        it, nsat = sim.Th.iter_stats.cpu().tolist()
        times[name], iters[name] = best, it / max(nsat, 1)
        sim.check_device_errors()
    print("12 thermodynamics updates, ms:", times, "secant iterations per saturated cell:", iters, "seed:", info)
    assert iters["seeded"] < iters["plain"]
    assert times["seeded"] < times["plain"]


@pytest.mark.parametrize("shape,gw,flagged", [((64, 64, 48), 4, 0.5), ((30, 22, 17), 3, 0.5),
                                               ((30, 22, 17), 3, 0.0), ((30, 22, 17), 3, 1.0)])
def test_tensor_core_refresh_matches_cpu_network(shape, gw, flagged):
    """pb_mlp_refresh_seed (tcgen05 products, FP32 accumulators in tensor
    memory) against the FP64 CPU evaluation of the same BF16 network: half
    of the cells flagged (several scan rounds per block), none and all, on a
    grid whose cell count is a multiple of the 128-cell tile and on a ragged
    one; cells not flagged get NaN.  Tolerance as the forward check: 3e-2 of
    the output's scale."""
    import ctypes

    from pycles_b200 import _capi
    from pycles_b200.learned import SeedMLP
    from pycles_b200.parallel import slab_dims
    mlp = SeedMLP(seed=5)
    dims = slab_dims(shape, gw, (35.0, 35.0, 5.0))
    npg, n2 = int(dims.npg), int(dims.nlg[2])
    g = torch.Generator(device="cuda").manual_seed(7)
    p0 = 9.0e4 + 5.0e3 * torch.rand(n2, device="cuda", dtype=torch.float64, generator=g)
    s = 6850.0 + 200.0 * torch.rand(npg, device="cuda", dtype=torch.float64, generator=g)
    qt = 0.025 * torch.rand(npg, device="cuda", dtype=torch.float64, generator=g)
    ql = torch.rand(npg, device="cuda", dtype=torch.float64, generator=g) - (1.0 - flagged)  # > 0: flagged
    if flagged == 1.0:
        ql += 1e-9
    y = torch.zeros(npg, dtype=torch.float32, device="cuda")
    st = mlp.struct()
    st.seed_y = y.data_ptr()
    _capi.check(_capi.load().pb_mlp_refresh_seed(ctypes.byref(st), ctypes.byref(dims), p0.data_ptr(), s.data_ptr(),
                                                 qt.data_ptr(), ql.data_ptr(), _capi.stream_handle(None)),
                "pb_mlp_refresh_seed")
    torch.cuda.synchronize()
    flag = (ql > 0).cpu().numpy()
    yg = y.cpu().numpy().astype(np.float64)
    assert np.isnan(yg[~flag]).all()
    P = p0.repeat(npg // n2)
    x = mlp.normalise(P, s, qt).cpu().numpy().astype(np.float64)
    if flagged == 0.0:
        assert not flag.any()
        return
    if flagged == 1.0:
        assert flag.all()
    yc, _ = _cpu_mlp(mlp.params.cpu().numpy(), x[flag], 0, 1, True)
    err = np.max(np.abs(yg[flag] - yc)) / max(1.0, float(np.max(np.abs(yc))))
    print("tensor-core refresh vs FP64 CPU network: max error", err, "flagged cells", int(flag.sum()))
    assert np.isfinite(yg[flag]).all()
    assert err < 3e-2
