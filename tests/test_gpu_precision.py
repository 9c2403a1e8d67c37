"""The precision form (FP32 WENO arithmetic on shifted stencils with FP64
flux assembly and divergence accumulation; FP32 FFTs with FP64 tridiagonal
solves and FP64-residual iterative refinement) against the FP64 oracle.

Tolerances (relative L2):
  * advection tendencies: 1e-5 (FP32 weights and candidate polynomials)
  * pressure without refinement: 1e-5; with the per-level horizontal mean
    (the mode the solver projects out) removed, one refinement sweep shrinks
    the difference to the FP64 solve by >= 1e4 and two reach 1e-12
  * prognostic fields after 5 steps of the whole hot path: 1e-6 against the
    FP64 oracle; after 1000 steps: 1e-5 against the FP64 plain form
"""
import numpy as np
import pytest

from helpers import gpu_dv, gpu_fields, gpu_sim, gpu_tends, host_case, oracle_sim, rel_l2

pytestmark = pytest.mark.gpu

MOIST = dict(case="bomex", nx=32, ny=32, nz=24, dx=100.0, dy=100.0, dz=40.0, gw=4, dt=1.0,
             scalar_order=7, momentum_order=5)


def _stir(f, seed=1, amp=0.3):
    rng = np.random.default_rng(seed)
    f = dict(f)
    for n in ("u", "v", "w"):
        f[n] = f[n] + amp * rng.standard_normal(f[n].shape)
    return f


# tiles of the one-pass kernels cut mid-domain: 33 rows (15 + 15 + 3), 40
# levels (31 + 9), an odd x extent
MOIST_TILES = dict(MOIST, nx=19, ny=33, nz=40)
# an odd number of ghosted levels (39 + 8): the fields' rows are not 16-byte
# multiples, so the momentum pass takes the kernel without TMA plane copies
MOIST_ODD_LEVELS = dict(MOIST, nx=19, ny=33, nz=39)


@pytest.mark.parametrize("cfg", [MOIST, MOIST_TILES, MOIST_ODD_LEVELS], ids=["small", "tiles", "odd_levels"])
def test_fp32_advection_tendencies(cfg):
    nl, rs, f = host_case(**cfg)
    f = _stir(f)
    o, g = oracle_sim(nl, rs, f), gpu_sim(nl, rs, f, precision="fp32")
    o.update_all_bcs()
    g.PV.Update_all_bcs(g.Gr)
    o.sa_update()
    o.ma_update()
    g.SA.update(g.Gr, g.RS, g.PV, g.DV)
    g.MA.update(g.Gr, g.RS, g.PV)
    gt = gpu_tends(g)
    for n in o.names:
        assert rel_l2(gt[n], o.tend(n)) < 1e-5, n


def test_fp32_scalar_fluxes():
    """Face fluxes of the precision form on the faces the divergence reads."""
    import torch
    nl, rs, f = host_case(**MOIST_TILES)
    f = _stir(f)
    nl["gpu"] = {"keep_scalar_fluxes": True}
    o, g = oracle_sim(nl, rs, f), gpu_sim(nl, rs, f, precision="fp32")
    g.SA.keep_fluxes = True
    g.SA.initialize(g.Gr, g.PV)
    o.update_all_bcs()
    g.PV.Update_all_bcs(g.Gr)
    o.sa_update()
    g.SA.update(g.Gr, g.RS, g.PV, g.DV)
    torch.cuda.synchronize()
    gf = g.SA.flux.cpu().numpy().reshape(2, 3, *g.Gr.shape)
    of = o.flux.reshape(2, 3, *g.Gr.shape)
    gw = nl["grid"]["gw"]
    sh = g.Gr.shape
    for d in range(3):
        sl = [slice(gw, sh[a] - gw) for a in range(3)]
        sl[d] = slice(gw - 1, sh[d] - gw)
        assert rel_l2(gf[(slice(None), d) + tuple(sl)], of[(slice(None), d) + tuple(sl)]) < 1e-7, d


def _levels_demeaned(p, d):
    """Interior of a ghosted field with its horizontal mean removed per level."""
    P = p.reshape(d.shape)[d.interior()]
    return P - P.mean(axis=(0, 1), keepdims=True)


MOIST_FFT_CT = dict(MOIST, nx=256, ny=128, nz=12)  # compile-time FFT kernels


@pytest.mark.parametrize("cfg", [MOIST, MOIST_FFT_CT], ids=["runtime_fft", "ct_fft"])
def test_fp32_pressure_refinement_converges(cfg):
    """Refinement computes the residual div - A p in FP64 and solves for the
    correction with the FP32 transforms.  The solver projects out the (0,0)
    horizontal mode (the reference zeroes it), so refinement cannot correct
    the per-level horizontal mean that the first FP32 inverse transform leaves
    in p (~1e-8 relative); that mean has no horizontal gradient and its
    vertical part only reaches the horizontal mean of w, which the next
    solve's remove_mean_u3 removes.  Everything else must converge to the FP64
    solution."""
    from helpers import oracle_dims
    nl, rs, f = host_case(**cfg)
    f = _stir(f)
    o = oracle_sim(nl, rs, f)
    o.update_all_bcs()
    o.pr_update()
    d = oracle_dims(nl)
    ref = o.dv["dynamic_pressure"]
    ref_dm = _levels_demeaned(ref, d)
    raw, demeaned = [], []
    for sweeps in (0, 1, 2):
        g = gpu_sim(nl, rs, f, precision="fp32")
        g.Pr.refine_sweeps = sweeps
        g.PV.Update_all_bcs(g.Gr)
        g.Pr.update(g.Gr, g.RS, g.DV, g.PV)
        p = gpu_dv(g)["dynamic_pressure"]
        raw.append(rel_l2(p, ref))
        demeaned.append(np.linalg.norm(_levels_demeaned(p, d) - ref_dm) / np.linalg.norm(ref_dm))
    print("pressure vs FP64 by refinement sweeps: raw", raw, "level means removed", demeaned)
    assert demeaned[0] < 1e-5
    assert demeaned[1] < demeaned[0] * 1e-4
    assert demeaned[2] < 1e-11  # FP64 level: the plain form's own pressure tolerance
    assert max(raw) < 1e-5 and raw[2] < 1e-7


def test_fp32_form_five_steps():
    nl, rs, f = host_case(**MOIST)
    o, g = oracle_sim(nl, rs, f), gpu_sim(nl, rs, f, precision="fp32")
    o.update_all_bcs()
    g.PV.Update_all_bcs(g.Gr)
    for _ in range(5):
        o.step()
        g.step()
    gf = gpu_fields(g)
    errs = {n: rel_l2(gf[n], o.var(n)) for n in o.names}
    print("precision form vs FP64 oracle after 5 steps:", errs)
    for n in ("s", "qt"):
        assert errs[n] < 1e-6, n
    for n in ("u", "v", "w"):
        # w and v start at rest: compare against the scale of the velocity field
        scale = np.linalg.norm(np.concatenate([o.var(m) for m in ("u", "v", "w")]))
        assert np.linalg.norm(gf[n] - o.var(n)) / scale < 1e-6, n


def test_fp32_form_1000_steps_against_fp64_form():
    """The accuracy budget of the precision form: relative L2
    error <= 1e-5 on s, qt and the velocities after 1000 steps.  The
    reference here is the FP64 plain form on the GPU (the oracle is too
    slow for 1000 steps; the plain form equals it to ~1e-13 after a step)."""
    nl, rs, f = host_case(**MOIST)
    runs = {}
    for precision in ("fp64", "fp32"):
        g = gpu_sim(nl, rs, f, precision=precision)
        g.run(1000)
        g.check_device_errors()
        runs[precision] = gpu_fields(g)
    a, b = runs["fp32"], runs["fp64"]
    vel = np.sqrt(sum(np.linalg.norm(b[m]) ** 2 for m in ("u", "v", "w")))
    errs = {n: np.linalg.norm(a[n] - b[n]) / (vel if n in ("u", "v", "w") else np.linalg.norm(b[n]))
            for n in b}
    print("precision form vs FP64 form after 1000 steps:", errs)
    for n in ("s", "qt", "u", "v", "w"):
        assert errs[n] < 1e-5, n


def test_fused_rk_step_equals_separate_passes():
    """The precision form's fused stepping (SSP-RK3 stage inside the momentum
    pass, new values in a second buffer, the scalars' stage out of place)
    gives the same state, bit for bit, as momentum advection followed by the
    separate RK3 pass: the same operations on the same values."""
    nl, rs, f = host_case(**MOIST_TILES)
    a = gpu_sim(nl, rs, f, precision="fp32")
    b = gpu_sim(nl, rs, f, precision="fp32")
    b.fuse_rk = False
    for g in (a, b):
        g.run(3)
    fa, fb = gpu_fields(a), gpu_fields(b)
    for n in fa:
        assert np.isfinite(fa[n]).all(), n
        assert np.array_equal(fa[n], fb[n]), n
    da, db = gpu_dv(a), gpu_dv(b)
    for n in ("temperature", "ql", "dynamic_pressure"):
        assert np.array_equal(da[n], db[n]), n



@pytest.mark.parametrize("stable", [False, True], ids=["swap", "stable_address"])
def test_reference_call_order_runs_fused_stages(stable):
    """A caller that keeps Simulation3d.run's calls per stage (Th.update,
    SA.update, MA.update, TS.update, PV.Update_all_bcs, Pr.update;
    Simulation3d.pyx:159-178) gets the fused stages: the advection is
    deferred into TS.update, which runs the passes that apply the SSP-RK3
    stage.  The state equals the driver's fused step bit for bit, every
    tendency is left at zero as the reference leaves it, and with
    PV.stable_values the device address of PV.values never changes."""
    import torch
    nl, rs, f = host_case(**MOIST_TILES)
    a = gpu_sim(nl, rs, f, precision="fp32")
    a.run(2)
    b = gpu_sim(nl, rs, f, precision="fp32")
    Gr, RS, PV, DV, TS = b.Gr, b.RS, b.PV, b.DV, b.TS
    PV.stable_values = stable
    PV.Update_all_bcs(Gr)
    b.Th.update(Gr, RS, PV, DV)
    addr = PV.values.data_ptr()
    for _ in range(2):
        for rk in range(3):
            TS.rk_step = rk
            b.Th.update(Gr, RS, PV, DV)
            b.SA.update(Gr, RS, PV, DV)
            b.MA.update(Gr, RS, PV)
            TS.update(Gr, PV)
            PV.Update_all_bcs(Gr)
            b.Pr.update(Gr, RS, DV, PV)
    assert TS.fused_stages == 6
    if stable:
        assert PV.values.data_ptr() == addr
    fa, fb = gpu_fields(a), gpu_fields(b)
    for n in fa:
        assert np.isfinite(fa[n]).all(), n
        assert np.array_equal(fa[n], fb[n]), n
    torch.cuda.synchronize()
    assert float(PV.tendencies.abs().max()) == 0.0


def test_deferred_advection_flushes_for_other_tendency_terms():
    """Deferred advection is launched as plain advection as soon as anything
    reads the tendencies before the time step (here a caller adding its own
    term), so the caller sees the reference's tendencies and the stage runs
    unfused."""
    import torch
    nl, rs, f = host_case(**MOIST_TILES)
    f = _stir(f)
    a = gpu_sim(nl, rs, f, precision="fp32")
    a.fuse_rk = False
    b = gpu_sim(nl, rs, f, precision="fp32")
    for g in (a, b):
        g.PV.Update_all_bcs(g.Gr)
    a.SA.update(a.Gr, a.RS, a.PV, a.DV)
    a.MA.update(a.Gr, a.RS, a.PV)
    b.PV.fuse_stages = True
    b.SA.update(b.Gr, b.RS, b.PV, b.DV)
    b.MA.update(b.Gr, b.RS, b.PV)
    assert b.PV._pending
    tb = b.PV.tendencies  # flushes
    assert not b.PV._pending
    torch.cuda.synchronize()
    assert torch.equal(a.PV.tendencies, tb)
    b.TS.update(b.Gr, b.PV)
    assert b.TS.fused_stages == 0
