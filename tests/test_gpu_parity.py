"""GPU parity: every hot-path component through the C ABI against the CPU
oracle (numpy restatement, itself pinned to the reference's compiled C) on
the same seeded inputs.

Tolerances (relative L2 per field):
  * advection tendencies, FP64 plain form: bit-identical (the FP64 advection
    is compiled without FMA contraction and keeps the reference's operations)
  * prognostic / diagnostic fields after one call, FP64 plain form: 1e-12
  * buoyancy (cancels ~3 digits of alpha) and buoyancy frequency (vertical
    differences): 1e-10
"""
import numpy as np
import pytest

from helpers import gpu_dv, gpu_fields, gpu_sim, gpu_tends, host_case, oracle_sim, rel_l2

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-12
DERIVED_TOL = 1e-10  # fields formed by cancellation or vertical differences

MOIST_SMALL = dict(case="bomex", nx=16, ny=12, nz=20, dx=100.0, dy=100.0, dz=40.0, gw=3, dt=1.0)
MOIST_W7 = dict(case="bomex", nx=12, ny=16, nz=18, dx=100.0, dy=100.0, dz=40.0, gw=4, dt=1.0,
                scalar_order=7, momentum_order=7)
DRY_SMALL = dict(case="dry_cbl", nx=16, ny=16, nz=16, dx=50.0, dy=50.0, dz=50.0, gw=3, dt=0.5)
ODD = dict(case="bomex", nx=12, ny=10, nz=14, dx=100.0, dy=100.0, dz=40.0, gw=3, dt=1.0)
# odd nx (no Nyquist column in the half spectrum) and odd nz (the last
# packed pair of levels of the x-FFT has one row)
ODD_XZ = dict(case="bomex", nx=9, ny=10, nz=13, dx=100.0, dy=100.0, dz=40.0, gw=3, dt=1.0)
# lengths with compile-time FFT kernels (128 ... 1024), odd nz
FFT_CT = dict(case="bomex", nx=256, ny=128, nz=7, dx=100.0, dy=100.0, dz=40.0, gw=3, dt=1.0)
FFT_CT_WIDE = dict(case="bomex", nx=512, ny=1024, nz=3, dx=100.0, dy=100.0, dz=40.0, gw=3, dt=1.0)


def _stir(fields, seed=1, amp=0.5):
    """Add seeded velocity structure so that every advection branch is hit."""
    rng = np.random.default_rng(seed)
    out = dict(fields)
    for n in ("u", "v", "w"):
        out[n] = fields[n] + amp * rng.standard_normal(fields[n].shape)
    return out


def _setup(cfg, stir=True, seed=0):
    nl, rs, f = host_case(**cfg, seed=seed)
    if stir:
        f = _stir(f)
    return nl, rs, f


def _bcs_both(o, g):
    o.update_all_bcs()
    g.PV.Update_all_bcs(g.Gr)


@pytest.mark.parametrize("cfg", [MOIST_SMALL, ODD, MOIST_W7], ids=["weno5", "odd", "weno7"])
def test_scalar_advection(cfg):
    nl, rs, f = _setup(cfg)
    o, g = oracle_sim(nl, rs, f), gpu_sim(nl, rs, f)
    _bcs_both(o, g)
    o.sa_update()
    g.SA.update(g.Gr, g.RS, g.PV, g.DV)
    gt = gpu_tends(g)
    print("scalar tendencies rel L2:", {n: rel_l2(gt[n], o.tend(n)) for n in ("s", "qt")})
    for n in ("s", "qt"):
        assert np.array_equal(gt[n], o.tend(n)), n


@pytest.mark.parametrize("cfg", [MOIST_SMALL, ODD, MOIST_W7], ids=["weno5", "odd", "weno7"])
def test_momentum_advection(cfg):
    nl, rs, f = _setup(cfg)
    o, g = oracle_sim(nl, rs, f), gpu_sim(nl, rs, f)
    _bcs_both(o, g)
    o.ma_update()
    g.MA.update(g.Gr, g.RS, g.PV)
    gt = gpu_tends(g)
    print("momentum tendencies rel L2:", {n: rel_l2(gt[n], o.tend(n)) for n in ("u", "v", "w")})
    for n in ("u", "v", "w"):
        assert np.array_equal(gt[n], o.tend(n)), n


def test_scalar_fluxes_exposed():
    """ScalarAdvection.flux on the faces the divergence reads."""
    import torch
    nl, rs, f = _setup(MOIST_SMALL)
    nl["gpu"] = {"keep_scalar_fluxes": True}
    o, g = oracle_sim(nl, rs, f), gpu_sim(nl, rs, f)
    g.SA.keep_fluxes = True
    g.SA.initialize(g.Gr, g.PV)
    _bcs_both(o, g)
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
        assert rel_l2(gf[(slice(None), d) + tuple(sl)], of[(slice(None), d) + tuple(sl)]) < 1e-13


def test_thermo_sa():
    nl, rs, f = _setup(MOIST_SMALL, stir=False)
    # raise qt so that part of the column is saturated
    f = dict(f)
    # saturate half of the domain (i < nx/2), leave the other half as it is
    qt = f["qt"].reshape(nl["grid"]["nx"] + 6, -1).copy()
    qt[: qt.shape[0] // 2] += 6e-3
    f["qt"] = qt.ravel()
    o, g = oracle_sim(nl, rs, f), gpu_sim(nl, rs, f)
    _bcs_both(o, g)
    o.th_update()
    g.Th.update(g.Gr, g.RS, g.PV, g.DV)
    gd, gt = gpu_dv(g), gpu_tends(g)
    assert (o.dv["ql"] > 0).any() and (o.dv["ql"] == 0).any()
    for n in ("temperature", "qv", "ql", "alpha", "theta_rho", "thetali"):
        assert rel_l2(gd[n], o.dv[n]) < FIELD_TOL, n
    # buoyancy cancels ~3 digits of alpha, bvf differentiates T in z
    for n in ("buoyancy", "buoyancy_frequency"):
        assert rel_l2(gd[n], o.dv[n]) < DERIVED_TOL, n
    assert rel_l2(gt["w"], o.tend("w")) < DERIVED_TOL
    assert np.array_equal(gd["qi"] == 0, o.dv["qi"] == 0)
    it = g.Th.iter_stats.cpu().numpy()
    assert it[1] == int((o.dv["ql"] > 0).sum()) or it[1] >= int((o.dv["ql"] > 0).sum())
    assert it[0] == int(o.secant_iters.sum())


def test_thermo_dry():
    nl, rs, f = _setup(DRY_SMALL, stir=False)
    o, g = oracle_sim(nl, rs, f), gpu_sim(nl, rs, f)
    _bcs_both(o, g)
    o.th_update()
    g.Th.update(g.Gr, g.RS, g.PV, g.DV)
    gd, gt = gpu_dv(g), gpu_tends(g)
    for n in ("temperature", "alpha", "theta"):
        assert rel_l2(gd[n], o.dv[n]) < FIELD_TOL, n
    for n in ("buoyancy", "buoyancy_frequency"):
        assert rel_l2(gd[n], o.dv[n]) < DERIVED_TOL, n
    assert rel_l2(gt["w"], o.tend("w")) < DERIVED_TOL


def test_ghost_fill_exact():
    nl, rs, f = _setup(ODD)
    o, g = oracle_sim(nl, rs, f), gpu_sim(nl, rs, f)
    _bcs_both(o, g)
    gf = gpu_fields(g)
    for n in o.names:
        assert np.array_equal(gf[n], o.var(n)), n


def test_rk3_stages():
    nl, rs, f = _setup(MOIST_SMALL)
    o, g = oracle_sim(nl, rs, f), gpu_sim(nl, rs, f)
    rng = np.random.default_rng(3)
    tend = rng.standard_normal(o.tendencies.shape)
    import torch
    for rk in range(3):
        o.tendencies[:] = tend * (rk + 1)
        g.PV.tendencies.copy_(torch.as_tensor(tend * (rk + 1)))
        o.ts_update(rk)
        g.TS.rk_step = rk
        g.TS.update(g.Gr, g.PV)
        gf = gpu_fields(g)
        for n in o.names:
            assert rel_l2(gf[n], o.var(n)) < 1e-15, (rk, n)
        assert float(g.PV.tendencies.abs().max()) == 0.0


@pytest.mark.parametrize("cfg", [MOIST_SMALL, ODD, ODD_XZ, DRY_SMALL, FFT_CT, FFT_CT_WIDE],
                         ids=["pow2ish", "odd", "odd_xz", "dry", "fft_ct", "fft_ct_wide"])
def test_pressure(cfg):
    nl, rs, f = _setup(cfg)
    o, g = oracle_sim(nl, rs, f), gpu_sim(nl, rs, f)
    _bcs_both(o, g)
    o.pr_update()
    g.Pr.update(g.Gr, g.RS, g.DV, g.PV)
    gf, gd = gpu_fields(g), gpu_dv(g)
    assert rel_l2(gd["divergence"], o.dv["divergence"]) < FIELD_TOL
    assert rel_l2(gd["dynamic_pressure"], o.dv["dynamic_pressure"]) < 1e-11
    for n in ("u", "v", "w"):
        assert rel_l2(gf[n], o.var(n)) < FIELD_TOL, n


@pytest.mark.parametrize("cfg", [MOIST_SMALL, DRY_SMALL, MOIST_W7], ids=["moist", "dry", "weno7"])
def test_one_step(cfg):
    """The plain-form gate: every prognostic field after one full step
    (three RK stages of the hot path) within 1e-12 relative L2."""
    nl, rs, f = _setup(cfg, stir=False)
    o, g = oracle_sim(nl, rs, f), gpu_sim(nl, rs, f)
    _bcs_both(o, g)
    o.step()
    g.step()
    gf = gpu_fields(g)
    print("one step rel L2:", {n: rel_l2(gf[n], o.var(n)) for n in o.names})
    for n in o.names:
        assert rel_l2(gf[n], o.var(n)) < FIELD_TOL, n


def test_run_matches_simulation3d_prologue():
    """run(): ghost fill + thermodynamics before the loop, as Simulation3d.run."""
    nl, rs, f = _setup(MOIST_SMALL, stir=False)
    o, g = oracle_sim(nl, rs, f), gpu_sim(nl, rs, f)
    o.update_all_bcs()
    o.th_update()
    o.step()
    o.step()
    g.run(2)
    gf = gpu_fields(g)
    for n in o.names:
        assert rel_l2(gf[n], o.var(n)) < FIELD_TOL, n


def test_device_error_flags():
    """Fault injection on the host side of the boundary: an out-of-table
    temperature and a secant cap of one iteration set the error word; the
    context stays usable."""
    from pycles_b200 import _capi
    nl, rs, f = _setup(MOIST_SMALL, stir=False)
    f = dict(f)
    f["qt"] = f["qt"] + 6e-3
    g = gpu_sim(nl, rs, f)
    g.PV.Update_all_bcs(g.Gr)
    _capi.clear_error()
    g.Th.max_secant_iter = 1
    g.Th.update(g.Gr, g.RS, g.PV, g.DV)
    assert _capi.get_error() & _capi.ERR_SECANT_CAP
    _capi.clear_error()
    g.Th.max_secant_iter = 100
    g.PV.field("s", g.Gr).add_(5000.0)  # far outside the pv* table
    g.Th.update(g.Gr, g.RS, g.PV, g.DV)
    assert _capi.get_error() & _capi.ERR_TABLE_RANGE
    _capi.clear_error()
    assert _capi.get_error() == 0


def test_step_host_equals_device_step():
    """HotPathSimulation.step_host (state in pinned host memory, copies in
    chunks overlapped with the first thermodynamics update and the last
    pressure solve) gives the device-resident step's state bit for bit, also
    when the chunking changes between steps and when a device step runs
    between two host steps."""
    import torch
    nl, rs, f = _setup(MOIST_SMALL, stir=False)
    a, b = gpu_sim(nl, rs, f), gpu_sim(nl, rs, f)
    for g in (a, b):
        g.PV.Update_all_bcs(g.Gr)
    host = torch.empty(b.PV.values.numel(), dtype=torch.float64, pin_memory=True)
    host.copy_(b.PV.values)
    for chunks in (4, 4, 1, 3):
        a.step()
        b.step_host(host, chunks_per_variable=chunks)
    # a device step between two host steps (ordered after the download, as
    # any work on the device copy must be): its result is replaced by the
    # host state's upload, which must wait for it, not race with it
    for cs in b.copy_streams():
        torch.cuda.current_stream().wait_stream(cs)
    b.step()
    a.step()
    b.step_host(host)
    torch.cuda.synchronize()
    ref = a.PV.values.cpu().numpy()
    assert np.all(np.isfinite(ref))
    assert np.array_equal(host.numpy(), ref)
