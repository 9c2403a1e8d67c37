"""Pins the oracle: the numpy restatement (oracle/port.py) against the
reference's own C kernels compiled from the reference tree (oracle/_ref),
the reference TDMA's known-answer test, and the committed golden fixtures
(tests/golden/*.npz, generated from the reference C by make_golden.py)."""
import os

import numpy as np
import pytest

from helpers import GOLDEN, host_case, oracle_dims, oracle_sim, rel_l2

from oracle import port, ref

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built (needs the reference tree)")

SMALL = dict(case="bomex", nx=10, ny=8, nz=14, dx=100.0, dy=100.0, dz=40.0, gw=3, dt=1.0)


def _stirred(cfg, qt_boost=6e-3):
    nl, rs, f = host_case(**cfg)
    rng = np.random.default_rng(7)
    f = dict(f)
    for n in ("u", "v", "w"):
        f[n] = f[n] + 0.5 * rng.standard_normal(f[n].shape)
    if "qt" in f:
        f["qt"] = f["qt"] + qt_boost
    return nl, rs, f


def test_tdma_known_answer():
    """SparseSolvers.pyx:49-60: a=[0,-1,-1,-1], b=4, c=[-1,-1,-1,0], d=[5,5,10,23] -> [2,3,5,7]."""
    a = np.array([0, -1, -1, -1], dtype=float)
    b = np.array([[4, 4, 4, 4]], dtype=float)
    c = np.array([-1, -1, -1, 0], dtype=float)
    d = np.array([[5, 5, 10, 23]], dtype=float)
    port.tdma(d, a, b, c)
    assert np.allclose(d[0], [2, 3, 5, 7], rtol=0, atol=1e-14)


@needs_ref
def test_tdma_port_matches_reference_cython():
    mod = ref.tdma_module()
    if mod is None:
        pytest.skip("reference SparseSolvers not cythonized")
    rng = np.random.default_rng(0)
    n = 37
    a = rng.standard_normal(n)
    c = rng.standard_normal(n)
    b = 6.0 + rng.standard_normal(n)
    x = rng.standard_normal(n)
    x_ref = x.copy()
    mod.tdma_solve(x_ref, a.copy(), b.copy(), c.copy())
    x_port = x.copy()[None, :]
    port.tdma(x_port, a, b[None, :], c)
    assert np.array_equal(x_port[0], x_ref)


@needs_ref
@pytest.mark.parametrize("order", [5, 7])
def test_advection_port_vs_reference(order):
    cfg = dict(SMALL, gw=4) if order == 7 else SMALL
    cfg = dict(cfg, scalar_order=order, momentum_order=order)
    nl, rs, f = _stirred(cfg)
    a, b = oracle_sim(nl, rs, f, "ref"), oracle_sim(nl, rs, f, "port")
    a.update_all_bcs()
    b.update_all_bcs()
    a.sa_update()
    b.sa_update()
    a.ma_update()
    b.ma_update()
    for n in a.names:
        assert rel_l2(b.tend(n), a.tend(n)) < 1e-14, n


@needs_ref
def test_thermo_port_vs_reference():
    nl, rs, f = _stirred(SMALL)
    a, b = oracle_sim(nl, rs, f, "ref"), oracle_sim(nl, rs, f, "port")
    a.update_all_bcs()
    b.update_all_bcs()
    a.th_update()
    b.th_update()
    assert (a.dv["ql"] > 0).any()
    # the port evaluates exp/log/pow with the C library and keeps the
    # reference's operation order: bit-identical
    for k in a.dv:
        assert np.array_equal(b.dv[k], a.dv[k]), k
    assert np.array_equal(b.tend("w"), a.tend("w"))


@needs_ref
def test_dry_thermo_port_vs_reference():
    nl, rs, f = host_case("dry_cbl", 8, 8, 12, 50.0, 50.0, 50.0)
    a, b = oracle_sim(nl, rs, f, "ref"), oracle_sim(nl, rs, f, "port")
    a.update_all_bcs()
    b.update_all_bcs()
    a.th_update()
    b.th_update()
    for k in a.dv:
        assert np.array_equal(b.dv[k], a.dv[k]), k
    assert np.array_equal(b.tend("w"), a.tend("w"))


@needs_ref
def test_halo_port_vs_reference_exact():
    nl, rs, f = _stirred(dict(SMALL, gw=4))
    a, b = oracle_sim(nl, rs, f, "ref"), oracle_sim(nl, rs, f, "port")
    a.update_all_bcs()
    b.update_all_bcs()
    assert np.array_equal(a.values, b.values)


@needs_ref
def test_reference_state_port_vs_reference():
    from oracle import glue
    from helpers import oracle_dims
    nl, _, _ = host_case(**SMALL)
    d = oracle_dims(nl)
    r1 = glue.reference_state(d, 1.015e5, 300.4, 0.02245, moist=True, backend="ref")
    r2 = glue.reference_state(d, 1.015e5, 300.4, 0.02245, moist=True, backend="port")
    for k in r1:
        assert rel_l2(r2[k], r1[k]) < 1e-14, k


def test_package_reference_state_matches_oracle():
    """The package's host-side reference-state integration (init only) agrees
    with the oracle's restatement of ReferenceState.initialize."""
    from oracle import glue
    from helpers import oracle_dims
    nl, rs, _ = host_case(**SMALL)
    d = oracle_dims(nl)
    r = glue.reference_state(d, 1.015e5, 300.4, 0.02245, moist=True, backend="port")
    for k in r:
        assert rel_l2(rs[k], r[k]) < 1e-13, k


@pytest.mark.parametrize("name", ["moist_w5", "moist_w7", "dry_w5"])
def test_golden_fixtures_port(name):
    """The numpy restatement reproduces the reference-generated goldens."""
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    cfg = eval(str(z["meta"][0]))  # the dict literal make_golden.py wrote
    from pycles_b200.simulation import namelist_for
    nl = namelist_for(**cfg)
    rs = {k[3:]: z[k] for k in z.files if k.startswith("rs_")}
    f = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    f0 = {k[4:]: z[k] for k in z.files if k.startswith("in0_")}

    def sim(fields=f):
        s = oracle_sim(nl, rs, fields, "port")
        s.update_all_bcs()
        return s

    s = sim()
    for k in s.names:
        assert np.array_equal(s.var(k), z["bcs_" + k]), k
    s.th_update()
    for k in s.dv:
        assert np.array_equal(s.dv[k], z["th_" + k]), k
    s = sim()
    s.sa_update()
    for k in s.names[3:]:
        assert rel_l2(s.tend(k), z["sa_" + k]) < 1e-14, k
    s = sim()
    s.ma_update()
    for k in ("u", "v", "w"):
        assert rel_l2(s.tend(k), z["ma_" + k]) < 1e-14, k
    s = sim()
    s.pr_update()
    assert rel_l2(s.dv["dynamic_pressure"], z["pr_p"]) < 1e-13
    for k in ("u", "v", "w"):
        assert rel_l2(s.var(k), z["pr_" + k]) < 1e-14, k
    # a whole time step, and Simulation3d.run's prologue + one step: bit-identical
    s = sim(f0)
    s.step()
    for k in s.names:
        assert np.array_equal(s.var(k), z["step_" + k]), k
    s = oracle_sim(nl, rs, f0, "port")
    s.update_all_bcs()
    s.th_update()
    s.step()
    for k in s.names:
        assert np.array_equal(s.var(k), z["run1_" + k]), k


# ---- surface fluxes (Surface.pyx, Csrc/surface.h) --------------------------
SURFACE_FIXTURES = ["surface_sullivan_patton", "surface_bomex", "surface_dycoms_rf01"]


@needs_ref
def test_surface_layer_functions_port_vs_reference():
    """compute_ustar (the reference runs its secant loop; the restatement
    returns the first iterate the reference returns), compute_windspeed and
    entropyflux_from_thetaflux_qtflux, bit for bit against the reference C."""
    rng = np.random.default_rng(11)
    n_stable = 0
    for t in range(2000):
        ws = 10 ** rng.uniform(-3, 1.3)
        bf = 0.0 if t % 40 == 0 else rng.choice([-1.0, 1.0]) * 10 ** rng.uniform(-6, -1)
        z0, zb = 10 ** rng.uniform(-4, -0.5), rng.uniform(1.0, 30.0)
        n_stable += bf < 0
        assert port.compute_ustar(ws, bf, z0, zb) == ref.compute_ustar(ws, bf, z0, zb), (ws, bf, z0, zb)
    assert 500 < n_stable < 1500  # both stability branches exercised
    nl, rs, f = _stirred(SMALL)
    d = oracle_dims(nl)
    a, b = np.zeros(d.nlg[0] * d.nlg[1]), np.zeros(d.nlg[0] * d.nlg[1])
    port.compute_windspeed(d, f["u"], f["v"], a, 0.7, -0.3, 0.001)
    ref.compute_windspeed(d, f["u"], f["v"], b, 0.7, -0.3, 0.001)
    assert np.array_equal(a, b)
    T = rng.uniform(280.0, 305.0, 64)
    qt = rng.uniform(1e-3, 2e-2, 64)
    qv = qt * rng.uniform(0.9, 1.0, 64)
    assert np.array_equal(port.entropyflux_from_thetaflux_qtflux(8e-3, 5.2e-5, 1.0e5, T, qt, qv),
                          ref.entropyflux_from_thetaflux_qtflux(8e-3, 5.2e-5, 1.0e5, T, qt, qv))


def _surface_fixture(name):
    from pycles_b200.simulation import namelist_for
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    cfg = eval(str(z["meta"][0]))  # dict literal written by make_golden.py
    scheme = str(z["meta"][1])
    nl = namelist_for(**cfg)
    rs = {k[3:]: z[k] for k in z.files if k.startswith("rs_")}
    f = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    f0 = {k[4:]: z[k] for k in z.files if k.startswith("in0_")}
    return z, scheme, nl, rs, f, f0


@pytest.mark.parametrize("name", SURFACE_FIXTURES)
def test_surface_golden_port(name):
    """The restated surface glue on the numpy restatement reproduces the
    reference-generated surface fixtures: the fluxes and tendencies bit for
    bit, one time step with the scheme to 1e-13."""
    from oracle.surface import OracleSurface
    z, scheme, nl, rs, f, f0 = _surface_fixture(name)
    d = oracle_dims(nl)
    s = oracle_sim(nl, rs, f, "port")
    s.update_all_bcs()
    s.th_update()
    s.tendencies[:] = 0.0
    s.surface = OracleSurface(scheme, d, u0=float(rs["u0"]), v0=float(rs["v0"]))
    s.surface.update(s)
    for n in OracleSurface.NAMES:
        assert np.array_equal(getattr(s.surface, n), z["sur_" + n]), n
    for k in s.names:
        assert np.array_equal(s.tend(k), z["surtend_" + k]), k
    from oracle.forcing import OracleForcing
    from pycles_b200.grid import Grid
    s = oracle_sim(nl, rs, f0, "port")
    s.surface = OracleSurface(scheme, d, u0=float(rs["u0"]), v0=float(rs["v0"]))
    s.forcing = OracleForcing(scheme, d, rs["p0_half"], Grid(nl).zl_half, u0=float(rs["u0"]), v0=float(rs["v0"]))
    if scheme == "DYCOMS_RF01":
        from oracle.radiation import OracleRadiation
        s.radiation = OracleRadiation(d, Grid(nl).z)
    s.update_all_bcs()
    s.step()
    for k in s.names:
        assert rel_l2(s.var(k), z["step_" + k]) < 1e-13, k


def test_surface_changes_the_step():
    """The surface fluxes reach the state: a step with the scheme differs
    from one without it at the first interior level (a planted omission of
    the surface update would pass the other checks of an unchanged field)."""
    z, scheme, nl, rs, f, f0 = _surface_fixture("surface_bomex")
    s = oracle_sim(nl, rs, f0, "port")
    s.update_all_bcs()
    s.step()
    d = oracle_dims(nl)
    for k in ("u", "s", "qt"):
        a = s.var(k).reshape(d.shape)[d.gw:-d.gw, d.gw:-d.gw, d.gw]
        b = z["step_" + k].reshape(d.shape)[d.gw:-d.gw, d.gw:-d.gw, d.gw]
        assert rel_l2(a, b) > 1e-9, k


# ---- subgrid scale and diffusion (SGS.pyx, Kinematics.pyx, *Diffusion.pyx) --
SGS_FIXTURES = ["sgs_smagorinsky_bomex", "sgs_smagorinsky_iles_bomex", "sgs_smagorinsky_wall_dry",
                "sgs_uniform_dycoms"]


def _sgs_fixture(name):
    from pycles_b200.simulation import namelist_for
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    cfg = eval(str(z["meta"][0]))  # dict literals written by make_golden.py
    extra = eval(str(z["meta"][1]))
    nl = dict(namelist_for(**cfg), **extra)
    rs = {k[3:]: z[k] for k in z.files if k.startswith("rs_")}
    f = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    f0 = {k[4:]: z[k] for k in z.files if k.startswith("in0_")}
    return z, nl, rs, f, f0


@pytest.mark.parametrize("name", SGS_FIXTURES)
def test_sgs_golden_port(name):
    """The restated SGS glue on the numpy restatement reproduces the
    reference-generated fixtures: strain-rate magnitude, viscosity and
    diffusivity (from the plane i = 2 on: at i = 1 the reference's strain
    stencil reads before its array) and the diffusion tendencies bit for bit,
    one time step to 1e-13."""
    from oracle.sgs import OracleSGS, scheme_from_namelist
    from oracle.surface import OracleSurface
    from pycles_b200.grid import Grid
    z, nl, rs, f, f0 = _sgs_fixture(name)
    d = oracle_dims(nl)
    conf = scheme_from_namelist(nl)
    casename = nl.get("meta", {}).get("casename")

    def attach(s):
        s.sgs = OracleSGS(conf, d, Grid(nl).zl_half)
        if casename:
            from oracle.forcing import OracleForcing
            s.surface = OracleSurface(casename, d, u0=float(rs["u0"]), v0=float(rs["v0"]))
            s.forcing = OracleForcing(casename, d, rs["p0_half"], Grid(nl).zl_half, u0=float(rs["u0"]),
                                      v0=float(rs["v0"]))
        return s

    s = attach(oracle_sim(nl, rs, f, "port"))
    s.update_all_bcs()
    s.sgs.ke_update(s)
    s.th_update()
    s.sgs.sgs_update(s)
    for n in ("strain_rate_mag", "viscosity", "diffusivity"):
        a = getattr(s.sgs, n).reshape(d.shape)[2:]
        b = z["sgs_" + n].reshape(d.shape)[2:]
        assert np.array_equal(a, b), n
    s.tendencies[:] = 0.0
    s.sgs.sd_update(s)
    for k in s.names:
        assert np.array_equal(s.tend(k), z["sdtend_" + k]), k
    s.tendencies[:] = 0.0
    s.sgs.md_update(s)
    for k in s.names:
        assert np.array_equal(s.tend(k), z["mdtend_" + k]), k
    s = attach(oracle_sim(nl, rs, f0, "port"))
    s.update_all_bcs()
    s.step()
    for k in s.names:
        assert rel_l2(s.var(k), z["step_" + k]) < 1e-13, k


def test_sgs_namelist_switches():
    """SGS.pyx:109-122: iles read after wall switches the wall adjustment off;
    the defaults cs = 0.17, prt = 1/3."""
    from oracle.sgs import scheme_from_namelist
    c = scheme_from_namelist({"sgs": {"scheme": "Smagorinsky", "Smagorinsky": {"wall": True, "iles": True}}})
    assert c["variant"] == "iles" and c["cs"] == 0.17 and c["prt"] == 1.0 / 3.0
    c = scheme_from_namelist({"sgs": {"scheme": "Smagorinsky", "Smagorinsky": {"wall": True}}})
    assert c["variant"] == "wall"
    c = scheme_from_namelist({"sgs": {"scheme": "UniformViscosity"}})
    assert c["viscosity"] == 0.0 and c["diffusivity"] == 0.0 and not c["qt_entropy_source"]


def test_horizontal_stat_restatement():
    """The sequential restatement of ParallelMPI's reductions against numpy
    reductions of the same interior columns (order aside, they agree), and
    HorizontalMean against the one the pressure glue uses."""
    nl, rs, f = host_case(**SMALL)
    d = oracle_dims(nl)
    rng = np.random.default_rng(2)
    a, b = f["s"], rng.standard_normal(d.npg)
    m = (rng.random(d.npg) < 0.5).astype(float)
    g_ = d.gw
    I = lambda x: x.reshape(d.shape)[g_:-g_, g_:-g_, :]
    assert rel_l2(port.horizontal_stat(d, "mean", a), port.horizontal_mean(d, a)) < 1e-15
    assert rel_l2(port.horizontal_stat(d, "squares", a, b), (I(a) * I(b)).mean(axis=(0, 1))) < 1e-13
    assert np.array_equal(port.horizontal_stat(d, "max", b), I(b).max(axis=(0, 1)))
    assert np.array_equal(port.horizontal_stat(d, "min", b), I(b).min(axis=(0, 1)))
    cond = (I(b) * I(m)).sum(axis=(0, 1)) / np.maximum(I(m).sum(axis=(0, 1)), 1.0)
    assert rel_l2(port.horizontal_stat(d, "conditional", b, mask=m), cond) < 1e-13


# ---- whole cases: surface + forcing (+ subgrid scale) ----------------------
CASE_FIXTURES = ["case_bomex", "case_dycoms_rf01", "case_sullivan_patton"]


@pytest.mark.parametrize("name", CASE_FIXTURES)
def test_case_golden_port(name):
    """The restated forcing (and surface, subgrid scale) on the numpy
    restatement reproduces the reference-generated case fixtures: the
    forcing tendencies bit for bit, one time step to 1e-13."""
    from oracle.forcing import OracleForcing
    from oracle.sgs import OracleSGS, scheme_from_namelist
    from oracle.surface import OracleSurface
    from pycles_b200.grid import Grid
    z, nl, rs, f, f0 = _sgs_fixture(name)
    d = oracle_dims(nl)
    casename = nl["meta"]["casename"]
    zl = Grid(nl).zl_half

    def attach(s):
        s.surface = OracleSurface(casename, d, u0=float(rs["u0"]), v0=float(rs["v0"]))
        s.forcing = OracleForcing(casename, d, rs["p0_half"], zl, u0=float(rs["u0"]), v0=float(rs["v0"]))
        if "sgs" in nl:
            s.sgs = OracleSGS(scheme_from_namelist(nl), d, zl)
        if casename == "DYCOMS_RF01":
            from oracle.radiation import OracleRadiation
            s.radiation = OracleRadiation(d, Grid(nl).z)
        return s

    s = attach(oracle_sim(nl, rs, f, "port"))
    s.update_all_bcs()
    s.th_update()
    s.tendencies[:] = 0.0
    s.forcing.update(s)
    for k in s.names:
        assert np.array_equal(s.tend(k), z["fotend_" + k]), k
    if s.radiation is not None:
        s.tendencies[:] = 0.0
        s.radiation.update(s)
        assert np.array_equal(s.tend("s"), z["ratend_s"])
        assert np.array_equal(s.radiation.heating_rate, z["ra_heating_rate"])
    s = attach(oracle_sim(nl, rs, f0, "port"))
    s.update_all_bcs()
    s.step()
    for k in s.names:
        assert rel_l2(s.var(k), z["step_" + k]) < 1e-13, k


@pytest.mark.parametrize("casename", ["SullivanPatton", "Bomex", "DYCOMS_RF01"])
def test_forcing_profiles_match_restatement(casename):
    """The package's host-side forcing profiles (pycles_b200/forcing.py) equal
    the oracle's restatement of the schemes' initialize, bit for bit."""
    from pycles_b200.forcing import ForcingFactory
    from pycles_b200.grid import Grid
    nl, rs, f = host_case(**SMALL)
    Gr = Grid(nl)
    Gr.device = "cpu"
    fo = ForcingFactory({"meta": {"casename": casename}})

    class RS:
        p0_half = rs["p0_half"]

    P = {k: np.zeros(len(Gr.zl_half)) for k in ("ug", "vg", "dtdt", "dqtdt", "subsidence")}
    fo._profiles(np.asarray(Gr.zl_half), np.asarray(RS.p0_half), P)
    O = port.forcing_profiles(casename, Gr.zl_half, rs["p0_half"])
    for k in P:
        assert np.array_equal(P[k], O[k]), k
    assert fo.coriolis_param == O["coriolis_param"]
