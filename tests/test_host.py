"""Host-side logic without a GPU: grid geometry against the reference's
DimStruct rules, variable bookkeeping, configurations, the learned seed's
parameter layout, and the precision-form pressure refinement restated on
the CPU with the oracle's pieces (FP32 transforms, FP64 residual)."""
import numpy as np
import pytest

from pycles_b200 import _capi
from pycles_b200.grid import Grid
from pycles_b200.simulation import CONFIGS, namelist_for
from pycles_b200.variables import DiagnosticVariables, PrognosticVariables


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_grid_dims_follow_reference_rules(name):
    """Grid.pyx:17-48 on one rank: nl = n, nlg = n + 2 gw, npg = prod(nlg),
    nbuffer[d] = gw * max over the other two ghosted extents' product."""
    from oracle.dims import Dims
    cfg = CONFIGS[name]
    nl = namelist_for(**cfg)
    d = Grid(nl).dims
    o = Dims((cfg["nx"], cfg["ny"], cfg["nz"]), cfg["gw"], (cfg["dx"], cfg["dy"], cfg["dz"]))
    oc = o.c()
    for f in ("n", "ng", "nl", "nlg", "nbuffer", "ghosted_stride"):
        assert list(getattr(d, f)) == list(getattr(oc, f)), f
    for f in ("npd", "npl", "npg", "gw", "dims"):
        assert getattr(d, f) == getattr(oc, f), f
    assert list(d.dx) == list(oc.dx) and list(d.dxi) == list(oc.dxi)
    g = Grid(nl)
    assert np.array_equal(g.z_half, o.z_half) and np.array_equal(g.z, o.z)


def test_c5_geometry_sizes():
    """512x512x256 with gw=4: 67,108,864 interior cells, 71,385,600 ghosted."""
    d = Grid(namelist_for(**CONFIGS["c5_dycoms"])).dims
    assert d.npl == 67_108_864 and d.npg == 71_385_600
    assert _capi.load().pb_pressure_workspace_bytes(d) > 0


def test_variable_bookkeeping_matches_reference():
    """add_variable (PrognosticVariables.pyx:34-64): name_index, bc_type
    (sym -> +1, asym -> -1), var_type (velocity 0, scalar 1)."""
    g = Grid(namelist_for(**CONFIGS["c1_dry_cbl"]))
    pv = PrognosticVariables(g)
    pv.add_variable("u", "m/s", "u", "", "sym", "velocity")
    pv.add_variable("v", "m/s", "v", "", "sym", "velocity")
    pv.add_variable("w", "m/s", "w", "", "asym", "velocity")
    pv.add_variable("s", "J/kg/K", "s", "", "sym", "scalar")
    for i, n in enumerate("uvw"):
        pv.set_velocity_direction(n, i)
    assert pv.name_index == {"u": 0, "v": 1, "w": 2, "s": 3}
    assert list(pv.bc_type) == [1.0, 1.0, -1.0, 1.0]
    assert list(pv.var_type) == [0, 0, 0, 1]
    assert pv.nv_velocities == 3 and pv.nv_scalars == 1
    assert list(pv.velocity_directions) == [0, 1, 2]
    assert pv.get_varshift(g, "s") == 3 * g.dims.npg
    with pytest.raises(ValueError):
        pv.add_variable("x", "", "", "", "periodic", "scalar")
    pv.initialize(g, device="cpu")
    assert pv.get_variable_array("w", g).shape == g.shape
    dv = DiagnosticVariables()
    dv.add_variables("T", "K", "T", "", "sym")
    dv.add_variables("T", "K", "T", "", "sym")  # repeated names are ignored, as the reference does
    dv.add_variables("bvf", "1/s^2", "N2", "", "sym")
    assert dv.nv == 2 and dv.name_index == {"T": 0, "bvf": 1}


def test_config_orders_and_ghost_widths():
    """WENO7 needs gw >= 4; every configuration satisfies gw >= (order+1)/2."""
    for cfg in CONFIGS.values():
        nl = namelist_for(**cfg)
        for key in ("scalar_transport", "momentum_transport"):
            assert nl["grid"]["gw"] >= (nl[key]["order"] + 1) // 2
    c5 = namelist_for(**CONFIGS["c5_dycoms"])
    assert c5["scalar_transport"]["order"] == 7 and c5["momentum_transport"]["order"] == 5
    assert c5["time_stepping"]["dt_initial"] == 0.25


def test_learned_seed_parameter_layout():
    """3 -> 64 -> 64 -> 1: W1 (64x3) b1 W2 (64x64) b2 W3 (64) b3, packed in
    the order the kernels read them; the count matches the header's."""
    from pycles_b200 import learned
    h = 64
    assert _capi.MLP_NPARAM == 3 * h + h + h * h + h + h + 1 == 4481
    assert learned.IN_LO == (5e4, 6800.0, 0.0) and learned.IN_HI == (1.02e5, 7100.0, 0.025)


def test_precision_form_refinement_algorithm_on_cpu():
    """The precision-form pressure algorithm with the oracle's building
    blocks: transforms in complex64, tridiagonal solves in FP64 on the FP32
    spectra, then sweeps p += solve32(div - A p) with the residual in FP64.
    The residual (its projected-out (0,0) mode removed) falls from ~1e-7 to
    FP64 level, and away from the per-level horizontal mean the solution
    equals the FP64 solve to ~1e-14."""
    from oracle import port
    from oracle.dims import Dims
    d = Dims((16, 16, 12), 3, (100.0, 100.0, 40.0))
    sh, gw = d.shape, d.gw
    rng = np.random.default_rng(3)
    z = d.z_half
    rho0 = 1.2 * np.exp(-np.concatenate([d.z, [d.z[-1] + d.dx[2]]])[:sh[2]] / 8000.0)
    rho0_half = 1.2 * np.exp(-z / 8000.0)
    I = tuple(slice(gw, n - gw) for n in sh)
    div = np.zeros(sh)
    div[I] = rng.standard_normal(div[I].shape)
    div[I] -= div[I].mean(axis=(0, 1), keepdims=True)
    div = div.reshape(-1)

    def apply_A(p):
        P = p.reshape(sh).copy()
        port.fill_ghosts(d, P.reshape(-1), 1.0)
        Pc = P[I]
        lap = rho0_half[None, None, gw:sh[2] - gw] * (
            (P[gw + 1:sh[0] - gw + 1, gw:-gw, gw:-gw] - 2 * Pc + P[gw - 1:sh[0] - gw - 1, gw:-gw, gw:-gw]) * d.dxi[0] ** 2
            + (P[gw:-gw, gw + 1:sh[1] - gw + 1, gw:-gw] - 2 * Pc + P[gw:-gw, gw - 1:sh[1] - gw - 1, gw:-gw]) * d.dxi[1] ** 2)
        kk = np.arange(gw, sh[2] - gw)
        up = P[gw:-gw, gw:-gw, gw + 1:sh[2] - gw + 1] - Pc
        dn = Pc - P[gw:-gw, gw:-gw, gw - 1:sh[2] - gw - 1]
        vert = (np.where(kk < sh[2] - gw - 1, rho0[kk], 0.0)[None, None, :] * up
                - np.where(kk > gw, rho0[kk - 1], 0.0)[None, None, :] * dn)
        out = np.zeros(sh)
        out[I] = lap + vert * d.dxi[2] ** 2
        return out.reshape(-1)

    def resid(p):
        r = (div - apply_A(p)).reshape(sh)[I]
        r = r - r.mean(axis=(0, 1), keepdims=True)
        return np.linalg.norm(r) / np.linalg.norm(div.reshape(sh)[I])

    kx2, ky2 = port.modified_wave_numbers(d)
    a, c = port.off_diagonals(d, rho0)
    b = port.diagonal(d, rho0, rho0_half, kx2[:, None] + ky2[None, :])

    def solve32(rhs):
        D = rhs.reshape(sh)[I].astype(np.float32).astype(np.complex64)
        H = np.fft.fft(np.fft.fft(D, axis=0), axis=1).astype(np.complex64)
        with np.errstate(all="ignore"):
            xr = port.tdma(np.ascontiguousarray(H.real, dtype=np.float64), a, b, c).astype(np.float32)
            xi = port.tdma(np.ascontiguousarray(H.imag, dtype=np.float64), a, b, c).astype(np.float32)
        Z = (xr + 1j * xi).astype(np.complex64)
        Z[0, 0, :] = 0
        Z = np.fft.ifft(np.fft.ifft(Z, axis=1), axis=0).astype(np.complex64)
        P = np.zeros(sh)
        P[I] = Z.real
        return P.reshape(-1)

    p64 = np.zeros(d.npg)
    port.poisson_solve(d, rho0, rho0_half, div, p64)
    assert resid(p64) < 1e-14
    q = solve32(div)
    res = [resid(q)]
    for _ in range(2):
        q = q + solve32(div - apply_A(q))
        res.append(resid(q))
    assert 1e-9 < res[0] < 1e-5
    assert res[1] < 1e-12 and res[2] < 1e-14
    dq = (q - p64).reshape(sh)[I]
    dq -= dq.mean(axis=(0, 1), keepdims=True)
    assert np.linalg.norm(dq) / np.linalg.norm(p64.reshape(sh)[I]) < 1e-12


def test_graph_step_counts():
    """How many time steps one CUDA graph of the step holds (host logic, no
    GPU): 1 for the plain form, 2 for the fused precision form (its stages
    swap the two value buffers, three swaps a step), 1 with stable value
    addresses, and whole learned-seed refresh periods with the seed."""
    from pycles_b200.learned import SeedMLP
    from pycles_b200.simulation import CONFIGS, HotPathSimulation, namelist_for
    small = dict(CONFIGS["c2_bomex"], nx=16, ny=16, nz=12)
    plain = HotPathSimulation(namelist_for(**small, precision="fp64"), device="cpu")
    assert plain.graph_steps() == 1
    prec = HotPathSimulation(namelist_for(**small, precision="fp32"), device="cpu")
    assert prec.graph_steps() == 2
    prec.PV.stable_values = True
    assert prec.graph_steps() == 1
    prec.PV.stable_values = False
    prec.Th.mlp = SeedMLP(device="cpu")
    for every, steps in ((12, 4), (6, 2), (3, 2), (5, 10), (1, 2)):
        prec.Th.seed_refresh_interval = every
        assert prec.graph_steps() == steps, every
