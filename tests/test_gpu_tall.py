"""The subgrid-scale, diffusion, forcing and radiation kernels on a tall,
ragged grid (7 x 5 x 140 cells, gw 4: more than one 128-level block along
k, odd horizontal extents) against the oracle's restatement on the same
state (relative L2 1e-12, plain form)."""
import numpy as np
import pytest

from helpers import gpu_sim, gpu_tends, host_case, oracle_dims, oracle_sim, rel_l2

pytestmark = pytest.mark.gpu

TALL = dict(case="dycoms", nx=7, ny=5, nz=140, dx=35.0, dy=35.0, dz=8.0, gw=4, dt=0.25, scalar_order=7,
            momentum_order=5)


def _stirred():
    nl, rs, f = host_case(**TALL)
    rng = np.random.default_rng(9)
    f = dict(f)
    for n in ("u", "v", "w"):
        f[n] = f[n] + 0.5 * rng.standard_normal(f[n].shape)
    return nl, rs, f


def test_tall_grid_sgs_forcing_radiation():
    import torch

    from oracle.forcing import OracleForcing
    from oracle.radiation import OracleRadiation
    from oracle.sgs import OracleSGS, scheme_from_namelist
    from pycles_b200.grid import Grid
    nl, rs, f = _stirred()
    nl = dict(nl, meta={"casename": "DYCOMS_RF01"}, sgs={"scheme": "Smagorinsky"},
              diffusion={"qt_entropy_source": True})
    d = oracle_dims(nl)
    Gr = Grid(nl)
    o = oracle_sim(nl, rs, f)
    o.sgs = OracleSGS(scheme_from_namelist(nl), d, Gr.zl_half)
    o.forcing = OracleForcing("DYCOMS_RF01", d, rs["p0_half"], Gr.zl_half, u0=rs["u0"], v0=rs["v0"])
    o.radiation = OracleRadiation(d, Gr.z)
    g = gpu_sim(nl, rs, f)
    o.update_all_bcs()
    g.PV.Update_all_bcs(g.Gr)
    o.sgs.ke_update(o)
    o.th_update()
    g.Th.update(g.Gr, g.RS, g.PV, g.DV)
    o.sgs.sgs_update(o)
    g.SGS.update(g.Gr, g.DV, g.PV, g.Ke)
    torch.cuda.synchronize()
    sh = d.shape
    assert rel_l2(g.Ke.strain_rate_mag.cpu().numpy().reshape(sh)[2:], o.sgs.strain_rate_mag.reshape(sh)[2:]) < 1e-12
    errs = {}
    for name, upd_o, upd_g in (
            ("sd", o.sgs.sd_update, lambda: g.SD.update(g.Gr, g.RS, g.PV, g.DV)),
            ("md", o.sgs.md_update, lambda: g.MD.update(g.Gr, g.RS, g.PV, g.DV, g.Ke)),
            ("forcing", o.forcing.update, lambda: (g.Fo.initialize(g.Gr, g.RS), g.Fo.update(g.Gr, g.RS, g.PV, g.DV))),
            ("radiation", o.radiation.update, lambda: g.Ra.update(g.Gr, g.RS, g.PV, g.DV))):
        o.tendencies[:] = 0.0
        g.PV.tendencies.zero_()
        upd_o(o)
        upd_g()
        gt = gpu_tends(g)
        for k in o.names:
            ref = o.tend(k)
            if np.any(ref):
                errs[f"{name}_{k}"] = rel_l2(gt[k], ref)
            else:
                assert not np.any(gt[k]), (name, k)
    print({k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < 1e-12, k
