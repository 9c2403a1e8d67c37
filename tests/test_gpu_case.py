"""Whole cases on the GPU against the fixtures generated from the
reference's own C (tests/golden/make_golden.py): the case forcing
(pb_forcing_update) after the thermodynamics, and one time step with the
case's surface, forcing, radiation and subgrid scale in the stage (Bomex;
DYCOMS_RF01 with its radiation and Smagorinsky; SullivanPatton with the
wall-adjusted Smagorinsky).  Tolerances (relative L2): forcing tendencies 1e-12 (plain
form; the horizontal means of u and v are summed in another order) and 1e-9
(precision form); one step 1e-12 (plain) and 1e-6 (precision)."""
import os

import numpy as np
import pytest

from helpers import GOLDEN, gpu_fields, gpu_sim, gpu_tends, rel_l2

pytestmark = pytest.mark.gpu

NAMES = ["case_bomex", "case_dycoms_rf01", "case_sullivan_patton"]


def _load(name):
    from pycles_b200.simulation import namelist_for
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    cfg = eval(str(z["meta"][0]))  # dict literals written by make_golden.py
    extra = eval(str(z["meta"][1]))
    nl = dict(namelist_for(**cfg), **extra)
    rs = {k[3:]: z[k] for k in z.files if k.startswith("rs_")}
    f = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    f0 = {k[4:]: z[k] for k in z.files if k.startswith("in0_")}
    return z, nl, rs, f, f0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", NAMES)
def test_forcing_vs_reference_golden(name, precision):
    z, nl, rs, f, _ = _load(name)
    g = gpu_sim(nl, rs, f, precision=precision)
    assert g.Fo.scheme != 0
    g.PV.Update_all_bcs(g.Gr)
    g.Th.update(g.Gr, g.RS, g.PV, g.DV)
    g.PV.tendencies.zero_()
    g.Fo.initialize(g.Gr, g.RS)
    g.Fo.update(g.Gr, g.RS, g.PV, g.DV)
    gt = gpu_tends(g)
    tol = 1e-12 if precision == "fp64" else 1e-9
    errs = {}
    for k in g.PV.index_name:
        if np.any(z["fotend_" + k]):
            errs[k] = rel_l2(gt[k], z["fotend_" + k])
        else:
            assert not np.any(gt[k]), k
    print(name, precision, {k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < tol, k


@pytest.mark.parametrize("name", NAMES)
def test_case_step_vs_reference_golden(name):
    z, nl, rs, _, f0 = _load(name)
    for precision, tol in (("fp64", 1e-12), ("fp32", 1e-6)):
        g = gpu_sim(nl, rs, f0, precision=precision)
        assert not g._fused()
        g.PV.Update_all_bcs(g.Gr)
        g.step()
        g.check_device_errors()
        gf = gpu_fields(g)
        vel = np.sqrt(sum(np.linalg.norm(z["step_" + m]) ** 2 for m in ("u", "v", "w")))
        errs = {k: (np.linalg.norm(gf[k] - z["step_" + k]) / vel if k in ("u", "v", "w")
                    else rel_l2(gf[k], z["step_" + k])) for k in g.PV.index_name}
        print(name, precision, "step:", {k: f"{v:.1e}" for k, v in errs.items()})
        for k, v in errs.items():
            assert v < tol, (precision, k)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_dycoms_radiation_vs_reference_golden(precision):
    """RadiationDyCOMS_RF01 (Radiation.pyx:230-353) after the thermodynamics:
    heating rate, temperature tendency and entropy tendency (1e-12 plain,
    1e-9 precision form)."""
    z, nl, rs, f, _ = _load("case_dycoms_rf01")
    g = gpu_sim(nl, rs, f, precision=precision)
    assert g.Ra.active
    g.PV.Update_all_bcs(g.Gr)
    g.Th.update(g.Gr, g.RS, g.PV, g.DV)
    g.PV.tendencies.zero_()
    g.Ra.update(g.Gr, g.RS, g.PV, g.DV)
    tol = 1e-12 if precision == "fp64" else 1e-9
    errs = {"s_tend": rel_l2(gpu_tends(g)["s"], z["ratend_s"]),
            "heating_rate": rel_l2(g.Ra.heating_rate.cpu().numpy(), z["ra_heating_rate"]),
            "dTdt_rad": rel_l2(g.Ra.dTdt_rad.cpu().numpy(), z["ra_dTdt_rad"])}
    print(precision, {k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < tol, k
