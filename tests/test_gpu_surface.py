"""Surface fluxes on the GPU (pb_surface_update) against the fixtures
generated from the reference's own C (tests/golden/make_golden.py):
SullivanPatton (dry), Bomex and DYCOMS_RF01, each on its case.

Tolerances (relative L2 per array): fluxes and first-level tendencies 1e-12
in the plain form (the lowest-level temperature mean is summed in a
different order, pow and atan are CUDA's), 1e-9 in the precision form
(its thermodynamics uses CUDA's exp/log); one time step with the scheme in
the stage 1e-12 (plain form) and 1e-6 (precision form, unfused stepping).
"""
import os

import numpy as np
import pytest

from helpers import GOLDEN, gpu_fields, gpu_sim, gpu_tends, rel_l2

pytestmark = pytest.mark.gpu

NAMES = ["surface_sullivan_patton", "surface_bomex", "surface_dycoms_rf01"]


def _load(name):
    from pycles_b200.simulation import namelist_for
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    cfg = eval(str(z["meta"][0]))  # dict literal written by make_golden.py
    nl = namelist_for(**cfg)
    nl["meta"] = {"casename": str(z["meta"][1])}
    rs = {k[3:]: z[k] for k in z.files if k.startswith("rs_")}
    f = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    f0 = {k[4:]: z[k] for k in z.files if k.startswith("in0_")}
    return z, nl, rs, f, f0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", NAMES)
def test_surface_update_vs_reference_golden(name, precision):
    import torch
    z, nl, rs, f, _ = _load(name)
    g = gpu_sim(nl, rs, f, precision=precision)
    assert g.Sur.scheme != 0
    g.PV.Update_all_bcs(g.Gr)
    g.Th.update(g.Gr, g.RS, g.PV, g.DV)
    g.PV.tendencies.zero_()
    g.Sur.update(g.Gr, g.RS, g.PV, g.DV)
    torch.cuda.synchronize()
    g.check_device_errors()
    tol = 1e-12 if precision == "fp64" else 1e-9
    errs = {}
    for n in ("u_flux", "v_flux", "qt_flux", "s_flux", "obukhov_length", "friction_velocity", "shf", "lhf",
              "b_flux", "windspeed"):
        a = g.Sur.fields[n].cpu().numpy()
        errs[n] = rel_l2(a, z["sur_" + n])
        assert np.isfinite(a).all(), n
    gt = gpu_tends(g)
    for k in g.PV.index_name:
        errs["tend_" + k] = rel_l2(gt[k], z["surtend_" + k])
    print(name, precision, {k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < tol, k


@pytest.mark.parametrize("name", NAMES)
def test_surface_step_vs_reference_golden(name):
    """One time step with the scheme (and the case's forcing, which the case
    name selects as well) between the advection and the SSP-RK3 stage
    (Simulation3d.pyx:165-175)."""
    z, nl, rs, _, f0 = _load(name)
    for precision, tol in (("fp64", 1e-12), ("fp32", 1e-6)):
        g = gpu_sim(nl, rs, f0, precision=precision)
        assert not g._fused()  # the surface sits between the advection and the stage
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
