"""Subgrid scale and diffusion on the GPU (pb_kinematics_sgs,
pb_scalar_diffusion, pb_momentum_diffusion) against the fixtures generated
from the reference's own C (tests/golden/make_golden.py): Smagorinsky with
the grid, ILES and wall length scales (the last with the SullivanPatton
surface), UniformViscosity on the DYCOMS case with WENO7 scalars.

Tolerances (relative L2 per array): strain-rate magnitude, viscosity,
diffusivity (from the plane i = 2 on) and the diffusion tendencies 1e-12 in
the plain form and 1e-9 in the precision form (its thermodynamics, which
feeds the buoyancy frequency and the temperature, uses CUDA's exp/log); one
time step with the subgrid scale in the stage 1e-12 (plain) and 1e-6
(precision, unfused stepping).
"""
import os

import numpy as np
import pytest

from helpers import GOLDEN, gpu_dv, gpu_fields, gpu_sim, gpu_tends, rel_l2

pytestmark = pytest.mark.gpu

NAMES = ["sgs_smagorinsky_bomex", "sgs_smagorinsky_iles_bomex", "sgs_smagorinsky_wall_dry", "sgs_uniform_dycoms"]


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
def test_sgs_and_diffusion_vs_reference_golden(name, precision):
    import torch
    z, nl, rs, f, _ = _load(name)
    g = gpu_sim(nl, rs, f, precision=precision)
    assert g.SGS is not None
    g.PV.Update_all_bcs(g.Gr)
    g.Th.update(g.Gr, g.RS, g.PV, g.DV)
    g.SGS.update(g.Gr, g.DV, g.PV, g.Ke)
    torch.cuda.synchronize()
    sh = g.Gr.shape
    tol = 1e-12 if precision == "fp64" else 1e-9
    errs = {"strain_rate_mag": rel_l2(g.Ke.strain_rate_mag.cpu().numpy().reshape(sh)[2:],
                                      z["sgs_strain_rate_mag"].reshape(sh)[2:])}
    gd = gpu_dv(g)
    for n in ("viscosity", "diffusivity"):
        errs[n] = rel_l2(gd[n].reshape(sh)[2:], z["sgs_" + n].reshape(sh)[2:])
    g.PV.tendencies.zero_()
    g.SD.update(g.Gr, g.RS, g.PV, g.DV)
    gt = gpu_tends(g)
    for k in g.PV.index_name:
        if np.any(z["sdtend_" + k]):
            errs["sd_" + k] = rel_l2(gt[k], z["sdtend_" + k])
        else:
            assert not np.any(gt[k]), k
    g.PV.tendencies.zero_()
    g.MD.update(g.Gr, g.RS, g.PV, g.DV, g.Ke)
    gt = gpu_tends(g)
    for k in g.PV.index_name:
        if np.any(z["mdtend_" + k]):
            errs["md_" + k] = rel_l2(gt[k], z["mdtend_" + k])
        else:
            assert not np.any(gt[k]), k
    g.check_device_errors()
    print(name, precision, {k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < tol, k


@pytest.mark.parametrize("name", NAMES)
def test_sgs_step_vs_reference_golden(name):
    """One time step with Ke/SGS/SD/MD in the stage (Simulation3d.pyx:159-175)."""
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
