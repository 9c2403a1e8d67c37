"""GPU path against the golden fixtures generated from the reference's own
C kernels (tests/golden/make_golden.py): the same seeded inputs, one call of
each component and one full time step.  Plain FP64 form.

Tolerances (relative L2 per field): advection tendencies bit-identical;
1e-12 for fields after a full step and for pressure-corrected velocities;
1e-10 for fields formed by cancellation (buoyancy) or vertical differences
(bvf)."""
import os

import numpy as np
import pytest

from helpers import GOLDEN, gpu_dv, gpu_fields, gpu_sim, gpu_tends, rel_l2

pytestmark = pytest.mark.gpu

NAMES = ["moist_w5", "moist_w7", "dry_w5"]


def _load(name):
    from pycles_b200.simulation import namelist_for
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    cfg = eval(str(z["meta"][0]))  # dict literal written by make_golden.py
    nl = namelist_for(**cfg)
    rs = {k[3:]: z[k] for k in z.files if k.startswith("rs_")}
    f = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    f0 = {k[4:]: z[k] for k in z.files if k.startswith("in0_")}
    return z, nl, rs, f, f0


def _sim(nl, rs, f):
    g = gpu_sim(nl, rs, f)
    g.PV.Update_all_bcs(g.Gr)
    return g


@pytest.mark.parametrize("name", NAMES)
def test_components_vs_reference_golden(name):
    z, nl, rs, f, _ = _load(name)
    g = _sim(nl, rs, f)
    gf = gpu_fields(g)
    for k in g.PV.index_name:
        assert np.array_equal(gf[k], z["bcs_" + k]), k
    g.Th.update(g.Gr, g.RS, g.PV, g.DV)
    gd = gpu_dv(g)
    print(name, "thermodynamics rel L2:",
          {k: rel_l2(gd[k], z["th_" + k]) for k in g.DV.index_name if "th_" + k in z.files})
    for k in g.DV.index_name:
        if "th_" + k not in z.files:
            continue
        tol = 1e-10 if k in ("buoyancy", "buoyancy_frequency") else 1e-12
        assert rel_l2(gd[k], z["th_" + k]) < tol, k
    g = _sim(nl, rs, f)
    g.SA.update(g.Gr, g.RS, g.PV, g.DV)
    g.MA.update(g.Gr, g.RS, g.PV)
    gt = gpu_tends(g)
    for k in g.PV.index_name[3:]:
        assert np.array_equal(gt[k], z["sa_" + k]), k
    for k in ("u", "v", "w"):
        assert np.array_equal(gt[k], z["ma_" + k]), k
    g = _sim(nl, rs, f)
    g.Pr.update(g.Gr, g.RS, g.DV, g.PV)
    gf, gd = gpu_fields(g), gpu_dv(g)
    print(name, "pressure rel L2: div", rel_l2(gd["divergence"], z["pr_div"]),
          "p", rel_l2(gd["dynamic_pressure"], z["pr_p"]),
          {k: rel_l2(gf[k], z["pr_" + k]) for k in ("u", "v", "w")})
    assert rel_l2(gd["divergence"], z["pr_div"]) < 1e-12
    assert rel_l2(gd["dynamic_pressure"], z["pr_p"]) < 1e-11
    for k in ("u", "v", "w"):
        assert rel_l2(gf[k], z["pr_" + k]) < 1e-12, k


@pytest.mark.parametrize("name", NAMES)
def test_one_step_vs_reference_golden(name):
    """Plain-form gate against the reference itself: <= 1e-12 per field."""
    z, nl, rs, _, f0 = _load(name)
    g = _sim(nl, rs, f0)
    g.step()
    gf = gpu_fields(g)
    print(name, "one step rel L2:", {k: rel_l2(gf[k], z["step_" + k]) for k in g.PV.index_name})
    for k in g.PV.index_name:
        assert rel_l2(gf[k], z["step_" + k]) < 1e-12, k
    g = gpu_sim(nl, rs, f0)
    g.run(1)
    gf = gpu_fields(g)
    for k in g.PV.index_name:
        assert rel_l2(gf[k], z["run1_" + k]) < 1e-12, k
