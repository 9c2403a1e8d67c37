"""Whole time steps recorded as one CUDA graph (HotPathSimulation.capture_steps)
and replayed give the eager steps' state bit for bit: the FP64 plain form
(no buffer swaps), the precision form (fused stages swap the two value
buffers: an even number of steps per graph) and the precision form with the
learned seed (a whole number of refresh periods per graph), on a moist
32 x 32 x 24 grid (TMA momentum planes)."""
import numpy as np
import pytest
import torch

from helpers import gpu_sim, host_case

pytestmark = pytest.mark.gpu

MOIST = dict(case="bomex", nx=32, ny=32, nz=24, dx=100.0, dy=100.0, dz=40.0, gw=4, dt=1.0,
             scalar_order=7, momentum_order=5)


@pytest.mark.parametrize("form", ["fp64", "fp32", "fp32+learned"])
def test_graph_replay_equals_eager_steps(form):
    from pycles_b200.learned import SeedMLP
    nl, rs, f = host_case(**MOIST)
    precision = "fp64" if form == "fp64" else "fp32"
    a, b = gpu_sim(nl, rs, f, precision=precision), gpu_sim(nl, rs, f, precision=precision)
    if form == "fp32+learned":
        mlp = SeedMLP(seed=3, out_mean=1.5, out_scale=2.0)
        a.Th.mlp = b.Th.mlp = mlp
    for g in (a, b):
        g.PV.Update_all_bcs(g.Gr)
        g.Th.update(g.Gr, g.RS, g.PV, g.DV)
    b.step()  # eagerly once: the lazily made buffers exist
    n = b.graph_steps()
    assert n == {"fp64": 1, "fp32": 2, "fp32+learned": 4}[form]
    graph = b.capture_steps()
    for _ in range(2):
        graph.replay()
    for _ in range(1 + 2 * n):
        a.step()
    torch.cuda.synchronize()
    assert torch.equal(a.PV.values, b.PV.values), form
    for name in ("temperature", "ql", "buoyancy"):
        assert torch.equal(a.DV.field(name, a.Gr), b.DV.field(name, b.Gr)), (form, name)
    assert np.isfinite(a.PV.values.cpu().numpy()).all()
    a.check_device_errors()
    b.check_device_errors()


def test_graph_step_counts_are_checked():
    nl, rs, f = host_case(**MOIST)
    g = gpu_sim(nl, rs, f, precision="fp32")
    with pytest.raises(RuntimeError):
        g.capture_steps()  # no eager step yet
    g.PV.Update_all_bcs(g.Gr)
    g.step()
    with pytest.raises(ValueError):
        g.capture_steps(3)  # the fused stages need an even count
