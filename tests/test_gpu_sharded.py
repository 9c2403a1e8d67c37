"""The hot path over x-slabs (pycles_b200.parallel) on one GPU: 1, 2 and 4
ranks run in one process (LocalComm), each rank's kernels on its own slab,
the collectives as copies between the ranks' tensors -- the same phase entry
points, transposes and halo exchanges a multi-GPU run issues, against the
one-GPU hot path from the same state.

Tolerances (relative L2 per field, three time steps from the seeded state;
the buoyancy of its perturbations drives a divergent flow that the pressure
solve removes): one rank reproduces the
one-GPU plain form bit for bit (the same kernels on the same values); with
several ranks the horizontal mean of w adds the ranks' sums, as the
reference's MPI_Allreduce does (ParallelMPI.pyx:229-230), which moves the
velocities at the rounding level: <= 1e-11 (plain form) and <= 1e-9
(precision form, whose one-GPU mean is a parallel sum).
"""
import numpy as np
import pytest

from helpers import gpu_fields, gpu_sim, host_case, rel_l2

pytestmark = pytest.mark.gpu

CFG = dict(case="bomex", nx=32, ny=16, nz=24, dx=100.0, dy=100.0, dz=40.0, gw=3, dt=1.0)


@pytest.mark.parametrize("world", [1, 2, 4])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_sharded_steps_match_one_gpu(world, precision):
    from pycles_b200 import _capi, parallel
    nl, rs, f = host_case(**CFG)
    _capi.clear_error()
    one = gpu_sim(nl, rs, f, precision=precision)
    one.run(3)
    one.check_device_errors()
    ref = gpu_fields(one)
    nl2 = dict(nl, gpu=dict(nl.get("gpu", {}), precision=precision))
    sh = parallel.ShardedSimulation(nl2, parallel.LocalComm(world), ["cuda"] * world)
    sh.load_global(rs, f)
    sh.run(3)
    for s in sh.sims:
        s.check_device_errors()
    gw = CFG["gw"]
    shape = one.Gr.shape
    errs = {}
    for n in ref:
        a = sh.gather_global(n)
        b = ref[n].reshape(shape)[gw:-gw]
        assert np.isfinite(a).all(), n
        errs[n] = rel_l2(a, b)
        if world == 1 and precision == "fp64":
            assert np.array_equal(a, b), n
    assert np.abs(sh.sims[0].DV.field("dynamic_pressure", sh.sims[0].Gr).cpu().numpy()).max() > 0
    print(world, precision, {k: f"{v:.1e}" for k, v in errs.items()})
    tol = 1e-11 if precision == "fp64" else 1e-9
    for n, v in errs.items():
        assert v < tol, n
