"""Horizontal statistics on the GPU (pb_horizontal_stat) against the
oracle's restatement of ParallelMPI's loops (sequential order,
ParallelMPI.pyx:196-540).  Sums: 1e-13 relative L2 (a fixed parallel order
against the sequential one); maximum and minimum: exact."""
import numpy as np
import pytest

from helpers import host_case, oracle_dims, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg", [dict(case="bomex", nx=12, ny=10, nz=16), dict(case="bomex", nx=37, ny=29, nz=9)],
                         ids=["small", "ragged"])
def test_horizontal_statistics(cfg):
    import torch

    from oracle import port
    from pycles_b200.grid import Grid
    from pycles_b200.statistics import HorizontalStatistics
    nl, rs, f = host_case(**cfg)
    d = oracle_dims(nl)
    rng = np.random.default_rng(3)
    a, b, c = f["s"], f["qt"] + 1e-3 * rng.standard_normal(d.npg), rng.standard_normal(d.npg)
    mask = (rng.random(d.npg) < 0.3).astype(np.float64)
    plane = rng.standard_normal(d.nlg[0] * d.nlg[1])
    Gr = Grid(nl)
    st = HorizontalStatistics(Gr)
    T = lambda x: torch.as_tensor(x, device="cuda")
    cases = {
        "mean": (st.HorizontalMean(Gr, T(a)), port.horizontal_stat(d, "mean", a)),
        "squares": (st.HorizontalMeanofSquares(Gr, T(a), T(b)), port.horizontal_stat(d, "squares", a, b)),
        "cubes": (st.HorizontalMeanofCubes(Gr, T(a), T(b), T(c)), port.horizontal_stat(d, "cubes", a, b, c)),
        "max": (st.HorizontalMaximum(Gr, T(c)), port.horizontal_stat(d, "max", c)),
        "min": (st.HorizontalMinimum(Gr, T(c)), port.horizontal_stat(d, "min", c)),
        "conditional": (st.HorizontalMeanConditional(Gr, T(b), T(mask)),
                        port.horizontal_stat(d, "conditional", b, mask=mask)),
        "squares_conditional": (st.HorizontalMeanofSquaresConditional(Gr, T(a), T(c), T(mask)),
                                port.horizontal_stat(d, "squares_conditional", a, c, mask=mask)),
    }
    for k, (g, o) in cases.items():
        g = g.cpu().numpy()
        assert g.shape == (d.nlg[2],), k
        if k in ("max", "min"):
            assert np.array_equal(g, o), k
        else:
            assert rel_l2(g, o) < 1e-13, k
    s = st.HorizontalMeanSurface(Gr, T(plane))
    assert abs(s - port.horizontal_stat(d, "surface", plane)) <= 1e-13 * np.abs(plane).max()
    # an all-zero mask gives 0 (the reference divides by max(sum, 1))
    z = st.HorizontalMeanConditional(Gr, T(b), T(np.zeros(d.npg))).cpu().numpy()
    assert not np.any(z)
