"""The allocation-free pressure entry point, pb_pressure_solve_noalloc.

Some callers cannot allocate device memory (a loop that cannot afford the
device-wide synchronisation an allocation may bring, an allocator policy that
forbids late device allocations, a host binding without a device
allocator); this entry point serves them by using
a fixed 64 MiB device array inside the library instead of a workspace.  This
file runs last (pytest collects it last) and checks, through the C ABI, that
two calls in a row give what pb_pressure_solve gives with a caller
workspace, and that grids too large for the fixed array are refused.
"""
import ctypes

import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _inputs(nx, ny, nz, seed):
    import torch

    from pycles_b200.grid import Grid
    from pycles_b200.simulation import namelist_for
    from pycles_b200.thermodynamics import ThermodynamicsSA
    from pycles_b200.reference_state import ReferenceState
    Gr = Grid(namelist_for("bomex", nx, ny, nz, 100.0, 100.0, 40.0))
    RS = ReferenceState(Gr)
    RS.Pg, RS.Tg, RS.qtg = 1.015e5, 300.4, 0.02245
    RS.initialize(Gr, ThermodynamicsSA({}), device="cuda")
    rng = np.random.default_rng(seed)
    vel = [torch.as_tensor(rng.standard_normal(Gr.npg), device="cuda") for _ in range(3)]
    return Gr, RS, vel


def _solve(Gr, RS, vel, noalloc):
    import torch

    from pycles_b200 import _capi
    L = _capi.load()
    u, v, w = (x.clone() for x in vel)
    div = torch.zeros(Gr.npg, dtype=torch.float64, device="cuda")
    p = torch.zeros(Gr.npg, dtype=torch.float64, device="cuda")
    args = [ctypes.byref(Gr.dims)] + [RS.d_rho0.data_ptr(), RS.d_rho0_half.data_ptr(), RS.d_alpha0.data_ptr(),
                                      RS.d_alpha0_half.data_ptr(), u.data_ptr(), v.data_ptr(), w.data_ptr(),
                                      div.data_ptr(), p.data_ptr()]
    stream = torch.cuda.current_stream().cuda_stream
    if noalloc:
        fn = L.pb_pressure_solve_noalloc
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.c_void_p] * 11
        rc = fn(*args, stream)
    else:
        nbytes = L.pb_pressure_workspace_bytes(ctypes.byref(Gr.dims))
        ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        _capi.check(L.pb_pressure_init(ctypes.byref(Gr.dims), ws.data_ptr(), nbytes), "pb_pressure_init")
        rc = L.pb_pressure_solve(*args, ws.data_ptr(), nbytes, 0, 0, stream)
    torch.cuda.synchronize()
    return rc, {n: t.cpu().numpy() for n, t in zip(("u", "v", "w", "div", "p"), (u, v, w, div, p))}


def test_noalloc_matches_workspace_entry_point_twice():
    from pycles_b200 import _capi
    Gr, RS, vel = _inputs(32, 24, 20, seed=5)
    rc, ref = _solve(Gr, RS, vel, noalloc=False)
    _capi.check(rc, "pb_pressure_solve")
    for call in range(2):  # the second call reuses the array the first one left behind
        rc, out = _solve(Gr, RS, vel, noalloc=True)
        _capi.check(rc, f"pb_pressure_solve_noalloc (call {call + 1})")
        for n in ref:
            assert rel_l2(out[n], ref[n]) <= 1e-12, (call, n)


def test_noalloc_alternating_grids_on_a_non_blocking_stream():
    """Two grids in turn on one non-blocking stream with no host sync between
    the calls: each grid change rewrites the shared constants, which must not
    reach a solve of the other grid still queued on the stream."""
    import torch

    from pycles_b200 import _capi
    L = _capi.load()
    fn = L.pb_pressure_solve_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p] * 11
    grids = [_inputs(32, 24, 20, seed=7), _inputs(64, 32, 16, seed=8)]
    refs = []
    for Gr, RS, vel in grids:
        rc, ref = _solve(Gr, RS, vel, noalloc=False)
        _capi.check(rc, "pb_pressure_solve")
        refs.append(ref)
    st = torch.cuda.Stream()
    assert st.cuda_stream != 0
    outs = []
    with torch.cuda.stream(st):
        for rnd in range(3):
            for Gr, RS, vel in grids:
                u, v, w = (x.clone() for x in vel)
                div = torch.zeros(Gr.npg, dtype=torch.float64, device="cuda")
                p = torch.zeros(Gr.npg, dtype=torch.float64, device="cuda")
                rc = fn(ctypes.byref(Gr.dims), RS.d_rho0.data_ptr(), RS.d_rho0_half.data_ptr(),
                        RS.d_alpha0.data_ptr(), RS.d_alpha0_half.data_ptr(), u.data_ptr(), v.data_ptr(),
                        w.data_ptr(), div.data_ptr(), p.data_ptr(), st.cuda_stream)
                _capi.check(rc, "pb_pressure_solve_noalloc")
                outs.append((u, v, w, div, p))
    st.synchronize()
    for idx, tensors in enumerate(outs):
        ref = refs[idx % 2]
        for n, t in zip(("u", "v", "w", "div", "p"), tensors):
            assert rel_l2(t.cpu().numpy(), ref[n]) <= 1e-12, (idx, n)


def test_noalloc_rejects_grids_beyond_its_array():
    from pycles_b200 import _capi
    from pycles_b200.grid import Grid
    from pycles_b200.simulation import namelist_for
    Gr = Grid(namelist_for("bomex", 256, 256, 128, 50.0, 50.0, 20.0))
    L = _capi.load()
    assert L.pb_pressure_workspace_bytes(ctypes.byref(Gr.dims)) > (64 << 20)
    fn = L.pb_pressure_solve_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p] * 11
    p = ctypes.c_void_p(256)  # never dereferenced: the size check comes first
    assert fn(ctypes.byref(Gr.dims), p, p, p, p, p, p, p, p, p, None) == _capi.PB_ERR_WORKSPACE
