"""The multi-GPU decomposition's host logic on the CPU: x-slabs with halo
exchanges and the pressure's transposes reproduce the one-rank layout
exactly.

* world_size-2 gloo process groups on 127.0.0.1 (DistComm: the same
  torch.distributed calls as NCCL between GPUs);
* LocalComm (every rank in one process) for 1, 2 and 4 ranks; a grid that
  does not divide into the slabs is refused.

The reference: halo exchange PrognosticVariables.pyx:199-233 (MPI_Sendrecv),
transposes ParallelMPI.pyx:542-1068 (MPI_Alltoallv).  The ghost fill of a
slab and of the whole domain is the oracle's restatement of
update_all_bcs; every comparison is bit for bit.
"""
import os
import sys

import numpy as np
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

N, GW, NV = (8, 6, 4), 2, 3
BC = np.array([1.0, 1.0, -1.0])


def _global_fields(seed=0):
    """Ghosted fields of the whole domain, ghosts filled as on one rank."""
    from oracle import port
    from oracle.dims import Dims
    d = Dims(N, GW, (1.0, 1.0, 1.0))
    rng = np.random.default_rng(seed)
    vals = rng.standard_normal(NV * d.npg)
    port.update_all_bcs(d, vals, BC)
    return d, vals.reshape(NV, *d.nlg)


def _slab_after_exchange(comm, ranks, world):
    """Each rank's slab, its x-ghosts spoiled, filled locally, then
    exchanged."""
    from oracle import port
    from oracle.dims import Dims
    from pycles_b200 import parallel
    _, G = _global_fields()
    sl = parallel.Slabs(*N, world)
    ds = Dims((sl.nxl, N[1], N[2]), GW, (1.0, 1.0, 1.0))
    fields, refs = [], []
    for r in ranks:
        x0 = sl.x0(r)
        ref = G[:, x0:x0 + sl.nxl + 2 * GW].copy()
        s = ref.copy()
        s[:, :GW] = np.nan
        s[:, -GW:] = np.nan
        flat = s.reshape(-1)
        port.update_all_bcs(ds, flat, BC)  # y and z ghosts; x-ghosts from the slab itself
        fields.append(torch.tensor(flat))
        refs.append(ref)
    parallel.exchange_x_halos(comm, fields, NV, ds.nlg, GW)
    return [f.numpy().reshape(refs[0].shape) for f in fields], refs


def _transposes(comm, ranks, world):
    from pycles_b200 import parallel
    sl = parallel.Slabs(*N, world)
    rng = np.random.default_rng(1)
    D = torch.tensor(rng.standard_normal(N))
    dense_x = [D[sl.x0(r):sl.x0(r) + sl.nxl].clone() for r in ranks]
    dz = parallel.x_to_z(comm, sl, dense_x)
    for r, z in zip(ranks, dz):
        assert torch.equal(z, D[:, :, sl.z0(r):sl.z0(r) + sl.nzl]), r
    back = parallel.z_to_x(comm, sl, dz)
    for a, b in zip(back, dense_x):
        assert torch.equal(a, b)
    nh = N[0] // 2 + 1
    W = torch.tensor(rng.standard_normal((N[2], N[1], nh, 2)), dtype=torch.float32)
    wz = [W[sl.z0(r):sl.z0(r) + sl.nzl].clone() for r in ranks]
    rows = parallel.z_to_rows(comm, sl, wz)
    for r, w in zip(ranks, rows):
        assert torch.equal(w, W[:, sl.y0(r):sl.y0(r) + sl.nyl]), r
    back = parallel.rows_to_z(comm, sl, rows)
    for a, b in zip(back, wz):
        assert torch.equal(a, b)
    sums = comm.allreduce_sum([torch.full((4,), float(r + 1), dtype=torch.float64) for r in ranks])
    for s in sums:
        assert torch.equal(s, torch.full((4,), float(sum(range(1, world + 1))), dtype=torch.float64))


def _worker(rank, world, port):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pycles_b200 import parallel
        comm = parallel.DistComm()
        got, ref = _slab_after_exchange(comm, comm.ranks, world)
        assert np.array_equal(got[0], ref[0]), rank
        _transposes(comm, comm.ranks, world)
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_slabs_gloo_world2():
    mp.start_processes(_worker, args=(2, _free_port()), nprocs=2, join=True, start_method="spawn")


def test_slabs_local_comm_1_and_2_ranks():
    from pycles_b200 import parallel
    for world in (1, 2):
        comm = parallel.LocalComm(world)
        got, ref = _slab_after_exchange(comm, comm.ranks, world)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
        _transposes(comm, comm.ranks, world)


def test_slabs_reject_uneven_splits():
    import pytest

    from pycles_b200 import parallel
    with pytest.raises(ValueError):
        parallel.Slabs(8, 6, 4, 3)


def test_slabs_local_comm_4_ranks():
    """4 slabs of a 16 x 8 x 8 domain (gw 2): halos and transposes."""
    global N
    saved = N
    N = (16, 8, 8)
    try:
        from pycles_b200 import parallel
        comm = parallel.LocalComm(4)
        got, ref = _slab_after_exchange(comm, comm.ranks, 4)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
        _transposes(comm, comm.ranks, 4)
    finally:
        N = saved
