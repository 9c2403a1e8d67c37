"""The hot path on several GPUs: the domain in x-slabs, full y and z columns
on every GPU.

The reference decomposes the domain over MPI ranks (ParallelMPI.pyx:20-160),
fills the halos between ranks with MPI_Sendrecv (PrognosticVariables.pyx:
199-233, build_buffer/buffer_to_values in Csrc/prognostic_variables.h) and
moves the pressure's spectral data between pencils with MPI_Alltoallv
(ParallelMPI.pyx:542-1068, PressureFFTParallel.pyx:150-219).  Here:

* the prognostic fields of a GPU are the ghosted arrays of its x-slab; every
  stencil component runs unchanged on them once the x-ghost planes hold the
  neighbours' edge planes (``exchange_x_halos``: the local ghost fill gives
  the y and z ghosts, then the gw interior planes at each x edge go to the
  neighbour, which stores them as its x-ghost planes; every ghost cell ends
  as the one-GPU ghost fill leaves it);
* the pressure solve (``ShardedPressure``) runs the library's phase entry
  points with three all-to-all transposes around them: x-slab -> z-slab (the
  horizontal FFTs need whole planes), z-slab -> row slab (the Thomas solves
  need whole columns) and back, each a single all-to-all of equal blocks;
  the horizontal mean of w adds the GPUs' per-level sums.

Communication goes through a communicator with two implementations that
take per-rank lists, so that the driver is one code path: ``DistComm``
(torch.distributed: NCCL between GPUs, gloo between CPU processes; one rank
per process) and ``LocalComm`` (all ranks in this process, one after the
other: the CPU tests and a one-GPU rehearsal of N GPUs).  Remote data always
lands in local memory before a kernel reads it.
"""
from __future__ import annotations

import copy
import ctypes

import numpy as np
import torch

from . import _capi


class Slabs:
    """x-slabs of nx/N columns; the pressure's z-slabs of nz/N levels and row
    slabs of ny/N rows.  The three extents must divide by the GPU count."""

    def __init__(self, nx, ny, nz, world):
        for name, n in (("nx", nx), ("ny", ny), ("nz", nz)):
            if n % world:
                raise ValueError(f"{name} = {n} does not divide into {world} slabs")
        self.nx, self.ny, self.nz, self.world = nx, ny, nz, world
        self.nxl, self.nyl, self.nzl = nx // world, ny // world, nz // world

    def x0(self, r):
        return r * self.nxl

    def y0(self, r):
        return r * self.nyl

    def z0(self, r):
        return r * self.nzl


def slab_dims(n, gw, dx, indx_lo=(0, 0, 0)):
    """pb_dims of one GPU's grid: n the local extents (nl == n, as the
    library's calls take them), dx the spacings, indx_lo the global offset."""
    d = _capi.PbDims()
    d.dims = 3
    d.gw = gw
    for i in range(3):
        d.n[i] = int(n[i])
        d.nl[i] = int(n[i])
        d.ng[i] = d.n[i] + 2 * gw
        d.nlg[i] = d.nl[i] + 2 * gw
        d.indx_lo[i] = int(indx_lo[i])
        d.indx_lo_g[i] = int(indx_lo[i])
        d.dx[i] = float(dx[i])
        d.dxi[i] = 1.0 / d.dx[i]
    d.npd = d.n[0] * d.n[1] * d.n[2]
    d.npl = d.npd
    d.npg = d.nlg[0] * d.nlg[1] * d.nlg[2]
    for i, (a, b) in enumerate(((1, 2), (0, 2), (0, 1))):
        d.nbuffer[i] = gw * max(d.nlg[a] * d.nlg[b], d.nlg[a], d.nlg[b])
    d.ghosted_stride[0] = d.nlg[1] * d.nlg[2]
    d.ghosted_stride[1] = d.nlg[0]
    d.ghosted_stride[2] = 1
    return d


# ---------------------------------------------------------------------------
# communicators
# ---------------------------------------------------------------------------
class LocalComm:
    """Every rank in this process.  Collectives are copies between the
    ranks' tensors; sums add the ranks' terms in rank order."""

    def __init__(self, world):
        self.world = world
        self.ranks = list(range(world))

    def alltoall(self, sends):
        """sends[i][q]: rank i's block for rank q -> recv[q][i]."""
        return [[sends[i][q].clone() for i in range(self.world)] for q in range(self.world)]

    def allreduce_sum(self, ts):
        s = ts[0].clone()
        for t in ts[1:]:
            s += t.to(s.device)
        return [s.to(t.device) for t in ts]

    def sendrecv_x(self, to_left, to_right):
        """Rank r sends to_left[r] to rank r-1 and to_right[r] to rank r+1
        (periodic); returns (from_right, from_left) per rank."""
        w = self.world
        from_right = [to_left[(r + 1) % w].to(to_left[r].device) for r in range(w)]
        from_left = [to_right[(r - 1) % w].to(to_right[r].device) for r in range(w)]
        return from_right, from_left


class DistComm:
    """One rank per process through torch.distributed (NCCL between GPUs,
    gloo between CPU processes).  Blocks of an all-to-all have equal sizes
    (the slabs divide evenly), so one all_to_all_single moves them."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.ranks = [self.rank]

    def alltoall(self, sends):
        blocks = sends[0]
        n = blocks[0].numel()
        if any(b.numel() != n for b in blocks):
            raise ValueError("all-to-all blocks must have equal sizes")
        inp = torch.cat([b.reshape(-1) for b in blocks])
        out = torch.empty_like(inp)
        self.dist.all_to_all_single(out, inp, group=self.group)
        return [[out[q * n:(q + 1) * n].view(blocks[q].shape) for q in range(self.world)]]

    def allreduce_sum(self, ts):
        t = ts[0].clone()
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return [t]

    def sendrecv_x(self, to_left, to_right):
        if self.world == 1:
            return [to_left[0].clone()], [to_right[0].clone()]
        dist = self.dist
        left = (self.rank - 1) % self.world
        right = (self.rank + 1) % self.world
        from_right = torch.empty_like(to_left[0])
        from_left = torch.empty_like(to_right[0])
        gl = dist.get_global_rank(self.group, left) if self.group is not None else left
        gr = dist.get_global_rank(self.group, right) if self.group is not None else right
        ops = [dist.P2POp(dist.isend, to_left[0], gl, self.group), dist.P2POp(dist.isend, to_right[0], gr, self.group),
               dist.P2POp(dist.irecv, from_right, gr, self.group), dist.P2POp(dist.irecv, from_left, gl, self.group)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        return [from_right], [from_left]


# ---------------------------------------------------------------------------
# halo exchange and transposes
# ---------------------------------------------------------------------------
def exchange_x_halos(comm, fields, nv, nlg, gw):
    """The x-ghost planes of every rank's ghosted fields (flat [v][i][j][k]
    tensors of nv variables, extents nlg) from its neighbours' edge planes:
    the first gw interior planes go to the left neighbour's right ghosts,
    the last gw to the right neighbour's left ghosts.  The local ghost fill
    runs first, so the planes carry their y and z ghosts."""
    n0, plane = int(nlg[0]), int(nlg[1]) * int(nlg[2])
    views = [f.view(nv, n0, plane) for f in fields]
    to_left = [v[:, gw:2 * gw].contiguous() for v in views]
    to_right = [v[:, n0 - 2 * gw:n0 - gw].contiguous() for v in views]
    from_right, from_left = comm.sendrecv_x(to_left, to_right)
    for v, fr, fl in zip(views, from_right, from_left):
        v[:, n0 - gw:] = fr
        v[:, :gw] = fl


def x_to_z(comm, sl, dense):
    """Dense x-slabs (nxl, ny, nz) -> dense z-slabs (nx, ny, nzl)."""
    nzl = sl.nzl
    sends = [[d[:, :, q * nzl:(q + 1) * nzl].contiguous() for q in range(sl.world)] for d in dense]
    recv = comm.alltoall(sends)
    return [torch.cat(blocks, dim=0) for blocks in recv]


def z_to_x(comm, sl, dense):
    """Dense z-slabs (nx, ny, nzl) -> dense x-slabs (nxl, ny, nz)."""
    nxl = sl.nxl
    sends = [[d[q * nxl:(q + 1) * nxl] for q in range(sl.world)] for d in dense]
    recv = comm.alltoall(sends)
    return [torch.cat(blocks, dim=2) for blocks in recv]


def z_to_rows(comm, sl, spec):
    """Spectra of z-slabs (nzl, ny, nh, 2) -> row slabs (nz, nyl, nh, 2)."""
    nyl = sl.nyl
    sends = [[w[:, q * nyl:(q + 1) * nyl].contiguous() for q in range(sl.world)] for w in spec]
    recv = comm.alltoall(sends)
    return [torch.cat(blocks, dim=0) for blocks in recv]


def rows_to_z(comm, sl, spec):
    """Spectra of row slabs (nz, nyl, nh, 2) -> z-slabs (nzl, ny, nh, 2)."""
    nzl = sl.nzl
    sends = [[w[q * nzl:(q + 1) * nzl] for q in range(sl.world)] for w in spec]
    recv = comm.alltoall(sends)
    return [torch.cat(blocks, dim=1) for blocks in recv]


# ---------------------------------------------------------------------------
# the sharded pressure solve
# ---------------------------------------------------------------------------
class ShardedPressure:
    """PressureSolver.update (PressureSolver.pyx:38-80) of a domain in
    x-slabs: the library's phase entry points between transposes; the
    precision form's refinement sweeps (no counterpart in the reference)
    repeat the solve on the residual and add the correction."""

    def __init__(self, comm, sl, gw, dx, precision, refine_sweeps, devices):
        self.comm, self.sl, self.gw, self.precision = comm, sl, gw, precision
        self.refine_sweeps = refine_sweeps if precision == _capi.PB_FP32 else 0
        L = _capi.load()
        self.L = L
        self.dims_x = slab_dims((sl.nxl, sl.ny, sl.nz), gw, dx)
        self.dims_rows = slab_dims((sl.nx, sl.nyl, sl.nz), gw, dx)
        self.dims_z, self.ws, self.spec_z, self.spec_rows, self.scratch = [], [], [], [], []
        self.cdtype = torch.float64 if precision == _capi.PB_FP64 else torch.float32
        nh = sl.nx // 2 + 1
        self.nh = nh
        for i, r in enumerate(comm.ranks):
            dz = slab_dims((sl.nx, sl.ny, sl.nzl), gw, dx, (0, 0, sl.z0(r)))
            nbytes = L.pb_pressure_workspace_bytes(ctypes.byref(dz))
            ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=devices[i])
            off = (-ws.data_ptr()) % 256
            ws = ws[off:off + nbytes]
            _capi.check(L.pb_pressure_init(ctypes.byref(dz), ws.data_ptr(), nbytes), "pb_pressure_init")
            so = L.pb_pressure_spectral_offset(ctypes.byref(dz))
            esz = 8 if self.cdtype == torch.float64 else 4
            sbytes = sl.nzl * sl.ny * nh * 2 * esz
            self.dims_z.append(dz)
            self.ws.append(ws)
            self.spec_z.append(ws[so:so + sbytes].view(self.cdtype).view(sl.nzl, sl.ny, nh, 2))
            self.spec_rows.append(torch.empty((sl.nz, sl.nyl, nh, 2), dtype=self.cdtype, device=devices[i]))
            self.scratch.append(torch.empty(sl.nz * sl.nyl * nh, dtype=torch.float64, device=devices[i]))

    def _solve(self, rhs_x, RS, streams):
        """The spectral solve of dense x-slab right-hand sides -> dense
        x-slab solutions."""
        sl, L = self.sl, self.L
        rhs_z = x_to_z(self.comm, sl, rhs_x)
        for i, r in enumerate(self.comm.ranks):
            _capi.check(L.pb_pressure_fft_forward(ctypes.byref(self.dims_z[i]), self.ws[i].data_ptr(),
                                                  self.ws[i].numel(), rhs_z[i].data_ptr(), self.precision,
                                                  streams[i]), "pb_pressure_fft_forward")
        rows = z_to_rows(self.comm, sl, self.spec_z)
        for i, r in enumerate(self.comm.ranks):
            self.spec_rows[i].copy_(rows[i])
            _capi.check(L.pb_pressure_fft_columns(
                ctypes.byref(self.dims_rows), _capi.ptr(RS[i].d_rho0), _capi.ptr(RS[i].d_rho0_half),
                ctypes.byref(self.dims_z[i]), self.ws[i].data_ptr(), self.spec_rows[i].data_ptr(),
                self.scratch[i].data_ptr(), sl.y0(r), self.precision, streams[i]), "pb_pressure_fft_columns")
        back = rows_to_z(self.comm, sl, self.spec_rows)
        out_z = []
        for i, r in enumerate(self.comm.ranks):
            self.spec_z[i].copy_(back[i])
            pz = torch.empty((sl.nx, sl.ny, sl.nzl), dtype=torch.float64, device=rhs_x[i].device)
            _capi.check(L.pb_pressure_fft_inverse(ctypes.byref(self.dims_z[i]), self.ws[i].data_ptr(),
                                                  self.ws[i].numel(), pz.data_ptr(), self.precision, streams[i]),
                        "pb_pressure_fft_inverse")
            out_z.append(pz)
        return z_to_x(self.comm, sl, out_z)

    def _fill(self, fields, nv, streams):
        bc = (ctypes.c_double * nv)(*([1.0] * nv))
        for i, f in enumerate(fields):
            _capi.check(self.L.pb_update_all_bcs(ctypes.byref(self.dims_x), _capi.ptr(f), bc, nv, streams[i]),
                        "pb_update_all_bcs")
        exchange_x_halos(self.comm, fields, nv, self.dims_x.nlg, self.gw)

    def update(self, RS, PV, DV, Gr, streams):
        """RS, PV, DV, Gr: per-rank lists of the x-slab simulations' objects."""
        sl, L, gw = self.sl, self.L, self.gw
        npg = self.dims_x.npg
        dx_ = self.dims_x
        nlg2 = dx_.nlg[2]
        # HorizontalMean of w: per-GPU sums, added across GPUs, scaled
        sums = []
        for i in range(len(PV)):
            s = torch.empty(nlg2, dtype=torch.float64, device=PV[i].values.device)
            _capi.check(L.pb_horizontal_sums(ctypes.byref(dx_), _capi.ptr(PV[i].values[2 * npg:]), s.data_ptr(),
                                             streams[i]), "pb_horizontal_sums")
            sums.append(s)
        means = [m * (1.0 / float(sl.ny * sl.nx)) for m in self.comm.allreduce_sum(sums)]
        dense = []
        for i in range(len(PV)):
            d = torch.empty((sl.nxl, sl.ny, sl.nz), dtype=torch.float64, device=PV[i].values.device)
            _capi.check(L.pb_pressure_divergence(
                ctypes.byref(dx_), _capi.ptr(RS[i].d_rho0), _capi.ptr(RS[i].d_rho0_half), _capi.ptr(RS[i].d_alpha0),
                _capi.ptr(RS[i].d_alpha0_half), _capi.ptr(PV[i].values[0:]), _capi.ptr(PV[i].values[npg:]),
                _capi.ptr(PV[i].values[2 * npg:]), means[i].data_ptr(), _capi.ptr(DV[i].field("divergence", Gr[i])),
                d.data_ptr(), self.precision, streams[i]), "pb_pressure_divergence")
            dense.append(d)
        px = self._solve(dense, RS, streams)
        p = [DV[i].field("dynamic_pressure", Gr[i]) for i in range(len(PV))]
        for i in range(len(PV)):
            p[i].view(*[int(n) for n in dx_.nlg])[gw:-gw, gw:-gw, gw:-gw] = px[i]
        self._fill(p, 1, streams)
        for _ in range(self.refine_sweeps):
            res = []
            for i in range(len(PV)):
                r_ = torch.empty((sl.nxl, sl.ny, sl.nz), dtype=torch.float64, device=PV[i].values.device)
                _capi.check(L.pb_pressure_residual(ctypes.byref(dx_), _capi.ptr(RS[i].d_rho0),
                                                   _capi.ptr(RS[i].d_rho0_half), _capi.ptr(p[i]),
                                                   _capi.ptr(DV[i].field("divergence", Gr[i])), r_.data_ptr(),
                                                   streams[i]), "pb_pressure_residual")
                res.append(r_)
            dp = self._solve(res, RS, streams)
            for i in range(len(PV)):
                p[i].view(*[int(n) for n in dx_.nlg])[gw:-gw, gw:-gw, gw:-gw] += dp[i]
            self._fill(p, 1, streams)
        for i in range(len(PV)):
            _capi.check(L.pb_pressure_correct(ctypes.byref(dx_), _capi.ptr(p[i]), _capi.ptr(PV[i].values[0:]),
                                              _capi.ptr(PV[i].values[npg:]), _capi.ptr(PV[i].values[2 * npg:]),
                                              means[i].data_ptr(), streams[i]), "pb_pressure_correct")


# ---------------------------------------------------------------------------
# the sharded hot path
# ---------------------------------------------------------------------------
class ShardedSimulation:
    """The hot path of Simulation3d.run over x-slabs: per GPU the one-GPU
    components (HotPathSimulation) on its slab, halo exchanges after every
    ghost fill, and the sharded pressure solve.  comm.ranks are the ranks
    this process drives (one with DistComm, all with LocalComm); devices[i]
    is the device of comm.ranks[i]."""

    def __init__(self, namelist, comm, devices):
        from .simulation import HotPathSimulation
        g = namelist["grid"]
        self.namelist = namelist
        self.comm = comm
        self.sl = Slabs(int(g["nx"]), int(g["ny"]), int(g["nz"]), comm.world)
        self.gw = int(g["gw"])
        self.dx = (float(g["dx"]), float(g["dy"]), float(g["dz"]))
        local = copy.deepcopy(namelist)
        local["grid"]["nx"] = self.sl.nxl
        self.sims = [HotPathSimulation(local, device=dev) for dev in devices]
        for sim in self.sims:
            if sim.Sur.scheme != _capi.PB_SURFACE_NONE or sim.SGS is not None or sim.Fo.scheme != 0 or sim.Ra.active:
                raise NotImplementedError("the sharded hot path runs without surface, subgrid-scale, forcing "
                                          "or radiation terms")
        s0 = self.sims[0]
        self.pressure = ShardedPressure(comm, self.sl, self.gw, self.dx, s0.Pr.precision, s0.Pr.refine_sweeps,
                                        devices)

    # state ------------------------------------------------------------------
    def load_global(self, rs, fields):
        """Reference-state profiles and the global ghosted fields (host
        arrays of the whole domain, flat [i][j][k]); each GPU takes its slab
        (with ghost planes, refilled by the first ghost fill)."""
        sl, gw = self.sl, self.gw
        shape = (sl.nx + 2 * gw, sl.ny + 2 * gw, sl.nz + 2 * gw)
        for i, r in enumerate(self.comm.ranks):
            sim = self.sims[i]
            sim.set_reference_state(rs)
            x0 = sl.x0(r)
            sim.load_fields({n: np.asarray(a).reshape(shape)[x0:x0 + sl.nxl + 2 * gw].ravel()
                             for n, a in fields.items()})

    def gather_global(self, name):
        """A prognostic field of the whole domain on the host (interior x
        planes of every slab; this process's slabs only with DistComm)."""
        sl, gw = self.sl, self.gw
        parts = []
        for i, r in enumerate(self.comm.ranks):
            sim = self.sims[i]
            f = sim.PV.field(name, sim.Gr).view(*sim.Gr.shape)
            parts.append(f[gw:gw + sl.nxl].cpu().numpy())
        return np.concatenate(parts, axis=0)

    def _streams(self):
        return [_capi.stream_handle(torch.cuda.current_stream(s.PV.values.device)) for s in self.sims]

    def fill_ghosts(self, first=0, count=None):
        """PV.Update_all_bcs of the variables first .. first+count-1 on every
        slab, then the x-halo exchange."""
        sims = self.sims
        nv = sims[0].PV.nv
        count = nv - first if count is None else count
        for s in sims:
            s.PV.update_bcs_range(s.Gr, first, count)
        npg = sims[0].Gr.dims.npg
        views = [s.PV.values[first * npg:(first + count) * npg] for s in sims]
        exchange_x_halos(self.comm, views, count, sims[0].Gr.dims.nlg, self.gw)

    # time stepping ------------------------------------------------------------
    def stage(self, rk_step):
        for s in self.sims:
            s.PV.fuse_stages = s._fused()
            s.TS.rk_step = rk_step
            s.Th.update(s.Gr, s.RS, s.PV, s.DV)
            s.SA.update(s.Gr, s.RS, s.PV, s.DV)
            s.MA.update(s.Gr, s.RS, s.PV)
            s.TS.update(s.Gr, s.PV)
        self.fill_ghosts()
        sims = self.sims
        self.pressure.update([s.RS for s in sims], [s.PV for s in sims], [s.DV for s in sims],
                             [s.Gr for s in sims], self._streams())
        vel = sorted(int(i) for i in sims[0].PV.velocity_directions)
        self.fill_ghosts(vel[0], len(vel))

    def step(self):
        for rk in range(3):
            self.stage(rk)

    def run(self, nsteps):
        """Simulation3d.run: ghost fill and a thermodynamics update before the
        loop, then nsteps time steps."""
        self.fill_ghosts()
        for s in self.sims:
            s.Th.update(s.Gr, s.RS, s.PV, s.DV)
        for _ in range(nsteps):
            self.step()
