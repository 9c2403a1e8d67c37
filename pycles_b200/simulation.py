"""Hot-path driver: Simulation3d.run (Simulation3d.pyx:140-189) restricted to
the components built here, in the reference's order per RK stage.

    sim = HotPathSimulation(namelist)
    sim.initialize()          # reference state + seeded initial condition
    sim.run(nsteps)           # as Simulation3d.run (pre-loop bcs + Th.update)
    sim.step()                # one time step = three RK stages
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi, cases
from .advection import MomentumAdvection, ScalarAdvection
from .grid import Grid
from .pressure import PressureSolver
from .reference_state import ReferenceState
from .forcing import ForcingFactory
from .radiation import RadiationFactory
from .sgs import SGS, Kinematics, MomentumDiffusion, ScalarDiffusion
from .surface import SurfaceFactory
from .thermodynamics import ThermodynamicsDry, ThermodynamicsSA
from .time_stepping import TimeStepping
from .variables import DiagnosticVariables, PrognosticVariables


def namelist_for(case: str, nx: int, ny: int, nz: int, dx: float, dy: float, dz: float, gw: int = 3,
                 dt: float = 1.0, scalar_order: int = 5, momentum_order: int = 5, precision: str = "fp64"):
    return {
        "case": case,
        "grid": {"dims": 3, "nx": nx, "ny": ny, "nz": nz, "gw": gw, "dx": dx, "dy": dy, "dz": dz},
        "scalar_transport": {"order": scalar_order},
        "momentum_transport": {"order": momentum_order},
        "time_stepping": {"ts_type": 3, "dt_initial": dt, "dt_max": dt, "t_max": 1e30},
        "thermodynamics": {"do_qt_clipping": True},
        "gpu": {"precision": precision},
    }


# the measured configurations (synthetic seeded states of these shapes)
CONFIGS = {
    "c1_dry_cbl": dict(case="dry_cbl", nx=32, ny=32, nz=32, dx=50.0, dy=50.0, dz=50.0, gw=3, dt=0.5),
    "c2_bomex": dict(case="bomex", nx=64, ny=64, nz=75, dx=100.0, dy=100.0, dz=40.0, gw=3, dt=1.0),
    "c3_bomex": dict(case="bomex", nx=256, ny=256, nz=128, dx=50.0, dy=50.0, dz=20.0, gw=3, dt=1.0),
    # the learned seed's measurement grid (256 x 256 x 128, WENO5 as above)
    # with a cloud-topped state: the BOMEX-like state above holds no
    # saturated cell, so its secant never runs; dz 10 m puts the 840 m
    # inversion and the cloud layer inside the 1280 m column
    "c4_dycoms": dict(case="dycoms", nx=256, ny=256, nz=128, dx=50.0, dy=50.0, dz=10.0, gw=3, dt=0.5),
    "c5_dycoms": dict(case="dycoms", nx=512, ny=512, nz=256, dx=35.0, dy=35.0, dz=5.0, gw=4, dt=0.25,
                      scalar_order=7, momentum_order=5),
}


class HotPathSimulation:
    def __init__(self, namelist, device="cuda"):
        self.namelist = namelist
        self.device = torch.device(device)
        self.case = namelist.get("case", "bomex")
        Gr = self.Gr = Grid(namelist)
        Gr.device = self.device
        self.PV = PrognosticVariables(Gr)
        self.DV = DiagnosticVariables()
        self.moist = self.case != "dry_cbl"
        self.Th = ThermodynamicsSA(namelist) if self.moist else ThermodynamicsDry(namelist)
        self.SA = ScalarAdvection(namelist)
        self.MA = MomentumAdvection(namelist)
        self.Pr = PressureSolver(namelist)
        self.TS = TimeStepping()
        self.RS = ReferenceState(Gr)
        self.Sur = SurfaceFactory(namelist)
        self.Fo = ForcingFactory(namelist)
        self.Ra = RadiationFactory(namelist)
        # subgrid scale and diffusion when the namelist has an sgs section
        # (the measured configurations have none)
        self.SGS = SGS(namelist) if "sgs" in namelist else None
        if self.SGS is not None:
            self.Ke = Kinematics()
            self.SD = ScalarDiffusion(namelist, None, self.DV)
            self.MD = MomentumDiffusion(self.DV)
        PV = self.PV
        PV.add_variable("u", "m/s", "u", "u velocity component", "sym", "velocity")
        PV.set_velocity_direction("u", 0)
        PV.add_variable("v", "m/s", "v", "v velocity component", "sym", "velocity")
        PV.set_velocity_direction("v", 1)
        PV.add_variable("w", "m/s", "w", "w velocity component", "asym", "velocity")
        PV.set_velocity_direction("w", 2)
        self.Th.initialize(Gr, PV, self.DV)
        self.Pr.initialize(namelist, Gr, self.RS, self.DV)
        PV.initialize(Gr, device=self.device)
        self.DV.initialize(Gr, device=self.device)
        self.Sur.initialize(Gr, self.RS)
        self._fo_ready = False
        self.Ra.initialize(Gr)
        if self.SGS is not None:
            self.Ke.initialize(Gr)
            self.SGS.initialize(Gr, PV)
        self.SA.initialize(Gr, PV)
        self.MA.initialize(Gr, PV)
        self.TS.initialize(namelist, PV)
        self.fuse_rk = True  # precision form: SSP-RK3 stage inside the momentum pass
        _capi.load()

    # state ---------------------------------------------------------------
    def initialize(self, seed=0):
        """Reference state + seeded initial condition of the case."""
        fields = cases.CASES[self.case](self.Gr, self.RS, self.Th, seed=seed)
        self.load_fields(fields)
        return fields

    def load_fields(self, fields: dict):
        for name, arr in fields.items():
            self.PV.field(name, self.Gr).copy_(torch.as_tensor(np.ascontiguousarray(arr), dtype=torch.float64))

    def set_reference_state(self, profiles: dict):
        self.RS.set_profiles(profiles, device=self.device)

    def host_fields(self) -> dict:
        return {n: self.PV.field(n, self.Gr).cpu().numpy() for n in self.PV.index_name}

    # time stepping ---------------------------------------------------------
    def stage(self, rk_step: int, stream=None, mark=None):
        """One RK stage with the reference's calls in the reference's order
        (Simulation3d.pyx:159-178).  In the precision form without surface,
        subgrid-scale, forcing or radiation terms, SA.update and MA.update
        are deferred and TS.update runs them fused with the SSP-RK3 stage
        (see PrognosticVariables); otherwise every call launches as called.
        mark(i), if given, is called at the component boundaries (i = 0
        before the thermodynamics, 1 after it, 2 after the scalar advection,
        3 after the momentum advection -- with the u, v, w stage when fused,
        with the surface, subgrid-scale, forcing and radiation terms when
        they are on --, 4 after the remaining RK3 stage and the ghost fill,
        5 after the pressure solve and its ghost fill)."""
        Gr, PV, DV, RS, TS = self.Gr, self.PV, self.DV, self.RS, self.TS
        m = mark if mark is not None else (lambda i: None)
        self._stages_run += 1
        fused = self._fused()
        PV.fuse_stages = fused
        TS.rk_step = rk_step
        m(0)
        self.Th.update(Gr, RS, PV, DV, stream=stream)
        m(1)
        self.SA.update(Gr, RS, PV, DV, stream=stream)
        if not fused:
            m(2)
        self.MA.update(Gr, RS, PV, stream=stream)
        # then Sur, SGS, SD and MD (Simulation3d.pyx:167-172); Ke.update
        # (:160) is folded into SGS.update: no velocity changes between
        self.Sur.update(Gr, RS, PV, DV, stream=stream)
        if self.SGS is not None:
            self.SGS.update(Gr, DV, PV, self.Ke, self.Sur, stream=stream)
            self.SD.update(Gr, RS, PV, DV, stream=stream)
            self.MD.update(Gr, RS, PV, DV, self.Ke, stream=stream)
        if self.Fo.scheme != _capi.PB_FORCING_NONE:  # Fo.update (:173)
            if not self._fo_ready:  # the profiles need the installed reference state
                self.Fo.initialize(Gr, RS)
                self._fo_ready = True
            self.Fo.update(Gr, RS, PV, DV, stream=stream)
        self.Ra.update(Gr, RS, PV, DV, self.Sur, TS, stream=stream)  # Ra.update (:174)
        if not fused:
            m(3)
        TS.update(Gr, PV, stream=stream, mark=m if fused else None)
        if self._scalar_ghosts_filled:
            # a mark hook filled the scalars' ghosts right after their pass
            self._scalar_ghosts_filled = False
            self._fill_velocity_ghosts(stream)
        else:
            PV.Update_all_bcs(Gr, stream=stream)
        m(4)
        # PressureSolver.update: the solve, then its ghost fill -- of the
        # velocities only, the one thing the correction changed (the
        # scalars' ghosts are the ones filled just above)
        self.Pr.solve(Gr, RS, DV, PV, stream=stream)
        self._fill_velocity_ghosts(stream)
        m(5)

    _scalar_ghosts_filled = False
    _stages_run = 0

    def _fused(self) -> bool:
        """The precision form steps with the SSP-RK3 stage fused into the
        advection passes (velocities u, v, w first, as this driver adds them)
        unless fuse_rk is off or a surface, subgrid-scale, forcing or
        radiation term adds tendencies between the advection and the stage."""
        return (self.fuse_rk and self.MA.precision == _capi.PB_FP32
                and self.Sur.scheme == _capi.PB_SURFACE_NONE and self.SGS is None
                and self.Fo.scheme == _capi.PB_FORCING_NONE and not self.Ra.active)

    def _fill_velocity_ghosts(self, stream=None):
        """Ghost fill of the velocities alone when they are the first
        prognostic variables (the usual order), else of all variables."""
        PV = self.PV
        vel = sorted(int(i) for i in PV.velocity_directions)
        if vel == list(range(len(vel))):
            PV.update_bcs_range(self.Gr, 0, len(vel), stream=stream)
        else:
            PV.Update_all_bcs(self.Gr, stream=stream)

    def step(self, stream=None):
        for rk in range(self.TS.n_rk_steps):
            self.stage(rk, stream=stream)

    def step_host(self, host_values, stream=None, chunks_per_variable=4):
        """One time step whose prognostic state lives in pinned host memory,
        as the reference keeps PV.values in host numpy arrays: the state is
        copied to the device before the step and back after it.

        The copies run on two copy streams (one per direction, so uploads
        and downloads use both directions of the link at once), in chunks of
        1/chunks_per_variable of a variable, each with its own event: the
        next call uploads a chunk as soon as this call's download of that
        chunk has finished, so a chunk's round trip is pipelined behind the
        download of the next one instead of waiting for a whole variable
        group.  The velocities' upload overlaps the first thermodynamics
        update (which reads only the scalars).  The scalars are final after
        the last stage's scalar pass: with fused stages their ghosts are
        filled right there and their download overlaps the momentum pass and
        the pressure solve (the stage's ghost fill and the solve's are then
        restricted to the velocities); otherwise it starts before the last
        pressure solve.  The next call's scalar upload overlaps this call's
        velocity download; the next call's uploads start as soon as their
        chunks are downloaded, without waiting for the end of this call's
        pressure solve.  Every host region is read only after the download
        that wrote it, and every device region is overwritten only after the
        download that read it and after the last kernel that writes it.
        Asynchronous: host_values holds the new state once
        `copy_streams()[1]` has finished.  Between two calls the device copy
        belongs to step_host: the next call may upload into PV.values before
        work queued on the stream between the calls has run, so read the
        state from host_values.  Work on the device copy between two calls
        must first wait for `copy_streams()` (the downloads still read it); a
        step or stage run between the calls makes the next call wait for the
        stream, as the first call does.
        host_values: pinned CPU float64 tensor of nv * npg values."""
        import torch
        Gr, PV = self.Gr, self.PV
        npg = Gr.dims.npg
        st = stream if stream is not None else torch.cuda.current_stream(PV.values.device)
        h2d, d2h = self.copy_streams()
        vel = sorted(int(i) for i in PV.velocity_directions)
        if vel != list(range(len(vel))):
            raise ValueError("step_host expects the velocities to be the first prognostic variables")
        nvel, nv = len(vel), PV.nv
        k = max(1, int(chunks_per_variable))

        def chunks(v0, v1):
            step = -(-npg // k)
            return [(v * npg + lo, v * npg + min(lo + step, npg)) for v in range(v0, v1) for lo in range(0, npg, step)]

        sc_chunks, vel_chunks = chunks(nvel, nv), chunks(0, nvel)

        def copy(dst, src, r):
            dst[r[0]:r[1]].copy_(src[r[0]:r[1]], non_blocking=True)

        def event(stream_):
            e = torch.cuda.Event()
            e.record(stream_)
            return e

        prev = getattr(self, "_host_events", None)
        free = getattr(self, "_host_free", None)
        if getattr(self, "_host_stages", None) != self._stages_run:
            prev = free = None  # stages ran since the last call: not a continuation
        if prev is None or free is None:
            h2d.wait_event(event(st))  # the work queued on PV.values so far
        else:
            # the previous call's last stage no longer writes the scalars
            # (recorded after its ghost fill); each chunk also waits for its
            # own download below, the velocities' after the pressure solve
            h2d.wait_event(free)
            if set(prev) != set(sc_chunks + vel_chunks):
                for e in prev.values():  # another chunking: wait for every download
                    h2d.wait_event(e)
                prev = None
        with torch.cuda.stream(h2d):
            for r in sc_chunks:
                if prev is not None:
                    h2d.wait_event(prev[r])  # the download of this chunk has left PV.values / filled host
                copy(PV.values, host_values, r)
            e_sc = event(h2d)
            for r in vel_chunks:
                if prev is not None:
                    h2d.wait_event(prev[r])
                copy(PV.values, host_values, r)
            e_all = event(h2d)
        st.wait_event(e_sc)
        last = self.TS.n_rk_steps - 1
        out = {}
        freed = [None]

        def download(rs, src=None):
            d2h.wait_event(event(st))
            with torch.cuda.stream(d2h):
                for r in rs:
                    copy(host_values, PV.values if src is None else src, r)
                    out[r] = event(d2h)

        def hooks(rk):
            def mark(i):
                if i == 1 and rk == 0:
                    st.wait_event(e_all)  # the velocities' upload, overlapped with the thermodynamics
                elif i == 2 and rk == last and self.TS.fused_values is not None and sc_chunks:
                    # the scalars' new values are complete in the fused stage's
                    # buffer: fill their ghosts and download them from there
                    buf = self.TS.fused_values
                    PV.update_bcs_range(Gr, nvel, nv - nvel, stream=st, values=buf)
                    self._scalar_ghosts_filled = True
                    download(sc_chunks, src=buf)
                    if not PV.stable_values:  # nothing writes the scalars after this point
                        self._host_free = freed[0] = event(st)
                elif i == 4 and rk == last:
                    if sc_chunks and sc_chunks[0] not in out:
                        download(sc_chunks)  # the scalars are final: download them during the pressure solve
                    if freed[0] is None:  # (with stable addresses: after the copy back)
                        self._host_free = event(st)
                elif i == 5 and rk == last:
                    download(vel_chunks)
            return mark

        for rk in range(self.TS.n_rk_steps):
            self.stage(rk, st, mark=hooks(rk))
        self._host_events = out
        self._host_stages = self._stages_run

    def copy_streams(self):
        """The (host->device, device->host) streams of step_host."""
        import torch
        if getattr(self, "_copy_streams", None) is None:
            dev = self.PV.values.device
            self._copy_streams = (torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev))
        return self._copy_streams

    def graph_steps(self) -> int:
        """The smallest number of time steps that one CUDA graph of the step
        (capture_steps) may hold: even when the fused stages swap the two
        value buffers (so that PV.values is the same buffer after the
        recorded steps), and a whole number of learned-seed refresh periods
        when the seed is on (so that every replay refreshes as the eager
        steps do)."""
        import math
        n = 2 if (self._fused() and not self.PV.stable_values) else 1
        if getattr(self.Th, "mlp", None) is not None:
            upd = self.TS.n_rk_steps
            every = int(self.Th.seed_refresh_interval)
            per = every // math.gcd(every, upd)
            n = n * per // math.gcd(n, per)
        return n

    def capture_steps(self, nsteps: int = 0):
        """Records nsteps device-resident time steps (`step`) as one CUDA
        graph and returns it (torch.cuda.CUDAGraph): `graph.replay()` runs
        them with one launch from the host.  For grids whose steps are bound
        by kernel launches (at 64x64x75 a step is ~150 kernels of a few
        microseconds).  nsteps = 0 takes graph_steps(); other counts must be
        multiples of it.  At least one step must have run eagerly (the lazily
        made buffers, workspaces and tables exist then); recording runs no
        kernel and does not advance the state.  The host-side time (TS.t)
        does not advance on replay, and the simulation must not change form,
        grid or learned seed while the graph is in use."""
        import torch
        unit = self.graph_steps()
        n = unit if nsteps == 0 else int(nsteps)
        if n < 1 or n % unit:
            raise ValueError(f"a graph of this simulation holds a multiple of {unit} steps, not {nsteps}")
        if self._stages_run < self.TS.n_rk_steps:
            raise RuntimeError("run one step eagerly before capturing the step in a graph")
        dev = self.PV.values.device
        g = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        t0 = self.TS.t
        with torch.cuda.graph(g, stream=side):
            for _ in range(n):
                self.step()
        self.TS.t = t0
        torch.cuda.current_stream(dev).wait_stream(side)
        return g

    def run(self, nsteps: int, stream=None):
        """Simulation3d.run: ghost fill and a thermodynamics update before the
        loop (its first output), then nsteps time steps."""
        self.PV.Update_all_bcs(self.Gr, stream=stream)
        self.Th.update(self.Gr, self.RS, self.PV, self.DV, stream=stream)
        for _ in range(nsteps):
            self.step(stream=stream)

    def check_device_errors(self):
        word = _capi.get_error()
        if word:
            raise _capi.PbError(f"device error word 0x{word:x} (table range=1, secant cap=2, non-finite=4)")
