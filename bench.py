"""Benchmark of the PyCLES hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c5_dycoms]
                    [--form both|fp64|fp32] [--impl ours|reference]

A step is one time step (three SSP-RK3 stages) of the hot path --
thermodynamics, scalar and momentum advection, RK update, ghost fill and the
pressure solve -- over the configuration's whole grid.  Metric: grid-cell
RK-stage updates/s = interior cells x 3 / time per step.

Workload (default): 512 x 512 x 256 cells, dx = dy = 35 m, dz = 5 m, gw = 4,
WENO7 scalars, WENO5 momentum, saturation adjustment, dt = 0.25 s, a seeded
synthetic DYCOMS-RF01-like stratocumulus state (no public data set is used).
The state (~19 GB FP64) is larger than L2, so no L2 flush is needed.

Multi-GPU: the domain is not split across GPUs here; N ranks run N
independent replicas (weak scaling), timed as the max over ranks.

``--impl reference`` times the reference's own CPU implementation of the
path (its C kernels compiled from source into oracle/_ref, driven by the
restated glue) on all host cores, each core stepping a bounded sub-domain
of the same configuration.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "grid-cell RK-stage updates/s"
UNIT = "cell-stage/s"
# algorithmic bytes and flops per interior cell per RK stage of the fused
# advection (read every prognostic field once, read-modify-write every
# tendency once): 24 B x nv; flops of WENO5/7 fluxes + divergence.
ADV_BYTES_PER_CELL = {5: 120, 4: 96}
ADV_FLOPS_PER_CELL = {("c5", 7): 3252, ("moist", 5): 2340, ("dry", 5): 1881}


def _ghost_bytes(nv, cfg):
    """Ghost fill: 16 B per ghost cell and variable, per interior cell."""
    gw, n = cfg["gw"], (cfg["nx"], cfg["ny"], cfg["nz"])
    npl = n[0] * n[1] * n[2]
    npg = (n[0] + 2 * gw) * (n[1] + 2 * gw) * (n[2] + 2 * gw)
    return 16.0 * nv * (npg - npl) / npl


# Compulsory (algorithmic) bytes per interior cell per RK stage of each timed
# component, FP64 storage: every array it must read once and write once.
# fused: the precision form's stepping, the u, v, w stage inside the
# momentum pass.
COMPONENT_BYTES_PER_CELL = {
    # moist: read s, qt, w-tendency; write qt, T, qv, ql, qi, alpha,
    # buoyancy, theta_rho, bvf, thetali, w-tendency.  dry: read s,
    # w-tendency; write T, alpha, buoyancy, theta, bvf, w-tendency.
    "thermo": lambda nv, cfg, fused: 112.0 if cfg["case"] != "dry_cbl" else 64.0,
    # read u, v, w and the scalars, read-modify-write the scalar tendencies;
    # fused: read u, v, w and the scalars, write the new scalars, write
    # (stage 0) or read the copies
    "scalar_adv": lambda nv, cfg, fused: 24.0 + 24.0 * (nv - 3) if fused else 8.0 * nv + 16.0 * (nv - 3),
    # read u, v, w, read-modify-write the three momentum tendencies; fused:
    # read u, v, w and the w tendency, write the new u, v, w, write (stage 0)
    # or read the copies, clear the w tendency
    "momentum_adv": lambda nv, cfg, fused: 88.0 if fused else 72.0,
    # SSP-RK3 stage (read value, tendency, copy; write value, copy,
    # zeroed tendency: 40 B per variable; fused: inside the advection
    # passes) + ghost fill
    "rk3+bcs": lambda nv, cfg, fused: (0.0 if fused else 40.0 * nv) + _ghost_bytes(nv, cfg),
    # read u, v, w; write u, v, w, divergence, pressure
    "pressure": lambda nv, cfg, fused: 64.0,
}
COMPONENT_KERNELS = {
    "thermo": "thermo_sa_kernel (saturation adjustment, buoyancy, bvf, thetali; one launch per stage)",
    "scalar_adv": "scalar_march x, y + scalar_z (WENO fluxes + divergence; 3 launches per stage and scalar "
                  "in the precision form, the scalars' SSP-RK3 stage in scalar_z; 3 per stage in the plain form)",
    "momentum_adv": "momentum_tma (y-z planes of u, v, w staged by TMA; momentum_tile on odd-level grids) with "
                    "the u, v, w SSP-RK3 stage in the precision form (1 launch per stage); "
                    "momentum_march x, y + momentum_z in the plain form (3 launches)",
    "rk3+bcs": "rk3_kernel + ghost_fill_kernel (the precision form: the ghost fill alone, its stage is "
               "inside the advection passes)",
    "pressure": "hmean_partial + hmean_final (hmean_serial, the reference's summation order, in the plain "
                "form), fft_x_fwd, fft_y, tdma, fft_x_inv (+ refinement), ghost_sym, correction",
}


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU side: reference implementation on bounded per-core samples
# ---------------------------------------------------------------------------
def _cpu_sample_shape(cfg):
    """Per-core sub-domain: the configuration's nz, gw and orders, with a
    horizontal extent sized for a few seconds of reference CPU work per step."""
    nz = cfg["nz"]
    nh = 64 if nz >= 128 else 48
    return nh, nh, nz


def _cpu_worker(args):
    """One process: build a sub-domain sample, run `nsteps` steps of the
    reference's C kernels + restated glue, return per-step wall times."""
    cfg, nsteps, backend, conn_barrier = args
    import numpy as np  # noqa: F401
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import host_case, oracle_sim
    nx, ny, nz = _cpu_sample_shape(cfg)
    nl, rs, f = host_case(cfg["case"], nx, ny, nz, cfg["dx"], cfg["dy"], cfg["dz"], gw=cfg["gw"], dt=cfg["dt"],
                          scalar_order=cfg.get("scalar_order", 5), momentum_order=cfg.get("momentum_order", 5))
    sim = oracle_sim(nl, rs, f, backend=backend)
    sim.update_all_bcs()
    times = []
    for _ in range(nsteps):
        if conn_barrier is not None:
            conn_barrier.wait()
        t0 = time.perf_counter()
        sim.step()
        times.append(time.perf_counter() - t0)
    # what this process actually ran: the compiled reference library mapped
    # into it, and the reference's cythonized TDMA for the pressure columns
    mapped = []
    try:
        with open("/proc/self/maps") as fh:
            mapped = sorted({ln.split()[-1] for ln in fh if "oracle/_ref/" in ln and ln.rstrip().endswith(".so")})
    except OSError:
        pass
    tdma = None
    if backend == "ref":
        from oracle import ref as oref
        tdma = oref.tdma_module() is not None
    return nx * ny * nz, times, {"backend": backend, "ref_libraries_mapped": [os.path.basename(m) for m in mapped],
                                 "reference_tdma": tdma}


def cpu_reference_run(cfg, nsteps, nwarm, backend="ref", cores=None):
    """Runs `cores` concurrent workers in lock-step; returns per-step aggregate
    throughput (cell-stage/s) and the description of the sample."""
    import multiprocessing as mp
    from oracle import ref as oref
    if backend == "ref" and not oref.available():
        backend = "port"
    cores = cores or len(os.sched_getaffinity(0))
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        barrier = mgr.Barrier(cores)
        with ctx.Pool(cores) as pool:
            res = pool.map(_cpu_worker, [(cfg, nsteps + nwarm, backend, barrier)] * cores)
    cells = res[0][0]
    ran = [r[2] for r in res]
    per_step = []
    for s in range(nwarm, nwarm + nsteps):
        wall = max(r[1][s] for r in res)
        per_step.append(cores * cells * 3 / wall)
    nx, ny, nz = _cpu_sample_shape(cfg)
    # the label follows what every worker reports it ran, not this process's check
    all_ref = all(r["backend"] == "ref" and "libpycles_ref.so" in r["ref_libraries_mapped"] for r in ran)
    kind = "reference" if all_ref else "port"
    sample = (f"{cores} concurrent processes, each one time step of a {nx}x{ny}x{nz} sub-domain "
              f"(gw={cfg['gw']}, WENO{cfg.get('scalar_order', 5)}/{cfg.get('momentum_order', 5)}) of the same case; "
              f"{'reference C kernels compiled from source + restated glue' if kind == 'reference' else 'numpy port'}"
              "; no halo exchange or pencil transposes between processes (MPI-free upper bound)")
    workers = {"backend": sorted({r["backend"] for r in ran}),
               "ref_libraries_mapped": sorted({m for r in ran for m in r["ref_libraries_mapped"]}),
               "workers_with_reference_library": sum("libpycles_ref.so" in r["ref_libraries_mapped"] for r in ran),
               "workers_with_reference_tdma": sum(bool(r["reference_tdma"]) for r in ran)}
    return per_step, {"kind": kind, "cores": cores, "sample": sample, "workers": workers}


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------
def max_over_ranks(ms: float, device, world: int) -> float:
    """The job's time: the slowest rank's device-timed region (the ranks are
    independent replicas; this is their only collective)."""
    if world <= 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _time_steps(sim, steps, local_rank, world):
    """Device-resident timed region: `steps` time steps with CUDA events around
    every component call on the launching stream."""
    import torch
    import torch.distributed as dist

    from pycles_b200 import _capi
    dev = sim.device
    stream = torch.cuda.current_stream(dev)
    comp = ["thermo", "scalar_adv", "momentum_adv", "rk3+bcs", "pressure"]
    ev = []
    clocks = ClockSampler(local_rank)
    clocks.start()
    L = _capi.load()
    n_launch0 = L.pb_launch_count()
    if sim.moist:
        sim.Th.iter_stats.zero_()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t_start.record(stream)
    for _ in range(steps):
        for rk in range(3):
            # the driver's own stage, with events at its component boundaries
            # (thermo | scalar advection | momentum advection [+ the u, v, w
            # RK3 stage when fused] | rest of the RK3 stage + ghost fill |
            # pressure + its ghost fill)
            e = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
            sim.stage(rk, stream, mark=lambda i, e=e: e[i].record(stream))
            ev.append(e)
    t_end.record(stream)
    torch.cuda.synchronize()
    launches = L.pb_launch_count() - n_launch0
    clock_info = clocks.stop()
    elapsed_ms = t_start.elapsed_time(t_end)
    comp_ms = {c: 0.0 for c in comp}
    for e in ev:
        for i, c in enumerate(comp):
            comp_ms[c] += e[i].elapsed_time(e[i + 1])
    elapsed_ms = max_over_ranks(elapsed_ms, dev, world)
    secant = None
    if sim.moist:
        st = sim.Th.iter_stats.cpu().tolist()
        secant = {"mean_iterations_per_saturated_cell": (st[0] / st[1]) if st[1] else 0.0,
                  "saturated_cells_per_stage": st[1] / (3 * steps)}
    return elapsed_ms, comp_ms, launches, clock_info, secant


# Training distribution of the learned seed: states of the moist BOMEX-like
# configurations (64x64x75 and 256x256x128, FP64 plain form, saved at the
# listed steps), each sampled cell jittered uniformly by these half-widths in
# (p0 [Pa], s [J/kg/K], qt [kg/kg]).  Those states hold no saturated cell
# (no surface fluxes build a cloud layer), so the spread is what reaches the
# saturated part of the network's input box; it also covers the
# stratocumulus (DYCOMS-like) states the network is then used on.
SEED_TRAIN_STATES = (("c2_bomex", (0, 20, 40)), ("c3_bomex", (0, 5)))
SEED_JITTER = (1500.0, 45.0, 5.0e-3)
SEED_PAIRS = 10_000_000


def _train_seed(sim, fields, log):
    """Learned seed for the secant (outside the timed region): 10^7 pairs
    from the plain FP64 secant on inputs drawn around states of the moist
    64x64x75 and 256x256x128 configurations, trained with the library's own
    tensor-core kernels, and evaluated on held-out pairs from the benchmark's
    own state (never trained on)."""
    import torch

    from pycles_b200 import learned
    from pycles_b200.simulation import CONFIGS, HotPathSimulation, namelist_for
    states = []
    for name, steps in SEED_TRAIN_STATES:
        src = HotPathSimulation(namelist_for(**CONFIGS[name], precision="fp64"), device=sim.device)
        src.initialize(seed=1)
        src.run(0)
        done = 0
        for s in steps:
            for _ in range(s - done):
                src.step()
            done = s
            states.append(tuple(t.clone() for t in learned.cell_inputs(src)))
        del src
    torch.cuda.empty_cache()
    Gr = sim.Gr
    n2 = Gr.dims.nlg[2]
    held = [(sim.RS.d_p0_half.repeat(Gr.npg // n2), torch.as_tensor(fields["s"], device=sim.device),
             torch.as_tensor(fields["qt"], device=sim.device))]
    mlp, info = learned.train_seed(sim.Th, states, n_pairs=SEED_PAIRS, jitter=SEED_JITTER, held_out_states=held,
                                   n_held_out=1_000_000, device=sim.device)
    info["trained_on"] = (f"inputs drawn around {len(states)} FP64 states of "
                          + ", ".join(f"{n} (steps {list(st)})" for n, st in SEED_TRAIN_STATES)
                          + f", uniform jitter +-{SEED_JITTER} in (p0, s, qt)")
    info["held_out_on"] = "the benchmark's own initial state (cells as they are, no jitter)"
    del states
    torch.cuda.empty_cache()
    log(f"learned seed: {info}")
    if mlp is None:
        return None
    return mlp, info


def _learned_at_c4(trained, dev, args, log):
    """The learned seed at 256x256x128 (cloud-topped state, the c4_dycoms
    configuration): precision form with and without the seed (the network
    trained for the headline, never on this state), device time per step and
    mean secant iterations per saturated cell over the timed steps."""
    import torch

    from pycles_b200.simulation import CONFIGS, HotPathSimulation, namelist_for
    cfg = CONFIGS["c4_dycoms"]
    out = {"workload": (f"c4_dycoms: {cfg['nx']}x{cfg['ny']}x{cfg['nz']} cells, dx={cfg['dx']} m, dz={cfg['dz']} m, "
                        f"WENO5, dt={cfg['dt']}, seeded DYCOMS-RF01-like state")}
    fields = rs = None
    for form, seeded in (("fp32", False), ("fp32+learned", True)):
        sim = HotPathSimulation(namelist_for(**cfg, precision="fp32"), device=dev)
        if fields is None:
            fields = sim.initialize(seed=0)
            rs = sim.RS.profiles()
        else:
            sim.set_reference_state(rs)
            sim.load_fields(fields)
        if seeded:
            sim.Th.mlp = trained[0]
        sim.run(0)
        for _ in range(args.warmup):
            sim.step()
        torch.cuda.synchronize()
        elapsed_ms, comp_ms, _, _, secant = _time_steps(sim, max(args.steps, 12), 0, 1)
        n = max(args.steps, 12)
        out[form] = {"ms_per_step": round(elapsed_ms / n, 4), "thermo_ms_per_step": round(comp_ms["thermo"] / n, 4),
                     "mean_secant_iterations_per_saturated_cell": secant["mean_iterations_per_saturated_cell"],
                     "saturated_cells_per_stage": secant["saturated_cells_per_stage"]}
        log(f"c4 {form}: {out[form]}")
        del sim
        torch.cuda.empty_cache()
    return out


# surface scheme of each configuration's case (Surface.pyx:39-74)
SURFACE_OF_CASE = {"dry_cbl": "SullivanPatton", "bomex": "Bomex", "dycoms": "DYCOMS_RF01"}


def _time_surface(sim, cfg, peak, calls=50, warm=3):
    """The surface scheme of the configuration's case on the timed state:
    CUDA-event time of pb_surface_update (its two kernels) over `calls`
    calls.  Algorithmic bytes per column: read u, v, T, qt, ql (qt, ql for
    the moist schemes); write the nine surface arrays and the wind speed;
    read and write the first-level tendencies of u, v, s (and qt).  Each 3-D
    field contributes one 8-byte value per column at k = gw, a strided
    access that moves a 32-byte sector per value."""
    import torch

    from pycles_b200.surface import SurfaceFactory
    scheme = SURFACE_OF_CASE[cfg["case"]]
    sur = SurfaceFactory({"meta": {"casename": scheme}})
    sur.initialize(sim.Gr, sim.RS)
    args = (sim.Gr, sim.RS, sim.PV, sim.DV)
    tend = sim.PV.tendencies.clone()
    for _ in range(warm):
        sur.update(*args)
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(calls):
        sur.update(*args)
    b.record(stream)
    torch.cuda.synchronize()
    sim.PV.tendencies.copy_(tend)
    us = a.elapsed_time(b) * 1e3 / calls
    moist = scheme != "SullivanPatton"
    cols = sim.Gr.dims.nlg[0] * sim.Gr.dims.nlg[1]
    nbytes_col = 8 * (5 if moist else 3) + 8 * 10 + 16 * (4 if moist else 3)
    ach = nbytes_col * cols / (us * 1e-6) / 1e9
    return {"scheme": scheme, "us_per_call": round(us, 2), "kernels_per_call": 2, "columns": cols,
            "algorithmic_bytes_per_column": nbytes_col, "achieved_gbs": round(ach, 1),
            "frac": round(ach / peak, 4)}


def _time_sgs(sim, peak, calls=10, warm=2):
    """Smagorinsky subgrid scale and diffusion on the timed state: CUDA-event
    time per launch of pb_kinematics_sgs (strain-rate magnitude + viscosity
    and diffusivity), pb_scalar_diffusion (all scalars) and
    pb_momentum_diffusion, with their algorithmic bytes per interior cell
    (each field read once, each result written once, tendencies read and
    written): 56, 8 + 24 per scalar, 112.  The tendencies are restored
    afterwards."""
    import ctypes

    import torch

    from pycles_b200 import _capi
    Gr, PV, DV, RS = sim.Gr, sim.PV, sim.DV, sim.RS
    L = _capi.load()
    npg, dev = Gr.dims.npg, PV.values.device
    smag, visc, diff = (torch.zeros(npg, dtype=torch.float64, device=dev) for _ in range(3))
    sgs = _capi.PbSgs(_capi.PB_SGS_SMAGORINSKY, _capi.PB_SGS_LENGTH_GRID, 0.17, 1.0 / 3.0, 0.0, 0.0)
    vel = [_capi.ptr(PV.values[int(PV.velocity_directions[d]) * npg:]) for d in range(3)]
    tvel = [_capi.ptr(PV.tendencies[int(PV.velocity_directions[d]) * npg:]) for d in range(3)]
    dvp = lambda n: _capi.ptr(DV.values[DV.get_varshift(Gr, n):])
    scal = [i for i in range(PV.nv) if PV.var_type[i] == 1]
    ns = len(scal)
    vals = (ctypes.c_void_p * ns)(*[_capi.ptr(PV.values[i * npg:]) for i in scal])
    tends = (ctypes.c_void_p * ns)(*[_capi.ptr(PV.tendencies[i * npg:]) for i in scal])
    s_t = _capi.ptr(PV.tendencies[PV.get_varshift(Gr, "s"):])
    st = _capi.stream_handle(None)
    d = ctypes.byref(Gr.dims)
    launches = {
        "kinematics_sgs": (lambda: L.pb_kinematics_sgs(d, ctypes.byref(sgs), *vel, dvp("buoyancy_frequency"), None,
                                                       _capi.ptr(smag), _capi.ptr(visc), _capi.ptr(diff), st), 56.0),
        "scalar_diffusion": (lambda: L.pb_scalar_diffusion(d, _capi.ptr(RS.d_rho0), _capi.ptr(RS.d_rho0_half),
                                                           _capi.ptr(RS.d_alpha0_half), _capi.ptr(diff), ns, vals,
                                                           tends, None, -1, -1, None, None, None, st),
                             8.0 + 24.0 * ns),
        "momentum_diffusion": (lambda: L.pb_momentum_diffusion(
            d, _capi.ptr(RS.d_rho0), _capi.ptr(RS.d_rho0_half), _capi.ptr(RS.d_alpha0), _capi.ptr(RS.d_alpha0_half),
            *vel, _capi.ptr(visc), _capi.ptr(smag), dvp("temperature"), *tvel, s_t, st), 112.0),
    }
    tend = PV.tendencies.clone()
    out = {}
    stream = torch.cuda.current_stream()
    for name, (fn, nbytes) in launches.items():
        for _ in range(warm):
            _capi.check(fn(), name)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(calls):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / calls
        ach = nbytes * Gr.dims.npl / (ms / 1e3) / 1e9
        out[name] = {"ms_per_launch": round(ms, 4), "algorithmic_bytes_per_cell": nbytes,
                     "achieved_gbs": round(ach, 1), "frac": round(ach / peak, 4)}
    PV.tendencies.copy_(tend)
    del smag, visc, diff, tend
    out["scheme"] = "Smagorinsky (grid length scale), FP64; one launch of each kernel per RK stage"
    return out


def _time_stats(sim, peak, calls=10, warm=2):
    """HorizontalMean of one prognostic field (the statistics' most common
    reduction) on the timed state: CUDA-event time per call (two launches)
    and the field's bytes over it."""
    import torch

    from pycles_b200.statistics import HorizontalStatistics
    st = HorizontalStatistics(sim.Gr)
    f = sim.PV.field("s", sim.Gr)
    for _ in range(warm):
        st.HorizontalMean(sim.Gr, f)
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(calls):
        st.HorizontalMean(sim.Gr, f)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / calls
    nbytes = 8.0 * sim.Gr.dims.npg
    ach = nbytes / (ms / 1e3) / 1e9
    return {"reduction": "HorizontalMean of s", "ms_per_call": round(ms, 4), "bytes_per_call": nbytes,
            "achieved_gbs": round(ach, 1), "frac": round(ach / peak, 4)}


def _time_forcing(sim, cfg, peak, calls=10, warm=2):
    """The case forcing of the configuration's case (DYCOMS_RF01 on the DYCOMS
    workload) on the timed state: CUDA-event time per call, with its
    algorithmic bytes per interior cell (read s, qt, u, v; read and write
    their tendencies: 96 B; Bomex also reads ql and T: 112 B; SullivanPatton
    u, v and their tendencies: 48 B).  The tendencies are restored."""
    import torch

    from pycles_b200.forcing import ForcingFactory
    scheme = SURFACE_OF_CASE[cfg["case"]]
    fo = ForcingFactory({"meta": {"casename": scheme}})
    fo.initialize(sim.Gr, sim.RS)
    args = (sim.Gr, sim.RS, sim.PV, sim.DV)
    tend = sim.PV.tendencies.clone()
    for _ in range(warm):
        fo.update(*args)
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(calls):
        fo.update(*args)
    b.record(stream)
    torch.cuda.synchronize()
    sim.PV.tendencies.copy_(tend)
    ms = a.elapsed_time(b) / calls
    nbytes = {"SullivanPatton": 48.0, "Bomex": 112.0, "DYCOMS_RF01": 96.0}[scheme]
    ach = nbytes * sim.Gr.dims.npl / (ms / 1e3) / 1e9
    out = {"scheme": scheme, "ms_per_call": round(ms, 4), "algorithmic_bytes_per_cell": nbytes,
           "achieved_gbs": round(ach, 1), "frac": round(ach / peak, 4)}
    if scheme == "DYCOMS_RF01":
        # its radiation (Radiation.pyx:230-353): read ql, qt (twice), T; read
        # and write the s tendency; write the heating rate and dT/dt: 64 B
        from pycles_b200.radiation import RadiationFactory
        ra = RadiationFactory({"meta": {"casename": scheme}})
        ra.initialize(sim.Gr)
        for _ in range(warm):
            ra.update(*args)
        a.record(stream)
        for _ in range(calls):
            ra.update(*args)
        b.record(stream)
        torch.cuda.synchronize()
        sim.PV.tendencies.copy_(tend)
        ms = a.elapsed_time(b) / calls
        ach = 64.0 * sim.Gr.dims.npl / (ms / 1e3) / 1e9
        out["radiation"] = {"ms_per_call": round(ms, 4), "algorithmic_bytes_per_cell": 64.0,
                            "achieved_gbs": round(ach, 1), "frac": round(ach / peak, 4)}
        del ra
    return out


def run_ours(args, rank, world, local_rank):
    import torch

    from pycles_b200 import _capi
    from pycles_b200.simulation import CONFIGS, HotPathSimulation, namelist_for

    cfg = dict(CONFIGS[args.config])
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    log = (lambda m: print(m, file=sys.stderr)) if rank == 0 else (lambda m: None)
    # (name, precision, learned seed); the last one is the headline
    forms = []
    if args.form in ("all", "fp64"):
        forms.append(("fp64", "fp64", False))
    if args.form in ("all", "fp32"):
        forms.append(("fp32", "fp32", False))
        if cfg["case"] != "dry_cbl" and not args.no_learned:
            forms.append(("fp32+learned", "fp32", True))
    results = {}
    fields = None
    rs = None
    headline_sim = None
    trained = None
    for form, precision, learned in forms:
        nl = namelist_for(**cfg, precision=precision)
        sim = HotPathSimulation(nl, device=dev)
        if fields is None:
            fields = sim.initialize(seed=rank)
            rs = sim.RS.profiles()
        else:
            sim.set_reference_state(rs)
            sim.load_fields(fields)
        seed_info = None
        if learned:
            if trained is None:
                trained = _train_seed(sim, fields, log)
            if trained is not None:
                sim.Th.mlp, seed_info = trained
                if args.seed_refresh_interval:
                    sim.Th.seed_refresh_interval = args.seed_refresh_interval
        sim.run(0)  # ghost fill + first thermodynamics update, as Simulation3d.run
        _capi.clear_error()
        for _ in range(args.warmup):
            sim.step()
        torch.cuda.synchronize()
        elapsed_ms, comp_ms, launches, clock_info, secant = _time_steps(sim, args.steps, local_rank, world)
        npl = sim.Gr.dims.npl
        results[form] = {
            "value": world * npl * 3 * args.steps / (elapsed_ms / 1e3),
            "ms_per_step": elapsed_ms / args.steps,
            "component_ms_per_step": {c: round(v / args.steps, 4) for c, v in comp_ms.items()},
            "gpu_launches": launches, "clocks": clock_info, "secant": secant,
            "device_error_word": _capi.get_error(),
            "learned_seed": seed_info,
            "pressure_refine_sweeps": sim.Pr.refine_sweeps if precision == "fp32" else None,
        }
        log(f"form {form}: {results[form]['ms_per_step']:.2f} ms/step")
        if precision == "fp32" and sim._fused() and not args.no_unfused:
            # the same form with every call launched as called (no advection
            # deferred into the time step): what a caller that switches the
            # fusion off, or adds tendency terms, gets
            sim.fuse_rk = False
            sim.step()
            torch.cuda.synchronize()
            un_ms, un_comp, _, _, _ = _time_steps(sim, args.steps, local_rank, world)
            sim.fuse_rk = True
            sim.step()
            torch.cuda.synchronize()
            results[form]["unfused_ms_per_step"] = un_ms / args.steps
            results[form]["unfused_component_ms_per_step"] = {c: round(v / args.steps, 4) for c, v in un_comp.items()}
            results[form]["stage_calls"] = ("the reference's call order per stage (Th, SA, MA, TS, bcs, Pr); "
                                            "SA and MA deferred into TS.update, which runs the fused passes")
            log(f"form {form} unfused: {results[form]['unfused_ms_per_step']:.2f} ms/step")
        if not args.no_graph:
            results[form]["graph"] = _time_graph(sim, args.steps, local_rank, world)
            log(f"form {form} as CUDA graphs: {results[form]['graph']['ms_per_step']:.2f} ms/step")
        if form == forms[-1][0]:
            headline_sim = sim
        else:
            del sim
            torch.cuda.empty_cache()
    c4 = None
    if trained is not None and args.config == "c5_dycoms" and not args.no_c4:
        c4 = _learned_at_c4(trained, dev, args, log)
    head = forms[-1][0]
    sim = headline_sim
    PV, Gr = sim.PV, sim.Gr
    npl = Gr.dims.npl

    # ---- end to end through the public API with host buffers ---------------
    e2e = None
    if not args.no_e2e:
        import torch.distributed as dist
        stream = torch.cuda.current_stream(dev)
        host = torch.empty(PV.values.numel(), dtype=torch.float64, pin_memory=True)
        host.copy_(PV.values)
        # untimed warm-up through the same host-memory path (first touch of
        # the pinned buffer, copy-stream set-up), as for the device timing
        for _ in range(args.warmup):
            sim.step_host(host, stream=stream)
        for cs in sim.copy_streams():
            stream.wait_stream(cs)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            sim.step_host(host, stream=stream)
        for cs in sim.copy_streams():
            stream.wait_stream(cs)
        b.record(stream)
        torch.cuda.synchronize()
        te_ms = max_over_ranks(a.elapsed_time(b), dev, world)
        nbytes = PV.values.numel() * 8
        link = _link_gbs(host, PV.values, sim.copy_streams())
        e2e = {"value": world * npl * 3 * args.steps / (te_ms / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "form": head, "link": link, "what": "full prognostic state copied host->device before and device->host "
                                     "after every step (the reference keeps it in host numpy arrays), "
                                     "through HotPathSimulation.step_host (copies in quarter-variable chunks, each "
                                     "uploaded as soon as its download is done; the scalars are downloaded "
                                     "right after their last pass, the velocities after the last pressure "
                                     "solve, and the velocities' upload overlaps the first thermodynamics "
                                     "update)"}
        del host

    # ---- roofline per component; the headline is the largest one ----------
    peak, peak_kind = _peaks()
    surface = _time_surface(sim, cfg, peak) if not args.no_surface else None
    sgs = _time_sgs(sim, peak) if not args.no_surface else None
    stats = _time_stats(sim, peak) if not args.no_surface else None
    forcing = _time_forcing(sim, cfg, peak) if not args.no_surface else None
    r = results[head]
    nv = PV.nv
    comps = {}
    for comp, ms_step in r["component_ms_per_step"].items():
        ms = ms_step / 3.0  # per RK stage
        nbytes = COMPONENT_BYTES_PER_CELL[comp](nv, cfg, "fp32" in head)
        ach = nbytes * npl / (ms / 1e3) / 1e9
        comps[comp] = {"ms_per_stage": round(ms, 4), "algorithmic_bytes_per_cell_stage": nbytes,
                       "achieved_gbs": round(ach, 1), "frac": round(ach / peak, 4),
                       "traffic_bytes_per_stage": _read_traffic(args.config, head, comp)}
    flops_key = ("c5", 7) if cfg.get("scalar_order", 5) == 7 else (("moist", 5) if nv == 5 else ("dry", 5))
    adv_ms = comps["scalar_adv"]["ms_per_stage"] + comps["momentum_adv"]["ms_per_stage"]
    comps["scalar_adv+momentum_adv"] = {
        "flops_per_cell_stage": ADV_FLOPS_PER_CELL[flops_key],
        "achieved_tflops": round(ADV_FLOPS_PER_CELL[flops_key] * npl / (adv_ms / 1e3) / 1e12, 2)}
    # the headline is the dominant kernel: the single-launch component (one
    # kernel per RK stage, so its CUDA-event time is that kernel's launch
    # duration) with the largest time; every component is in "components"
    single = [c for c in r["component_ms_per_step"] if c == "thermo" or (c == "momentum_adv" and "fp32" in head)]
    top = max(single, key=lambda c: r["component_ms_per_step"][c])
    roofline = {"bound": "hbm", "achieved": comps[top]["achieved_gbs"], "peak": peak, "unit": "GB/s",
                "frac": comps[top]["frac"], "traffic": comps[top]["traffic_bytes_per_stage"],
                "peak_source": peak_kind, "kernel": COMPONENT_KERNELS[top],
                "algorithmic_bytes_per_cell_stage": comps[top]["algorithmic_bytes_per_cell_stage"],
                "launch_ms": comps[top]["ms_per_stage"],
                "note": ("bytes are compulsory bytes per launch over the CUDA-event launch time; "
                         + ("the thermodynamics is bound by its FP64 transcendentals, not by HBM"
                            if top == "thermo" else "the fused advection is bound by instruction issue")),
                "components": comps}

    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if head == "fp64" else "f32 fluxes/FFT, f64 accumulation, TDMA, secant",
            "data": "synthetic (seeded DYCOMS-RF01-like state)" if cfg["case"] == "dycoms" else "synthetic (seeded)",
            "config": {"workload": f"{args.config}: {cfg['nx']}x{cfg['ny']}x{cfg['nz']} cells, "
                                   f"gw={cfg['gw']}, WENO{cfg.get('scalar_order', 5)} scalars / "
                                   f"WENO{cfg.get('momentum_order', 5)} momentum, case={cfg['case']}, "
                                   f"dt={cfg['dt']}",
                       "form": head,
                       "cells": npl, "l2": "inputs larger than L2 (no flush needed)",
                       "parallelism": f"replicas x{world}"},
            "forms": results,
            "speedup_vs_fp64_plain": ({f: results[f]["value"] / results["fp64"]["value"] for f in results}
                                      if "fp64" in results else None),
            "component_ms_per_step": r["component_ms_per_step"],
            "roofline": roofline,
            "e2e": e2e,
            "learned_seed_c4": c4,
            "surface": surface,
            "sgs": sgs,
            "statistics": stats,
            "forcing": forcing,
            "gpu_launches": r["gpu_launches"],
            "clocks": r["clocks"],
            "device_error_word": r["device_error_word"],
        }
    return out, sim


def run_slabs(args, cfg, rank, world, local_rank):
    """The precision form over x-slabs of the configuration's domain (one
    slab per GPU; pycles_b200.parallel): device time of K steps after W
    warm-up steps, the slowest rank's, for the whole domain."""
    import torch

    from pycles_b200 import _capi, cases, parallel
    from pycles_b200.grid import Grid
    from pycles_b200.reference_state import ReferenceState
    from pycles_b200.simulation import namelist_for
    from pycles_b200.thermodynamics import ThermodynamicsDry, ThermodynamicsSA
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    nl = namelist_for(**cfg, precision="fp32")
    # the whole domain's seeded state, built the same way on every rank (host)
    Gr = Grid(nl)
    Gr.device = "cpu"
    RS = ReferenceState(Gr)
    Th = ThermodynamicsSA(nl) if cfg["case"] != "dry_cbl" else ThermodynamicsDry(nl)
    fields = cases.CASES[cfg["case"]](Gr, RS, Th, seed=0)
    comm = parallel.DistComm() if world > 1 else parallel.LocalComm(1)
    sh = parallel.ShardedSimulation(nl, comm, [dev])
    sh.load_global(RS.profiles(), fields)
    del fields
    sh.run(0)
    _capi.clear_error()
    for _ in range(args.warmup):
        sh.step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    stream = torch.cuda.current_stream(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    L = _capi.load()
    n0 = L.pb_launch_count()
    a.record(stream)
    for _ in range(args.steps):
        sh.step()
    b.record(stream)
    torch.cuda.synchronize()
    launches = L.pb_launch_count() - n0
    ms = max_over_ranks(a.elapsed_time(b), dev, world)
    npl = cfg["nx"] * cfg["ny"] * cfg["nz"]
    return {"metric": METRIC, "value": npl * 3 * args.steps / (ms / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32 fluxes/FFT, f64 accumulation, TDMA, secant",
            "data": "synthetic (seeded)",
            "config": {"workload": f"{args.config}: {cfg['nx']}x{cfg['ny']}x{cfg['nz']} cells in {world} x-slabs",
                       "form": "fp32", "cells": npl, "l2": "inputs larger than L2 (no flush needed)",
                       "parallelism": f"x-slabs x{world}"},
            "e2e": None, "gpu_launches": launches, "device_error_word": _capi.get_error()}


def _time_graph(sim, steps, local_rank, world):
    """The same steps recorded as CUDA graphs (HotPathSimulation.capture_steps:
    graph_steps() time steps per graph, one host launch per replay) and
    replayed: ms per step over the replays that fit in `steps`, at least
    one; the state advances as with eager steps."""
    import torch
    n = sim.graph_steps()
    g = sim.capture_steps()
    g.replay()  # warm-up
    torch.cuda.synchronize()
    reps = max(1, steps // n)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        g.replay()
    b.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(a.elapsed_time(b), torch.device("cuda", local_rank), world) / (reps * n)
    del g
    return {"ms_per_step": ms, "steps_per_graph": n, "replays": reps,
            "value": world * sim.Gr.dims.npl * 3 / (ms / 1e3)}


def _link_gbs(host, dev_buf, streams, reps=3):
    """Host<->device copy bandwidth of the state's own pinned buffer, GB/s:
    each direction alone and both at once (the two copy streams of
    step_host), best of `reps`; what bounds the end-to-end step."""
    import torch
    h2d, d2h = streams
    nbytes = dev_buf.numel() * 8
    scratch = torch.empty_like(host, pin_memory=True)
    out = {}
    for name, jobs in (("h2d", ((h2d, dev_buf, host),)), ("d2h", ((d2h, scratch, dev_buf),)),
                       ("both", ((h2d, dev_buf, host), (d2h, scratch, dev_buf)))):
        best = 0.0
        for _ in range(reps):
            torch.cuda.synchronize()
            start = torch.cuda.Event(enable_timing=True)
            start.record(torch.cuda.current_stream())
            ends = []
            for st, dst, src in jobs:
                st.wait_event(start)
                with torch.cuda.stream(st):
                    dst.copy_(src, non_blocking=True)
                e = torch.cuda.Event(enable_timing=True)
                e.record(st)
                ends.append(e)
            torch.cuda.synchronize()
            ms = max(start.elapsed_time(e) for e in ends)
            best = max(best, len(jobs) * nbytes / (ms / 1e3) / 1e9)
        out[name + "_gbs"] = round(best, 1)
    out["bytes_per_copy"] = nbytes
    del scratch
    return out


def run_accuracy(args, cfg):
    """Error of the precision forms against the FP64 plain form: the three
    forms start from the same seeded state and run N steps; per field the
    relative L2 difference after 1 and N steps.  (The plain form equals the
    reference's FP64 path to ~1e-13 after one step on the parity grids.)"""
    import numpy as np
    import torch

    from pycles_b200.simulation import HotPathSimulation, namelist_for
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    log = lambda m: print(m, file=sys.stderr)
    n = args.accuracy_steps
    forms = [("fp64", "fp64", False), ("fp32", "fp32", False)]
    if cfg["case"] != "dry_cbl" and not args.no_learned:
        forms.append(("fp32+learned", "fp32", True))
    fields, rs, trained = None, None, None
    snaps = {}
    for form, precision, learned in forms:
        sim = HotPathSimulation(namelist_for(**cfg, precision=precision), device=dev)
        if fields is None:
            fields = sim.initialize(seed=0)
            rs = sim.RS.profiles()
        else:
            sim.set_reference_state(rs)
            sim.load_fields(fields)
        if learned:
            trained = trained or _train_seed(sim, fields, log)
            if trained is not None:
                sim.Th.mlp = trained[0]
                if args.seed_refresh_interval:
                    sim.Th.seed_refresh_interval = args.seed_refresh_interval
        sim.run(0)
        sim.step()
        snaps[form] = {1: sim.host_fields()}
        t0 = time.time()
        for _ in range(n - 1):
            sim.step()
        snaps[form][n] = sim.host_fields()
        sim.check_device_errors()
        log(f"{form}: {n} steps in {time.time() - t0:.1f} s")
        del sim
        torch.cuda.empty_cache()
    err = {}
    for form in snaps:
        if form == "fp64":
            continue
        err[form] = {}
        for step in (1, n):
            a, b = snaps[form][step], snaps["fp64"][step]
            e = {name: float(np.linalg.norm(a[name] - b[name]) / np.linalg.norm(b[name])) for name in b}
            vel = np.sqrt(sum(np.linalg.norm(b[m]) ** 2 for m in ("u", "v", "w")))
            e["velocity_pooled"] = float(np.sqrt(sum(np.linalg.norm(a[m] - b[m]) ** 2 for m in ("u", "v", "w")))
                                         / vel)
            err[form][f"after_{step}_steps"] = e
    return {"accuracy": err, "reference_form": "fp64 plain", "steps": n,
            "config": {"workload": f"{args.config}: {cfg['nx']}x{cfg['ny']}x{cfg['nz']} cells", **cfg},
            "norm": ("relative L2 per field, each field against its own norm; velocity_pooled: the difference "
                     "of (u, v, w) against the norm of the whole velocity field")}


def _read_traffic(config, form, component):
    """DRAM bytes per RK stage of a component's kernels, from the committed
    ncu summaries (profiles/*.md lines
    'traffic_bytes_per_stage[<config>,<form>,<component>]: N'), or None."""
    import glob
    import re
    key = rf"traffic_bytes_per_stage\[{re.escape(config)},{re.escape(form)},{re.escape(component)}\]:\s*([0-9.eE+]+)"
    for p in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        try:
            txt = open(p).read()
        except OSError:
            continue
        m = re.search(key, txt)
        if m:
            return float(m.group(1))
    return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c5_dycoms")
    ap.add_argument("--form", default="all", choices=["all", "fp64", "fp32"],
                    help="fp64: plain form; fp32: precision form without and with the learned seed; "
                         "all: every form, headline the last (fp32+learned)")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-unfused", action="store_true",
                    help="skip timing the precision forms with every call launched as called")
    ap.add_argument("--no-c4", action="store_true",
                    help="skip the learned seed's measurement at 256x256x128 (c4_dycoms)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--decomposition", default="replicas", choices=["replicas", "slabs"],
                    help="replicas: every GPU steps its own copy of the configuration (weak scaling); "
                         "slabs: the configuration's domain split in x-slabs across the GPUs, halo "
                         "exchanges and the pressure's transposes over NCCL (strong scaling)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-graph", action="store_true",
                    help="skip the per-form timing of the steps recorded as CUDA graphs")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-surface", action="store_true",
                    help="skip the timings of the case's surface scheme and forcing, of the Smagorinsky "
                         "subgrid scale and diffusion and of a horizontal mean (reported beside the step)")
    ap.add_argument("--cpu-cores", type=int, default=None)
    ap.add_argument("--seed-refresh-interval", type=int, default=0,
                    help="thermodynamics updates between refreshes of the learned seed (default: the "
                         "library's, gpu.seed_refresh_interval)")
    ap.add_argument("--accuracy-steps", type=int, default=0,
                    help="instead of timing: run every form N steps from the same state and report each "
                         "field's relative L2 error against the FP64 plain form after 1 and N steps")
    ap.add_argument("--grid", default=None, metavar="NXxNYxNZ",
                    help="override the configuration's cell counts (orders, gw, case and spacing kept), "
                         "e.g. a reduced case for profiler captures")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    from pycles_b200.simulation import CONFIGS
    if args.grid:
        nx, ny, nz = (int(t) for t in args.grid.lower().split("x"))
        CONFIGS[args.config] = dict(CONFIGS[args.config], nx=nx, ny=ny, nz=nz)
    cfg = dict(CONFIGS[args.config])

    if args.accuracy_steps > 0:
        print(json.dumps(run_accuracy(args, cfg)))
        return 0

    if args.impl == "reference":
        if rank != 0:
            return 0
        per_step, info = cpu_reference_run(cfg, args.steps, args.warmup, backend="ref", cores=args.cpu_cores)
        value = statistics.mean(per_step)
        info["value"] = value
        info["unit"] = UNIT
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": f"{args.config}: per-core sub-domains of the same configuration",
                       "parallelism": f"{info['cores']} host processes"},
            "cpu_baseline": info,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return 0

    # CPU baseline first (spawned workers, before any CUDA context exists)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            per_step, info = cpu_reference_run(cfg, 1, 1, backend="ref", cores=args.cpu_cores)
            info["value"] = per_step[0]
            info["unit"] = UNIT
            cpu = info
        except Exception as e:  # reported, not fatal
            cpu = {"error": str(e)[:200]}

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    if args.decomposition == "slabs":
        out = run_slabs(args, cfg, rank, world, local_rank)
    else:
        out, _ = run_ours(args, rank, world, local_rank)
    if rank == 0:
        out["cpu_baseline"] = cpu
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
