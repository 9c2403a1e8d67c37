"""Shared test helpers: seeded states, oracle and GPU simulations built from
the same inputs, and the relative-L2 metric used by every parity check."""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    num = np.linalg.norm(a - b)
    return num / den if den > 0 else num


def host_case(case="bomex", nx=12, ny=10, nz=16, dx=100.0, dy=100.0, dz=40.0, gw=3, dt=1.0,
              scalar_order=5, momentum_order=5, seed=0):
    """Seeded initial state built on the host (no GPU): returns
    (namelist, reference-state profiles, {field: flat array})."""
    import torch  # noqa: F401  (package import needs torch)
    from pycles_b200 import cases
    from pycles_b200.grid import Grid
    from pycles_b200.reference_state import ReferenceState
    from pycles_b200.simulation import namelist_for
    from pycles_b200.thermodynamics import ThermodynamicsDry, ThermodynamicsSA

    nl = namelist_for(case, nx, ny, nz, dx, dy, dz, gw=gw, dt=dt, scalar_order=scalar_order,
                      momentum_order=momentum_order)
    Gr = Grid(nl)
    Gr.device = "cpu"
    RS = ReferenceState(Gr)
    Th = ThermodynamicsSA(nl) if case != "dry_cbl" else ThermodynamicsDry(nl)
    fields = cases.CASES[case](Gr, RS, Th, seed=seed)
    return nl, RS.profiles(), fields


def oracle_dims(nl):
    from oracle.dims import Dims
    g = nl["grid"]
    return Dims((g["nx"], g["ny"], g["nz"]), g["gw"], (g["dx"], g["dy"], g["dz"]))


def oracle_sim(nl, rs, fields, backend="port"):
    from oracle.glue import OracleSim
    d = oracle_dims(nl)
    sim = OracleSim(d, rs, moist=nl["case"] != "dry_cbl", scalar_order=nl["scalar_transport"]["order"],
                    momentum_order=nl["momentum_transport"]["order"], dt=nl["time_stepping"]["dt_initial"],
                    backend=backend)
    for name, arr in fields.items():
        sim.var(name)[:] = arr
    return sim


def gpu_sim(nl, rs, fields, precision="fp64"):
    from pycles_b200.simulation import HotPathSimulation
    nl = dict(nl)
    nl["gpu"] = dict(nl.get("gpu", {}), precision=precision)
    sim = HotPathSimulation(nl, device="cuda")
    sim.set_reference_state(rs)
    sim.load_fields(fields)
    return sim


def gpu_fields(sim):
    import torch
    torch.cuda.synchronize()
    return {n: sim.PV.field(n, sim.Gr).cpu().numpy() for n in sim.PV.index_name}


def gpu_tends(sim):
    return {n: sim.PV.tendency(n, sim.Gr).cpu().numpy() for n in sim.PV.index_name}


def gpu_dv(sim):
    return {n: sim.DV.field(n, sim.Gr).cpu().numpy() for n in sim.DV.index_name}
