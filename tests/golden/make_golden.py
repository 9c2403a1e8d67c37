"""Generate the golden fixtures of the hot path from the reference's own C.

    python tests/golden/make_golden.py [fixture names]

Needs oracle/_ref (the reference's C kernels and its Cython TDMA compiled
from the reference tree by oracle/build_ref.py).  For each case it stores
the seeded input state and reference-state profiles, and the outputs of the
reference kernels driven by the restated glue (oracle.glue, backend "ref"):
thermodynamics, scalar advection, momentum advection, pressure, one full
time step, and Simulation3d.run's prologue + one step.  The surface
fixtures hold, per surface scheme, the scheme's update after the
thermodynamics and one time step with the scheme in the stage; the sgs
fixtures the strain-rate magnitude, viscosity and diffusivity, the scalar
and momentum diffusion tendencies and one time step with them; the case
fixtures the case forcing's tendencies and one time step of the whole case
(surface, forcing, subgrid scale).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

CASES = {
    "moist_w5": dict(case="bomex", nx=12, ny=10, nz=16, dx=100.0, dy=100.0, dz=40.0, gw=3, dt=1.0),
    "moist_w7": dict(case="bomex", nx=8, ny=12, nz=14, dx=100.0, dy=100.0, dz=40.0, gw=4, dt=1.0,
                     scalar_order=7, momentum_order=7),
    "dry_w5": dict(case="dry_cbl", nx=8, ny=8, nz=12, dx=50.0, dy=50.0, dz=50.0, gw=3, dt=0.5),
}


def stir(fields, seed=1, amp=0.5):
    rng = np.random.default_rng(seed)
    out = dict(fields)
    for n in ("u", "v", "w"):
        out[n] = fields[n] + amp * rng.standard_normal(fields[n].shape)
    if "qt" in out:
        out["qt"] = fields["qt"] + 6e-3  # part of the column saturated
    return out


def make(name, cfg):
    from helpers import host_case, oracle_sim
    from oracle import ref
    assert ref.available(), "oracle/_ref missing: run oracle/build_ref.py"
    nl, rs, f0 = host_case(**cfg)
    f = stir(f0)
    out = {"rs_" + k: v for k, v in rs.items()}
    for k, v in f.items():
        out["in_" + k] = v
    # whole-step outputs start from the unstirred state (white-noise
    # velocities are not a state a time step should be asked to take)
    for k, v in f0.items():
        out["in0_" + k] = v

    def sim(fields=f):
        s = oracle_sim(nl, rs, fields, backend="ref")
        s.update_all_bcs()
        return s

    s = sim()
    for k in s.names:
        out["bcs_" + k] = s.var(k).copy()
    s.th_update()
    for k, v in s.dv.items():
        out["th_" + k] = v.copy()
    out["th_wtend"] = s.tend("w").copy()
    s = sim()
    s.sa_update()
    for k in s.names[3:]:
        out["sa_" + k] = s.tend(k).copy()
    s = sim()
    s.ma_update()
    for k in ("u", "v", "w"):
        out["ma_" + k] = s.tend(k).copy()
    s = sim()
    s.pr_update()
    for k in ("u", "v", "w"):
        out["pr_" + k] = s.var(k).copy()
    out["pr_p"] = s.dv["dynamic_pressure"].copy()
    out["pr_div"] = s.dv["divergence"].copy()
    s = sim(f0)
    s.step()
    for k in s.names:
        out["step_" + k] = s.var(k).copy()
    s = oracle_sim(nl, rs, f0, backend="ref")
    s.update_all_bcs()
    s.th_update()
    s.step()
    for k in s.names:
        out["run1_" + k] = s.var(k).copy()
    meta = np.array([repr(cfg)])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=meta, **out)


# surface schemes (Surface.pyx) on the case each belongs to
SURFACE_CASES = {
    "surface_sullivan_patton": ("SullivanPatton", dict(case="dry_cbl", nx=8, ny=8, nz=12, dx=50.0, dy=50.0,
                                                       dz=50.0, gw=3, dt=0.5)),
    "surface_bomex": ("Bomex", dict(case="bomex", nx=12, ny=10, nz=16, dx=100.0, dy=100.0, dz=40.0, gw=3,
                                    dt=1.0)),
    "surface_dycoms_rf01": ("DYCOMS_RF01", dict(case="dycoms", nx=8, ny=10, nz=16, dx=35.0, dy=35.0, dz=60.0,
                                                gw=4, dt=0.25, scalar_order=7, momentum_order=5)),
}


def make_surface(name, scheme, cfg):
    """The surface scheme's update after the thermodynamics (fluxes and the
    tendencies of the first interior level), and one time step with the
    scheme and the case's forcing in the stage, from the reference's C driven
    by the restated glue."""
    from helpers import host_case, oracle_dims, oracle_sim
    from oracle import ref
    from oracle.surface import OracleSurface
    assert ref.available(), "oracle/_ref missing: run oracle/build_ref.py"
    nl, rs, f0 = host_case(**cfg)
    f = stir(f0)
    d = oracle_dims(nl)
    out = {"rs_" + k: np.asarray(v) for k, v in rs.items()}
    for k, v in f.items():
        out["in_" + k] = v
    for k, v in f0.items():
        out["in0_" + k] = v
    s = oracle_sim(nl, rs, f, backend="ref")
    s.update_all_bcs()
    s.th_update()
    s.tendencies[:] = 0.0
    s.surface = OracleSurface(scheme, d, u0=rs["u0"], v0=rs["v0"])
    s.surface.update(s)
    for n in OracleSurface.NAMES:
        out["sur_" + n] = getattr(s.surface, n).copy()
    for k in s.names:
        out["surtend_" + k] = s.tend(k).copy()
    # the case name selects the forcing too (Forcing.pyx:29-67)
    from oracle.forcing import OracleForcing
    from pycles_b200.grid import Grid
    s = oracle_sim(nl, rs, f0, backend="ref")
    s.surface = OracleSurface(scheme, d, u0=rs["u0"], v0=rs["v0"])
    s.forcing = OracleForcing(scheme, d, rs["p0_half"], Grid(nl).zl_half, u0=rs["u0"], v0=rs["v0"])
    if scheme == "DYCOMS_RF01":  # RadiationFactory (Radiation.pyx:30-57)
        from oracle.radiation import OracleRadiation
        s.radiation = OracleRadiation(d, Grid(nl).z)
    s.update_all_bcs()
    s.step()
    for k in s.names:
        out["step_" + k] = s.var(k).copy()
    meta = np.array([repr(cfg), scheme])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=meta, **out)


# subgrid scale and diffusion (SGS.pyx, Kinematics.pyx, ScalarDiffusion.pyx,
# MomentumDiffusion.pyx): namelist sections as the reference reads them
SGS_CASES = {
    "sgs_smagorinsky_bomex": (dict(case="bomex", nx=12, ny=10, nz=16, dx=100.0, dy=100.0, dz=40.0, gw=3, dt=1.0),
                              {"sgs": {"scheme": "Smagorinsky"}, "diffusion": {"qt_entropy_source": True}}),
    "sgs_smagorinsky_iles_bomex": (dict(case="bomex", nx=10, ny=12, nz=14, dx=100.0, dy=100.0, dz=40.0, gw=3,
                                        dt=1.0),
                                   {"sgs": {"scheme": "Smagorinsky", "Smagorinsky": {"iles": True, "cs": 0.2}}}),
    "sgs_smagorinsky_wall_dry": (dict(case="dry_cbl", nx=8, ny=8, nz=12, dx=50.0, dy=50.0, dz=50.0, gw=3, dt=0.5),
                                 {"sgs": {"scheme": "Smagorinsky", "Smagorinsky": {"wall": True}},
                                  "meta": {"casename": "SullivanPatton"}}),
    "sgs_uniform_dycoms": (dict(case="dycoms", nx=8, ny=10, nz=16, dx=35.0, dy=35.0, dz=60.0, gw=4, dt=0.25,
                                scalar_order=7, momentum_order=5),
                           {"sgs": {"scheme": "UniformViscosity",
                                    "UniformViscosity": {"viscosity": 75.0, "diffusivity": 75.0}}}),
}


def make_sgs(name, cfg, extra):
    """Kinematics + SGS after the thermodynamics, the scalar and momentum
    diffusion tendencies, and one time step with them (and the case's
    surface scheme when the namelist names one), from the reference's C
    driven by the restated glue."""
    from helpers import host_case, oracle_dims, oracle_sim
    from oracle import ref
    from oracle.sgs import OracleSGS, scheme_from_namelist
    from oracle.surface import OracleSurface
    from pycles_b200.grid import Grid
    assert ref.available(), "oracle/_ref missing: run oracle/build_ref.py"
    nl, rs, f0 = host_case(**cfg)
    nl = dict(nl, **extra)
    f = stir(f0)
    d = oracle_dims(nl)
    zl_half = Grid(nl).zl_half
    conf = scheme_from_namelist(nl)
    casename = extra.get("meta", {}).get("casename")

    def attach(s):
        s.sgs = OracleSGS(conf, d, zl_half)
        if casename:
            from oracle.forcing import OracleForcing
            s.surface = OracleSurface(casename, d, u0=rs["u0"], v0=rs["v0"])
            s.forcing = OracleForcing(casename, d, rs["p0_half"], zl_half, u0=rs["u0"], v0=rs["v0"])
        return s

    out = {"rs_" + k: np.asarray(v) for k, v in rs.items()}
    for k, v in f.items():
        out["in_" + k] = v
    for k, v in f0.items():
        out["in0_" + k] = v
    s = attach(oracle_sim(nl, rs, f, backend="ref"))
    s.update_all_bcs()
    s.sgs.ke_update(s)
    s.th_update()
    s.sgs.sgs_update(s)
    out["sgs_strain_rate_mag"] = s.sgs.strain_rate_mag.copy()
    out["sgs_viscosity"] = s.sgs.viscosity.copy()
    out["sgs_diffusivity"] = s.sgs.diffusivity.copy()
    s.tendencies[:] = 0.0
    s.sgs.sd_update(s)
    for k in s.names:
        out["sdtend_" + k] = s.tend(k).copy()
    s.tendencies[:] = 0.0
    s.sgs.md_update(s)
    for k in s.names:
        out["mdtend_" + k] = s.tend(k).copy()
    s = attach(oracle_sim(nl, rs, f0, backend="ref"))
    s.update_all_bcs()
    s.step()
    for k in s.names:
        out["step_" + k] = s.var(k).copy()
    meta = np.array([repr(cfg), repr(extra)])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=meta, **out)


# whole cases: the case's surface scheme and forcing (and, where given, the
# subgrid scale), chosen by meta.casename as the reference does
FORCING_CASES = {
    "case_bomex": (dict(case="bomex", nx=12, ny=10, nz=16, dx=100.0, dy=100.0, dz=40.0, gw=3, dt=1.0),
                   {"meta": {"casename": "Bomex"}}),
    "case_dycoms_rf01": (dict(case="dycoms", nx=8, ny=10, nz=16, dx=35.0, dy=35.0, dz=60.0, gw=4, dt=0.25,
                              scalar_order=7, momentum_order=5),
                         {"meta": {"casename": "DYCOMS_RF01"}, "sgs": {"scheme": "Smagorinsky"}}),
    "case_sullivan_patton": (dict(case="dry_cbl", nx=8, ny=8, nz=12, dx=50.0, dy=50.0, dz=50.0, gw=3, dt=0.5),
                             {"meta": {"casename": "SullivanPatton"},
                              "sgs": {"scheme": "Smagorinsky", "Smagorinsky": {"wall": True}}}),
}


def make_case(name, cfg, extra):
    """The case forcing's tendencies after the thermodynamics, and one time
    step with the case's surface, forcing and subgrid scale in the stage."""
    from helpers import host_case, oracle_dims, oracle_sim
    from oracle import ref
    from oracle.forcing import OracleForcing
    from oracle.sgs import OracleSGS, scheme_from_namelist
    from oracle.surface import OracleSurface
    from pycles_b200.grid import Grid
    assert ref.available(), "oracle/_ref missing: run oracle/build_ref.py"
    nl, rs, f0 = host_case(**cfg)
    nl = dict(nl, **extra)
    f = stir(f0)
    d = oracle_dims(nl)
    zl_half = Grid(nl).zl_half
    casename = extra["meta"]["casename"]

    def attach(s):
        s.surface = OracleSurface(casename, d, u0=rs["u0"], v0=rs["v0"])
        s.forcing = OracleForcing(casename, d, rs["p0_half"], zl_half, u0=rs["u0"], v0=rs["v0"])
        if "sgs" in nl:
            s.sgs = OracleSGS(scheme_from_namelist(nl), d, zl_half)
        if casename == "DYCOMS_RF01":  # RadiationFactory (Radiation.pyx:30-57)
            from oracle.radiation import OracleRadiation
            s.radiation = OracleRadiation(d, Grid(nl).z)
        return s

    out = {"rs_" + k: np.asarray(v) for k, v in rs.items()}
    for k, v in f.items():
        out["in_" + k] = v
    for k, v in f0.items():
        out["in0_" + k] = v
    s = attach(oracle_sim(nl, rs, f, backend="ref"))
    s.update_all_bcs()
    s.th_update()
    s.tendencies[:] = 0.0
    s.forcing.update(s)
    for k in s.names:
        out["fotend_" + k] = s.tend(k).copy()
    if s.radiation is not None:
        s.tendencies[:] = 0.0
        s.radiation.update(s)
        out["ratend_s"] = s.tend("s").copy()
        out["ra_heating_rate"] = s.radiation.heating_rate.copy()
        out["ra_dTdt_rad"] = s.radiation.dTdt_rad.copy()
    s = attach(oracle_sim(nl, rs, f0, backend="ref"))
    s.update_all_bcs()
    s.step()
    for k in s.names:
        out["step_" + k] = s.var(k).copy()
    meta = np.array([repr(cfg), repr(extra)])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=meta, **out)


def main(names=None):
    for name, cfg in CASES.items():
        if not names or name in names:
            make(name, cfg)
            print("wrote", name)
    for name, (scheme, cfg) in SURFACE_CASES.items():
        if not names or name in names:
            make_surface(name, scheme, cfg)
            print("wrote", name)
    for name, (cfg, extra) in SGS_CASES.items():
        if not names or name in names:
            make_sgs(name, cfg, extra)
            print("wrote", name)
    for name, (cfg, extra) in FORCING_CASES.items():
        if not names or name in names:
            make_case(name, cfg, extra)
            print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1:])
