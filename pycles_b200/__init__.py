"""pycles_b200: the PyCLES per-timestep hot path on NVIDIA B200 (sm_100a).

Components keep the reference's Python-side API (``update`` signatures of
ScalarAdvection, MomentumAdvection, PressureSolver, ThermodynamicsSA/Dry,
TimeStepping, PrognosticVariables.Update_all_bcs) and run through the C ABI
of ``include/pycles_b200.h`` implemented in ``csrc/``.
"""
from ._capi import PbError, load  # noqa: F401
from .advection import MomentumAdvection, ScalarAdvection  # noqa: F401
from .grid import Grid  # noqa: F401
from .pressure import PressureSolver  # noqa: F401
from .reference_state import ReferenceState  # noqa: F401
from .simulation import CONFIGS, HotPathSimulation, namelist_for  # noqa: F401
from .thermodynamics import ClausiusClapeyron, ThermodynamicsDry, ThermodynamicsSA  # noqa: F401
from .time_stepping import TimeStepping  # noqa: F401
from .variables import DiagnosticVariables, PrognosticVariables  # noqa: F401
