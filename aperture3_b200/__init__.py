"""aperture3_b200: the Aperture3 particle update for NVIDIA B200 (sm_100a).

The Vay push fused with charge-conserving (Esirkepov) current deposition,
the per-step tile counting sort and the Yee FDTD field update, as
hand-written CUDA kernels in libaperture_b200.so behind a C ABI
(include/aperture_b200.h). This package is the host-side mirror of the
reference's lab-facing classes (ptc_updater, field_solver, sim_environment,
sim_data) over that ABI. There is no CPU fallback: importing the classes
loads the library and fails if it is missing.
"""
from . import _lib  # noqa: F401
from .sim import (Batch, FLAG_IGNORE_CURRENT, FLAG_IGNORE_EM, ELECTRON, ION, POSITRON, FieldSolver,
                  FieldSolver1dGap, FieldSolverLogsph, PtcUpdater, PtcUpdater1dGap,
                  PtcUpdaterLogsph, SimData, SimEnvironment, SimParams, field_solver,
                  field_solver_1dgap, field_solver_1dgr, field_solver_logsph, inverse_compton,
                  ptc_updater, ptc_updater_1dgap, ptc_updater_1dgr, ptc_updater_logsph,
                  radiative_transfer, species_flag)

__all__ = [
    "Batch", "SimParams", "SimEnvironment", "SimData", "ptc_updater", "field_solver", "PtcUpdater",
    "FieldSolver", "ptc_updater_logsph", "field_solver_logsph", "PtcUpdaterLogsph",
    "FieldSolverLogsph", "ptc_updater_1dgap", "field_solver_1dgap", "PtcUpdater1dGap",
    "FieldSolver1dGap", "ptc_updater_1dgr", "field_solver_1dgr", "radiative_transfer",
    "inverse_compton", "species_flag", "ELECTRON",
    "POSITRON", "ION", "FLAG_IGNORE_EM", "FLAG_IGNORE_CURRENT",
]
