"""B200-native FDM micromagnetic time-stepper (Exchange + Demag + Zeeman + LLG).

The compute path is libfullmag_fdm.so.0 (fullmag_b200/csrc, sm_100a), a
drop-in for the reference's C ABI (include/fullmag_fdm.h).  This package holds
its build recipe and the Python host binding.
"""
from .native_fdm import (  # noqa: F401
    FdmPlan, NativeFdmBackend, RunError, is_available, load_library, newell_spectra,
    MU0, HEUN, DP45, PRECISION_SINGLE, PRECISION_DOUBLE,
    OBS_M, OBS_H_EX, OBS_H_DEMAG, OBS_H_EXT, OBS_H_EFF, DEMAG_FROM_PLAN, DEMAG_NEWELL,
)
